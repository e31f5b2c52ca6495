// engine.cuh -- the step engine class behind include/meu.h (implementation in
// engine.cu) and its launch counter / per-kernel timer.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/meu.h"
#include "fft.cuh"
#include "landau_fused.cuh"

namespace meu {
// proportional-moduli polarization coefficients, passed by value to k_el_x_prop
// (W = double) and to the fused row kernel (W = the field precision)
template <typename W>
struct ElxCoef {
  W c0[36], c1[36], ebar[6];
  W ep[MEU_MAX_VAR][6];
  W av[MEU_MAX_VAR];   // alpha of the variant's phase, 0 for phase-1 variants
  W inc[MEU_MAX_VAR];  // 1 when the variant counts toward sum P (phase >= 2)
  int nvar;
  template <typename U>
  void assign(const ElxCoef<U>& o) {
    for (int i = 0; i < 36; ++i) {
      c0[i] = (W)o.c0[i];
      c1[i] = (W)o.c1[i];
    }
    for (int m = 0; m < 6; ++m) ebar[m] = (W)o.ebar[m];
    for (int v = 0; v < MEU_MAX_VAR; ++v) {
      for (int m = 0; m < 6; ++m) ep[v][m] = (W)o.ep[v][m];
      av[v] = (W)o.av[v];
      inc[v] = (W)o.inc[v];
    }
    nvar = o.nvar;
  }
};
using ElxProp = ElxCoef<double>;
// proportional-moduli elastic-energy coefficients, passed by value to k_elener_prop
struct ElenProp {
  double c1[36], s1[36], emean[6];
  double tp[MEU_MAX_VAR][6];  // trans_ppt (tensor shear)
  double av[MEU_MAX_VAR];     // alpha of the variant's phase, 0 for phase-1 variants
  int use[MEU_MAX_VAR];       // phase >= 2 and use_var: gets an energy share and a driving force
  int nvar;
};
// x-direction work of one elastic iteration in one pass (el_rows.cu): x C2R of the six
// strain spectra, polarisation, x R2C into the same spectra; row length nx/2 a power
// of two in 32..512 (el_rows_ok)
bool el_rows_ok(int nx);
template <typename R>
void el_rows_launch(const FFT3& f, const PtrList<cplx<R>>& sp, const R* pphi, const ElxCoef<R>& E, bool ortho,
                    double cfac, int* err, cudaStream_t st);
}  // namespace meu

namespace meu {

// ==========================================================================
// Launch counter and per-kernel CUDA-event timing (off unless requested).
class Profiler : public LaunchHook {
 public:
  int64_t launches = 0;
  bool on = false;
  struct Stat { int64_t n = 0; double ms = 0, bytes = 0; };
  std::vector<std::string> names;
  std::vector<Stat> stats;
  ~Profiler() override {
    for (auto& q : pend) { cudaEventDestroy(q.a); cudaEventDestroy(q.b); }
    for (auto e : pool) cudaEventDestroy(e);
  }
  void begin(const char* n, double b, cudaStream_t st) override {
    ++launches;
    if (!on) return;
    cur_id = id_of(n);
    cur_bytes = b;
    cur_a = get();
    MEU_CUDA(cudaEventRecord(cur_a, st));
  }
  bool timing() const override { return on; }
  void end(cudaStream_t st) override {
    if (!on) return;
    cudaEvent_t e = get();
    MEU_CUDA(cudaEventRecord(e, st));
    pend.push_back({cur_id, cur_bytes, cur_a, e});
  }
  void resolve() {
    for (auto& q : pend) {
      MEU_CUDA(cudaEventSynchronize(q.b));
      float ms = 0;
      MEU_CUDA(cudaEventElapsedTime(&ms, q.a, q.b));
      stats[q.id].n += 1;
      stats[q.id].ms += ms;
      stats[q.id].bytes += q.bytes;
      pool.push_back(q.a);
      pool.push_back(q.b);
    }
    pend.clear();
  }
  void reset() {
    resolve();
    names.clear();
    stats.clear();
  }

 private:
  struct Pend { int id; double bytes; cudaEvent_t a, b; };
  std::vector<Pend> pend;
  std::vector<cudaEvent_t> pool;
  int cur_id = 0;
  double cur_bytes = 0;
  cudaEvent_t cur_a = nullptr;
  int id_of(const char* n) {
    for (size_t i = 0; i < names.size(); ++i)
      if (names[i] == n) return (int)i;
    names.push_back(n);
    stats.push_back(Stat());
    return (int)names.size() - 1;
  }
  cudaEvent_t get() {
    if (pool.empty()) {
      cudaEvent_t e;
      MEU_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
};

#define KLAUNCH(name, bytes, ...)  \
  do {                             \
    prof.begin(name, bytes, st);   \
    __VA_ARGS__;                   \
    MEU_CHECK_LAUNCH();            \
    prof.end(st);                  \
  } while (0)

// ==========================================================================
struct EngineBase {
  virtual ~EngineBase() {}
  virtual void set_fields(const double* cons, const double* phi, const double* ustate) = 0;
  virtual void add_noise(const double* incr) = 0;
  virtual void run(int nsteps, meu_diag* diag) = 0;
  // nsteps steps with the Langevin increments of the noisy steps drawn on a host
  // thread from the caller's ran_2 state while the previous step runs
  virtual void run_noise(int nsteps, meu_ran2_state* rng, double sd, meu_diag* diag) = 0;
  virtual void get_fields(double* cons, double* phi, double* el_en, double* ustate) = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual bool schedule(int32_t* out3) const = 0;
  virtual void set_schedule(const int32_t* in3) = 0;
  // loss and gradient of the last of nsteps steps from the current fields (adjoint.cu)
  virtual void adjoint(int nsteps, int checkpoint_every, const double* cons_tgt, const double* phi_tgt, double* loss,
                       double* dparams, double* dphi0) = 0;
  int64_t step = 0;
  std::string err;
  Profiler prof;
};

template <typename R>
class EnsembleT;
template <typename R>
struct AdjBuffers;
template <typename R>
void adj_buffers_free(AdjBuffers<R>* b);

template <typename R>
class Engine : public EngineBase {
  using C = cplx<R>;
  friend class EnsembleT<R>;

 public:
  explicit Engine(const meu_params& p);
  ~Engine() override;
  void set_fields(const double* cons, const double* phi, const double* ustate) override;
  void add_noise(const double* incr) override;
  void run(int nsteps, meu_diag* diag) override;
  void run_noise(int nsteps, meu_ran2_state* rng, double sd, meu_diag* diag) override;
  void get_fields(double* cons, double* phi, double* el_en, double* ustate) override;
  void set_stream(cudaStream_t s) override { st = s ? s : own_st; }
  bool schedule(int32_t* out3) const override {
    if (!fused) {  // generic path: radix plan and column-tile factor of its transforms
      out3[0] = fft->pv;
      out3[1] = 0;
      out3[2] = fft->ct;
      return true;
    }
    out3[0] = sched.pv;
    out3[1] = sched.ntp;
    out3[2] = sched.tm ? sched.tm : (sizeof(R) == 4 ? 16 : 8);
    return true;
  }
  void set_schedule(const int32_t* in3) override;
  void adjoint(int nsteps, int checkpoint_every, const double* cons_tgt, const double* phi_tgt, double* loss,
               double* dparams, double* dphi0) override;

 private:
  meu_params P;
  DevConst hK;
  DevConst* dK = nullptr;
  LanFusedConst* dF = nullptr;  // constants of the fused Landau step (when it applies)
  bool fused = false;
  std::unique_ptr<FFT3> fft;
  cudaStream_t st = nullptr, own_st = nullptr;
  int V, E;
  int64_t n3, nk;
  // device buffers
  R *c = nullptr, *c2 = nullptr, *phi = nullptr, *noise = nullptr, *pphi = nullptr, *wr = nullptr, *fd = nullptr,
    *fc = nullptr, *el_en = nullptr, *strain = nullptr, *xs = nullptr;
  C *sp = nullptr, *uk = nullptr;
  int NS = 0, NWR = 0;
  double *partials = nullptr, *results = nullptr, *h_results = nullptr;
  int* d_ops = nullptr;
  int* d_err = nullptr;
  int* h_err = nullptr;
  double* stage = nullptr;  // AoS staging (double)
  // run_noise: two pinned host buffers of one step's increments (Fortran layout), their
  // device copy, and the events that free a host buffer once its copy has run
  double* noise_host[2] = {nullptr, nullptr};
  double* noise_dev = nullptr;
  cudaEvent_t noise_ev[2] = {nullptr, nullptr};
  void upload_noise(const double* dev_incr);
  int64_t stage_elems = 0;
  std::vector<void*> allocs;
  // reference quirk state: values written on the next fort.98 line
  double prev_min = 1.0, prev_max = 0.0, prev_phimax = 0.0, prev_solid = 0.0;
  bool el_ready = false;  // u^ / strain hold a valid elastic state
  int last_iters = 0;

  template <typename T> T* dalloc(int64_t n) {
    void* ptr = nullptr;
    MEU_CUDA(cudaMalloc(&ptr, (size_t)std::max<int64_t>(n, 1) * sizeof(T)));
    allocs.push_back(ptr);
    return (T*)ptr;
  }
  R* field(R* base, int f) const { return base + (int64_t)f * n3; }
  C* spec(int f) const { return sp + (int64_t)f * nk; }
  unsigned gridk() const { return grid_for(nk, 256); }
  unsigned gridr() const { return grid_for(n3, 256); }

  // Batched transforms of any number of fields, issued in groups of at most
  // MAXF (the pointer lists the transform kernels take by value hold MAXF entries).
  void fwd(std::initializer_list<const R*> in, int s0) { fwd_list(std::vector<const R*>(in), s0); }
  void fwd_list(const std::vector<const R*>& in, int s0) {
    for (size_t g0 = 0; g0 < in.size(); g0 += MAXF) {
      PtrList<const R> a{};
      PtrList<C> b{};
      int n = 0;
      for (size_t i = g0; i < in.size() && n < MAXF; ++i, ++n) {
        a.p[n] = in[i];
        b.p[n] = spec(s0 + (int)i);
      }
      fft->forward<R>(a, b, n, st);
    }
  }
  void inv_list(int s0, const std::vector<R*>& out) {
    for (size_t g0 = 0; g0 < out.size(); g0 += MAXF) {
      PtrList<C> a{};
      PtrList<R> b{};
      int n = 0;
      for (size_t i = g0; i < out.size() && n < MAXF; ++i, ++n) {
        a.p[n] = spec(s0 + (int)i);
        b.p[n] = out[i];
      }
      fft->inverse<R>(a, b, n, st);
    }
  }
  PtrList<C> specs(int s0, int n) const {
    if (n > MAXF) throw CudaError("internal: more than MAXF spectra in one kernel argument", MEU_ERR_UNSUPPORTED);
    PtrList<C> l{};
    for (int i = 0; i < n; ++i) l.p[i] = spec(s0 + i);
    return l;
  }
  void check_err();
  void finalize(int q0, int nq, double* out = nullptr, const int* nbs = nullptr);
  void elastic(const R* ph_for_ppr, R* elg, int mode, bool zeroth_only);
  void kks_step(meu_diag* d);
  void landau_step(meu_diag* d);
  void landau_step_fused();
  LanFusedArgs<R> fused_args() const;
  void sync_args();           // upload fused_args() into dA when it changed
  void fused_steps(int n);    // n fused steps (CUDA graphs of 8, 4, 2 and 1 steps where possible)
  void fused_step_launches(); // launches of one fused step (stream or capture)
  void capture_graph(int slot);  // 2^slot fused steps into gexec[slot], not run
  void drop_graphs();
  C *keta = nullptr, *kc = nullptr;  // spectral state of the Landau step
  R* gtab = nullptr;  // Green-operator table of the fused step (homogeneous elasticity)
  // fused Landau path: schedule, device argument record, history row counter
  LanSched sched;
  LanFusedArgs<R>* dA = nullptr;
  LanFusedArgs<R> hA{};
  bool hA_valid = false;
  int* d_row = nullptr;
  int* d_ticket = nullptr;
  int fnb[Q_TOTAL] = {0};
  static constexpr int GRAPH_SLOTS = 4;   // graphs of 1, 2, 4 and 8 steps
  // grids of grid-stride reduction kernels sized to the blocks that fit at once (a
  // partial second wave would redo a whole share of the loop); <= RED_BLOCKS
  int g_el_k = RED_BLOCKS, g_elener = RED_BLOCKS, g_lan_k1 = RED_BLOCKS, g_el_x = RED_BLOCKS;
  ElxProp el_prop{};  // proportional-moduli polarization coefficients (host-built)
  ElxCoef<R> el_prop_r{};  // the same in the field precision (fused row kernel)
  ElenProp en_prop{};  // proportional-moduli energy coefficients (host-built)
  // the instantiation of the proportional kernels for this stiffness form
  void (*fn_el_x)(ElxProp, int64_t, const R*, const R*, R*, double, int*) = nullptr;
  void (*fn_elener)(ElenProp, int64_t, const R*, const R*, const R*, R*, R*, int, int, double*, int*) = nullptr;
  size_t sm_el_x = 0, sm_elener = 0;  // their dynamic shared memory (prefetch tiles)
  bool el_ortho = false;              // stiffnesses with decoupled normal / shear blocks
  bool el_ortho_gen = false;          // general moduli: C0 and every phase's compliance in that pattern
  bool el_fused_rows = false;         // iterations run the x passes and el_x as one kernel
  bool fused_warm = false;
  bool q_checked = false;  // Q(k) of the fused step tested (LS_QCHECK on its first step)
  bool theta_ready = false;  // sp holds theta^ of the current fields (written by the last step's PI)
  bool fields_set = false;  // the spectral-state layout is fixed from the first upload on
  std::unique_ptr<AdjBuffers<R>, void (*)(AdjBuffers<R>*)> adjb{nullptr, adj_buffers_free<R>};
  void reset_fused_state();
  void tune_transforms();  // generic path: pick FFT3::pv by timing
  cudaGraphExec_t gexec[GRAPH_SLOTS] = {nullptr, nullptr, nullptr, nullptr};
  int64_t graph_launches[GRAPH_SLOTS] = {0, 0, 0, 0};  // kernels in each graph
  void end_step(meu_diag* d, int clip);
  void flush_hist(meu_diag* diag);
  static constexpr int HIST_MAX = 4096;
  double* hist = nullptr;  // per-step reductions [HIST_MAX][Q_STEP_COUNT]
  double* cmean_acc = nullptr;
  int hist_n = 0;
  std::vector<int64_t> hist_step = std::vector<int64_t>(HIST_MAX);
  std::vector<int> hist_iters = std::vector<int>(HIST_MAX);
};

}  // namespace meu
