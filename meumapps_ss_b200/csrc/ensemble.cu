// ensemble.cu -- many independent fused Landau simulations ("members") stepped
// together.  Members with the same grid size, variant count, precision and
// energy flag form a bucket; every kernel of the fused step covers all members
// of its bucket in one launch (blockIdx.z = member), the buckets run as parallel
// branches, and runs of 8, 4, 2 or 1 whole-ensemble steps replay CUDA graphs.
// An optional autotuner picks each bucket's schedule (radix plan, plane threads,
// column tile) by timing the candidates on the bucket before the fields are set.
// With MEU_ENS_PERSISTENT the warm steps of every member instead run as work items of
// one persistent launch per run of up to PK_MAX_STEPS steps (ens_persist.cuh).
#include <algorithm>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "engine.cuh"
#include "ens_persist.cuh"

namespace meu {

struct EnsembleBase {
  virtual ~EnsembleBase() {}
  virtual void set_fields(int m, const double* cons, const double* phi) = 0;
  virtual void get_fields(int m, double* cons, double* phi, double* el_en) = 0;
  virtual void run(int nsteps, meu_diag* diag) = 0;
  virtual void schedule(int m, int32_t* out) const = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual int64_t launch_count() const = 0;
  int64_t step = 0;
  int members = 0;
  Profiler prof;
};

template <typename R>
class EnsembleT : public EnsembleBase {
 public:
  EnsembleT(int n, const meu_params* ps, int flags);
  ~EnsembleT() override;
  void set_fields(int m, const double* cons, const double* phi) override;
  void get_fields(int m, double* cons, double* phi, double* el_en) override;
  void run(int nsteps, meu_diag* diag) override;
  void schedule(int m, int32_t* out) const override;
  void set_stream(cudaStream_t s) override { st = s ? s : own_st; }
  int64_t launch_count() const override {
    int64_t n = prof.launches;
    for (const auto& e : mem) n += e->prof.launches;
    return n;
  }

 private:
  static constexpr int GRAPH_SLOTS = Engine<R>::GRAPH_SLOTS;
  struct Bucket {
    int N = 0, V = 0;
    bool energy = false;
    LanSched sched;
    std::vector<int> idx;
    LanFusedArgs<R>* dA = nullptr;
    std::vector<LanFusedArgs<R>> hA;
    int nb[Q_TOTAL] = {0};
    cudaStream_t bst = nullptr;
    cudaEvent_t done = nullptr;
    bool theta_ready = false;  // the members' M holds theta^ of their current fields
    bool q_checked = false;    // Q(k) tested (LS_QCHECK on the first, never captured, step)
  };
  std::vector<std::unique_ptr<Engine<R>>> mem;
  std::vector<Bucket> bk;
  std::vector<int> bucket_of;
  cudaStream_t st = nullptr, own_st = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t gexec[GRAPH_SLOTS] = {};   // 2^slot whole-ensemble steps
  int64_t graph_launches[GRAPH_SLOTS] = {};  // kernels in each graph
  bool warm = false;
  // persistent mode: argument records of all members (member order), the work list of
  // one step, and the launch's counters
  bool persist = false;
  std::vector<LanFusedArgs<R>> hAll;
  LanFusedArgs<R>* dAll = nullptr;
  PkMember* dMt = nullptr;
  uint32_t* dItems = nullptr;
  int* dNeed = nullptr;
  int* dCtrl = nullptr;
  int pkL = 0;

  void sync_args();
  void step_launches();
  bool homog_stable(int n) const;
  bool can_replay() const;
  void capture_graph(int slot);  // captured and instantiated, not run
};

template <typename R>
EnsembleT<R>::EnsembleT(int n, const meu_params* ps, int flags) {
  if (n < 1 || !ps) throw CudaError("ensemble needs at least one member", MEU_ERR_BADARG);
  members = n;
  step = ps[0].step;
  std::map<std::tuple<int, int, int>, int> key2b;
  for (int m = 0; m < n; ++m) {
    const meu_params& p = ps[m];
    if (p.precision != ps[0].precision) throw CudaError("ensemble members must share one precision", MEU_ERR_BADARG);
    if (p.step != ps[0].step) throw CudaError("ensemble members must start at the same step", MEU_ERR_BADARG);
    if (!lan_fused_supported(p) || (p.flags & MEU_FLAG_GENERIC))
      throw CudaError("ensemble member " + std::to_string(m) +
                          ": members are Landau decks on cubic grids N in {32,48,64,96,128} with 1-4 variants, "
                          "eta^2 coupling and homogeneous or no elasticity",
                      MEU_ERR_UNSUPPORTED);
    meu_params q = p;
    q.flags &= ~MEU_FLAG_AUTOTUNE;  // tuned per bucket below
    mem.emplace_back(new Engine<R>(q));
    const auto key = std::make_tuple(p.nx, p.nvar, p.diag_energy != 0 ? 1 : 0);
    auto it = key2b.find(key);
    int b;
    if (it == key2b.end()) {
      b = (int)bk.size();
      key2b[key] = b;
      bk.emplace_back();
      bk[b].N = p.nx;
      bk[b].V = p.nvar;
      bk[b].energy = p.diag_energy != 0;
    } else {
      b = it->second;
    }
    if (bk[b].idx.size() >= 65535) throw CudaError("more than 65535 members of one size", MEU_ERR_UNSUPPORTED);
    bk[b].idx.push_back(m);
    bucket_of.push_back(b);
  }
  persist = (flags & MEU_ENS_PERSISTENT) != 0;
  if (persist) {
    if (n > PK_MAX_MEMBERS) throw CudaError("persistent ensemble: too many members", MEU_ERR_UNSUPPORTED);
    for (int m = 0; m < n; ++m)
      if (ps[m].nvar != PK_V)
        throw CudaError("persistent ensemble member " + std::to_string(m) + ": one order parameter per member",
                        MEU_ERR_UNSUPPORTED);
  }
  MEU_CUDA(cudaStreamCreateWithFlags(&own_st, cudaStreamNonBlocking));
  st = own_st;
  MEU_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (Bucket& b : bk) {
    MEU_CUDA(cudaStreamCreateWithFlags(&b.bst, cudaStreamNonBlocking));
    MEU_CUDA(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    MEU_CUDA(cudaMalloc(&b.dA, sizeof(LanFusedArgs<R>) * b.idx.size()));
  }
  if (persist) {
    // one schedule for every size: the persistent kernel's
    for (Bucket& b : bk) {
      b.sched.pv = PK_PV;
      b.sched.ntp = PK_NTP;
      b.sched.tm = pk_tm<R>();
    }
    std::vector<int> Ns(n), en(n);
    for (int m = 0; m < n; ++m) {
      Ns[m] = ps[m].nx;
      en[m] = ps[m].diag_energy != 0 ? 1 : 0;
    }
    const PkPlan pl = pk_plan(Ns, en, sizeof(R) == 8);
    pkL = (int)pl.items.size();
    MEU_CUDA(cudaMalloc(&dAll, sizeof(LanFusedArgs<R>) * n));
    MEU_CUDA(cudaMalloc(&dMt, sizeof(PkMember) * n));
    MEU_CUDA(cudaMalloc(&dItems, sizeof(uint32_t) * pkL));
    MEU_CUDA(cudaMalloc(&dNeed, sizeof(int) * pkL));
    MEU_CUDA(cudaMalloc(&dCtrl, sizeof(int) * (2 + (size_t)n)));
    MEU_CUDA(cudaMemcpy(dMt, pl.mt.data(), sizeof(PkMember) * n, cudaMemcpyHostToDevice));
    MEU_CUDA(cudaMemcpy(dItems, pl.items.data(), sizeof(uint32_t) * pkL, cudaMemcpyHostToDevice));
    MEU_CUDA(cudaMemcpy(dNeed, pl.need.data(), sizeof(int) * pkL, cudaMemcpyHostToDevice));
  }
  for (auto& e : mem) MEU_CUDA(cudaStreamSynchronize(e->st));
  sync_args();
  if ((flags & MEU_ENS_AUTOTUNE) && !persist) {
    for (Bucket& b : bk)
      b.sched = lan_autotune<R>(b.N, b.V, b.dA, (int)b.idx.size(), b.energy, st, nullptr);
    MEU_CUDA(cudaStreamSynchronize(st));
    for (auto& e : mem) e->reset_fused_state();
    for (Bucket& b : bk) b.theta_ready = false;
  }
  for (Bucket& b : bk)
    for (int m : b.idx) mem[m]->sched = b.sched;  // the spectral-state layout follows the radix plan
}

template <typename R>
EnsembleT<R>::~EnsembleT() {
  if (st) cudaStreamSynchronize(st);
  for (cudaGraphExec_t g : gexec)
    if (g) cudaGraphExecDestroy(g);
  for (Bucket& b : bk) {
    if (b.bst) cudaStreamSynchronize(b.bst);
    if (b.dA) cudaFree(b.dA);
    if (b.done) cudaEventDestroy(b.done);
    if (b.bst) cudaStreamDestroy(b.bst);
  }
  if (fork) cudaEventDestroy(fork);
  for (void* q : {(void*)dAll, (void*)dMt, (void*)dItems, (void*)dNeed, (void*)dCtrl})
    if (q) cudaFree(q);
  prof.reset();
  mem.clear();
  if (own_st) cudaStreamDestroy(own_st);
}

// per-member argument records of every bucket, uploaded when one changed
template <typename R>
void EnsembleT<R>::sync_args() {
  for (Bucket& b : bk) {
    std::vector<LanFusedArgs<R>> a;
    for (int m : b.idx) {
      mem[m]->step = step;
      a.push_back(mem[m]->fused_args());
    }
    if (a.size() == b.hA.size() && memcmp(a.data(), b.hA.data(), sizeof(LanFusedArgs<R>) * a.size()) == 0) continue;
    b.hA = a;
    MEU_CUDA(cudaMemcpyAsync(b.dA, b.hA.data(), sizeof(LanFusedArgs<R>) * b.hA.size(), cudaMemcpyHostToDevice, st));
    MEU_CUDA(cudaStreamSynchronize(st));
  }
  if (!persist) return;
  std::vector<LanFusedArgs<R>> all(members);
  for (const Bucket& b : bk)
    for (size_t j = 0; j < b.idx.size(); ++j) all[b.idx[j]] = b.hA[j];
  if (all.size() == hAll.size() && memcmp(all.data(), hAll.data(), sizeof(LanFusedArgs<R>) * all.size()) == 0) return;
  hAll = all;
  MEU_CUDA(cudaMemcpyAsync(dAll, hAll.data(), sizeof(LanFusedArgs<R>) * hAll.size(), cudaMemcpyHostToDevice, st));
  MEU_CUDA(cudaStreamSynchronize(st));
}

// Work list of one step of the persistent kernel (see ens_persist.cuh): pass-major,
// members of larger grids first within a pass.  need = the member's items of its earlier
// passes: Z1 0, PB T, Z2 T + N, PI and PC 2T + N, END 2T + 3N (T column tiles).
PkPlan pk_plan(const std::vector<int>& N, const std::vector<int>& energy, bool f64) {
  PkPlan p;
  const int n = (int)N.size(), tm = f64 ? pk_tm<double>() : pk_tm<float>();
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return N[a] > N[b]; });
  p.mt.resize(n);
  for (int m = 0; m < n; ++m) {
    const int nn = N[m], t = nn * (nn / 2 + 1) / tm;
    PkMember& q = p.mt[m];
    q.N = nn;
    q.per_step = 2 * t + 3 * nn + 1;
    for (int k = 0; k < Q_TOTAL; ++k) q.nb.nb[k] = 0;
    q.nb.nb[Q_FCH] = energy[m] ? nn : 0;
    q.nb.nb[Q_FINT] = q.nb.nb[Q_ELEN] = q.nb.nb[Q_FINT2] = t;
    q.nb.nb[Q_CMIN] = q.nb.nb[Q_CMAX] = q.nb.nb[Q_PHIMAX] = q.nb.nb[Q_SOLID] = q.nb.nb[Q_CSUM0] = nn * (PK_V + 1);
  }
  for (int kind = PK_Z1; kind <= PK_END; ++kind)
    for (int m : order) {
      const int nn = N[m], t = nn * (nn / 2 + 1) / tm;
      const int count = (kind == PK_Z1 || kind == PK_Z2) ? t : kind == PK_END ? 1 : nn;
      const int need = kind == PK_Z1 ? 0 : kind == PK_PB ? t : kind == PK_Z2 ? t + nn : kind == PK_END ? 2 * t + 3 * nn
                                                                                                        : 2 * t + nn;
      for (int i = 0; i < count; ++i) {
        p.items.push_back(pk_item(m, kind, i));
        p.need.push_back(need);
      }
    }
  return p;
}

// one ensemble step: fork to the bucket streams, batched step, join
template <typename R>
void EnsembleT<R>::step_launches() {
  MEU_CUDA(cudaEventRecord(fork, st));
  for (Bucket& b : bk) {
    MEU_CUDA(cudaStreamWaitEvent(b.bst, fork, 0));
    const int nm = (int)b.idx.size();
    const int opts = (b.energy ? LS_ENERGY : 0) | (b.theta_ready ? LS_THETA_READY : 0) | (b.q_checked ? 0 : LS_QCHECK);
    if (!lan_fused_step<R>(b.N, b.V, b.sched, b.dA, nm, opts, b.bst, &prof, b.nb))
      throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
    b.theta_ready = true;
    b.q_checked = true;
    MEU_CUDA(cudaEventRecord(b.done, b.bst));
    MEU_CUDA(cudaStreamWaitEvent(st, b.done, 0));
  }
}

// the elastic flag (homog) of every member stays the same over the next n steps
template <typename R>
bool EnsembleT<R>::homog_stable(int n) const {
  for (const auto& e : mem) {
    if (e->P.elastic == MEU_ELAST_NONE) continue;
    if ((step >= e->P.elastep0) != (step + n - 1 >= e->P.elastep0)) return false;
  }
  return true;
}

// the step is warm, every bucket's theta^ is current, the per-kernel timer is off and
// the stream can be captured
template <typename R>
bool EnsembleT<R>::can_replay() const {
  if (!warm || prof.on || st == nullptr) return false;
  for (const Bucket& b : bk)
    if (!b.theta_ready) return false;
  return true;
}

template <typename R>
void EnsembleT<R>::capture_graph(int slot) {
  const int64_t l0 = prof.launches;
  cudaGraph_t g = nullptr;
  MEU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    for (int s = 0; s < (1 << slot); ++s) step_launches();
  } catch (...) {
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  MEU_CUDA(cudaStreamEndCapture(st, &g));
  const cudaError_t e = cudaGraphInstantiate(&gexec[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    gexec[slot] = nullptr;
    throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e), MEU_ERR_CUDA);
  }
  graph_launches[slot] = prof.launches - l0;
  prof.launches = l0;
}

// Once warm, runs of steps with one elastic state replay graphs of 8, 4, 2 and 1 steps
// (largest first).  The graphs are captured at the end of the first call that leaves the
// ensemble able to replay them, so a later call of any length only replays.
template <typename R>
void EnsembleT<R>::run(int nsteps, meu_diag* diag) {
  if (nsteps < 0) throw CudaError("negative step count", MEU_ERR_BADARG);
  for (auto& e : mem) MEU_CUDA(cudaStreamSynchronize(e->st));
  constexpr int HM = Engine<R>::HIST_MAX;
  int done = 0;
  while (done < nsteps) {
    const int chunk = std::min(nsteps - done, HM);
    for (auto& e : mem) {
      MEU_CUDA(cudaMemsetAsync(e->d_row, 0, 2 * sizeof(int), st));
      e->hist_n = 0;
    }
    int i = 0;
    while (i < chunk) {
      sync_args();
      int slot = -1;
      if (can_replay())
        for (int sl = GRAPH_SLOTS - 1; sl >= 0; --sl)
          if (chunk - i >= (1 << sl) && homog_stable(1 << sl)) {
            slot = sl;
            break;
          }
      int k = 1;
      if (persist && can_replay()) {
        k = std::min(chunk - i, PK_MAX_STEPS);
        while (k > 1 && !homog_stable(k)) --k;
        pk_launch<R>(dAll, dMt, dItems, dNeed, pkL, k, members, dCtrl, st);
        prof.launches += 1;
      } else if (slot >= 0) {
        if (!gexec[slot]) capture_graph(slot);
        MEU_CUDA(cudaGraphLaunch(gexec[slot], st));
        prof.launches += graph_launches[slot];
        k = 1 << slot;
      } else {
        step_launches();
        warm = true;
      }
      for (int s = 0; s < k; ++s) {
        for (auto& e : mem) {
          e->hist_step[e->hist_n] = step;
          e->hist_iters[e->hist_n] = 0;
          e->hist_n += 1;
        }
        step += 1;
      }
      i += k;
    }
    MEU_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < members; ++m) {
      Engine<R>& e = *mem[m];
      e.step = step;
      e.check_err();
      e.flush_hist(diag ? diag + (int64_t)m * nsteps + done : nullptr);
    }
    done += chunk;
  }
  if (can_replay() && !persist)
    for (int sl = 0; sl < GRAPH_SLOTS; ++sl)
      if (!gexec[sl]) capture_graph(sl);
}

template <typename R>
void EnsembleT<R>::set_fields(int m, const double* cons, const double* phi) {
  if (m < 0 || m >= members) throw CudaError("member index out of range", MEU_ERR_BADARG);
  MEU_CUDA(cudaStreamSynchronize(st));
  mem[m]->step = step;
  mem[m]->set_fields(cons, phi, nullptr);
  bk[bucket_of[m]].theta_ready = false;
  MEU_CUDA(cudaStreamSynchronize(mem[m]->st));
}

template <typename R>
void EnsembleT<R>::get_fields(int m, double* cons, double* phi, double* el_en) {
  if (m < 0 || m >= members) throw CudaError("member index out of range", MEU_ERR_BADARG);
  MEU_CUDA(cudaStreamSynchronize(st));
  mem[m]->get_fields(cons, phi, el_en, nullptr);
}

template <typename R>
void EnsembleT<R>::schedule(int m, int32_t* out) const {
  if (m < 0 || m >= members) throw CudaError("member index out of range", MEU_ERR_BADARG);
  const LanSched& s = bk[bucket_of[m]].sched;
  const int tm = s.tm ? s.tm : (sizeof(R) == 4 ? 16 : 8);
  out[0] = s.pv;
  out[1] = s.ntp;
  out[2] = tm;
  out[3] = bucket_of[m];
}

template class EnsembleT<float>;
template class EnsembleT<double>;

}  // namespace meu

// =============================================================== C-ABI
struct meu_ensemble {
  std::unique_ptr<meu::EnsembleBase> ens;
  std::string err;
};

static thread_local std::string g_ens_create_err;

#define MEU_ENS_TRY(e, body)                         \
  try {                                              \
    body;                                            \
  } catch (const meu::CudaError& x) {                \
    e->err = x.what();                               \
    return x.code;                                   \
  } catch (const std::bad_alloc&) {                  \
    e->err = "host allocation failed";               \
    return MEU_ERR_NOMEM;                            \
  } catch (const std::exception& x) {                \
    e->err = x.what();                               \
    return MEU_ERR_CUDA;                             \
  }

extern "C" {

int meu_ensemble_create(int32_t n_members, const meu_params* params, int32_t flags, meu_ensemble** out) {
  if (!params || !out || n_members < 1) return MEU_ERR_BADARG;
  *out = nullptr;
  meu_ensemble* e = new (std::nothrow) meu_ensemble();
  if (!e) return MEU_ERR_NOMEM;
  try {
    if (params[0].precision == MEU_PREC_F64) e->ens.reset(new meu::EnsembleT<double>(n_members, params, flags));
    else if (params[0].precision == MEU_PREC_F32) e->ens.reset(new meu::EnsembleT<float>(n_members, params, flags));
    else throw meu::CudaError("unknown precision", MEU_ERR_BADARG);
  } catch (const meu::CudaError& x) {
    g_ens_create_err = x.what();
    delete e;
    return x.code;
  } catch (const std::exception& x) {
    g_ens_create_err = x.what();
    delete e;
    return MEU_ERR_CUDA;
  }
  *out = e;
  return MEU_OK;
}

int meu_ensemble_set_fields(meu_ensemble* e, int32_t member, const double* cons, const double* phi) {
  if (!e) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, e->ens->set_fields(member, cons, phi));
  return MEU_OK;
}

int meu_ensemble_run(meu_ensemble* e, int32_t nsteps, meu_diag* diag) {
  if (!e) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, e->ens->run(nsteps, diag));
  return MEU_OK;
}

int meu_ensemble_get_fields(meu_ensemble* e, int32_t member, double* cons, double* phi, double* el_en) {
  if (!e) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, e->ens->get_fields(member, cons, phi, el_en));
  return MEU_OK;
}

int64_t meu_ensemble_get_step(const meu_ensemble* e) { return e ? e->ens->step : -1; }

int meu_ensemble_schedule(meu_ensemble* e, int32_t member, int32_t* out4) {
  if (!e || !out4) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, e->ens->schedule(member, out4));
  return MEU_OK;
}

int meu_ensemble_set_stream(meu_ensemble* e, void* cuda_stream) {
  if (!e) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, e->ens->set_stream((cudaStream_t)cuda_stream));
  return MEU_OK;
}

int meu_ensemble_timing(meu_ensemble* e, int32_t enable) {
  if (!e) return MEU_ERR_BADARG;
  MEU_ENS_TRY(e, {
    e->ens->prof.reset();
    e->ens->prof.on = enable != 0;
  });
  return MEU_OK;
}

int32_t meu_ensemble_timing_report(meu_ensemble* e, int32_t max, char* names, int64_t* counts, double* total_ms,
                                   double* bytes) {
  if (!e || max < 0) return -MEU_ERR_BADARG;
  try {
    meu::Profiler& pr = e->ens->prof;
    pr.resolve();
    const int n = (int)pr.names.size();
    for (int i = 0; i < n && i < max; ++i) {
      if (names) {
        memset(names + 32 * i, 0, 32);
        strncpy(names + 32 * i, pr.names[i].c_str(), 31);
      }
      if (counts) counts[i] = pr.stats[i].n;
      if (total_ms) total_ms[i] = pr.stats[i].ms;
      if (bytes) bytes[i] = pr.stats[i].bytes;
    }
    return n;
  } catch (const meu::CudaError& x) {
    e->err = x.what();
    return -x.code;
  }
}

int64_t meu_ensemble_launch_count(const meu_ensemble* e) { return e ? e->ens->launch_count() : -1; }

const char* meu_ensemble_last_error(const meu_ensemble* e) { return e ? e->err.c_str() : g_ens_create_err.c_str(); }

int meu_ensemble_destroy(meu_ensemble* e) {
  if (!e) return MEU_ERR_BADARG;
  delete e;
  return MEU_OK;
}

}  // extern "C"
