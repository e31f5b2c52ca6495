// landau_fused.cu -- size dispatch, per-step finalisation and schedule
// autotuning of the fused Landau step (kernels: landau_fused_kernels.cuh,
// instantiated per (precision, N) in lf_inst_*.cu).
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include "landau_fused.cuh"

namespace meu {

namespace {
// Fixed-order reduction of member blockIdx.y's partials into its history row.
// The last of the member's blocks advances the member's row counter, so graph
// replays of the step need no host-side row index.
template <typename R>
__global__ void __launch_bounds__(256) k_lf_finalize(const LanFusedArgs<R>* __restrict__ A, NbList nb,
                                                     const int* __restrict__ ops) {
  const LanFusedArgs<R>& a = A[blockIdx.y];
  const int q = blockIdx.x, op = ops[q];
  const int row = *a.hist_row;
  double acc = op == 0 ? 0.0 : op == 1 ? -1.0e308 : 1.0e308;
  for (int i = threadIdx.x; i < nb.nb[q]; i += blockDim.x) {
    const double v = a.partials[(int64_t)q * PSTRIDE + i];
    acc = op == 0 ? acc + v : op == 1 ? fmax(acc, v) : fmin(acc, v);
  }
  const double x = block_reduce_value(acc, op);
  if (threadIdx.x == 0) {
    if (row < a.hist_rows) a.hist[(int64_t)row * Q_STEP_COUNT + q] = x;
    __threadfence();
    if (atomicAdd(a.ticket, 1) == (int)gridDim.x - 1) {
      *a.ticket = 0;
      *a.hist_row = row + 1;
    }
  }
}
}  // namespace

bool lan_fused_supported(const meu_params& p) {
  const int n = p.nx;
  const bool size_ok = (n == 32 || n == 48 || n == 64 || n == 96 || n == 128) && p.ny == n && p.nz == n;
  return size_ok && p.model == MEU_MODEL_LANDAU && p.nvar >= 1 && p.nvar <= 4 && p.numel == 1 &&
         p.eig_coupling == MEU_EIG_ETA2 && (p.elastic == MEU_ELAST_NONE || p.elastic == MEU_ELAST_HOMOG);
}

template <typename R>
bool lan_fused_step(int N, int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, bool energy,
                    cudaStream_t st, LaunchHook* hook, int* nb) {
  if (members < 1 || members > 65535) return false;
  switch (N) {
    case 32: return lf_step_n<R, 32>(V, s, dA, members, energy, st, hook, nb);
    case 48: return lf_step_n<R, 48>(V, s, dA, members, energy, st, hook, nb);
    case 64: return lf_step_n<R, 64>(V, s, dA, members, energy, st, hook, nb);
    case 96: return lf_step_n<R, 96>(V, s, dA, members, energy, st, hook, nb);
    case 128: return lf_step_n<R, 128>(V, s, dA, members, energy, st, hook, nb);
    default: return false;
  }
}

template <typename R>
bool lan_fused_init(int N, int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, cudaStream_t st,
                    LaunchHook* hook) {
  if (members < 1 || members > 65535) return false;
  switch (N) {
    case 32: return lf_init_n<R, 32>(V, s, dA, members, st, hook);
    case 48: return lf_init_n<R, 48>(V, s, dA, members, st, hook);
    case 64: return lf_init_n<R, 64>(V, s, dA, members, st, hook);
    case 96: return lf_init_n<R, 96>(V, s, dA, members, st, hook);
    case 128: return lf_init_n<R, 128>(V, s, dA, members, st, hook);
    default: return false;
  }
}

template <typename R>
void lan_fused_finalize(const LanFusedArgs<R>* dA, int members, const int* nb, const int* ops, cudaStream_t st,
                        LaunchHook* hook) {
  NbList l;
  for (int q = 0; q < Q_TOTAL; ++q) l.nb[q] = q < Q_STEP_COUNT ? nb[q] : 0;
  double bytes = 0;
  for (int q = 0; q < Q_STEP_COUNT; ++q) bytes += 8.0 * nb[q];
  if (hook) hook->begin("finalize", bytes * members, st);
  k_lf_finalize<R><<<dim3(Q_STEP_COUNT, members), 256, 0, st>>>(dA, l, ops);
  MEU_CHECK_LAUNCH();
  if (hook) hook->end(st);
}

std::vector<LanSched> lan_sched_candidates(int N, bool f64) {
  std::vector<LanSched> v;
  const int wide = f64 ? 8 : 16;
  const int cols = N * (N / 2 + 1);
  for (int pv = 0; pv < 2; ++pv)
    for (int ntp : {512, 256})
      for (int tm : {wide, wide / 2}) {
        if (cols % tm != 0 || cols / tm > PSTRIDE) continue;
        LanSched s;
        s.pv = pv;
        s.ntp = ntp;
        s.tm = tm;
        v.push_back(s);
      }
  return v;
}

namespace {
std::mutex g_tune_mu;
std::map<std::string, LanSched> g_tune;
bool g_tune_loaded = false;

std::string tune_key(bool f64, int N, int V, int members, bool energy) {
  std::ostringstream o;
  o << (f64 ? "f64" : "f32") << ' ' << N << ' ' << V << ' ' << members << ' ' << (energy ? 1 : 0);
  return o.str();
}
void tune_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("MEU_AUTOTUNE_CACHE");
  if (!path || !*path) return;
  std::ifstream f(path);
  std::string prec;
  int N, V, members, energy;
  LanSched s;
  while (f >> prec >> N >> V >> members >> energy >> s.pv >> s.ntp >> s.tm) {
    std::string rest;
    std::getline(f, rest);
    g_tune[tune_key(prec == "f64", N, V, members, energy != 0)] = s;
  }
}
void tune_store(const std::string& key, const LanSched& s, double ms) {
  const char* path = std::getenv("MEU_AUTOTUNE_CACHE");
  if (!path || !*path) return;
  std::ofstream f(path, std::ios::app);
  f << key << ' ' << s.pv << ' ' << s.ntp << ' ' << s.tm << ' ' << ms << '\n';
}
}  // namespace

template <typename R>
LanSched lan_autotune(int N, int V, const LanFusedArgs<R>* dA, int members, bool energy, const int* d_ops,
                      cudaStream_t st, double* best_ms) {
  const bool f64 = sizeof(R) == 8;
  const std::string key = tune_key(f64, N, V, members, energy);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      if (best_ms) *best_ms = -1.0;
      return it->second;
    }
  }
  constexpr int WARM = 2, TIMED = 5;
  cudaEvent_t e0, e1;
  MEU_CUDA(cudaEventCreate(&e0));
  MEU_CUDA(cudaEventCreate(&e1));
  LanSched best;
  double best_t = 1e300;
  int nb[Q_TOTAL];
  for (const LanSched& s : lan_sched_candidates(N, f64)) {
    for (int i = 0; i < WARM + TIMED; ++i) {
      if (i == WARM) MEU_CUDA(cudaEventRecord(e0, st));
      if (!lan_fused_step<R>(N, V, s, dA, members, energy, st, nullptr, nb)) break;
      lan_fused_finalize<R>(dA, members, nb, d_ops, st, nullptr);
    }
    MEU_CUDA(cudaEventRecord(e1, st));
    MEU_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MEU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / TIMED < best_t) {
      best_t = ms / TIMED;
      best = s;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_ms) *best_ms = best_t;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  tune_store(key, best, best_t);
  return best;
}

template bool lan_fused_init<float>(int, int, const LanSched&, const LanFusedArgs<float>*, int, cudaStream_t, LaunchHook*);
template bool lan_fused_init<double>(int, int, const LanSched&, const LanFusedArgs<double>*, int, cudaStream_t, LaunchHook*);
template bool lan_fused_step<float>(int, int, const LanSched&, const LanFusedArgs<float>*, int, bool, cudaStream_t,
                                    LaunchHook*, int*);
template bool lan_fused_step<double>(int, int, const LanSched&, const LanFusedArgs<double>*, int, bool, cudaStream_t,
                                     LaunchHook*, int*);
template void lan_fused_finalize<float>(const LanFusedArgs<float>*, int, const int*, const int*, cudaStream_t, LaunchHook*);
template void lan_fused_finalize<double>(const LanFusedArgs<double>*, int, const int*, const int*, cudaStream_t,
                                         LaunchHook*);
template LanSched lan_autotune<float>(int, int, const LanFusedArgs<float>*, int, bool, const int*, cudaStream_t, double*);
template LanSched lan_autotune<double>(int, int, const LanFusedArgs<double>*, int, bool, const int*, cudaStream_t,
                                       double*);

}  // namespace meu
