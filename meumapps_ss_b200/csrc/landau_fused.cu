// landau_fused.cu -- size dispatch and schedule autotuning of the fused
// Landau step (kernels: landau_fused_kernels.cuh,
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

bool lan_fused_supported(const meu_params& p) {
  const int n = p.nx;
  const bool size_ok = (n == 32 || n == 48 || n == 64 || n == 96 || n == 128) && p.ny == n && p.nz == n;
  return size_ok && p.model == MEU_MODEL_LANDAU && p.nvar >= 1 && p.nvar <= 4 && p.numel == 1 &&
         p.eig_coupling == MEU_EIG_ETA2 && (p.elastic == MEU_ELAST_NONE || p.elastic == MEU_ELAST_HOMOG);
}

template <typename R>
bool lan_fused_step(int N, int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, int opts,
                    cudaStream_t st, LaunchHook* hook, int* nb) {
  if (members < 1 || members > 65535) return false;
  switch (N) {
    case 32: return lf_step_n<R, 32>(V, s, dA, members, opts, st, hook, nb);
    case 48: return lf_step_n<R, 48>(V, s, dA, members, opts, st, hook, nb);
    case 64: return lf_step_n<R, 64>(V, s, dA, members, opts, st, hook, nb);
    case 96: return lf_step_n<R, 96>(V, s, dA, members, opts, st, hook, nb);
    case 128: return lf_step_n<R, 128>(V, s, dA, members, opts, st, hook, nb);
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

std::vector<LanSched> lan_sched_candidates(int N, bool f64) {
  std::vector<LanSched> v;
  const int wide = f64 ? 8 : 16;
  const int cols = N * (N / 2 + 1);
  for (int pv = 0; pv < 3; ++pv)
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
LanSched lan_autotune(int N, int V, const LanFusedArgs<R>* dA, int members, bool energy, cudaStream_t st,
                      double* best_ms) {
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
  // Each candidate is timed the way a run executes it: a CUDA graph of GSTEPS steps
  // (programmatic dependent launch inside), best of REPS replays after one warm replay.
  // A stream that cannot be captured (the legacy default stream) times eager launches.
  constexpr int WARM = 3, GSTEPS = 8, REPS = 3;
  cudaEvent_t e0, e1;
  MEU_CUDA(cudaEventCreate(&e0));
  MEU_CUDA(cudaEventCreate(&e1));
  LanSched best;
  double best_t = 1e300;
  int nb[Q_TOTAL];
  const int eopt = energy ? LS_ENERGY : 0;
  const int sopt = eopt | LS_THETA_READY;
  for (const LanSched& s : lan_sched_candidates(N, f64)) {
    bool ok = true;
    for (int i = 0; i < WARM && ok; ++i)
      ok = lan_fused_step<R>(N, V, s, dA, members, eopt | (i ? LS_THETA_READY : 0), st, nullptr, nb);
    if (!ok) continue;
    cudaGraphExec_t ge = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      cudaGraph_t g = nullptr;
      try {
        for (int i = 0; i < GSTEPS; ++i) lan_fused_step<R>(N, V, s, dA, members, sopt, st, nullptr, nb);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      if (cudaStreamEndCapture(st, &g) == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
        ge = nullptr;
      if (g) cudaGraphDestroy(g);
    }
    (void)cudaGetLastError();  // a refused capture leaves its (non-sticky) error behind
    auto steps = [&]() {
      if (ge) {
        MEU_CUDA(cudaGraphLaunch(ge, st));
      } else {
        for (int i = 0; i < GSTEPS; ++i) lan_fused_step<R>(N, V, s, dA, members, sopt, st, nullptr, nb);
      }
    };
    try {
      steps();
      for (int r = 0; r < REPS; ++r) {
        MEU_CUDA(cudaEventRecord(e0, st));
        steps();
        MEU_CUDA(cudaEventRecord(e1, st));
        MEU_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MEU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms / GSTEPS < best_t) {
          best_t = ms / GSTEPS;
          best = s;
        }
      }
    } catch (...) {
      if (ge) cudaGraphExecDestroy(ge);
      throw;
    }
    if (ge) cudaGraphExecDestroy(ge);
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
template bool lan_fused_step<float>(int, int, const LanSched&, const LanFusedArgs<float>*, int, int, cudaStream_t,
                                    LaunchHook*, int*);
template bool lan_fused_step<double>(int, int, const LanSched&, const LanFusedArgs<double>*, int, int, cudaStream_t,
                                     LaunchHook*, int*);
template LanSched lan_autotune<float>(int, int, const LanFusedArgs<float>*, int, bool, cudaStream_t, double*);
template LanSched lan_autotune<double>(int, int, const LanFusedArgs<double>*, int, bool, cudaStream_t, double*);

}  // namespace meu
