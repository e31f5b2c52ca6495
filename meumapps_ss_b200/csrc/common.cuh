// common.cuh -- complex arithmetic, launch helpers and error handling shared by
// the MEUMAPPS-SS step kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace meu {

template <typename R> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename R> using cplx = typename CplxOf<R>::type;

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
  return mk(a.x * s, a.y * s);
}
// multiply by i*s (s = +1 or -1)
template <int S, typename C> __host__ __device__ __forceinline__ C cmul_is(C a) {
  return S > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

#define MEU_CUDA(x)                                                                              \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess)                                                                       \
      throw ::meu::CudaError(std::string(#x) + ": " + cudaGetErrorString(e_) + " at " __FILE__ ":" \
                                 + std::to_string(__LINE__),                                     \
                             101);                                                               \
  } while (0)

#define MEU_CHECK_LAUNCH() MEU_CUDA(cudaGetLastError())

inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 16) {
  int64_t g = (n + block - 1) / block;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// Message returned by meu_last_error(NULL) for calls that have no handle.
void set_thread_error(const std::string& msg);

// Observer of kernel launches (launch counting and per-kernel event timing).
// bytes = algorithmic bytes the launch must move (compulsory reads + writes).
struct LaunchHook {
  virtual ~LaunchHook() {}
  virtual void begin(const char* name, double bytes, cudaStream_t st) = 0;
  virtual void end(cudaStream_t st) = 0;
  virtual bool timing() const { return false; }  // events around every kernel
};

// Up to MAXF field pointers passed by value to batched kernels.
constexpr int MAXF = 32;
template <typename T> struct PtrList {
  T* p[MAXF];
};

// Raise a kernel's dynamic shared-memory limit to the opt-in maximum (227 KB per block
// on sm_100 minus the kernel's static shared memory), once per kernel and device, and
// return that limit.  Raising it to the maximum (not to one launch's need) keeps every
// later launch of the kernel valid whatever size it asks for.
inline int smem_optin(const void* fn) {
  static thread_local std::vector<std::pair<const void*, int>> done;  // (kernel, device)
  int dev = 0;
  MEU_CUDA(cudaGetDevice(&dev));
  static thread_local std::vector<int> lims;
  for (size_t i = 0; i < done.size(); ++i)
    if (done[i].first == fn && done[i].second == dev) return lims[i];
  int optin = 0;
  MEU_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  MEU_CUDA(cudaFuncGetAttributes(&fa, fn));
  const int lim = optin - (int)fa.sharedSizeBytes;
  MEU_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  done.push_back({fn, dev});
  lims.push_back(lim);
  return lim;
}

}  // namespace meu
