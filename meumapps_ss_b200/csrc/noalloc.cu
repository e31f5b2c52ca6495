// noalloc.cu -- the transform round trip without any device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran driver whose device memory is
// owned by its OpenACC/managed-memory runtime, a framework whose allocator has
// already reserved the GPU's memory, or code that must not add the implicit
// device synchronisation of cudaMalloc/cudaFree to its stream.  They pass their
// own device arrays, and the library's working memory (transform tables and the
// working spectrum) comes from the fixed array below, which every GPU that loads
// the library holds until the process exits.
#include <cstdint>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/meu.h"
#include "fft.cuh"

namespace {

constexpr size_t kTableBytes = 192u << 10;  // twiddle + digit tables of any admissible grid
constexpr size_t kWorkBytes = (size_t)MEU_NOALLOC_MAX_POINTS * 12 + 512;
constexpr size_t kScratchBytes = kTableBytes + kWorkBytes;

// Shared by every call on a device; keeps the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the symbol name
// is only a host-side stand-in, so the address is looked up once per device,
// with that device current.
std::mutex g_mu;
void* g_addr[64] = {nullptr};

void* scratch_address() {
  int dev = 0;
  MEU_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw meu::CudaError("device index out of range", MEU_ERR_UNSUPPORTED);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw meu::CudaError(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e), MEU_ERR_CUDA);
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

template <typename A, typename B>
__global__ void k_copy_convert(const A* __restrict__ src, B* __restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (B)src[i];
}

}  // namespace

extern "C" int meu_fft_roundtrip_noalloc(int32_t nx, int32_t ny, int32_t nz, int32_t precision,
                                         const double* in_dev, double* spec_dev, double* back_dev) {
  using namespace meu;
  try {
    if (!in_dev || !spec_dev || !back_dev) {
      set_thread_error("meu_fft_roundtrip_noalloc: NULL array");
      return MEU_ERR_BADARG;
    }
    if (!fft_size_ok(nx, true) || !fft_size_ok(ny, false) || !fft_size_ok(nz, false)) {
      set_thread_error("meu_fft_roundtrip_noalloc: grid sizes must be 2^a 3^b with Nx even");
      return MEU_ERR_UNSUPPORTED;
    }
    const int64_t n3 = (int64_t)nx * ny * nz;
    if (n3 > MEU_NOALLOC_MAX_POINTS) {
      set_thread_error("meu_fft_roundtrip_noalloc: " + std::to_string(n3) + " grid points exceed the maximum of " +
                       std::to_string((long long)MEU_NOALLOC_MAX_POINTS) + " of the static working memory");
      return MEU_ERR_UNSUPPORTED;
    }
    const bool f64 = precision == MEU_PREC_F64;
    if (!f64 && precision != MEU_PREC_F32) {
      set_thread_error("meu_fft_roundtrip_noalloc: unknown precision");
      return MEU_ERR_BADARG;
    }
    // FP64 transforms read and write the caller's arrays as 16-byte (re,im) pairs and
    // 16-byte asynchronous copies; the FP32 path reads and writes single doubles
    const uintptr_t align = f64 ? 16 : 8;
    if ((((uintptr_t)in_dev | (uintptr_t)spec_dev | (uintptr_t)back_dev) & (align - 1)) != 0) {
      set_thread_error(std::string("meu_fft_roundtrip_noalloc: in_dev, spec_dev and back_dev must be ") +
                       (f64 ? "16-byte aligned in FP64" : "8-byte aligned in FP32"));
      return MEU_ERR_BADARG;
    }
    unsigned char* base = (unsigned char*)scratch_address();
    FFT3 f(nx, ny, nz, f64, base, kTableBytes);
    unsigned char* work = base + kTableBytes;
    const int64_t nk = f.nk();
    cudaStream_t st = 0;
    const unsigned g1 = grid_for(n3, 256), g2 = grid_for(2 * nk, 256);
    if (f64) {
      // forward straight into the caller's spectrum; the inverse consumes a copy
      PtrList<const double> a{};
      PtrList<double2> b{};
      a.p[0] = in_dev;
      b.p[0] = (double2*)spec_dev;
      f.forward<double>(a, b, 1, st);
      double2* wspec = (double2*)work;
      MEU_CUDA(cudaMemcpyAsync(wspec, spec_dev, sizeof(double2) * nk, cudaMemcpyDeviceToDevice, st));
      PtrList<double2> c{};
      PtrList<double> d{};
      c.p[0] = wspec;
      d.p[0] = back_dev;
      f.inverse<double>(c, d, 1, st);
    } else {
      float* wreal = (float*)work;
      float2* wspec = (float2*)(work + (((size_t)n3 * sizeof(float) + 255) & ~(size_t)255));
      k_copy_convert<double, float><<<g1, 256, 0, st>>>(in_dev, wreal, n3);
      MEU_CHECK_LAUNCH();
      PtrList<const float> a{};
      PtrList<float2> b{};
      a.p[0] = wreal;
      b.p[0] = wspec;
      f.forward<float>(a, b, 1, st);
      k_copy_convert<float, double><<<g2, 256, 0, st>>>((const float*)wspec, spec_dev, 2 * nk);
      MEU_CHECK_LAUNCH();
      PtrList<float2> c{};
      PtrList<float> d{};
      c.p[0] = wspec;
      d.p[0] = wreal;
      f.inverse<float>(c, d, 1, st);
      k_copy_convert<float, double><<<g1, 256, 0, st>>>(wreal, back_dev, n3);
      MEU_CHECK_LAUNCH();
    }
    MEU_CUDA(cudaStreamSynchronize(st));
  } catch (const CudaError& e) {
    set_thread_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_thread_error("meu_fft_roundtrip_noalloc: host allocation failed");
    return MEU_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_thread_error(std::string("meu_fft_roundtrip_noalloc: ") + e.what());
    return MEU_ERR_CUDA;
  }
  return MEU_OK;
}
