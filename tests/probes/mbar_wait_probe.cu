// mbar_wait_probe.cu -- test-only kernels for the bounded bulk-copy wait of the plane
// kernels (fz::mbar_init1, fz::bulk_load, fz::mbar_wait in csrc/fused.cuh).
//
//   mode 0: one block bulk-copies n bytes of `in` into shared memory on its mbarrier,
//           waits (bounded), and writes the shared copy to `out`: the normal path.
//   mode 1: the mbarrier expects 16 bytes of transactions that no copy ever delivers
//           (nothing is issued), so the bounded wait runs out; the block records
//           MEU_ERR_TIMEOUT in *err and returns.  No memory operation is invalid and
//           nothing is in flight when the block exits.
//
// Entry: probe_mbar(mode, polls, in, out, n, err, ms) -- in/out: device arrays of n bytes
// (n a multiple of 16, at most 32 KB); err: device int; ms: kernel time (CUDA events).
#include <cuda_runtime.h>

#include "../../meumapps_ss_b200/csrc/fused.cuh"

namespace {

__global__ void k_mbar(int mode, int polls, const float4* __restrict__ in, float4* __restrict__ out, int n, int* err) {
  __shared__ __align__(16) float4 sm[32 * 1024 / 16];
  __shared__ uint64_t mb;
  if (threadIdx.x == 0) meu::fz::mbar_init1(&mb);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (mode == 0) {
      meu::fz::bulk_load(sm, in, (unsigned)n, &mb);
    } else {
      const unsigned a = meu::fz::smem_u32(&mb);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(16u) : "memory");
    }
  }
  if (!meu::fz::mbar_wait(&mb, 0, polls)) {
    if (threadIdx.x == 0) atomicMax(err, MEU_ERR_TIMEOUT);
    return;
  }
  for (int i = threadIdx.x; i < n / 16; i += blockDim.x) out[i] = sm[i];
}

}  // namespace

extern "C" int probe_mbar(int mode, int polls, const void* in, void* out, int n, int* err, float* ms) {
  if (n % 16 != 0 || n <= 0 || n > 32 * 1024) return 1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  k_mbar<<<1, 256>>>(mode, polls, (const float4*)in, (float4*)out, n, err);
  cudaEventRecord(b);
  const cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  *ms = t;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 2;
}
