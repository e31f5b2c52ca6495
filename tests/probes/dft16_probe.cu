// dft16_probe.cu -- test-only measurement: one radix-16 DFT stage on the tensor pipe
// against the same stage on the CUDA cores (the butterfly the fused transforms use).
//
// Both kernels run `reps` passes of y = DFT16(x) / 4 over a tile of 256 lines x 16
// points held in shared memory (read tile -> compute -> write tile -> barrier), so the
// time per pass is the cost of one radix-16 stage from and to shared memory, the unit
// of work of the shared-memory FFT stages.  The 1/4 keeps the tile's norm (DFT16 / 4
// is unitary).  Layout: tile[p][l], point p in [0,16), line l in [0,256).
//
//   mode 0: CUDA cores -- one line per thread, Dft<16> (4 x 4 radix-4 form).
//   mode 1: tensor pipe -- the stage as a real GEMM Y = W X with
//           W = [[Re F, -Im F], [Im F, Re F]] (32 x 32), X = [Re x; Im x] (32 x lines),
//           mma.sync.m16n8k8 in TF32 with the 3xTF32 split (x = hi + lo, W = hi + lo,
//           Y = Whi Xhi + Whi Xlo + Wlo Xhi) for FP32-level accuracy.  A warp takes
//           8 lines per 24 MMAs (2 row tiles x 4 k tiles x 3 products).
//
// Entry: probe_dft16(mode, nblocks, reps, in, out, ms) -- in/out: nblocks tiles of
// 16 x 256 float2 in device memory; ms: kernel time from CUDA events.
#include <cuda_runtime.h>

#include "../../meumapps_ss_b200/csrc/fft.cuh"

namespace {

constexpr int LINES = 256, PTS = 16, NT = 256;

__constant__ float c_whi[32 * 32];
__constant__ float c_wlo[32 * 32];

__global__ void __launch_bounds__(NT) k_cuda(const float2* __restrict__ in, float2* __restrict__ out, int reps) {
  __shared__ float2 tile[PTS][LINES];
  const float2* src = in + (size_t)blockIdx.x * PTS * LINES;
  for (int i = threadIdx.x; i < PTS * LINES; i += NT) tile[i / LINES][i % LINES] = src[i];
  __syncthreads();
  for (int r = 0; r < reps; ++r) {
    // each pass takes another line, so the tile really goes through shared memory
    const int l = (threadIdx.x + r * 37) % LINES;
    float2 x[PTS];
#pragma unroll
    for (int p = 0; p < PTS; ++p) x[p] = tile[p][l];
    meu::Dft<16, -1, float2>::run(x);
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PTS; ++p) tile[p][l] = make_float2(0.25f * x[p].x, 0.25f * x[p].y);
    __syncthreads();
  }
  float2* dst = out + (size_t)blockIdx.x * PTS * LINES;
  for (int i = threadIdx.x; i < PTS * LINES; i += NT) dst[i] = tile[i / LINES][i % LINES];
}

__device__ __forceinline__ unsigned tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(NT) k_mma(const float2* __restrict__ in, float2* __restrict__ out, int reps) {
  __shared__ float2 tile[PTS][LINES];
  const float2* src = in + (size_t)blockIdx.x * PTS * LINES;
  for (int i = threadIdx.x; i < PTS * LINES; i += NT) tile[i / LINES][i % LINES] = src[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  // A fragments of W (m16n8k8, row-major A): a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4)
  unsigned ahi[2][4][4], alo[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const int r0 = mt * 16 + g, c0 = kt * 8 + t;
      const int rows[4] = {r0, r0 + 8, r0, r0 + 8}, cols[4] = {c0, c0, c0 + 4, c0 + 4};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        ahi[mt][kt][i] = __float_as_uint(c_whi[rows[i] * 32 + cols[i]]);
        alo[mt][kt][i] = __float_as_uint(c_wlo[rows[i] * 32 + cols[i]]);
      }
    }
  __syncthreads();
  for (int r = 0; r < reps; ++r) {
    // 8 warps x 4 groups of 8 lines = 256 lines; B fragments (col-major 8 x 8):
    // b0 (row t, col g), b1 (row t+4, col g): rows 0-15 Re x_p, 16-31 Im x_p
    float d[4][2][4];
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
      const int l = ((warp * 4 + grp) * 8 + g + r * 37) % LINES;
      unsigned bhi[4][2], blo[4][2];
#pragma unroll
      for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = kt * 8 + t + 4 * h;
          const float2 v = tile[row & 15][l];
          const float x = row < 16 ? v.x : v.y;
          bhi[kt][h] = tf32(x);
          blo[kt][h] = tf32(x - __uint_as_float(bhi[kt][h]));
        }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
        for (int i = 0; i < 4; ++i) d[grp][mt][i] = 0.f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          mma_tf32(d[grp][mt], alo[mt][kt], bhi[kt]);
          mma_tf32(d[grp][mt], ahi[mt][kt], blo[kt]);
          mma_tf32(d[grp][mt], ahi[mt][kt], bhi[kt]);
        }
      }
    }
    __syncthreads();
    // D fragments: d0 (g, 2t), d1 (g, 2t+1), d2 (g+8, 2t), d3 (g+8, 2t+1); rows = output
    // points (tile 0: Re, tile 1: Im), columns = the group's lines
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
      const int lb = (warp * 4 + grp) * 8;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int p = g + (i >= 2 ? 8 : 0), col = 2 * t + (i & 1);
        const int l = (lb + col + r * 37) % LINES;
        tile[p][l] = make_float2(0.25f * d[grp][0][i], 0.25f * d[grp][1][i]);
      }
    }
    __syncthreads();
  }
  float2* dst = out + (size_t)blockIdx.x * PTS * LINES;
  for (int i = threadIdx.x; i < PTS * LINES; i += NT) dst[i] = tile[i / LINES][i % LINES];
}

}  // namespace

extern "C" int probe_dft16(int mode, int nblocks, int reps, const float2* in, float2* out, float* ms) {
  static bool init = false;
  if (!init) {
    float whi[32 * 32], wlo[32 * 32];
    for (int q = 0; q < 32; ++q)
      for (int c = 0; c < 32; ++c) {
        const int qp = q & 15, cp = c & 15;
        const double ang = -2.0 * 3.14159265358979323846 * (double)(qp * cp % 16) / 16.0;
        const double re = __builtin_cos(ang), im = __builtin_sin(ang);
        // [[Re F, -Im F], [Im F, Re F]]
        const double w = (q < 16) ? (c < 16 ? re : -im) : (c < 16 ? im : re);
        unsigned hb;
        const float wf = (float)w;
        __builtin_memcpy(&hb, &wf, 4);
        hb &= 0xffffe000u;  // the TF32 head (truncated mantissa); the remainder is exact in FP32
        float hi;
        __builtin_memcpy(&hi, &hb, 4);
        whi[q * 32 + c] = hi;
        wlo[q * 32 + c] = (float)(w - (double)hi);
      }
    if (cudaMemcpyToSymbol(c_whi, whi, sizeof(whi)) != cudaSuccess) return 1;
    if (cudaMemcpyToSymbol(c_wlo, wlo, sizeof(wlo)) != cudaSuccess) return 1;
    init = true;
  }
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  if (mode == 0) k_cuda<<<nblocks, NT>>>(in, out, reps);
  else k_mma<<<nblocks, NT>>>(in, out, reps);
  cudaEventRecord(b);
  const cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  *ms = t;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 2;
}
