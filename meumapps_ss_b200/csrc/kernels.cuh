// kernels.cuh -- pointwise and k-space kernels of the MEUMAPPS-SS step.
//
// Real fields are structure-of-arrays a[f][z][y][x]; spectra are [kz][ky][kx]
// with kx in [0, Nx/2] (natural order).  All per-k operators rebuild the
// reference's k-vectors on the fly (k_space, ModInitials.f:348-409):
//   kf = i*b   (b = 2 pi m / N, zeroed at the Nyquist index)
//   kf_sq = -a^2 (a = 2 pi m / N, Nyquist kept)
// Reductions are deterministic: per-block FP64 partials, then a fixed-order
// finalisation.
#pragma once
#include "../../include/meu.h"
#include "common.cuh"

namespace meu {

constexpr int RED_BLOCKS = 592;  // 4 per SM on 148 SMs
constexpr int RED_THREADS = 256;

// Constants of one engine, resident in device memory.
struct DevConst {
  meu_params p;
  int nx, ny, nz, nxh;
  int64_t n3, nk;
  int var_phase[MEU_MAX_VAR];          // 1-based phase of each variant
  int ph_lo[MEU_MAX_PH + 1], ph_hi[MEU_MAX_PH + 1];  // 0-based [lo,hi) variants of phase n
  int zdim;
  double zconst[144], zr_const[12];    // constant rows of Zintf / Zr (Multi_MEUMAPPS.f:426-448)
  double sig0[MEU_MAX_VAR][6];         // eigenstress of variant v with its phase's moduli (tensor Voigt)
  double eps_eng[MEU_MAX_VAR][6];      // eigenstrain, engineering shear
  double A[MEU_MAX_VAR][MEU_MAX_VAR];  // eps0_p : C : eps0_q (Landau homogeneous)
  double sig0_ebar[MEU_MAX_VAR];       // sig0_v : e_mean
  double ebar_eng[6];                  // e_mean with engineering shear
  double c0m[36];                      // C0 = CEla(:,:,2) (column-major)
  // Q(k) as 6 unique entries (11,22,33,23,13,12): Q_m = sum_n qcoef[m][n] Kv_n,
  // Kv = (a1^2, a2^2, a3^2, b2 b3, b1 b3, b1 b2) (the fused Landau kernels' form)
  double qcoef[6][6];
  int use_var[MEU_MAX_VAR];            // elener: variant contributes (transsum > 1e-9)
  // prop_moduli: every phase's compliance is alpha[n] * SEla(:,:,1), so the mixed
  // stiffness (sum_v P_v S_n(v) + w S_1)^-1 is CEla(:,:,1) / (sum_v alpha P_v + w)
  int prop_moduli;
  double alpha[MEU_MAX_PH];
  double c_mean[MEU_MAX_EL];           // conserved mean of each solute (k = 0 mode), FP64
  // 1: the stored concentration is the fluctuation c - c_mean (Landau decks).  The
  // mean is exactly conserved, so it is kept in FP64 and the bulk FP32 field and
  // its transforms only carry the fluctuation.
  int c_shift;
};

enum RedQ : int {
  Q_FCH = 0, Q_FW, Q_FINT, Q_ELEN, Q_CMIN, Q_CMAX, Q_PHIMAX, Q_SOLID, Q_CSUM0,
  // gradient energy of the fields a step produces (the next step's start-of-step value)
  Q_FINT2 = Q_CSUM0 + MEU_MAX_EL,
  Q_STEP_COUNT,
  // elastic convergence sums, separate finalisation
  Q_ERR0 = Q_STEP_COUNT, Q_TOTAL = Q_ERR0 + 6
};
// row length of the partials array: quantity q of block b at partials[q * PSTRIDE + b]
constexpr int PSTRIDE = 2048;
struct NbList {
  int nb[Q_TOTAL];
};

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// op: 0 sum, 1 max, 2 min.  Stores the block result to out (thread 0).
// block reduction whose result is valid in thread 0
__device__ __forceinline__ double block_reduce_value(double v, int op) {
  __shared__ double shv[32];
  v = op == 0 ? warp_sum(v) : op == 1 ? warp_max(v) : warp_min(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) shv[w] = v;
  __syncthreads();
  double x = op == 0 ? 0.0 : op == 1 ? -1.0e308 : 1.0e308;
  if (w == 0) {
    x = lane < nw ? shv[lane] : x;
    x = op == 0 ? warp_sum(x) : op == 1 ? warp_max(x) : warp_min(x);
  }
  return x;
}

__device__ __forceinline__ void block_reduce_store(double v, int op, double* out) {
  __shared__ double sh[32];
  v = op == 0 ? warp_sum(v) : op == 1 ? warp_max(v) : warp_min(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double init = op == 0 ? 0.0 : op == 1 ? -1.0e308 : 1.0e308;
    double x = lane < nw ? sh[lane] : init;
    x = op == 0 ? warp_sum(x) : op == 1 ? warp_max(x) : warp_min(x);
    if (lane == 0) *out = x;
  }
}


// --------------------------------------------------------------- k helpers
__device__ __forceinline__ void kdecode(const DevConst& K, int64_t id, int& kx, int& ky, int& kz) {
  if (K.nk < ((int64_t)1 << 31)) {
    // 32-bit division (a 64-bit one is a long software sequence on the GPU)
    const unsigned u = (unsigned)id, nxh = (unsigned)K.nxh, ny = (unsigned)K.ny;
    const unsigned r = u / nxh;
    kx = (int)(u - r * nxh);
    kz = (int)(r / ny);
    ky = (int)(r - (unsigned)kz * ny);
    return;
  }
  kx = (int)(id % K.nxh);
  int64_t r = id / K.nxh;
  ky = (int)(r % K.ny);
  kz = (int)(r / K.ny);
}
__device__ __forceinline__ void kvec(const DevConst& K, int kx, int ky, int kz, double a[3], double b[3]) {
  const double twopi = 6.283185307179586476925286766559;
  const int n[3] = {K.nx, K.ny, K.nz}, m[3] = {kx, ky, kz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int mm = (m[d] <= n[d] / 2) ? m[d] : m[d] - n[d];
    a[d] = (double)mm * (twopi / (double)n[d]);
    b[d] = (2 * m[d] == n[d]) ? 0.0 : a[d];
  }
}
__device__ __forceinline__ double hweight(const DevConst& K, int kx) {
  return (kx == 0 || 2 * kx == K.nx) ? 1.0 : 2.0;
}
// -(the reference's grad_coeff multiplier) = k.kappa.k with kf_sq on the diagonal
__device__ __forceinline__ double kkappak(const double* g, const double a[3], const double b[3]) {
  // g column-major 3x3
  return g[0] * a[0] * a[0] + g[4] * a[1] * a[1] + g[8] * a[2] * a[2] + (g[3] + g[1]) * b[0] * b[1] +
         (g[7] + g[5]) * b[1] * b[2] + (g[2] + g[6]) * b[2] * b[0];
}
// k.kappa.k with Nyquist-zeroed vectors everywhere (gradient energy, f_int form)
__device__ __forceinline__ double kkappak_b(const double* g, const double b[3]) {
  return g[0] * b[0] * b[0] + g[4] * b[1] * b[1] + g[8] * b[2] * b[2] + (g[3] + g[1]) * b[0] * b[1] +
         (g[7] + g[5]) * b[1] * b[2] + (g[2] + g[6]) * b[2] * b[0];
}

__device__ __forceinline__ int voigt(int i, int j) { return i == j ? i : 9 - i - j; }

// Q(k) of ModElastic.f:119-158 with C0 = CEla(:,:,2) (column-major 3x3)
__device__ __forceinline__ void build_q(const DevConst& K, const double a[3], const double b[3], double Q[9]) {
#pragma unroll
  for (int i = 0; i < 9; ++i) Q[i] = 0;
#pragma unroll
  for (int i = 1; i <= 3; ++i)
#pragma unroll
    for (int j = 1; j <= 3; ++j) {
      const int ij = voigt(i, j);
#pragma unroll
      for (int k = 1; k <= 3; ++k)
#pragma unroll
        for (int l = 1; l <= 3; ++l) {
          const int kl = voigt(k, l);
          const double kpr = (k == j) ? -(a[k - 1] * a[k - 1]) : -(b[k - 1] * b[j - 1]);
          Q[(i - 1) + (l - 1) * 3] += K.c0m[(ij - 1) + (kl - 1) * 6] * kpr;
        }
    }
}

// General small inverse (ModFunc.f:44-72): Gauss-Jordan with partial pivoting,
// reciprocal 1-norm condition test.  Returns 0 or flag.  a is column-major.
template <int NMAX>
__device__ int invert_small(double* a, int n, int flag) {
  double anorm = 0;
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += fabs(a[i + j * n]);
    anorm = fmax(anorm, s);
  }
  int piv[NMAX];
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(a[k + k * n]);
    for (int i = k + 1; i < n; ++i) {
      double v = fabs(a[i + k * n]);
      if (v > best) { best = v; p = i; }
    }
    if (best == 0.0) return flag;
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        double t = a[k + j * n]; a[k + j * n] = a[p + j * n]; a[p + j * n] = t;
      }
      int t = piv[k]; piv[k] = piv[p]; piv[p] = t;
    }
    const double d = 1.0 / a[k + k * n];
    a[k + k * n] = 1.0;
    for (int j = 0; j < n; ++j) a[k + j * n] *= d;
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const double f = a[i + k * n];
      if (f == 0.0) continue;
      a[i + k * n] = 0.0;
      for (int j = 0; j < n; ++j) a[i + j * n] -= f * a[k + j * n];
    }
  }
  // undo the row permutation as a column permutation
  double w[NMAX * NMAX];
  for (int i = 0; i < n * n; ++i) w[i] = a[i];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + piv[j] * n] = w[i + j * n];
  double inorm = 0;
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += fabs(a[i + j * n]);
    inorm = fmax(inorm, s);
  }
  if (!(anorm * inorm < 1e16)) return flag;  // rcond = 1 / (|A| |A^-1|) > 1e-16
  return 0;
}

// 6x6 inverse by Gauss-Jordan without pivoting, fully unrolled so the matrix
// stays in registers (the compliance mixes inverted per voxel are symmetric
// positive definite).  Returns false when a pivot is not safely positive; the
// caller then falls back to invert_small (partial pivoting).
__device__ __forceinline__ bool invert6_spd(double* a) {
  double amax = 0;
#pragma unroll
  for (int i = 0; i < 36; ++i) amax = fmax(amax, fabs(a[i]));
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double pv = a[k + k * 6];
    ok = ok && (pv > 1e-13 * amax);
    const double d = 1.0 / pv;
    a[k + k * 6] = 1.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) a[k + j * 6] *= d;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (i == k) continue;
      const double f = a[i + k * 6];
      a[i + k * 6] = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) a[i + j * 6] -= f * a[k + j * 6];
    }
  }
  return ok;
}

// Inverse of a per-voxel 6x6 mix with the reference's singularity test
// (ModFunc.f:44-72): fast unrolled path, pivoting fallback.
__device__ __forceinline__ int invert6(double* a, int flag) {
  double b[36];
#pragma unroll
  for (int i = 0; i < 36; ++i) b[i] = a[i];
  if (invert6_spd(b)) {
    double anorm = 0, inorm = 0;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double sa = 0, si = 0;
#pragma unroll
      for (int i = 0; i < 6; ++i) { sa += fabs(a[i + j * 6]); si += fabs(b[i + j * 6]); }
      anorm = fmax(anorm, sa);
      inorm = fmax(inorm, si);
    }
    if (anorm * inorm < 1e16) {  // rcond > 1e-16
#pragma unroll
      for (int i = 0; i < 36; ++i) a[i] = b[i];
      return 0;
    }
  }
  return invert_small<6>(a, 6, flag);
}

// Inverse of a 6x6 (column-major) whose normal and shear parts decouple and whose shears
// are independent (nonzero only at i, j < 3 or i == j: every cubic or orthotropic
// compliance mix in the crystal frame): the 3x3 normal block by its adjugate, the three
// shears by their reciprocals.  The same singularity test as invert6, on the exact
// 1-norms of the block-diagonal matrix and of its inverse; a zero determinant or shear
// returns flag with a unchanged.
__device__ __forceinline__ int invert6_ortho(double* a, int flag) {
  const double b00 = a[0], b10 = a[1], b20 = a[2], b01 = a[6], b11 = a[7], b21 = a[8];
  const double b02 = a[12], b12 = a[13], b22 = a[14];
  const double s3 = a[21], s4 = a[28], s5 = a[35];
  const double c00 = b11 * b22 - b12 * b21, c01 = b02 * b21 - b01 * b22, c02 = b01 * b12 - b02 * b11;
  const double c10 = b12 * b20 - b10 * b22, c11 = b00 * b22 - b02 * b20, c12 = b02 * b10 - b00 * b12;
  const double c20 = b10 * b21 - b11 * b20, c21 = b01 * b20 - b00 * b21, c22 = b00 * b11 - b01 * b10;
  const double det = b00 * c00 + b01 * c10 + b02 * c20;
  if (det == 0.0 || s3 == 0.0 || s4 == 0.0 || s5 == 0.0) return flag;
  const double anorm = fmax(fmax(fabs(b00) + fabs(b10) + fabs(b20), fabs(b01) + fabs(b11) + fabs(b21)),
                            fmax(fabs(b02) + fabs(b12) + fabs(b22), fmax(fabs(s3), fmax(fabs(s4), fabs(s5)))));
  const double r = 1.0 / det;
  a[0] = c00 * r; a[6] = c01 * r; a[12] = c02 * r;
  a[1] = c10 * r; a[7] = c11 * r; a[13] = c12 * r;
  a[2] = c20 * r; a[8] = c21 * r; a[14] = c22 * r;
  a[21] = 1.0 / s3; a[28] = 1.0 / s4; a[35] = 1.0 / s5;
  const double inorm = fmax(fmax(fabs(a[0]) + fabs(a[1]) + fabs(a[2]), fabs(a[6]) + fabs(a[7]) + fabs(a[8])),
                            fmax(fabs(a[12]) + fabs(a[13]) + fabs(a[14]),
                                 fmax(fabs(a[21]), fmax(fabs(a[28]), fabs(a[35])))));
  // rcond = 1 / (|A| |A^-1|) <= 1e-16 stops, as the reference's rcond .le. 1e-16 does; a
  // mix of non-finite values (NaN) fails that comparison there and here alike, so it
  // goes on to the step's non-finite check (MEU_ERR_NOT_FINITE) instead
  if (anorm * inorm >= 1e16) return flag;
  return 0;
}
// nonzero pattern of invert6_ortho's matrices (column-major index i + 6 j)
__host__ __device__ constexpr bool ortho_nz(int k) { return (k % 6 < 3 && k / 6 < 3) || k % 6 == k / 6; }

// 3x3 inverse in closed form (adjugate), column-major; returns 0 or flag.
__device__ __forceinline__ int invert3(double* q, int flag) {
  const double a = q[0], b = q[3], c = q[6], d = q[1], e = q[4], f = q[7], g = q[2], h = q[5], i = q[8];
  const double A = e * i - f * h, B = -(d * i - f * g), Cc = d * h - e * g;
  const double det = a * A + b * B + c * Cc;
  const double anorm = fmax(fabs(a) + fabs(d) + fabs(g), fmax(fabs(b) + fabs(e) + fabs(h), fabs(c) + fabs(f) + fabs(i)));
  if (det == 0.0) return flag;
  const double r = 1.0 / det;
  double o[9];
  o[0] = A * r; o[3] = -(b * i - c * h) * r; o[6] = (b * f - c * e) * r;
  o[1] = B * r; o[4] = (a * i - c * g) * r; o[7] = -(a * f - c * d) * r;
  o[2] = Cc * r; o[5] = -(a * h - b * g) * r; o[8] = (a * e - b * d) * r;
  const double inorm = fmax(fabs(o[0]) + fabs(o[1]) + fabs(o[2]), fmax(fabs(o[3]) + fabs(o[4]) + fabs(o[5]), fabs(o[6]) + fabs(o[7]) + fabs(o[8])));
  for (int k = 0; k < 9; ++k) q[k] = o[k];
  // rcond = 1 / (|Q| |Q^-1|) > 1e-16, tested without a second division
  if (!(anorm * inorm < 1e16)) return flag;
  return 0;
}

}  // namespace meu
