// step_kernels.cuh -- the kernels of one time step (templated on the bulk
// precision R: double for the plain FP64 path, float for the FP32 path; every
// per-k operator and every reduction computes in FP64).
#pragma once
#include "kernels.cuh"

namespace meu {

__device__ __forceinline__ void set_err(int* err, int code) {
  if (code) atomicMax(err, code);
}

template <typename C>
__device__ __forceinline__ void ld2(const C& v, double& re, double& im) {
  re = (double)v.x;
  im = (double)v.y;
}

// ------------------------------------------------------------ KKS: gradients
// dft_grad_{x,y,z} = kf * phi^, dft_k_del_sq = phi^ * (grad_coeff multiplier)
// (Multi_MEUMAPPS.f:581-605).  in: V spectra at in0 + v*nk; out: 4V spectra at
// out0 + (4v+c)*nk (contiguous, so any variant count fits one launch).
template <typename R>
__global__ void __launch_bounds__(256) k_kks_grad(const DevConst* __restrict__ Kp, const cplx<R>* __restrict__ in0,
                                                  cplx<R>* __restrict__ out0, int V) {
  const DevConst& K = *Kp;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    for (int v = 0; v < V; ++v) {
      const cplx<R> val = in0[v * K.nk + id];
      const double re = val.x, im = val.y;
#pragma unroll
      for (int c = 0; c < 3; ++c) out0[(4 * v + c) * K.nk + id] = mk((R)(-b[c] * im), (R)(b[c] * re));
      const double m = -kkappak(K.p.grad_coeff[v], a, b);
      out0[(4 * v + 3) * K.nk + id] = mk((R)(re * m), (R)(im * m));
    }
  }
}

// ------------------------------------------------- KKS: local driving force
// Multi_MEUMAPPS.f:634-845 per voxel.  g4 = [gx_v, gy_v, gz_v, kds_v] per v.
// Fields in R; the local solve and the energies in FP64.  NPH, NEL > 0: the phase and
// solute counts are compile-time (the common decks), so the zdim x zdim composition
// system and its inverse live in registers; 0, 0: any counts, arrays sized for the
// largest system (local memory).
template <typename R, int NPH = 0, int NEL = 0>
__global__ void __launch_bounds__(RED_THREADS) k_kks_point(const DevConst* __restrict__ Kp, const R* __restrict__ phi,
                                                           const R* __restrict__ cons, const R* __restrict__ g4,
                                                           R* __restrict__ pphi, R* __restrict__ fdiff,
                                                           R* __restrict__ fc, double* partials, int* err) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  constexpr bool FIX = NPH > 0 && NEL > 0;
  constexpr int ZM = FIX ? NPH * NEL : 12;  // largest zdim the arrays hold
  const int V = p.nvar, numel = FIX ? NEL : p.numel, numph = FIX ? NPH : p.numph, zdim = FIX ? ZM : K.zdim;
  const int64_t n3 = K.n3;
  double fch = 0, fw = 0, fint = 0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
    double Pph[MEU_MAX_PH], Gph[MEU_MAX_PH], Ppr[MEU_MAX_VAR], fgrad[MEU_MAX_VAR], ph[MEU_MAX_VAR];
    for (int n = 0; n < MEU_MAX_PH; ++n) { Pph[n] = 0; Gph[n] = 0; }
    for (int v = 0; v < V; ++v) ph[v] = (double)phi[v * n3 + id];
    for (int n = 2; n <= numph; ++n)
      for (int v = K.ph_lo[n]; v < K.ph_hi[n]; ++v) {
        const double fi = ph[v], fi_sq = fi * fi;
        const double pl = fi_sq * fi * (6.0 * fi_sq - 15.0 * fi + 10.0);
        pphi[v * n3 + id] = (R)pl;
        Ppr[v] = 30.0 * fi_sq * (fi_sq - 2.0 * fi + 1.0);
        Pph[0] += pl;
        Pph[n - 1] += pl;
        Gph[n - 1] += fi_sq * (1.0 - fi) * (1.0 - fi);
        for (int u = 0; u < V; ++u)
          if (u != v) Gph[0] += fi_sq * ph[u] * ph[u];
      }
    Pph[0] = 1.0 - Pph[0];
    // interface compositions (:677-710)
    double Z[ZM * ZM], Zr[ZM], X[MEU_MAX_EL][MEU_MAX_PH], Gib[MEU_MAX_PH], MuC[MEU_MAX_EL];
    for (int i = 0; i < zdim * zdim; ++i) Z[i] = K.zconst[i];
    for (int i = 0; i < zdim; ++i) Zr[i] = K.zr_const[i];
    for (int e = 1; e <= numel; ++e) {
      const int i0 = zdim - numel + e;
      Zr[i0 - 1] = (double)cons[(e - 1) * n3 + id];
      for (int n = 1; n <= numph; ++n) Z[(i0 - 1) + (numph * (e - 1) + n - 1) * zdim] = Pph[n - 1];
    }
    set_err(err, invert_small<ZM>(Z, zdim, MEU_ERR_Z_SINGULAR));
    for (int n = 1; n <= numph; ++n)
      for (int e = 1; e <= numel; ++e) {
        const int i0 = numph * (e - 1) + n;
        double acc = 0;
        for (int j0 = 1; j0 <= zdim; ++j0) acc += Z[(i0 - 1) + (j0 - 1) * zdim] * Zr[j0 - 1];
        X[e - 1][n - 1] = acc;
      }
#define GP(j, n) p.gparams[(n) - 1][(j) - 1]
    for (int n = 1; n <= numph; ++n) {
      double g = 0;
      for (int e = 1; e <= numel; ++e) {
        const double d = X[e - 1][n - 1] - GP(e + numel + 1, n);
        g += GP(e, n) * d * d;
      }
      Gib[n - 1] = g + GP(numel + 1, n);
    }
    for (int e = 1; e <= numel; ++e) MuC[e - 1] = 2.0 * GP(e, 1) * (X[e - 1][0] - GP(e + numel + 1, 1));
#undef GP
    double fchloc = Pph[0] * Gib[0], fwloc = p.wellph[0] * Gph[0];
    double fcl[3 * MEU_MAX_EL];
    for (int i = 0; i < 3 * numel; ++i) fcl[i] = 0;
    for (int n = 2; n <= numph; ++n) {
      for (int v = K.ph_lo[n]; v < K.ph_hi[n]; ++v) {
        const double* g = p.grad_coeff[v];
        const double gx = (double)g4[(4 * v + 0) * n3 + id], gy = (double)g4[(4 * v + 1) * n3 + id];
        const double gz = (double)g4[(4 * v + 2) * n3 + id];
        const double term = g[0] * gx * gx + g[4] * gy * gy + g[8] * gz * gz + (g[3] + g[1]) * gx * gy +
                            (g[6] + g[2]) * gx * gz + (g[7] + g[5]) * gy * gz;
        fint += 0.5 * term;
        const double fi = ph[v];
        double termch = Gib[n - 1] - Gib[0];
        for (int e = 0; e < numel; ++e) {
          const double xd = X[e][0] - X[e][n - 1];
          termch += MuC[e] * xd;
          const double t = Ppr[v] * xd;
          fcl[3 * e + 0] += t * gx;
          fcl[3 * e + 1] += t * gy;
          fcl[3 * e + 2] += t * gz;
        }
        double well = 2.0 * p.wellph[n - 1] * fi * (1.0 - fi) * (1.0 - 2.0 * fi);
        for (int u = 0; u < V; ++u)
          if (u != v) well += 4.0 * p.wellph[0] * fi * ph[u] * ph[u];
        fgrad[v] = termch * Ppr[v] + well;
      }
      fchloc += Pph[n - 1] * Gib[n - 1];
      fwloc += p.wellph[n - 1] * Gph[n - 1];
    }
    fch += fchloc;
    fw += fwloc;
    for (int i = 0; i < 3 * numel; ++i) fc[(int64_t)i * n3 + id] = (R)fcl[i];
    // n_tilda projection (:824-841)
    for (int jv = 0; jv < V; ++jv) {
      double term11 = 0;
      int nt = 1;
      if (ph[jv] > 0.0)
        for (int iv = 0; iv < V; ++iv)
          if (ph[iv] > 0.0 && iv != jv) {
            term11 += fgrad[iv] - (double)g4[(4 * iv + 3) * n3 + id];
            nt += 1;
          }
      fdiff[jv * n3 + id] = (R)(fgrad[jv] - term11 / (double)nt);
    }
  }
  block_reduce_store(fch, 0, partials + Q_FCH * PSTRIDE + blockIdx.x);
  block_reduce_store(fw, 0, partials + Q_FW * PSTRIDE + blockIdx.x);
  block_reduce_store(fint, 0, partials + Q_FINT * PSTRIDE + blockIdx.x);
}

// ------------------------------------------------------ elastic: zeroth order
// ModElastic.f:115-236: u^ = Q^-1 R, R_i = sum_j kf_j sum_v P^_v sig0_v(ij); the
// engineering strain gamma^ of u^ goes to g[0..6).
template <typename R>
__global__ void __launch_bounds__(256) k_el_zeroth(const DevConst* __restrict__ Kp, PtrList<cplx<R>> pk, int V,
                                                   cplx<R>* __restrict__ uk, PtrList<cplx<R>> g, int* err) {
  const DevConst& K = *Kp;
  const int64_t nk = K.nk;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    double sr[6] = {0, 0, 0, 0, 0, 0}, si[6] = {0, 0, 0, 0, 0, 0};
    for (int v = 0; v < V; ++v) {
      double re, im;
      ld2(pk.p[v][id], re, im);
#pragma unroll
      for (int m = 0; m < 6; ++m) { sr[m] += re * K.sig0[v][m]; si[m] += im * K.sig0[v][m]; }
    }
    // R_i = i sum_j b_j S_ij  (S symmetric, Voigt m = voigt(i,j))
    double Rr[3], Ri[3];
#pragma unroll
    for (int i = 1; i <= 3; ++i) {
      double tr = 0, ti = 0;
#pragma unroll
      for (int j = 1; j <= 3; ++j) { const int m = voigt(i, j) - 1; tr += b[j - 1] * sr[m]; ti += b[j - 1] * si[m]; }
      Rr[i - 1] = -ti;
      Ri[i - 1] = tr;
    }
    double ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
    if (id != 0) {
      double Q[9];
      build_q(K, a, b, Q);
      set_err(err, invert3(Q, MEU_ERR_Q_SINGULAR));
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        ur[i] = Q[i] * Rr[0] + Q[i + 3] * Rr[1] + Q[i + 6] * Rr[2];
        ui[i] = Q[i] * Ri[0] + Q[i + 3] * Ri[1] + Q[i + 6] * Ri[2];
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) uk[(int64_t)i * nk + id] = mk((R)ur[i], (R)ui[i]);
    // gamma = i*(b (x) u) symmetrised, engineering Voigt order 11,22,33,23,13,12
    const int I1[6] = {0, 1, 2, 1, 0, 0}, J1[6] = {0, 1, 2, 2, 2, 1};
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const int i = I1[m], j = J1[m];
      double gr, gi;
      if (m < 3) { gr = -b[i] * ui[i]; gi = b[i] * ur[i]; }
      else { gr = -(b[i] * ui[j] + b[j] * ui[i]); gi = b[i] * ur[j] + b[j] * ur[i]; }
      g.p[m][id] = mk((R)gr, (R)gi);
    }
  }
}

// --------------------------------------------------- elastic: polarisation x
// ModElastic.f:248-327.  strain = engineering gamma (6), xs out (6).  General
// moduli: the per-voxel mixed compliance is inverted (6x6); the proportional case
// goes through k_el_x_prop below.  ORTHO: every phase's compliance and C0 have the
// decoupled normal / shear pattern (cubic or orthotropic in the crystal frame), so the
// mix is inverted as a 3x3 block and three shears and the zero entries are skipped.
template <typename R, bool ORTHO = false>
__global__ void __launch_bounds__(256, ORTHO ? 3 : 1) k_el_x(const DevConst* __restrict__ Kp, const R* __restrict__ pphi,
                                              const R* __restrict__ strain, R* __restrict__ xs, double cfac, int* err) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  const int64_t n3 = K.n3;
  const int V = p.nvar;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
    double Cm[36], e0[6] = {0, 0, 0, 0, 0, 0}, psum = 0;
    for (int v = 0; v < V; ++v) {
      const double pv = (double)pphi[v * n3 + id];
#pragma unroll
      for (int m = 0; m < 6; ++m) e0[m] += pv * K.eps_eng[v][m];
    }
    {
#pragma unroll
      for (int i = 0; i < 36; ++i) Cm[i] = 0;
      for (int n = 2; n <= p.numph; ++n)
        for (int v = K.ph_lo[n]; v < K.ph_hi[n]; ++v) {
          const double pv = (double)pphi[v * n3 + id];
          psum += pv;
#pragma unroll
          for (int i = 0; i < 36; ++i)
            if (!ORTHO || ortho_nz(i)) Cm[i] += pv * p.sela[n - 1][i];
        }
      if (psum < 1.0) {
#pragma unroll
        for (int i = 0; i < 36; ++i)
          if (!ORTHO || ortho_nz(i)) Cm[i] += (1.0 - psum) * p.sela[0][i];
      }
      set_err(err, ORTHO ? invert6_ortho(Cm, MEU_ERR_C_SINGULAR) : invert6(Cm, MEU_ERR_C_SINGULAR));
    }
    double gam[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) gam[m] = (double)strain[(int64_t)m * n3 + id] + K.ebar_eng[m];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double s = 0;
#pragma unroll
      for (int m = 0; m < 6; ++m) {
        if (ORTHO && !ortho_nz(r + m * 6)) continue;
        const double c = Cm[r + m * 6];
        s += cfac * (K.c0m[r + m * 6] - c) * gam[m] + c * e0[m];
      }
      xs[(int64_t)r * n3 + id] = (R)s;
    }
  }
}

// 6x6 (column-major) times 6-vector.  ORTHO: normal and shear parts decouple and the
// shears are independent (C[i][j] = 0 for i < 3 <= j, j < 3 <= i and 3 <= i != j,
// every cubic or orthotropic stiffness in its crystal frame).  The skipped terms are
// exact zeros, so the sums are bit-identical to the full product.
template <bool ORTHO, typename W>
__device__ __forceinline__ void mv6(const W* __restrict__ c, const W* x, W* y) {
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    W a = 0;
#pragma unroll
    for (int m = 0; m < 6; ++m)
      if (!ORTHO || (i < 3 && m < 3) || i == m) a += c[i + m * 6] * x[m];
    y[i] = a;
  }
}

// Per-voxel prefetch through shared memory: each thread copies its own voxel's
// values of the next tile with cp.async while it works on the current one, so the
// loads of a whole tile are in flight during the FP64 work without holding
// registers.  Per element (VEC = false): thread i copies and uses voxel i of every
// tile, no barrier needed.  VEC (n3 a multiple of 16 bytes of R): the tile moves in
// 16-byte copies spread over the block, and barriers order copies and uses.
constexpr int PF_TILE = 256;
template <typename R>
__device__ __forceinline__ void pf_copy(R* smem, const R* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(R) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void pf_copy16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void pf_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void pf_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Proportional moduli (K.prop_moduli): C(x) = C_1 / s(x), so
// x = cfac C0 gamma + (C_1 / s)(e0 - cfac gamma), s = sum_v alpha_v P_v (+ 1 - sum P).
// The coefficients travel as a kernel parameter, so the FP64 products read their
// constants straight from the parameter bank.  Dynamic shared memory:
// 2 * (6 + V) * PF_TILE elements of R (double-buffered tiles, field-major).
template <typename R, bool ORTHO, bool VEC>
__global__ void __launch_bounds__(PF_TILE, 4) k_el_x_prop(const __grid_constant__ ElxProp E, int64_t n3,
                                                          const R* __restrict__ pphi, const R* __restrict__ strain,
                                                          R* __restrict__ xs, double cfac, int* err) {
  constexpr int NV = MEU_MAX_VAR;
  const int V = E.nvar;
  const int NF = 6 + V;
  extern __shared__ __align__(16) unsigned char pf_raw[];
  R* buf = (R*)pf_raw;
  const int tid = threadIdx.x;
  auto issue = [&](int64_t tile, int slot) {
    if constexpr (VEC) {
      constexpr int PER = 16 / (int)sizeof(R), CPF = PF_TILE / PER;
      const int64_t base = tile * PF_TILE;
      R* b = buf + (int64_t)slot * NF * PF_TILE;
      for (int c = tid; c < NF * CPF; c += PF_TILE) {
        const int f = c / CPF, j = (c - f * CPF) * PER;
        const R* src = f < 6 ? strain + (int64_t)f * n3 : pphi + (int64_t)(f - 6) * n3;
        if (base + j < n3) pf_copy16(b + f * PF_TILE + j, src + base + j);
      }
    } else {
      const int64_t id = tile * PF_TILE + tid;
      R* b = buf + (int64_t)slot * NF * PF_TILE + tid;
      if (id < n3) {
#pragma unroll
        for (int m = 0; m < 6; ++m) pf_copy(b + m * PF_TILE, strain + (int64_t)m * n3 + id);
#pragma unroll
        for (int v = 0; v < NV; ++v)
          if (v < V) pf_copy(b + (6 + v) * PF_TILE, pphi + (int64_t)v * n3 + id);
      }
    }
    pf_commit();
  };
  const int64_t ntiles = (n3 + PF_TILE - 1) / PF_TILE;
  int64_t tile = blockIdx.x;
  issue(tile, 0);
  for (int k = 0; tile < ntiles; tile += gridDim.x, ++k) {
    if (VEC) __syncthreads();  // every thread is done with the slot the next copies fill
    issue(tile + gridDim.x, (k + 1) & 1);
    pf_wait_prev();
    if (VEC) __syncthreads();  // the other threads' copies of this tile have landed
    const int64_t id = tile * PF_TILE + tid;
    if (id >= n3) continue;
    const R* b = buf + (int64_t)(k & 1) * NF * PF_TILE + tid;
    double e0[6] = {0, 0, 0, 0, 0, 0}, psum = 0, sc = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v >= V) break;
      const double q = (double)b[(6 + v) * PF_TILE];
      psum += E.inc[v] * q;
      sc += E.av[v] * q;
#pragma unroll
      for (int m = 0; m < 6; ++m) e0[m] += q * E.ep[v][m];
    }
    if (psum < 1.0) sc += 1.0 - psum;
    if (!(sc != 0.0)) set_err(err, MEU_ERR_C_SINGULAR);
    const double r = 1.0 / sc;
    double gam[6], d[6], a0[6], a1[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      gam[m] = (double)b[m * PF_TILE] + E.ebar[m];
      d[m] = e0[m] - cfac * gam[m];
    }
    mv6<ORTHO>(E.c0, gam, a0);
    mv6<ORTHO>(E.c1, d, a1);
#pragma unroll
    for (int i = 0; i < 6; ++i) xs[(int64_t)i * n3 + id] = (R)(cfac * a0[i] + r * a1[i]);
  }
}

// ------------------------------------------------- elastic: Green operator
// ModElastic.f:340-394: u^ = Qinv (kf . x^), gamma^ of u^ written over x^.
// Convergence sums (ModElastic.f:413-430) by Parseval against the previous u^.
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_el_k(const DevConst* __restrict__ Kp, PtrList<cplx<R>> xk,
                                                      cplx<R>* __restrict__ uk, double* partials, int* err) {
  using C = cplx<R>;
  const DevConst& K = *Kp;
  const int64_t nk = K.nk, stride = (int64_t)gridDim.x * blockDim.x;
  double e[6] = {0, 0, 0, 0, 0, 0};
  // software pipeline: the next k's nine loads are in flight during this k's FP64 work
  int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  C x[6], u[3];
  if (id < nk) {
#pragma unroll
    for (int m = 0; m < 6; ++m) x[m] = xk.p[m][id];
#pragma unroll
    for (int i = 0; i < 3; ++i) u[i] = uk[(int64_t)i * nk + id];
  }
  for (; id < nk; id += stride) {
    const int64_t nid = id + stride;
    C xn[6], un[3];
    if (nid < nk) {
#pragma unroll
      for (int m = 0; m < 6; ++m) xn[m] = xk.p[m][nid];
#pragma unroll
      for (int i = 0; i < 3; ++i) un[i] = uk[(int64_t)i * nk + nid];
    }
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    double xr[6], xi[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) { xr[m] = (double)x[m].x; xi[m] = (double)x[m].y; }
    // R = kf . x (Voigt 1..6 -> x1 x2 x3 x4 x5 x6)
    const double tr1 = xr[0] * b[0] + xr[5] * b[1] + xr[4] * b[2], ti1 = xi[0] * b[0] + xi[5] * b[1] + xi[4] * b[2];
    const double tr2 = xr[5] * b[0] + xr[1] * b[1] + xr[3] * b[2], ti2 = xi[5] * b[0] + xi[1] * b[1] + xi[3] * b[2];
    const double tr3 = xr[4] * b[0] + xr[3] * b[1] + xr[2] * b[2], ti3 = xi[4] * b[0] + xi[3] * b[1] + xi[2] * b[2];
    const double Rr[3] = {-ti1, -ti2, -ti3}, Ri[3] = {tr1, tr2, tr3};
    double ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
    if (id != 0) {
      double Q[9];
      build_q(K, a, b, Q);
      set_err(err, invert3(Q, MEU_ERR_Q_SINGULAR));
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        ur[i] = Q[i] * Rr[0] + Q[i + 3] * Rr[1] + Q[i + 6] * Rr[2];
        ui[i] = Q[i] * Ri[0] + Q[i + 3] * Ri[1] + Q[i + 6] * Ri[2];
      }
    }
    const double w = hweight(K, kx);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double orr = (double)u[i].x, oi = (double)u[i].y;
      const double dr = ur[i] - orr, di = ui[i] - oi;
      e[2 * i] += w * (dr * dr + di * di);
      e[2 * i + 1] += w * (orr * orr + oi * oi);
      uk[(int64_t)i * nk + id] = mk((R)ur[i], (R)ui[i]);
    }
    const int I1[6] = {0, 1, 2, 1, 0, 0}, J1[6] = {0, 1, 2, 2, 2, 1};
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const int i = I1[m], j = J1[m];
      double gr, gi;
      if (m < 3) { gr = -b[i] * ui[i]; gi = b[i] * ur[i]; }
      else { gr = -(b[i] * ui[j] + b[j] * ui[i]); gi = b[i] * ur[j] + b[j] * ur[i]; }
      xk.p[m][id] = mk((R)gr, (R)gi);
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) x[m] = xn[m];
#pragma unroll
    for (int i = 0; i < 3; ++i) u[i] = un[i];
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) block_reduce_store(e[q], 0, partials + (Q_ERR0 + q) * PSTRIDE + blockIdx.x);
}

// -------------------------------------------------------------- elener
// ModElastic.f:540-687.  mode 0 (KKS): fdiff += el_grad; mode 1 (Landau): elg = el_grad.
// theta' = 30 f^2 (f^2 - 2f + 1) (KKS and Landau h coupling) or 2 eta (eta^2 coupling).
template <typename R, bool ORTHO = false>
__global__ void __launch_bounds__(RED_THREADS, ORTHO ? 3 : 1) k_elener(const DevConst* __restrict__ Kp, const R* __restrict__ phi,
                                                        const R* __restrict__ pphi, const R* __restrict__ strain,
                                                        R* __restrict__ el_en, R* __restrict__ elg, int mode, int eta2,
                                                        double* partials, int* err) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  const int64_t n3 = K.n3;
  const int V = p.nvar;
  double esum = 0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
    double te[6] = {0, 0, 0, 0, 0, 0}, psum = 0, P[MEU_MAX_VAR];
    for (int v = 0; v < V; ++v) {
      P[v] = (double)pphi[v * n3 + id];
      psum += P[v];
#pragma unroll
      for (int m = 0; m < 6; ++m) te[m] += P[v] * p.trans_ppt[v][m];
    }
    double eps[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const double gm = (double)strain[(int64_t)m * n3 + id];
      eps[m] = (m < 3) ? (p.e_mean[m] + gm - te[m]) : (2.0 * p.e_mean[m] + gm - 2.0 * te[m]);
    }
    double Cm[36], sig[6];
    {
#pragma unroll
      for (int i = 0; i < 36; ++i) Cm[i] = (!ORTHO || ortho_nz(i)) ? (1.0 - psum) * p.sela[0][i] : 0.0;
      for (int n = 2; n <= p.numph; ++n)
        for (int v = K.ph_lo[n]; v < K.ph_hi[n]; ++v) {
#pragma unroll
          for (int i = 0; i < 36; ++i)
            if (!ORTHO || ortho_nz(i)) Cm[i] += P[v] * p.sela[n - 1][i];
        }
      set_err(err, ORTHO ? invert6_ortho(Cm, MEU_ERR_C_ELENER_SINGULAR) : invert6(Cm, MEU_ERR_C_ELENER_SINGULAR));
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j)
          if (!ORTHO || ortho_nz(i + j * 6)) s += Cm[i + j * 6] * eps[j];
        sig[i] = s;
      }
    }
    double elmat = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double em = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j)
        if (!ORTHO || ortho_nz(i + j * 6)) em += p.sela[0][i + j * 6] * sig[j];
      elmat += sig[i] * em;
    }
    elmat *= 0.5;
    double en = (1.0 - psum) * elmat;
    for (int n = 2; n <= p.numph; ++n)
      for (int v = K.ph_lo[n]; v < K.ph_hi[n]; ++v) {
        if (!K.use_var[v]) continue;
        double elp = 0;
        {
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            double ep = 0;
#pragma unroll
            for (int j = 0; j < 6; ++j)
              if (!ORTHO || ortho_nz(i + j * 6)) ep += p.sela[n - 1][i + j * 6] * sig[j];
            elp += sig[i] * ep;
          }
          elp *= 0.5;
        }
        en += elp * P[v];
        const double* t = p.trans_ppt[v];
        const double g = sig[0] * t[0] + sig[1] * t[1] + sig[2] * t[2] + 2.0 * (sig[3] * t[3] + sig[4] * t[4] + sig[5] * t[5]);
        const double f = (double)phi[v * n3 + id];
        const double pr = eta2 ? 2.0 * f : 30.0 * f * f * (f * f - 2.0 * f + 1.0);
        const double eg = pr * (elmat - elp) - g * pr;
        if (mode == 0) elg[v * n3 + id] += (R)eg;
        else elg[v * n3 + id] = (R)eg;
      }
    el_en[id] = (R)en;
    esum += en;
  }
  block_reduce_store(esum, 0, partials + Q_ELEN * PSTRIDE + blockIdx.x);
}

// Proportional moduli (K.prop_moduli) form of k_elener: sigma = (C_1 eps) / s with
// s = 1 - sum P + sum_v alpha_v P_v, and each variant's energy alpha_v * elmat.
// Coefficients as a kernel parameter; ORTHO as in mv6.  Loads prefetched through
// shared memory as in k_el_x_prop: dynamic shared memory 2 * (6 + 2V) * PF_TILE
// elements of R.
template <typename R, bool ORTHO, bool VEC>
__global__ void __launch_bounds__(PF_TILE, 3) k_elener_prop(const __grid_constant__ ElenProp E, int64_t n3,
                                                            const R* __restrict__ phi, const R* __restrict__ pphi,
                                                            const R* __restrict__ strain, R* __restrict__ el_en,
                                                            R* __restrict__ elg, int mode, int eta2, double* partials,
                                                            int* err) {
  static_assert(PF_TILE == RED_THREADS, "one voxel per reduction thread");
  constexpr int NV = MEU_MAX_VAR;
  const int V = E.nvar;
  const int NF = 6 + 2 * V;
  extern __shared__ __align__(16) unsigned char pf_raw[];
  R* buf = (R*)pf_raw;
  const int tid = threadIdx.x;
  auto issue = [&](int64_t tile, int slot) {
    if constexpr (VEC) {
      constexpr int PER = 16 / (int)sizeof(R), CPF = PF_TILE / PER;
      const int64_t base = tile * PF_TILE;
      R* b = buf + (int64_t)slot * NF * PF_TILE;
      for (int c = tid; c < NF * CPF; c += PF_TILE) {
        const int f = c / CPF, j = (c - f * CPF) * PER;
        const R* src = f < 6 ? strain + (int64_t)f * n3
                             : (f < 6 + V ? pphi + (int64_t)(f - 6) * n3 : phi + (int64_t)(f - 6 - V) * n3);
        if (base + j < n3 && (f < 6 + V || E.use[f - 6 - V])) pf_copy16(b + f * PF_TILE + j, src + base + j);
      }
    } else {
      const int64_t id = tile * PF_TILE + tid;
      R* b = buf + (int64_t)slot * NF * PF_TILE + tid;
      if (id < n3) {
#pragma unroll
        for (int m = 0; m < 6; ++m) pf_copy(b + m * PF_TILE, strain + (int64_t)m * n3 + id);
#pragma unroll
        for (int v = 0; v < NV; ++v)
          if (v < V) {
            pf_copy(b + (6 + v) * PF_TILE, pphi + (int64_t)v * n3 + id);
            if (E.use[v]) pf_copy(b + (6 + V + v) * PF_TILE, phi + (int64_t)v * n3 + id);
          }
      }
    }
    pf_commit();
  };
  double esum = 0;
  const int64_t ntiles = (n3 + PF_TILE - 1) / PF_TILE;
  int64_t tile = blockIdx.x;
  issue(tile, 0);
  for (int k = 0; tile < ntiles; tile += gridDim.x, ++k) {
    if (VEC) __syncthreads();  // every thread is done with the slot the next copies fill
    issue(tile + gridDim.x, (k + 1) & 1);
    pf_wait_prev();
    if (VEC) __syncthreads();  // the other threads' copies of this tile have landed
    const int64_t id = tile * PF_TILE + tid;
    if (id >= n3) continue;
    const R* b = buf + (int64_t)(k & 1) * NF * PF_TILE + tid;
    double te[6] = {0, 0, 0, 0, 0, 0}, psum = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v >= V) break;
      const double q = (double)b[(6 + v) * PF_TILE];
      psum += q;
#pragma unroll
      for (int m = 0; m < 6; ++m) te[m] += q * E.tp[v][m];
    }
    double eps[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const double gm = (double)b[m * PF_TILE];
      eps[m] = (m < 3) ? (E.emean[m] + gm - te[m]) : (2.0 * E.emean[m] + gm - 2.0 * te[m]);
    }
    double sc = 1.0 - psum;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v >= V) break;
      sc += E.av[v] * (double)b[(6 + v) * PF_TILE];
    }
    if (!(sc != 0.0)) set_err(err, MEU_ERR_C_ELENER_SINGULAR);
    const double r = 1.0 / sc;
    double sig[6], em[6];
    mv6<ORTHO>(E.c1, eps, sig);
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[i] *= r;
    mv6<ORTHO>(E.s1, sig, em);
    double elmat = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) elmat += sig[i] * em[i];
    elmat *= 0.5;
    double en = (1.0 - psum) * elmat;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (v >= V) break;
      if (!E.use[v]) continue;
      const double elp = E.av[v] * elmat;
      en += elp * (double)b[(6 + v) * PF_TILE];
      const double* t = E.tp[v];
      const double g = sig[0] * t[0] + sig[1] * t[1] + sig[2] * t[2] + 2.0 * (sig[3] * t[3] + sig[4] * t[4] + sig[5] * t[5]);
      const double f = (double)b[(6 + V + v) * PF_TILE];
      const double pr = eta2 ? 2.0 * f : 30.0 * f * f * (f * f - 2.0 * f + 1.0);
      const double eg = pr * (elmat - elp) - g * pr;
      if (mode == 0) elg[v * n3 + id] += (R)eg;
      else elg[v * n3 + id] = (R)eg;
    }
    el_en[id] = (R)en;
    esum += en;
  }
  block_reduce_store(esum, 0, partials + Q_ELEN * PSTRIDE + blockIdx.x);
}

// --------------------------------------------------- KKS: diffusion update
// Multi_MEUMAPPS.f:924-943 on spectra [c, fx, fy, fz] of one solute.
template <typename R>
__global__ void __launch_bounds__(256) k_kks_ch(const DevConst* __restrict__ Kp, cplx<R>* __restrict__ ck,
                                                const cplx<R>* __restrict__ fx, const cplx<R>* __restrict__ fy,
                                                const cplx<R>* __restrict__ fz, double dm) {
  const DevConst& K = *Kp;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    const double ksq = -a[0] * a[0] - a[1] * a[1] - a[2] * a[2];
    double cr, ci, xr, xi, yr, yi, zr, zi;
    ld2(ck[id], cr, ci);
    ld2(fx[id], xr, xi);
    ld2(fy[id], yr, yi);
    ld2(fz[id], zr, zi);
    // term1 = i (b . F)
    const double t1r = -(b[0] * xi + b[1] * yi + b[2] * zi), t1i = b[0] * xr + b[1] * yr + b[2] * zr;
    const double term2 = 1.0 - dm * ksq;
    ck[id] = mk((R)((cr + dm * t1r) / term2), (R)((ci + dm * t1i) / term2));
  }
}

// TDGL right-hand side in real space: w = phi - dt L f_diff + dt noise
// (by linearity equal to the three transforms of Multi_MEUMAPPS.f:957-987).
template <typename R>
__global__ void k_tdgl_pre(const R* __restrict__ phi, const R* __restrict__ fdiff, const R* __restrict__ noise,
                           R* __restrict__ w, int64_t n, double dtl, double dt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    w[i] = (R)((double)phi[i] - dtl * (double)fdiff[i] + dt * (double)noise[i]);
}

// TDGL divide (Multi_MEUMAPPS.f:979-987): w^ /= 1 + dt L k.kappa.k
template <typename R>
__global__ void __launch_bounds__(256) k_tdgl(const DevConst* __restrict__ Kp, PtrList<cplx<R>> sp, int V, double dtl) {
  const DevConst& K = *Kp;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    for (int v = 0; v < V; ++v) {
      const double den = 1.0 + dtl * kkappak(K.p.grad_coeff[v], a, b);
      double re, im;
      ld2(sp.p[v][id], re, im);
      sp.p[v][id] = mk((R)(re / den), (R)(im / den));
    }
  }
}

// TDGL update of the spectral state: eta^ <- (eta^ - dt L g^) / (1 + dt L k.kappa.k);
// the new spectrum is also written to sp (the inverse transform consumes it).
template <typename R>
__global__ void __launch_bounds__(256) k_tdgl_state(const DevConst* __restrict__ Kp, PtrList<cplx<R>> sp, int V,
                                                    cplx<R>* __restrict__ keta, double dtl) {
  const DevConst& K = *Kp;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    for (int v = 0; v < V; ++v) {
      const double den = 1.0 + dtl * kkappak(K.p.grad_coeff[v], a, b);
      double gr, gi, hr, hi;
      ld2(sp.p[v][id], gr, gi);
      ld2(keta[(int64_t)v * K.nk + id], hr, hi);
      const cplx<R> o = mk((R)((hr - dtl * gr) / den), (R)((hi - dtl * gi) / den));
      keta[(int64_t)v * K.nk + id] = o;
      sp.p[v][id] = o;
    }
  }
}

// -------------------------------------------------------------- Landau
// theta_v, mu_c and the bulk free energy
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_lan_a(const DevConst* __restrict__ Kp, const R* __restrict__ c,
                                                       const R* __restrict__ eta, R* __restrict__ theta,
                                                       R* __restrict__ mu, double* partials) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  const int64_t n3 = K.n3;
  const int V = p.nvar;
  const int hcp = p.eig_coupling == MEU_EIG_H;
  double fch = 0;
  const double cbar = K.c_shift ? K.c_mean[0] : 0.0;
  // mu is transformed only to be multiplied by k^2: its constant part A (cbar - c1) is dropped
  const double mu0 = K.c_shift ? p.lan_a * (cbar - p.lan_c1) : 0.0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
    const double cv = cbar + (double)c[id];
    double s2 = 0, s4 = 0, s6 = 0;
    for (int v = 0; v < V; ++v) {
      const double e = (double)eta[v * n3 + id], e2 = e * e;
      s2 += e2; s4 += e2 * e2; s6 += e2 * e2 * e2;
      theta[v * n3 + id] = (R)(hcp ? e2 * e * (6.0 * e2 - 15.0 * e + 10.0) : e2);
    }
    // sum_{u != v} eta_u^2 eta_v^2 = s2^2 - s4
    const double cross = s2 * s2 - s4;
    fch += 0.5 * p.lan_a * (cv - p.lan_c1) * (cv - p.lan_c1) + 0.5 * p.lan_b * (p.lan_c2 - cv) * s2 - 0.25 * p.lan_c * s4 +
           p.lan_d / 6.0 * s6 + p.cross_w * cross;
    mu[id] = (R)((p.lan_a * (cv - p.lan_c1) - mu0) - 0.5 * p.lan_b * s2);
  }
  block_reduce_store(fch, 0, partials + Q_FCH * PSTRIDE + blockIdx.x);
}

// Landau k-space kernel: gradient energy (Parseval), homogeneous Green
// operator phi^_p = sum_q (sig0_p b).Omega.(sig0_q b) theta^_q with
// Omega = -Q^-1 (the reference's Q, ModElastic.f:119-158), its exact elastic
// energy, and the Cahn-Hilliard update of the spectral state
//   dc^ <- (dc^ - dt M k^2 mu^) / (1 + dt M kappa_c k^4),  dc^(0) = 0.
// sp: [theta_0..V-1, mu] on entry; [phi_0..V-1 (homog), dc_new] on exit.
// kc: dc^ state (read, updated); keta: eta^ state (read for the energy).
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_lan_k1(const DevConst* __restrict__ Kp, PtrList<cplx<R>> sp, int V,
                                                        cplx<R>* __restrict__ kc, const cplx<R>* __restrict__ keta,
                                                        int homog, int energy, double* partials, int* err) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  const int64_t nk = K.nk;
  const double dm = p.dt * p.cmobs[0];
  double fint = 0, elen = 0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    const double w = hweight(K, kx);
    double cr, ci, mr, mi;
    ld2(kc[id], cr, ci);
    ld2(sp.p[V][id], mr, mi);
    if (energy) {
      const double bb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
      double f = p.kappa_c * bb * (cr * cr + ci * ci);
      for (int v = 0; v < V; ++v) {
        double er, ei;
        ld2(keta[(int64_t)v * nk + id], er, ei);
        f += kkappak_b(p.grad_coeff[v], b) * (er * er + ei * ei);
      }
      fint += 0.5 * w * f;
    }
    if (homog) {
      double tr[MEU_MAX_VAR], ti[MEU_MAX_VAR];
      double sr[6] = {0, 0, 0, 0, 0, 0}, si[6] = {0, 0, 0, 0, 0, 0};
      for (int v = 0; v < V; ++v) {
        ld2(sp.p[v][id], tr[v], ti[v]);
#pragma unroll
        for (int m = 0; m < 6; ++m) { sr[m] += tr[v] * K.sig0[v][m]; si[m] += ti[v] * K.sig0[v][m]; }
      }
      double ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
      if (id != 0) {
        double Rr[3], Ri[3];
#pragma unroll
        for (int i = 1; i <= 3; ++i) {
          double t_r = 0, t_i = 0;
#pragma unroll
          for (int j = 1; j <= 3; ++j) { const int m = voigt(i, j) - 1; t_r += b[j - 1] * sr[m]; t_i += b[j - 1] * si[m]; }
          Rr[i - 1] = -t_i;
          Ri[i - 1] = t_r;
        }
        double Q[9];
        build_q(K, a, b, Q);
        set_err(err, invert3(Q, MEU_ERR_Q_SINGULAR));
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          ur[i] = Q[i] * Rr[0] + Q[i + 3] * Rr[1] + Q[i + 6] * Rr[2];
          ui[i] = Q[i] * Ri[0] + Q[i + 3] * Ri[1] + Q[i + 6] * Ri[2];
        }
      }
      // phi^_p = sig0_p : sym(i b (x) u^) = i (sig0_p b) . u^
      for (int v = 0; v < V; ++v) {
        double sb[3];
#pragma unroll
        for (int i = 1; i <= 3; ++i) {
          double t = 0;
#pragma unroll
          for (int j = 1; j <= 3; ++j) t += K.sig0[v][voigt(i, j) - 1] * b[j - 1];
          sb[i - 1] = t;
        }
        const double dr = sb[0] * ur[0] + sb[1] * ur[1] + sb[2] * ur[2];
        const double di = sb[0] * ui[0] + sb[1] * ui[1] + sb[2] * ui[2];
        sp.p[v][id] = mk((R)(-di), (R)dr);
      }
      if (energy) {
        // engineering elastic strain e = gamma(u^) - sum_q theta^_q eps0_q (+ e_mean at k = 0)
        const int I1[6] = {0, 1, 2, 1, 0, 0}, J1[6] = {0, 1, 2, 2, 2, 1};
        double er[6], ei[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          const int i = I1[m], j = J1[m];
          double gr, gi;
          if (m < 3) { gr = -b[i] * ui[i]; gi = b[i] * ur[i]; }
          else { gr = -(b[i] * ui[j] + b[j] * ui[i]); gi = b[i] * ur[j] + b[j] * ur[i]; }
          for (int v = 0; v < V; ++v) { gr -= tr[v] * K.eps_eng[v][m]; gi -= ti[v] * K.eps_eng[v][m]; }
          if (id == 0) gr += K.ebar_eng[m];
          er[m] = gr;
          ei[m] = gi;
        }
        double q = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          double cr2 = 0, ci2 = 0;
#pragma unroll
          for (int j = 0; j < 6; ++j) { cr2 += K.c0m[i + j * 6] * er[j]; ci2 += K.c0m[i + j * 6] * ei[j]; }
          q += er[i] * cr2 + ei[i] * ci2;
        }
        elen += 0.5 * w * q;
      }
    }
    // Cahn-Hilliard on the spectral state of the fluctuation
    const double k2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    double nr = 0.0, ni = 0.0;
    if (id != 0) {
      const double den = 1.0 + dm * p.kappa_c * k2 * k2;
      nr = (cr - dm * k2 * mr) / den;
      ni = (ci - dm * k2 * mi) / den;
    }
    const cplx<R> o = mk((R)nr, (R)ni);
    kc[id] = o;
    sp.p[V][id] = o;
  }
  block_reduce_store(fint, 0, partials + Q_FINT * PSTRIDE + blockIdx.x);
  if (homog) block_reduce_store(elen, 0, partials + Q_ELEN * PSTRIDE + blockIdx.x);
}

// Landau TDGL driving force g_v = df/deta_v + el_grad_v
// homog: el_grad_v = -theta'_v (sig0_v:e_mean + phi_v - sum_q A_vq theta_q); else el from elener.
template <typename R>
__global__ void __launch_bounds__(256) k_lan_b(const DevConst* __restrict__ Kp, const R* __restrict__ c,
                                               const R* __restrict__ eta, const R* __restrict__ el, int homog,
                                               R* __restrict__ w) {
  const DevConst& K = *Kp;
  const meu_params& p = K.p;
  const int64_t n3 = K.n3;
  const int V = p.nvar;
  const int hcp = p.eig_coupling == MEU_EIG_H;
  const double cbar = K.c_shift ? K.c_mean[0] : 0.0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
    const double cv = cbar + (double)c[id];
    double e[MEU_MAX_VAR], th[MEU_MAX_VAR], s2 = 0;
    for (int v = 0; v < V; ++v) {
      e[v] = (double)eta[v * n3 + id];
      const double e2 = e[v] * e[v];
      s2 += e2;
      th[v] = hcp ? e2 * e[v] * (6.0 * e2 - 15.0 * e[v] + 10.0) : e2;
    }
    for (int v = 0; v < V; ++v) {
      const double ev = e[v], e2 = ev * ev;
      double g = p.lan_b * (p.lan_c2 - cv) * ev - p.lan_c * e2 * ev + p.lan_d * e2 * e2 * ev +
                 4.0 * p.cross_w * ev * (s2 - e2);
      if (el) {
        if (homog) {
          const double tp = hcp ? 30.0 * e2 * (e2 - 2.0 * ev + 1.0) : 2.0 * ev;
          double s = K.sig0_ebar[v] + (double)el[v * n3 + id];
          for (int q = 0; q < V; ++q) s -= K.A[v][q] * th[q];
          g += -tp * s;
        } else {
          g += (double)el[v * n3 + id];
        }
      }
      w[v * n3 + id] = (R)g;
    }
  }
}

// ---------------------------------------------------- end-of-step reductions
// Multi_MEUMAPPS.f:1008-1043: clip phi (KKS), min/max C (initial 1.0 / 0.0),
// max phi (initial 0.0), solid fraction (sum of phi>0; Landau: sum eta^2), sum C.
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_stats(const DevConst* __restrict__ Kp, const R* __restrict__ c,
                                                       R* __restrict__ phi, int clip, double* partials) {
  const DevConst& K = *Kp;
  const int64_t n3 = K.n3;
  const int V = K.p.nvar, E = K.p.numel;
  double cmin = 1.0, cmax = 0.0, pmax = 0.0, solid = 0.0, cs[MEU_MAX_EL] = {0, 0, 0};
#pragma unroll 4
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n3; id += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int e = 0; e < MEU_MAX_EL; ++e) {
      if (e >= E) break;
      const double v = (K.c_shift ? K.c_mean[e] : 0.0) + (double)c[(int64_t)e * n3 + id];
      cmin = fmin(cmin, v);
      cmax = fmax(cmax, v);
      cs[e] += v;
    }
    for (int v = 0; v < V; ++v) {
      double f = (double)phi[v * n3 + id];
      if (clip) {
        if (f < 0.0) f = 0.0;
        if (f > 1.0) f = 1.0;
        phi[v * n3 + id] = (R)f;
        if (f > 0.0) solid += f;
      } else {
        solid += f * f;
      }
      pmax = fmax(pmax, f);
    }
  }
  block_reduce_store(cmin, 2, partials + Q_CMIN * PSTRIDE + blockIdx.x);
  block_reduce_store(cmax, 1, partials + Q_CMAX * PSTRIDE + blockIdx.x);
  block_reduce_store(pmax, 1, partials + Q_PHIMAX * PSTRIDE + blockIdx.x);
  block_reduce_store(solid, 0, partials + Q_SOLID * PSTRIDE + blockIdx.x);
  for (int e = 0; e < MEU_MAX_EL; ++e) block_reduce_store(cs[e], 0, partials + (Q_CSUM0 + e) * PSTRIDE + blockIdx.x);
}

}  // namespace meu
