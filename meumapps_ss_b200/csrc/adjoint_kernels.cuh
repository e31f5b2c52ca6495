// adjoint_kernels.cuh -- kernels of the adjoint step (see adjoint.cuh).
#pragma once
#include "adjoint.cuh"

namespace meu {
namespace adj {

using lf::NT;
constexpr int NTP = 512;
constexpr int PV = 0;

// g(k) = -(sig0 b)^T Omega (sig0 b) for one variant (same Q as the forward Green operator)
__device__ __forceinline__ double green_scalar(const LanFusedConst& F, const double av[3], const double b[3]) {
  const double* sg = F.sig0[0];
  const double t0 = sg[0] * b[0] + sg[5] * b[1] + sg[4] * b[2];
  const double t1 = sg[5] * b[0] + sg[1] * b[1] + sg[3] * b[2];
  const double t2 = sg[4] * b[0] + sg[3] * b[1] + sg[2] * b[2];
  const double Kv[6] = {av[0] * av[0], av[1] * av[1], av[2] * av[2], b[1] * b[2], b[0] * b[2], b[0] * b[1]};
  double Qs[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double acc = 0;
#pragma unroll
    for (int n = 0; n < 6; ++n) acc += F.qcoef[q][n] * Kv[n];
    Qs[q] = acc;
  }
  const double qa = Qs[0], qb = Qs[1], qc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
  const double i00 = qb * qc - qf * qf, i01 = qe * qf - qc * qd, i02 = qd * qf - qb * qe;
  const double i11 = qa * qc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
  const double det = qa * i00 + qd * i01 + qe * i02;
  const double quad = t0 * (i00 * t0 + i01 * t1 + i02 * t2) + t1 * (i01 * t0 + i11 * t1 + i12 * t2) +
                      t2 * (i02 * t0 + i12 * t1 + i22 * t2);
  return det != 0.0 ? -quad / det : 0.0;
}

// k.kappa_eta.k as in the forward eta update
__device__ __forceinline__ double kk_eta(const double* gv, const double av[3], const double b[3]) {
  return gv[0] * av[0] * av[0] + gv[4] * av[1] * av[1] + gv[8] * av[2] * av[2] + (gv[3] + gv[1]) * b[0] * b[1] +
         (gv[7] + gv[5]) * b[1] * b[2] + (gv[2] + gv[6]) * b[2] * b[0];
}

// ------------------------------------------------------------------ EA
template <typename R, int N>
__global__ void __launch_bounds__(NT) k_ad_ea(AdjArgs<R> a) {
  using C = cplx<R>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;  // [N][TM]
  C* tw = buf + N * TM;
  __shared__ LanFusedConst F;
  const int64_t m0 = (int64_t)blockIdx.x * TM;
  lf::tile_load<C, N, TM>(buf, TM, 0, a.from_seed ? a.lam_seed : a.M, NK, PL, m0, 1);
  for (int i = threadIdx.x; i < (int)(sizeof(LanFusedConst) / 8); i += NT) ((double*)&F)[i] = ((const double*)a.F)[i];
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  fz::cp_async_wait_all();
  __syncthreads();
  if (!a.from_seed) fz::dif<C, N, TM, 1, TM, NT, PV>(buf, tw);
  const double s = a.from_seed ? 1.0 : 1.0 / ((double)N * N * N);
  double X = 0, Y = 0, Z = 0;
  for (int i = threadIdx.x; i < N * TM; i += NT) {
    const int p = i / TM, c = i - p * TM;
    const int64_t m = m0 + c, id = p * PL + m;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
    double av[3], b[3];
    lf::kvec_n<N>(kx, ky, kz, av, b);
    const double wk = (kx == 0 || 2 * kx == N) ? 1.0 : 2.0;
    const bool k0 = (kx == 0 && ky == 0 && kz == 0);
    const double lr = (double)buf[i].x * s, li = (double)buf[i].y * s;
    const double kk = kk_eta(F.g[0], av, b);
    const double H = 1.0 / (1.0 + F.dtl * kk);
    const C e1 = a.eta_k1[id];
    X += wk * kk * H * (lr * (double)e1.x + li * (double)e1.y);
    if (!k0) {
      const double k2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
      const double P = 1.0 / (1.0 + F.dm * F.kappa_c * k2 * k2);
      const C n1 = a.nu[id], c1 = a.c_k1[id], c0 = a.c_k0[id], t0 = a.theta_k0[id];
      const double nr = (double)n1.x, ni = (double)n1.y;
      Y += wk * k2 * k2 * P * (nr * (double)c1.x + ni * (double)c1.y);
      const double mr = F.lan_a * (double)c0.x - 0.5 * F.lan_b * (double)t0.x;
      const double mi = F.lan_a * (double)c0.y - 0.5 * F.lan_b * (double)t0.y;
      Z += wk * P * k2 * (nr * mr + ni * mi);
    }
    buf[i] = mk((R)(H * lr), (R)(H * li));
  }
  __syncthreads();
  fz::dit<C, N, TM, 1, TM, NT, PV>(buf, tw);
  lf::tile_store<C, N, TM>(buf, TM, 0, a.M, NK, PL, m0, 1);
  block_reduce_store(X, 0, a.partials + AQ_X * PSTRIDE + blockIdx.x);
  block_reduce_store(Y, 0, a.partials + AQ_Y * PSTRIDE + blockIdx.x);
  block_reduce_store(Z, 0, a.partials + AQ_Z * PSTRIDE + blockIdx.x);
}

// ------------------------------------------------------------------ B
template <typename R, int N>
__global__ void __launch_bounds__(NTP) k_ad_b(AdjArgs<R> a) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x;
  constexpr int64_t PL = (int64_t)N * N;
  C* mp = a.M + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  const LanFusedConst& F = *a.F;
  const double dtl = F.dtl, cbar = F.cbar, s0 = F.sig0_ebar[0], A11 = F.A[0][0];
  double wg = 0, ea = 0;
  const int64_t off = z * PL;
  // pointwise adjoint between the x transform's inverse and forward stage 0
  P::template x_stage0<true>(buf, tws, [&](int y, int n0, int dn, C* x) {
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) {
      const int n = n0 + r * dn;
      const int64_t g = off + (int64_t)y * N + 2 * n;
      const C wv = x[r];
      const C ev = *(const C*)(a.eta + g), cv = *(const C*)(a.c + g), pv = *(const C*)(a.phi + g);
      const double w2[2] = {(double)wv.x, (double)wv.y}, e2v[2] = {(double)ev.x, (double)ev.y};
      const double c2v[2] = {cbar + (double)cv.x, cbar + (double)cv.y}, p2v[2] = {(double)pv.x, (double)pv.y};
      double ao[2], ho[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double e = e2v[h], e2 = e * e, cc = c2v[h], ph = p2v[h], w = w2[h];
        double G = F.lan_b * (F.lan_c2 - cc) * e - F.lan_c * e2 * e + F.lan_d * e2 * e2 * e;
        double dG = F.lan_b * (F.lan_c2 - cc) - 3.0 * F.lan_c * e2 + 5.0 * F.lan_d * e2 * e2;
        if (a.homog) {
          G += -2.0 * e * (s0 + ph - A11 * e2);
          dG += -2.0 * (s0 + ph) + 6.0 * A11 * e2;
          ea += -dtl * w * (-2.0 * e * (s0 + 2.0 * ph - 2.0 * A11 * e2));
        }
        wg += w * G;
        ao[h] = w * (1.0 - dtl * dG);
        ho[h] = dtl * e * w;
      }
      *(C*)(a.aw + g) = mk((R)ao[0], (R)ao[1]);
      x[r] = mk((R)ho[0], (R)ho[1]);
    }
  });
  P::forward_tail(buf, tws, mp);
  block_reduce_store(wg, 0, a.partials + AQ_WG * PSTRIDE + z);
  block_reduce_store(ea, 0, a.partials + AQ_EA * PSTRIDE + z);
}

// ------------------------------------------------------------------ C
template <typename R, int N>
__global__ void __launch_bounds__(NT) k_ad_c(AdjArgs<R> a) {
  using C = cplx<R>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tw = buf + N * TM;
  __shared__ LanFusedConst F;
  const int64_t m0 = (int64_t)blockIdx.x * TM;
  lf::tile_load<C, N, TM>(buf, TM, 0, a.M, NK, PL, m0, 1);
  for (int i = threadIdx.x; i < (int)(sizeof(LanFusedConst) / 8); i += NT) ((double*)&F)[i] = ((const double*)a.F)[i];
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  fz::cp_async_wait_all();
  __syncthreads();
  fz::dif<C, N, TM, 1, TM, NT, PV>(buf, tw);
  const double s = 1.0 / ((double)N * N * N);
  for (int i = threadIdx.x; i < N * TM; i += NT) {
    const int p = i / TM, c = i - p * TM;
    const int64_t m = m0 + c, id = p * PL + m;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
    double av[3], b[3];
    lf::kvec_n<N>(kx, ky, kz, av, b);
    const bool k0 = (kx == 0 && ky == 0 && kz == 0);
    const double hr = (double)buf[i].x * s, hi = (double)buf[i].y * s;
    const C n1 = a.nu[id];
    double rr = 0, ri = 0, nr = F.lan_b * hr, ni = F.lan_b * hi;
    if (!k0) {
      const double k2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
      const double P = 1.0 / (1.0 + F.dm * F.kappa_c * k2 * k2);
      const double P1 = P * (1.0 - F.dm * F.lan_a * k2), P2 = P * F.dm * k2 * 0.5 * F.lan_b;
      const double g = a.homog ? green_scalar(F, av, b) : 0.0;
      rr = 2.0 * g * hr + P2 * (double)n1.x;
      ri = 2.0 * g * hi + P2 * (double)n1.y;
      nr += P1 * (double)n1.x;
      ni += P1 * (double)n1.y;
    }
    a.nu[id] = mk((R)nr, (R)ni);
    buf[i] = mk((R)rr, (R)ri);
  }
  __syncthreads();
  fz::dit<C, N, TM, 1, TM, NT, PV>(buf, tw);
  lf::tile_store<C, N, TM>(buf, TM, 0, a.M, NK, PL, m0, 1);
}

// ------------------------------------------------------------------ D
template <typename R, int N>
__global__ void __launch_bounds__(NTP) k_ad_d(AdjArgs<R> a) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x;
  constexpr int64_t PL = (int64_t)N * N;
  C* mp = a.M + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  const int64_t off = z * PL;
  auto lam = [&](int y, int n0, int dn, C* x) {
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) {
      const int64_t g = off + (int64_t)y * N + 2 * (n0 + r * dn);
      const C rv = x[r];
      const C av = *(const C*)(a.aw + g), ev = *(const C*)(a.eta + g);
      x[r] = mk((R)((double)av.x + 2.0 * (double)ev.x * (double)rv.x),
                (R)((double)av.y + 2.0 * (double)ev.y * (double)rv.y));
    }
  };
  if (a.lam_out) {
    // lambda of the initial state: real space out, no forward transform
    P::template x_stage0<false>(buf, tws, [&](int y, int n0, int dn, C* x) {
      lam(y, n0, dn, x);
#pragma unroll
      for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r)
        *(C*)(a.lam_out + off + (int64_t)y * N + 2 * (n0 + r * dn)) = x[r];
    });
    return;
  }
  P::template x_stage0<true>(buf, tws, lam);
  P::forward_tail(buf, tws, mp);
}

// =================================================== V variants (V >= 2)
// Q^-1 of the forward Green operator (FP64), as the adjugate over the determinant
__device__ __forceinline__ void q_inverse(const LanFusedConst& F, const double av[3], const double b[3],
                                          double qi[6], bool& ok) {
  const double Kv[6] = {av[0] * av[0], av[1] * av[1], av[2] * av[2], b[1] * b[2], b[0] * b[2], b[0] * b[1]};
  double Qs[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double acc = 0;
#pragma unroll
    for (int n = 0; n < 6; ++n) acc += F.qcoef[q][n] * Kv[n];
    Qs[q] = acc;
  }
  const double qa = Qs[0], qb = Qs[1], qc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
  const double i00 = qb * qc - qf * qf, i01 = qe * qf - qc * qd, i02 = qd * qf - qb * qe;
  const double i11 = qa * qc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
  const double det = qa * i00 + qd * i01 + qe * i02;
  ok = det != 0.0;
  const double rd = ok ? 1.0 / det : 0.0;
  // symmetric: (00, 11, 22, 01, 02, 12)
  qi[0] = i00 * rd; qi[1] = i11 * rd; qi[2] = i22 * rd; qi[3] = i01 * rd; qi[4] = i02 * rd; qi[5] = i12 * rd;
}

// sig0_v b (Voigt 11,22,33,23,13,12)
__device__ __forceinline__ void sig_b(const double* sg, const double b[3], double t[3]) {
  t[0] = sg[0] * b[0] + sg[5] * b[1] + sg[4] * b[2];
  t[1] = sg[5] * b[0] + sg[1] * b[1] + sg[3] * b[2];
  t[2] = sg[4] * b[0] + sg[3] * b[1] + sg[2] * b[2];
}

// EA_v: z FFT of lam_{v,n+1} -> w^_v = H_v lam^_v (+ X, Y, Z sums) -> z iFFT, V fields
template <typename R, int N, int V>
__global__ void __launch_bounds__(NT) k_ad_ea_v(AdjArgs<R> a) {
  using C = cplx<R>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1, LN = V * TM;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;  // [N][V][TM]
  C* tw = buf + N * LN;
  __shared__ LanFusedConst F;
  const int64_t m0 = (int64_t)blockIdx.x * TM;
  lf::tile_load<C, N, TM>(buf, LN, 0, a.from_seed ? a.lam_seed : a.M, NK, PL, m0, V);
  for (int i = threadIdx.x; i < (int)(sizeof(LanFusedConst) / 8); i += NT) ((double*)&F)[i] = ((const double*)a.F)[i];
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  fz::cp_async_wait_all();
  __syncthreads();
  if (!a.from_seed) fz::dif<C, N, LN, 1, LN, NT, PV>(buf, tw);
  const double s = a.from_seed ? 1.0 : 1.0 / ((double)N * N * N);
  double X = 0, Y = 0, Z = 0;
  for (int i = threadIdx.x; i < N * TM; i += NT) {
    const int p = i / TM, c = i - p * TM;
    const int64_t m = m0 + c, id = p * PL + m;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
    double av[3], b[3];
    lf::kvec_n<N>(kx, ky, kz, av, b);
    const double wk = (kx == 0 || 2 * kx == N) ? 1.0 : 2.0;
    const bool k0 = (kx == 0 && ky == 0 && kz == 0);
    double tr = 0, ti = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      C* e = buf + p * LN + v * TM + c;
      const double lr = (double)e->x * s, li = (double)e->y * s;
      const double kk = kk_eta(F.g[v], av, b);
      const double H = 1.0 / (1.0 + F.dtl * kk);
      const C e1 = a.eta_k1[v * NK + id];
      X += wk * kk * H * (lr * (double)e1.x + li * (double)e1.y);
      *e = mk((R)(H * lr), (R)(H * li));
      const C t0 = a.theta_k0[v * NK + id];
      tr += (double)t0.x;
      ti += (double)t0.y;
    }
    if (!k0) {
      const double k2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
      const double P = 1.0 / (1.0 + F.dm * F.kappa_c * k2 * k2);
      const C n1 = a.nu[id], c1 = a.c_k1[id], c0 = a.c_k0[id];
      const double nr = (double)n1.x, ni = (double)n1.y;
      Y += wk * k2 * k2 * P * (nr * (double)c1.x + ni * (double)c1.y);
      const double mr = F.lan_a * (double)c0.x - 0.5 * F.lan_b * tr;
      const double mi = F.lan_a * (double)c0.y - 0.5 * F.lan_b * ti;
      Z += wk * P * k2 * (nr * mr + ni * mi);
    }
  }
  __syncthreads();
  fz::dit<C, N, LN, 1, LN, NT, PV>(buf, tw);
  lf::tile_store<C, N, TM>(buf, LN, 0, a.M, NK, PL, m0, V);
  block_reduce_store(X, 0, a.partials + AQ_X * PSTRIDE + blockIdx.x);
  block_reduce_store(Y, 0, a.partials + AQ_Y * PSTRIDE + blockIdx.x);
  block_reduce_store(Z, 0, a.partials + AQ_Z * PSTRIDE + blockIdx.x);
}

// B1_v: plane (z, v): xy iFFT of w^_v -> real w_v
template <typename R, int N>
__global__ void __launch_bounds__(NTP) k_ad_b1_v(AdjArgs<R> a) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x, v = blockIdx.y;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  __syncthreads();
  P::inverse_head(buf, tws, a.M + v * NK + z * (int64_t)N * P::NXH, a.err);
  R* dst = a.wv + v * N3 + z * PL;
  P::template x_stage0<false>(buf, tws, [&](int y, int n0, int dn, C* x) {
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) ((C*)(dst + (int64_t)y * N))[n0 + r * dn] = x[r];
  });
}

// B2_v: pointwise, every variant at a voxel: a_u, h_v, <w, G> and the d/d(alpha) sum
template <typename R, int V>
__global__ void __launch_bounds__(RED_THREADS) k_ad_b2_v(AdjArgs<R> a, int64_t n3) {
  __shared__ double Fa[V][V], s0[V];
  __shared__ double cst[9];
  if (threadIdx.x == 0) {
    const LanFusedConst& F = *a.F;
    for (int v = 0; v < V; ++v) {
      s0[v] = F.sig0_ebar[v];
      for (int q = 0; q < V; ++q) Fa[v][q] = F.A[v][q];
    }
    cst[0] = F.dtl; cst[1] = F.cbar; cst[2] = F.lan_b; cst[3] = F.lan_c2; cst[4] = F.lan_c; cst[5] = F.lan_d;
    cst[6] = F.cross_w;
  }
  __syncthreads();
  const double dtl = cst[0], cbar = cst[1], lb = cst[2], lc2 = cst[3], lc = cst[4], ld = cst[5], cw = cst[6];
  const bool homog = a.homog != 0;
  double wg = 0, ea = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
    double e[V], w[V], ph[V], Ae[V];
    double s2 = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      e[v] = (double)a.eta[v * n3 + i];
      w[v] = (double)a.wv[v * n3 + i];
      ph[v] = (double)a.phi[v * n3 + i];
      s2 += e[v] * e[v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double acc = 0;
#pragma unroll
      for (int q = 0; q < V; ++q) acc += Fa[v][q] * e[q] * e[q];
      Ae[v] = acc;  // sum_q A_vq eta_q^2
    }
    const double cc = cbar + (double)a.c[i];
    double z[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double ev = e[v], e2 = ev * ev;
      double G = lb * (lc2 - cc) * ev - lc * e2 * ev + ld * e2 * e2 * ev + 4.0 * cw * ev * (s2 - e2);
      if (homog) G += -2.0 * ev * (s0[v] + ph[v] - Ae[v]);
      wg += w[v] * G;
      z[v] = -dtl * w[v];
      if (homog) ea += z[v] * (-2.0 * ev * (s0[v] + 2.0 * ph[v] - 2.0 * Ae[v]));
    }
#pragma unroll
    for (int u = 0; u < V; ++u) {
      double au = w[u];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        double d;
        if (u == v) {
          const double e2 = e[v] * e[v];
          d = lb * (lc2 - cc) - 3.0 * lc * e2 + 5.0 * ld * e2 * e2 + 4.0 * cw * (s2 - e2);
          if (homog) d += -2.0 * (s0[v] + ph[v] - Ae[v]) + 4.0 * Fa[v][v] * e2;
        } else {
          d = 8.0 * cw * e[v] * e[u];
          if (homog) d += 4.0 * Fa[v][u] * e[v] * e[u];
        }
        au += z[v] * d;
      }
      a.aw[u * n3 + i] = (R)au;
      a.hv[u * n3 + i] = (R)(-e[u] * z[u]);
    }
  }
  block_reduce_store(wg, 0, a.partials + AQ_WG * PSTRIDE + blockIdx.x);
  block_reduce_store(ea, 0, a.partials + AQ_EA * PSTRIDE + blockIdx.x);
}

// B3_v: plane (z, v): xy FFT of the real h_v -> M-form field v
template <typename R, int N>
__global__ void __launch_bounds__(NTP) k_ad_b3_v(AdjArgs<R> a) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x, v = blockIdx.y;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  P::load_real(buf, a.hv + v * N3 + z * PL);
  P::load_tw(tws, a.twx, a.twy, a.post);
  fz::cp_async_wait_all();
  __syncthreads();
  P::x_forward0(buf, tws, [](int, int, int, C*) {});
  P::forward_tail(buf, tws, a.M + v * NK + z * (int64_t)N * P::NXH);
}

// C_v: z FFT of h^_v -> nu^ update (B sum_v h^_v), r^_q -> z iFFT, V fields
template <typename R, int N, int V>
__global__ void __launch_bounds__(NT) k_ad_c_v(AdjArgs<R> a) {
  using C = cplx<R>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1, LN = V * TM;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tw = buf + N * LN;
  __shared__ LanFusedConst F;
  const int64_t m0 = (int64_t)blockIdx.x * TM;
  lf::tile_load<C, N, TM>(buf, LN, 0, a.M, NK, PL, m0, V);
  for (int i = threadIdx.x; i < (int)(sizeof(LanFusedConst) / 8); i += NT) ((double*)&F)[i] = ((const double*)a.F)[i];
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  fz::cp_async_wait_all();
  __syncthreads();
  fz::dif<C, N, LN, 1, LN, NT, PV>(buf, tw);
  const double s = 1.0 / ((double)N * N * N);
  for (int i = threadIdx.x; i < N * TM; i += NT) {
    const int p = i / TM, c = i - p * TM;
    const int64_t m = m0 + c, id = p * PL + m;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
    double av[3], b[3];
    lf::kvec_n<N>(kx, ky, kz, av, b);
    const bool k0 = (kx == 0 && ky == 0 && kz == 0);
    double hr[V], hi[V], shr = 0, shi = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const C h = buf[p * LN + v * TM + c];
      hr[v] = (double)h.x * s;
      hi[v] = (double)h.y * s;
      shr += hr[v];
      shi += hi[v];
    }
    const C n1 = a.nu[id];
    double nr = F.lan_b * shr, ni = F.lan_b * shi;
    double rr[V], ri[V];
#pragma unroll
    for (int v = 0; v < V; ++v) rr[v] = ri[v] = 0;
    if (!k0) {
      const double k2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
      const double P = 1.0 / (1.0 + F.dm * F.kappa_c * k2 * k2);
      const double P1 = P * (1.0 - F.dm * F.lan_a * k2), P2 = P * F.dm * k2 * 0.5 * F.lan_b;
      double ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
      if (a.homog) {
        double qi[6];
        bool ok;
        q_inverse(F, av, b, qi, ok);
        double Sr[3] = {0, 0, 0}, Si[3] = {0, 0, 0};
#pragma unroll
        for (int v = 0; v < V; ++v) {
          double t[3];
          sig_b(F.sig0[v], b, t);
#pragma unroll
          for (int d = 0; d < 3; ++d) { Sr[d] += t[d] * hr[v]; Si[d] += t[d] * hi[v]; }
        }
        // u = Q^-1 S
        ur[0] = qi[0] * Sr[0] + qi[3] * Sr[1] + qi[4] * Sr[2];
        ur[1] = qi[3] * Sr[0] + qi[1] * Sr[1] + qi[5] * Sr[2];
        ur[2] = qi[4] * Sr[0] + qi[5] * Sr[1] + qi[2] * Sr[2];
        ui[0] = qi[0] * Si[0] + qi[3] * Si[1] + qi[4] * Si[2];
        ui[1] = qi[3] * Si[0] + qi[1] * Si[1] + qi[5] * Si[2];
        ui[2] = qi[4] * Si[0] + qi[5] * Si[1] + qi[2] * Si[2];
      }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        double t[3];
        sig_b(F.sig0[q], b, t);
        rr[q] = -2.0 * (t[0] * ur[0] + t[1] * ur[1] + t[2] * ur[2]) + P2 * (double)n1.x;
        ri[q] = -2.0 * (t[0] * ui[0] + t[1] * ui[1] + t[2] * ui[2]) + P2 * (double)n1.y;
      }
      nr += P1 * (double)n1.x;
      ni += P1 * (double)n1.y;
    }
    a.nu[id] = mk((R)nr, (R)ni);
#pragma unroll
    for (int q = 0; q < V; ++q) buf[p * LN + q * TM + c] = mk((R)rr[q], (R)ri[q]);
  }
  __syncthreads();
  fz::dit<C, N, LN, 1, LN, NT, PV>(buf, tw);
  lf::tile_store<C, N, TM>(buf, LN, 0, a.M, NK, PL, m0, V);
}

// D_v: plane (z, q): xy iFFT of r_q -> lam_q = a_q + 2 eta_q r_q -> xy FFT (or lam_0 out)
template <typename R, int N>
__global__ void __launch_bounds__(NTP) k_ad_d_v(AdjArgs<R> a) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x, q = blockIdx.y;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  C* mp = a.M + q * NK + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  const int64_t off = q * N3 + z * PL;
  auto lam = [&](int y, int n0, int dn, C* x) {
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) {
      const int64_t g = off + (int64_t)y * N + 2 * (n0 + r * dn);
      const C rv = x[r];
      const C av = *(const C*)(a.aw + g), ev = *(const C*)(a.eta + g);
      x[r] = mk((R)((double)av.x + 2.0 * (double)ev.x * (double)rv.x),
                (R)((double)av.y + 2.0 * (double)ev.y * (double)rv.y));
    }
  };
  if (a.lam_out) {
    P::template x_stage0<false>(buf, tws, [&](int y, int n0, int dn, C* x) {
      lam(y, n0, dn, x);
#pragma unroll
      for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r)
        *(C*)(a.lam_out + off + (int64_t)y * N + 2 * (n0 + r * dn)) = x[r];
    });
    return;
  }
  P::template x_stage0<true>(buf, tws, lam);
  P::forward_tail(buf, tws, mp);
}

}  // namespace adj
}  // namespace meu
