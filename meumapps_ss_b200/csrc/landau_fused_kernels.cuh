// landau_fused_kernels.cuh -- kernels of the fused Landau step (see
// landau_fused.cuh for the data flow) and their launch sequence for one (R, N).
// Included by the per-(R, N) translation units lf_inst_*.cu, which instantiate
// every (V, schedule) for their grid size.
//
// Every kernel serves a batch of members: blockIdx.z selects the member's
// argument record.
#pragma once
#include <type_traits>
#include <utility>
#include <vector>

#include "landau_fused.cuh"

namespace meu {
namespace lf {

constexpr int NT = 256;   // column kernels
constexpr double TWO_PI = 6.283185307179586476925286766559;

template <int N>
__device__ __forceinline__ void kvec_n(int kx, int ky, int kz, double a[3], double b[3]) {
  const int m[3] = {kx, ky, kz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int mm = (m[d] <= N / 2) ? m[d] : m[d] - N;
    a[d] = (double)mm * (TWO_PI / (double)N);
    b[d] = (2 * m[d] == N) ? 0.0 : a[d];
  }
}

// the same k-vectors in the working precision W of the step (float for FP32 fields)
template <int N, typename W>
__device__ __forceinline__ void kvec_w(int kx, int ky, int kz, W a[3], W b[3]) {
  const int m[3] = {kx, ky, kz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int mm = (m[d] <= N / 2) ? m[d] : m[d] - N;
    a[d] = (W)mm * (W)(TWO_PI / (double)N);
    b[d] = (2 * m[d] == N) ? (W)0 : a[d];
  }
}

// x * r for a per-step damping factor r computed in FP64.  The factor multiplies
// the state every step, so in FP32 it is applied as r_hi + r_lo (a rounded
// factor would bias every mode the same way each step and the bias would compound).
template <typename W>
struct Damp {
  W hi, lo;
  __device__ __forceinline__ explicit Damp(double r) : hi((W)r), lo((W)(r - (double)(W)r)) {}
  __device__ __forceinline__ W operator()(W x) const { return x * hi + x * lo; }
};

// 1/x for x >= 1 in FP64: a single-precision estimate refined by two Newton-Raphson
// steps r <- r + r (1 - x r), each of which squares the relative error (2^-22 ->
// 2^-44 -> below FP64 rounding).  Used for the semi-implicit factors 1/(1 + ...).
__device__ __forceinline__ double recip_ge1(double x) {
  double r = (double)__fdividef(1.0f, (float)x);
  r = fma(r, fma(-x, r, 1.0), r);
  r = fma(r, fma(-x, r, 1.0), r);
  return r;
}

// 1/x in FP64 for any x whose reciprocal is a normal single: a single-precision
// estimate and two Newton-Raphson steps (relative error 2^-22 -> 2^-44 -> FP64
// rounding); other x take the FP64 division.
__device__ __forceinline__ double recip_nr(double x) {
  double r = (double)__fdividef(1.0f, (float)x);
  if (!(fabs(r) < 1.0e37 && fabs(r) > 1.0e-37)) return 1.0 / x;
  r = fma(r, fma(-x, r, 1.0), r);
  r = fma(r, fma(-x, r, 1.0), r);
  return r;
}

// one component of the k-vector a (m wrapped into (-N/2, N/2]); b = a except at Nyquist
template <int N>
__device__ __forceinline__ double kcomp(int m) {
  return (double)((m <= N / 2) ? m : m - N) * (TWO_PI / (double)N);
}

template <typename R> constexpr int col_tile_default() { return sizeof(R) == 4 ? 16 : 8; }

// Programmatic dependent launch of the four per-step kernels (Z1, PB, Z2, PI): each is
// launched while its predecessor in the stream still runs, so its blocks take the slots
// the predecessor's last wave leaves free and load their constants and twiddles there.
// step_dep_wait() blocks until the predecessor grid has completed and its writes are
// visible; nothing the predecessor writes is read before it.  step_dep_release() comes
// after the wait, so a successor's blocks start only once this grid's predecessor has
// completed: a prologue overlaps one kernel at most (the one right before it).  A kernel
// launched without the attribute passes both at once.
__device__ __forceinline__ void step_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void step_dep_release() { asm volatile("griddepcontrol.launch_dependents;\n"); }

// Column tile of nf fields: smem [z][slot][TM] with LN complex per z row, global
// M-form (or state) field f at G + f*NK, row z at + z*PL, columns m0 .. m0+TM.
// tile_load only issues cp.async copies; the caller waits.
template <typename C, int N, int TM>
__device__ __forceinline__ void tile_load(C* buf, int LN, int slot0, const C* G, int64_t NK, int64_t PL, int64_t m0,
                                          int nf) {
  constexpr int PER = 16 / sizeof(C);
  const int per_row = nf * TM / PER;
  for (int i = threadIdx.x; i < N * per_row; i += NT) {
    const int zz = i / per_row, r = (i - zz * per_row) * PER, f = r / TM, c = r - f * TM;
    fz::cp_async16(buf + zz * LN + (slot0 + f) * TM + c, G + f * NK + zz * PL + m0 + c);
  }
}
template <typename C, int N, int TM>
__device__ __forceinline__ void tile_store(const C* buf, int LN, int slot0, C* G, int64_t NK, int64_t PL, int64_t m0,
                                           int nf) {
  constexpr int PER = 16 / sizeof(C);
  const int per_row = nf * TM / PER;
  for (int i = threadIdx.x; i < N * per_row; i += NT) {
    const int zz = i / per_row, r = (i - zz * per_row) * PER, f = r / TM, c = r - f * TM;
    *(float4*)(G + f * NK + zz * PL + m0 + c) = *(const float4*)(buf + zz * LN + (slot0 + f) * TM + c);
  }
}

// ------------------------------------------------------------------ PF
// raw = 0: fields theta_v (f < V).
// raw = 1: fields eta_v (f < V) and dc (f == V), for the spectral state.
template <typename R, int N, int PV, int NTP>
__global__ void __launch_bounds__(NTP) k_lf_pf(const LanFusedArgs<R>* __restrict__ A, int V, int raw) {
  using P = fz::Plane<R, N, NTP, PV>;
  const LanFusedArgs<R> a = A[blockIdx.z];
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  const int z = blockIdx.x, f = blockIdx.y;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  const R* ez = a.eta + z * PL;
  const R* cz = a.c + z * PL;
  P::load_real(buf, f < V ? ez + f * N3 : cz);
  P::load_tw(tws, a.twx, a.twy, a.post);
  fz::cp_async_wait_all();
  __syncthreads();
  // theta_v = eta_v^2 (raw: the fields themselves), then the same forward path as
  // PI's theta transform, so a step after new fields sees bit-identical theta^
  const bool square = f < V && !raw;
  P::x_forward0(buf, tws, [&](int, int, int, C* x) {
    if (square) {
#pragma unroll
      for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r)
        x[r] = mk((R)((double)x[r].x * (double)x[r].x), (R)((double)x[r].y * (double)x[r].y));
    }
  });
  P::forward_tail(buf, tws, a.M + f * NK + z * (int64_t)N * P::NXH);
}

// ------------------------------------------------------------------ Z0
// set-up: z FFT of eta_v (f < V) and dc (f == V) into the spectral state
template <typename R, int N, int V, int PV, int TM>
__global__ void __launch_bounds__(NT) k_lf_z0(const LanFusedArgs<R>* __restrict__ A) {
  using C = cplx<R>;
  const LanFusedArgs<R> a = A[blockIdx.z];
  constexpr int NF = V + 1, NXH = N / 2 + 1, LN = NF * TM;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tw = buf + N * LN;
  const int64_t m0 = (int64_t)blockIdx.x * TM;
  tile_load<C, N, TM>(buf, LN, 0, a.M, NK, PL, m0, NF);
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  fz::cp_async_wait_all();
  __syncthreads();
  fz::dif<C, N, LN, 1, LN, NT, PV>(buf, tw);
  const double s = 1.0 / ((double)N * N * N);
  for (int i = threadIdx.x; i < N * LN; i += NT) {
    const int p = i / LN, r = i - p * LN, f = r / TM, c = r - f * TM;
    const C v = buf[i];
    C o = mk((R)((double)v.x * s), (R)((double)v.y * s));
    if (f == V && p == 0 && m0 + c == 0) o = mk((R)0, (R)0);  // dc has no k = 0 mode
    C* dst = (f < V) ? a.Keta + f * NK : a.Kc;
    dst[p * PL + m0 + c] = o;
  }
}

// Z1's tile row stride: NF*TM complex padded so that (stride * words) mod 32 = 16, i.e.
// consecutive rows start half the 32 banks apart
template <typename R, int N, int V, int TM>
constexpr int z1_row_stride() {
  constexpr int W = 2 * (int)sizeof(R) / 4, LN = (V + 1) * TM;
  int ls = LN;
  while ((ls * W) % 32 != 16) ++ls;
  return ls;
}

// a shared-memory load the compiler keeps in place (it is not moved across barriers)
template <typename T>
__device__ __forceinline__ T lds(const T* p);
template <>
__device__ __forceinline__ float lds<float>(const float* p) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
  return v;
}
template <>
__device__ __forceinline__ double lds<double>(const double* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];\n" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
  return v;
}

// With one variant, Z1 stages its tile of the Green-operator table and of the dc^ state
// in shared memory (cp.async, issued before it waits for its predecessor) when both fit
// beside the transform tile within a third of the SM's shared memory (three blocks per SM)
template <typename R, int N, int V, int TM>
constexpr size_t z1_smem_base() {
  return sizeof(cplx<R>) * ((size_t)N * z1_row_stride<R, N, V, TM>() + N * Tw<cplx<R>>::K);
}
template <typename R, int N, int V, int TM>
constexpr size_t z1_smem_stage() {
  return sizeof(R) * (size_t)(V * (V + 1) / 2) * N * TM + sizeof(cplx<R>) * (size_t)N * TM;
}
template <typename R, int N, int V, int TM>
constexpr bool z1_prefetch() {
  return V == 1 && z1_smem_base<R, N, V, TM>() + z1_smem_stage<R, N, V, TM>() <= 74 * 1024;
}

// ------------------------------------------------------------------ QCHECK
// Q(k) of every k (natural order) against the reference's rcond <= 1e-16 stop
// (ModFunc.f:55-67 via ModElastic.f:187), on the exact 1-norm condition number from
// the adjugate: ||Q|| ||adj Q|| >= 1e16 |det Q| sets MEU_ERR_Q_SINGULAR.  Q(k) does not
// change in time, so the step tests it once (its first step) and Z1 only inverts.
template <typename R, int N>
__global__ void __launch_bounds__(256) k_lf_qcheck(const LanFusedArgs<R>* __restrict__ A) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  const LanFusedConst& F = *a.F;
  if (F.elastic_on == 0.0) return;
  constexpr int NXH = N / 2 + 1;
  constexpr int64_t NKK = (int64_t)N * N * NXH;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < NKK; id += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(id % NXH), ky = (int)((id / NXH) % N), kz = (int)(id / ((int64_t)NXH * N));
    if (kx == 0 && ky == 0 && kz == 0) continue;
    double ad[3], bd[3];
    kvec_n<N>(kx, ky, kz, ad, bd);
    const double Kv[6] = {ad[0] * ad[0], ad[1] * ad[1], ad[2] * ad[2], bd[1] * bd[2], bd[0] * bd[2], bd[0] * bd[1]};
    double Qs[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double acc = 0;
#pragma unroll
      for (int n = 0; n < 6; ++n) acc += F.qcoef[q][n] * Kv[n];
      Qs[q] = acc;
    }
    const double qa = Qs[0], qb = Qs[1], qcc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
    const double i00 = qb * qcc - qf * qf, i01 = qe * qf - qcc * qd, i02 = qd * qf - qb * qe;
    const double i11 = qa * qcc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
    const double det = qa * i00 + qd * i01 + qe * i02;
    const double qn = fmax(fabs(qa) + fabs(qd) + fabs(qe), fmax(fabs(qd) + fabs(qb) + fabs(qf), fabs(qe) + fabs(qf) + fabs(qcc)));
    const double an = fmax(fabs(i00) + fabs(i01) + fabs(i02), fmax(fabs(i01) + fabs(i11) + fabs(i12), fabs(i02) + fabs(i12) + fabs(i22)));
    if (!(qn * an < 1e16 * fabs(det))) atomicMax(a.err, (int)MEU_ERR_Q_SINGULAR);
  }
}

// ------------------------------------------------------------------ GTAB
// The Green operator of homogeneous elasticity as a table, built once per upload in FP64
// and stored in the field precision (used by the one-variant step).  With u^ = Omega(k) R, R = i sum_u theta^_u s_u,
// s_v = sig0_v b and phi^_v = i s_v . u^, the elastic potential is
//   phi^_v = sum_u T_vu theta^_u,   T_vu = -s_v . Omega(k) s_u   (real, symmetric),
// Omega = Q(k)^-1.  Entry (v <= u) in pair order q goes to gtab[q * NK + p * PL + m],
// the layout of the dc^ state (p: z row in the column kernels' digit-reversed order,
// m: spectral column), so Z1 reads it beside dc^.  Q(k) and the moduli do not change in
// time; k = 0 is left zero (Z1 does not read it).  Singular Q(k) is k_lf_qcheck's error.
template <typename R, int N, int V, int PV>
__global__ void __launch_bounds__(256) k_lf_gtab(const LanFusedArgs<R>* __restrict__ A) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  if (a.gtab == nullptr) return;
  const LanFusedConst& F = *a.F;
  constexpr int NXH = N / 2 + 1;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < NK; id += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(id / PL);
    const int64_t m = id - (int64_t)p * PL;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
    double T[V][V];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int u = 0; u < V; ++u) T[v][u] = 0.0;
    if (kx != 0 || ky != 0 || kz != 0) {
      double ad[3], bd[3];
      kvec_n<N>(kx, ky, kz, ad, bd);
      const double Kv[6] = {ad[0] * ad[0], ad[1] * ad[1], ad[2] * ad[2], bd[1] * bd[2], bd[0] * bd[2], bd[0] * bd[1]};
      double Qs[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        double acc = 0;
#pragma unroll
        for (int n = 0; n < 6; ++n) acc += F.qcoef[q][n] * Kv[n];
        Qs[q] = acc;
      }
      const double qa = Qs[0], qb = Qs[1], qcc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
      const double i00 = qb * qcc - qf * qf, i01 = qe * qf - qcc * qd, i02 = qd * qf - qb * qe;
      const double i11 = qa * qcc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
      const double det = qa * i00 + qd * i01 + qe * i02;
      const double Om[3][3] = {{i00 / det, i01 / det, i02 / det},
                               {i01 / det, i11 / det, i12 / det},
                               {i02 / det, i12 / det, i22 / det}};
      double sb[V][3];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double* sg = F.sig0[v];
        sb[v][0] = sg[0] * bd[0] + sg[5] * bd[1] + sg[4] * bd[2];
        sb[v][1] = sg[5] * bd[0] + sg[1] * bd[1] + sg[3] * bd[2];
        sb[v][2] = sg[4] * bd[0] + sg[3] * bd[1] + sg[2] * bd[2];
      }
#pragma unroll
      for (int u = 0; u < V; ++u) {
        double w[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) w[r] = Om[r][0] * sb[u][0] + Om[r][1] * sb[u][1] + Om[r][2] * sb[u][2];
#pragma unroll
        for (int v = 0; v < V; ++v) T[v][u] = -(sb[v][0] * w[0] + sb[v][1] * w[1] + sb[v][2] * w[2]);
      }
    }
    int q = 0;
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int u = v; u < V; ++u) {
        // symmetric to rounding; the pair's mean keeps T_vu = T_uv exactly
        a.gtab[q * NK + id] = (R)(0.5 * (T[v][u] + T[u][v]));
        ++q;
      }
  }
}

// Elastic energy density 0.5 e*.C0.e (without the w factor) of one k on a Nyquist plane
// or at k = 0, where the quadratic form in theta^ does not hold: u^ = Omega(k) R with
// R_i = i sum_j b_j S_ij, S = sum_v theta^_v sig0_v (Voigt 11,22,33,23,13,12), then the
// engineering strain e = gamma(u^) - sum_v theta^_v eps0_v (+ e_mean at k = 0).
template <typename W, int V>
__device__ __forceinline__ W nyq_strain_energy(const W* tr, const W* ti, const W* b, const double* ad, const double* bd,
                                            bool k0, bool green, const W (*sgW)[6], const W (*epW)[6], const W* c0W,
                                            const W* ebW, const double (*qc)[6]) {
  W ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
  if (green) {
    W Sr[6] = {0, 0, 0, 0, 0, 0}, Si[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int q = 0; q < 6; ++q) { Sr[q] += tr[v] * sgW[v][q]; Si[q] += ti[v] * sgW[v][q]; }
    const W t1r = b[0] * Sr[0] + b[1] * Sr[5] + b[2] * Sr[4], t1i = b[0] * Si[0] + b[1] * Si[5] + b[2] * Si[4];
    const W t2r = b[0] * Sr[5] + b[1] * Sr[1] + b[2] * Sr[3], t2i = b[0] * Si[5] + b[1] * Si[1] + b[2] * Si[3];
    const W t3r = b[0] * Sr[4] + b[1] * Sr[3] + b[2] * Sr[2], t3i = b[0] * Si[4] + b[1] * Si[3] + b[2] * Si[2];
    const W Rr[3] = {-t1i, -t2i, -t3i}, Ri[3] = {t1r, t2r, t3r};
    const double Kv[6] = {ad[0] * ad[0], ad[1] * ad[1], ad[2] * ad[2], bd[1] * bd[2], bd[0] * bd[2], bd[0] * bd[1]};
    double Qs[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double acc = 0;
#pragma unroll
      for (int n = 0; n < 6; ++n) acc += qc[q][n] * Kv[n];
      Qs[q] = acc;
    }
    const double qa = Qs[0], qb = Qs[1], qcc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
    const double i00 = qb * qcc - qf * qf, i01 = qe * qf - qcc * qd, i02 = qd * qf - qb * qe;
    const double i11 = qa * qcc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
    const double rd = 1.0 / (qa * i00 + qd * i01 + qe * i02);
    const W Qi[3][3] = {{(W)(i00 * rd), (W)(i01 * rd), (W)(i02 * rd)},
                        {(W)(i01 * rd), (W)(i11 * rd), (W)(i12 * rd)},
                        {(W)(i02 * rd), (W)(i12 * rd), (W)(i22 * rd)}};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      ur[r] = Qi[r][0] * Rr[0] + Qi[r][1] * Rr[1] + Qi[r][2] * Rr[2];
      ui[r] = Qi[r][0] * Ri[0] + Qi[r][1] * Ri[1] + Qi[r][2] * Ri[2];
    }
  }
  // engineering elastic strain e = gamma(u^) - sum_v theta^_v eps0_v (+ e_mean at k = 0)
  const int I1[6] = {0, 1, 2, 1, 0, 0}, J1[6] = {0, 1, 2, 2, 2, 1};
  W er[6], ei[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int ii = I1[q], jj = J1[q];
    W gr, gi;
    if (q < 3) { gr = -b[ii] * ui[ii]; gi = b[ii] * ur[ii]; }
    else { gr = -(b[ii] * ui[jj] + b[jj] * ui[ii]); gi = b[ii] * ur[jj] + b[jj] * ur[ii]; }
#pragma unroll
    for (int v = 0; v < V; ++v) { gr -= tr[v] * epW[v][q]; gi -= ti[v] * epW[v][q]; }
    if (k0) gr += ebW[q];
    er[q] = gr;
    ei[q] = gi;
  }
  W qq = 0;
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    W cr2 = 0, ci2 = 0;
#pragma unroll
    for (int j = 0; j < 6; ++j) { cr2 += c0W[r + j * 6] * er[j]; ci2 += c0W[r + j * 6] * ei[j]; }
    qq += er[r] * cr2 + ei[r] * ci2;
  }
  return qq;
}

// ------------------------------------------------------------------ Z1
// z FFT of theta^_v (the first DIF stage straight from global memory), Green
// operator and Cahn-Hilliard update of the dc^ state (read and written in global
// memory by the k-space pass), z iFFT of phi^_v and dc^ (the last DIT stage
// straight to global memory).
// resident Z1 blocks per SM it is compiled for: as many as its shared memory allows
// (dynamic tile, 2 KB for its static arrays, 1 KB the runtime reserves per block), at
// most 3 (80 registers a thread).  A bound above what fits would cap the registers for
// nothing (FP64, 3 variants: 2 blocks fit, and a 3-block bound spilled 480 bytes)
template <typename R, int N, int V, int TM>
constexpr int z1_min_blocks() {
  constexpr size_t bytes = z1_smem_base<R, N, V, TM>() + (z1_prefetch<R, N, V, TM>() ? z1_smem_stage<R, N, V, TM>() : 0);
  constexpr int by_smem = (int)((228 * 1024) / (bytes + 1024 + 2048));
  return by_smem < 1 ? 1 : (by_smem < 3 ? by_smem : 3);
}

// Z1 of column tile bx of one member (the kernel's body; the persistent ensemble kernel
// runs it as one of its work items)
template <typename R, int N, int V, int PV, int TM>
__device__ __forceinline__ void lf_z1_body(const LanFusedArgs<R>& a, const int bx) {
  using C = cplx<R>;
  constexpr int NF = V + 1, NXH = N / 2 + 1, LN = NF * TM, LV = V * TM;
  // row stride of the tile: LN padded so that consecutive rows start half the banks apart
  // (the k-space pass reads TM columns of several rows per warp)
  constexpr int LS = z1_row_stride<R, N, V, TM>();
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  constexpr int NS = fz::rplan(N, PV).ns;
  static_assert(NS >= 2, "the column kernels need a radix plan of two stages or more");
  using S0 = fz::StageOf<N, 0, PV>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;  // [N][LS >= NF*TM]: theta^_v in slots 0..V-1, dc^ in slot V
  C* tw = buf + N * LS;
  // FP64 only for Omega(k) = Q^-1; every other k-space product in the field precision W
  using W = R;
  __shared__ double qc[6][6];
  __shared__ W sgW[V][6], epW[V][6], c0W[36], ebW[6], aW[V][V];
  const int64_t m0 = (int64_t)bx * TM;
  {
    const LanFusedConst& G = *a.F;
    for (int i = threadIdx.x; i < 36; i += NT) {
      qc[i / 6][i % 6] = G.qcoef[i / 6][i % 6];
      c0W[i] = (W)G.c0m[i];
    }
    for (int i = threadIdx.x; i < V * 6; i += NT) {
      sgW[i / 6][i % 6] = (W)G.sig0[i / 6][i % 6];
      epW[i / 6][i % 6] = (W)G.eps_eng[i / 6][i % 6];
    }
    for (int i = threadIdx.x; i < V * V; i += NT) aW[i / V][i % V] = (W)G.A[i / V][i % V];
    if (threadIdx.x < 6) ebW[threadIdx.x] = (W)G.ebar_eng[threadIdx.x];
  }
  const double kapcd = a.F->kappa_c, dmd = a.F->dm;
  const bool qcub = a.F->q_cubic != 0.0;
  const double q_own = a.F->q_own, q_other = a.F->q_other, q_off = a.F->q_off;
  const W kapc = (W)kapcd, lan_a = (W)a.F->lan_a, hlb = (W)(0.5 * a.F->lan_b);
  // staged tiles: table [q][z][TM] and dc^ state [z][TM].  Neither is written by the
  // kernels this launch may overlap: the table only at upload, dc^ by the previous Z1,
  // which has completed once this block runs (the predecessor released it after its wait)
  // one variant: the Green operator from the table (one real per k); more variants:
  // Omega(k) per k in FP64 (the table's V(V+1)/2 reals per k cost more than the solve)
  constexpr bool TAB = V == 1;
  constexpr bool PRE = TAB && z1_prefetch<R, N, V, TM>();
  constexpr int NQ = V * (V + 1) / 2;
  R* gts = (R*)(tw + N * Tw<C>::K);
  C* kcs = (C*)(gts + NQ * N * TM);
  if constexpr (PRE) {
    constexpr int PR = 16 / sizeof(R), PC = 16 / sizeof(C);
    if (a.homog) {
      for (int i = threadIdx.x; i < NQ * N * (TM / PR); i += NT) {
        const int row = i / (TM / PR), c = (i - row * (TM / PR)) * PR, q = row / N, z = row - q * N;
        fz::cp_async16(gts + (q * N + z) * TM + c, a.gtab + q * NK + z * PL + m0 + c);
      }
    }
    for (int i = threadIdx.x; i < N * (TM / PC); i += NT) {
      const int z = i / (TM / PC), c = (i - z * (TM / PC)) * PC;
      fz::cp_async16(kcs + z * TM + c, a.Kc + z * PL + m0 + c);
    }
    fz::cp_async_commit();
  }
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  step_dep_wait();
  step_dep_release();
  __syncthreads();
#pragma unroll 1
  for (int t = threadIdx.x; t < LV * S0::M; t += NT) {
    const int line = t % LV, j = t / LV, f = line / TM, c = line - f * TM;
    const C* src = a.M + f * NK + m0 + c;
    C x[S0::R];
#pragma unroll
    for (int r = 0; r < S0::R; ++r) x[r] = src[(int64_t)(j + r * S0::M) * PL];
    fz::dif_regs<C, N, 0, PV>(x, tw, j);
#pragma unroll
    for (int q = 0; q < S0::R; ++q) buf[(j + q * S0::M) * LS + line] = x[q];
  }
  __syncthreads();
  // the staged tiles are complete and visible after the barrier that ends the DIF stages
  if constexpr (PRE) fz::cp_async_wait_all();
  fz::dif_range<C, N, LV, 1, LS, NT, PV, 1, NS>(buf, tw);
  const W s = (W)(1.0 / ((double)N * N * N));
  double fint = 0, elen = 0;
  if constexpr (TAB) {
    // Two passes over the tile's k-points, each thread on the same points in both (no
    // barrier between them): the Cahn-Hilliard update reads theta^ and writes slot V, then
    // the elastic pass overwrites theta^ with phi^.  Split, each pass keeps fewer values live.
    // ---- Cahn-Hilliard on the fluctuation state: mu^ = A dc^ - B/2 sum theta^
#pragma unroll 1
    for (int i = threadIdx.x; i < N * TM; i += NT) {
      const int p = i / TM, c = i - p * TM;
      const int64_t m = m0 + c;
      const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
      const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
      C* e = buf + p * LS + c;
      W str = 0, sti = 0;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const W tr = (W)e[v * TM].x * s, ti = (W)e[v * TM].y * s;
        str += tr;
        sti += ti;
        if (a.rec_theta) a.rec_theta[v * NK + p * PL + m] = mk((R)tr, (R)ti);
      }
      const C cs = PRE ? kcs[p * TM + c] : a.Kc[p * PL + m];
      const W cr = (W)cs.x, ci = (W)cs.y;
      const bool k0 = (kx == 0 && ky == 0 && kz == 0);
      if (a.energy) {
        W av[3], b[3];
        kvec_w<N, W>(kx, ky, kz, av, b);
        const W w = (kx == 0 || 2 * kx == N) ? (W)1 : (W)2;
        fint += (double)((W)0.5 * w * kapc * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) * (cr * cr + ci * ci));
      }
      W nr = 0, ni = 0;
      if (!k0) {
        const double a0 = kcomp<N>(kx), a1 = kcomp<N>(ky), a2 = kcomp<N>(kz);
        const double k2d = a0 * a0 + a1 * a1 + a2 * a2;
        const Damp<W> rden(recip_ge1(1.0 + dmd * kapcd * k2d * k2d));
        const W dk2 = (W)(dmd * k2d);
        const W mr = lan_a * cr - hlb * str, mi = lan_a * ci - hlb * sti;
        nr = rden(cr - dk2 * mr);
        ni = rden(ci - dk2 * mi);
      }
      const C cn = mk((R)nr, (R)ni);
      a.Kc_out[p * PL + m] = cn;
      e[V * TM] = cn;
    }
    // ---- homogeneous elasticity: phi^_v = sum_u T_vu theta^_u from the Green-operator table
#pragma unroll 1
    for (int i = threadIdx.x; i < N * TM; i += NT) {
      const int p = i / TM, c = i - p * TM;
      C* e = buf + p * LS + c;
      if (!a.homog) {
#pragma unroll
        for (int v = 0; v < V; ++v) e[v * TM] = mk((R)0, (R)0);
        continue;
      }
      const int64_t m = m0 + c;
      const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
      const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
      const bool k0 = (kx == 0 && ky == 0 && kz == 0);
      W tr[V], ti[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        tr[v] = (W)e[v * TM].x * s;
        ti[v] = (W)e[v * TM].y * s;
      }
      W phr[V], phi_[V];
      {
        W T[V][V];
        int q = 0;
#pragma unroll
        for (int v = 0; v < V; ++v)
#pragma unroll
          for (int u = v; u < V; ++u) {
            const W t = k0 ? (W)0 : PRE ? (W)lds<R>(gts + (q * N + p) * TM + c) : (W)__ldg(a.gtab + q * NK + p * PL + m);
            T[v][u] = t;
            T[u][v] = t;
            ++q;
          }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          W pr = 0, pi = 0;
#pragma unroll
          for (int u = 0; u < V; ++u) {
            pr += T[v][u] * tr[u];
            pi += T[v][u] * ti[u];
          }
          phr[v] = pr;
          phi_[v] = pi;
          e[v * TM] = mk((R)pr, (R)pi);
        }
      }
      if (!a.energy) continue;
      const W w = (kx == 0 || 2 * kx == N) ? (W)1 : (W)2;
      const bool nyq = 2 * kx == N || 2 * ky == N || 2 * kz == N;
      if (!k0 && !nyq) {
        // Khachaturyan's quadratic form: with equilibrium u^ and homogeneous C0,
        // e*.C0.e = sum_pq A_pq Re(theta^_p* theta^_q) - sum_p Re(theta^_p* phi^_p),
        // A_pq = eps0_p.C0.eps0_q.  It needs the strain's and Q(k)'s k-vectors to agree,
        // which they do off the Nyquist planes (k_space zeroes b there but not a).
        W qq = 0;
#pragma unroll
        for (int pv = 0; pv < V; ++pv) {
          qq -= tr[pv] * phr[pv] + ti[pv] * phi_[pv];
#pragma unroll
          for (int qv = 0; qv < V; ++qv) qq += aW[pv][qv] * (tr[pv] * tr[qv] + ti[pv] * ti[qv]);
        }
        elen += (double)((W)0.5 * w * qq);
      } else {
        // Nyquist planes and k = 0: the strain itself
        W av[3], b[3];
        kvec_w<N, W>(kx, ky, kz, av, b);
        double ad[3], bd[3];
        kvec_n<N>(kx, ky, kz, ad, bd);
        const W qq = nyq_strain_energy<W, V>(tr, ti, b, ad, bd, k0, !k0, sgW, epW, c0W, ebW, qc);
        elen += (double)((W)0.5 * w * qq);
      }
    }
  } else {
    // one pass: theta^ sums and Cahn-Hilliard, Omega(k) = Q(k)^-1 in FP64 per k, phi^_v
    for (int i = threadIdx.x; i < N * TM; i += NT) {
      const int p = i / TM, c = i - p * TM;
      const int64_t m = m0 + c;
      const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
      const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py), kz = fz::rev<N, PV>(p);
      W av[3], b[3];
      kvec_w<N, W>(kx, ky, kz, av, b);
      const W w = (kx == 0 || 2 * kx == N) ? (W)1 : (W)2;
      C* e = buf + p * LS + c;
      W tr[V], ti[V], str = 0, sti = 0;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        tr[v] = (W)e[v * TM].x * s;
        ti[v] = (W)e[v * TM].y * s;
        str += tr[v];
        sti += ti[v];
      }
      if (a.rec_theta) {
#pragma unroll
        for (int v = 0; v < V; ++v) a.rec_theta[v * NK + p * PL + m] = mk((R)tr[v], (R)ti[v]);
      }
      const C cs = a.Kc[p * PL + m];
      const W cr = (W)cs.x, ci = (W)cs.y;
      const bool k0 = (kx == 0 && ky == 0 && kz == 0);
      const bool nyq = 2 * kx == N || 2 * ky == N || 2 * kz == N;
      double ad[3], bd[3];
      kvec_n<N>(kx, ky, kz, ad, bd);
      if (a.energy) fint += (double)((W)0.5 * w * kapc * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) * (cr * cr + ci * ci));
      // ---- homogeneous elasticity: u^ = Q^-1 R, phi^_v = i (sig0_v b) . u^
      W ur[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
      if (a.homog && !k0) {
        W Sr[6] = {0, 0, 0, 0, 0, 0}, Si[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int v = 0; v < V; ++v)
#pragma unroll
          for (int q = 0; q < 6; ++q) { Sr[q] += tr[v] * sgW[v][q]; Si[q] += ti[v] * sgW[v][q]; }
        // R_i = i sum_j b_j S_ij (Voigt: 11,22,33,23,13,12)
        const W t1r = b[0] * Sr[0] + b[1] * Sr[5] + b[2] * Sr[4], t1i = b[0] * Si[0] + b[1] * Si[5] + b[2] * Si[4];
        const W t2r = b[0] * Sr[5] + b[1] * Sr[1] + b[2] * Sr[3], t2i = b[0] * Si[5] + b[1] * Si[1] + b[2] * Si[3];
        const W t3r = b[0] * Sr[4] + b[1] * Sr[3] + b[2] * Sr[2], t3i = b[0] * Si[4] + b[1] * Si[3] + b[2] * Si[2];
        const W Rr[3] = {-t1i, -t2i, -t3i}, Ri[3] = {t1r, t2r, t3r};
        // Omega(k) in FP64 from the double k-vectors
        const double Kv[6] = {ad[0] * ad[0], ad[1] * ad[1], ad[2] * ad[2], bd[1] * bd[2], bd[0] * bd[2], bd[0] * bd[1]};
        double Qs[6];
        if (qcub) {
          const double s2 = Kv[0] + Kv[1] + Kv[2];
#pragma unroll
          for (int q = 0; q < 3; ++q) Qs[q] = q_other * s2 + (q_own - q_other) * Kv[q];
#pragma unroll
          for (int q = 3; q < 6; ++q) Qs[q] = q_off * Kv[q];
        } else {
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            double acc = 0;
#pragma unroll
            for (int n = 0; n < 6; ++n) acc += qc[q][n] * Kv[n];
            Qs[q] = acc;
          }
        }
        // symmetric [[a,d,e],[d,b,f],[e,f,c]] with a=Q11 b=Q22 c=Q33 d=Q12 e=Q13 f=Q23
        const double qa = Qs[0], qb = Qs[1], qcc = Qs[2], qf = Qs[3], qe = Qs[4], qd = Qs[5];
        const double i00 = qb * qcc - qf * qf, i01 = qe * qf - qcc * qd, i02 = qd * qf - qb * qe;
        const double i11 = qa * qcc - qe * qe, i12 = qd * qe - qa * qf, i22 = qa * qb - qd * qd;
        const double det = qa * i00 + qd * i01 + qe * i02;  // singular Q(k): k_lf_qcheck's error
        const double rd = recip_nr(det);
        const W Qi[3][3] = {{(W)(i00 * rd), (W)(i01 * rd), (W)(i02 * rd)},
                            {(W)(i01 * rd), (W)(i11 * rd), (W)(i12 * rd)},
                            {(W)(i02 * rd), (W)(i12 * rd), (W)(i22 * rd)}};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          ur[r] = Qi[r][0] * Rr[0] + Qi[r][1] * Rr[1] + Qi[r][2] * Rr[2];
          ui[r] = Qi[r][0] * Ri[0] + Qi[r][1] * Ri[1] + Qi[r][2] * Ri[2];
        }
      }
      W phr[V], phi_[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        W pr = 0, pi = 0;
        if (a.homog && !k0) {
          const W* sg = sgW[v];
          const W sb0 = sg[0] * b[0] + sg[5] * b[1] + sg[4] * b[2];
          const W sb1 = sg[5] * b[0] + sg[1] * b[1] + sg[3] * b[2];
          const W sb2 = sg[4] * b[0] + sg[3] * b[1] + sg[2] * b[2];
          const W dr = sb0 * ur[0] + sb1 * ur[1] + sb2 * ur[2];
          const W di = sb0 * ui[0] + sb1 * ui[1] + sb2 * ui[2];
          pr = -di;
          pi = dr;
        }
        phr[v] = pr;
        phi_[v] = pi;
        e[v * TM] = mk((R)pr, (R)pi);
      }
      if (a.homog && a.energy && !k0 && !nyq) {
        // Khachaturyan's quadratic form: with equilibrium u^ and homogeneous C0,
        // e*.C0.e = sum_pq A_pq Re(theta^_p* theta^_q) - sum_p Re(theta^_p* phi^_p),
        // A_pq = eps0_p.C0.eps0_q.  It needs the strain's and Q(k)'s k-vectors to agree,
        // which they do off the Nyquist planes (k_space zeroes b there but not a).
        W qq = 0;
#pragma unroll
        for (int pv = 0; pv < V; ++pv) {
          qq -= tr[pv] * phr[pv] + ti[pv] * phi_[pv];
#pragma unroll
          for (int qv = 0; qv < V; ++qv) qq += aW[pv][qv] * (tr[pv] * tr[qv] + ti[pv] * ti[qv]);
        }
        elen += (double)((W)0.5 * w * qq);
      } else if (a.homog && a.energy) {
        // engineering elastic strain e = gamma(u^) - sum_v theta^_v eps0_v (+ e_mean at k = 0)
        const int I1[6] = {0, 1, 2, 1, 0, 0}, J1[6] = {0, 1, 2, 2, 2, 1};
        W er[6], ei[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const int ii = I1[q], jj = J1[q];
          W gr, gi;
          if (q < 3) { gr = -b[ii] * ui[ii]; gi = b[ii] * ur[ii]; }
          else { gr = -(b[ii] * ui[jj] + b[jj] * ui[ii]); gi = b[ii] * ur[jj] + b[jj] * ur[ii]; }
#pragma unroll
          for (int v = 0; v < V; ++v) { gr -= tr[v] * epW[v][q]; gi -= ti[v] * epW[v][q]; }
          if (k0) gr += ebW[q];
          er[q] = gr;
          ei[q] = gi;
        }
        W qq = 0;
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          W cr2 = 0, ci2 = 0;
#pragma unroll
          for (int j = 0; j < 6; ++j) { cr2 += c0W[r + j * 6] * er[j]; ci2 += c0W[r + j * 6] * ei[j]; }
          qq += er[r] * cr2 + ei[r] * ci2;
        }
        elen += (double)((W)0.5 * w * qq);
      }
      // ---- Cahn-Hilliard on the fluctuation state: mu^ = A dc^ - B/2 sum theta^
      W nr = 0, ni = 0;
      if (!k0) {
        const double k2d = ad[0] * ad[0] + ad[1] * ad[1] + ad[2] * ad[2];
        const Damp<W> rden(recip_ge1(1.0 + dmd * kapcd * k2d * k2d));
        const W dk2 = (W)(dmd * k2d);
        const W mr = lan_a * cr - hlb * str, mi = lan_a * ci - hlb * sti;
        nr = rden(cr - dk2 * mr);
        ni = rden(ci - dk2 * mi);
      }
      const C cn = mk((R)nr, (R)ni);
      a.Kc_out[p * PL + m] = cn;
      e[V * TM] = cn;
    }
  }
  __syncthreads();
  fz::dit_range<C, N, LN, 1, LS, NT, PV, 1, NS - 1>(buf, tw);
#pragma unroll 1
  for (int t = threadIdx.x; t < LN * S0::M; t += NT) {
    const int line = t % LN, j = t / LN, f = line / TM, c = line - f * TM;
    C x[S0::R];
#pragma unroll
    for (int q = 0; q < S0::R; ++q) x[q] = buf[(j + q * S0::M) * LS + line];
    fz::dit_regs<C, N, 0, PV>(x, tw, j);
    C* dst = a.M + f * NK + m0 + c;
#pragma unroll
    for (int r = 0; r < S0::R; ++r) dst[(int64_t)(j + r * S0::M) * PL] = x[r];
  }
  block_reduce_store(fint, 0, a.partials + LQ_FINT * PSTRIDE + bx);
  block_reduce_store(elen, 0, a.partials + LQ_ELEN * PSTRIDE + bx);
}
template <typename R, int N, int V, int PV, int TM>
__global__ void __launch_bounds__(NT, (z1_min_blocks<R, N, V, TM>())) k_lf_z1(const LanFusedArgs<R>* __restrict__ A) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  lf_z1_body<R, N, V, PV, TM>(a, blockIdx.x);
}

// ------------------------------------------------------------------ PB
// Block (f, z): phi_f of plane z -> g_f -> forward transform.  The pointwise work
// runs between the x transform's inverse and forward stage 0 on each butterfly's
// registers (Plane::x_stage0); its inputs (eta_0..V-1 and dc of this plane) are
// read straight from global memory (mostly L2).
constexpr size_t SM_SMEM = 228 * 1024, BLOCK_RESERVED = 1024;

template <typename R, int N, int V, int PV, int NTP>
constexpr size_t pb_smem() {
  return fz::Plane<R, N, NTP, PV>::smem_bytes();
}

// resident blocks per SM the plane kernels are compiled for: as many as shared memory
// allows, at most 4 of 256 threads (64 registers a thread; 128^3 FP32 planes fit 3, so
// 80) or 2 of 512 (64).  Four 256-thread blocks on the 32^3-96^3 planes: deck 3
// 1.798 -> 1.752 ms per step
template <typename R, int N, int PV, int NTP>
constexpr int plane_min_blocks() {
  constexpr size_t per = fz::Plane<R, N, NTP, PV>::smem_bytes() + BLOCK_RESERVED;
  constexpr int by_smem = (int)(SM_SMEM / per);
  constexpr int by_threads = NTP >= 512 ? 2 : 4;
  return by_smem < 1 ? 1 : (by_smem < by_threads ? by_smem : by_threads);
}

// PB of variant f, plane z of one member.  COH: the eta and dc planes may have been
// written earlier in the same launch (the persistent ensemble kernel), so they are read
// with coherent loads instead of the read-only path.
template <typename R, int N, int V, int PV, int NTP, bool COH = false>
__device__ __forceinline__ void lf_pb_body(const LanFusedArgs<R>& a, const int f, const int z) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  C* mp = a.M + f * NK + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  step_dep_wait();
  step_dep_release();
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  // constants of the driving force in registers; pointwise math in the field precision W
  using W = R;
  const LanFusedConst& F = *a.F;
  const W cbar = (W)F.cbar, lb = (W)F.lan_b, lc2 = (W)F.lan_c2, lc = (W)F.lan_c, ld = (W)F.lan_d;
  const W cw4 = (W)(4.0 * F.cross_w), s0f = (W)F.sig0_ebar[f];
  W Af[V];
#pragma unroll
  for (int q = 0; q < V; ++q) Af[q] = (W)F.A[f][q];
  const bool homog = a.homog != 0;
  // bulk free energy of the start-of-step fields, summed by the f == 0 block of each plane
  const bool bulk = a.energy && f == 0;
  const W la2 = (W)(0.5 * F.lan_a), lc1 = (W)F.lan_c1, lb2 = (W)(0.5 * F.lan_b), lc4 = (W)(0.25 * F.lan_c);
  const W ld6 = (W)(F.lan_d / 6.0), cw = (W)F.cross_w;
  double fch = 0;
  auto bulk_energy = [&](const C* ev, C dcv) {
    W acc = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      W s2 = 0, s4 = 0, s6 = 0;
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const W x = h ? ev[q].y : ev[q].x, e2 = x * x;
        s2 += e2;
        s4 += e2 * e2;
        s6 += e2 * e2 * e2;
      }
      const W cv = cbar + (W)(h ? dcv.y : dcv.x), dc1 = cv - lc1;
      acc += la2 * dc1 * dc1 + lb2 * (lc2 - cv) * s2 - lc4 * s4 + ld6 * s6 + cw * (s2 * s2 - s4);
    }
    fch += (double)acc;
  };
  // g_f at the pair (x, x+1) of row y from eta_q (q < V), dc and phi_f
  auto point = [&](const C* ev, C dcv, C ph) -> C {
    W e2q[2][V], s2[2] = {0, 0}, ef[2];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const W x = ev[q].x, yv = ev[q].y;
      e2q[0][q] = x * x;
      e2q[1][q] = yv * yv;
      s2[0] += e2q[0][q];
      s2[1] += e2q[1][q];
      if (q == f) { ef[0] = x; ef[1] = yv; }
    }
    const W cv[2] = {cbar + (W)dcv.x, cbar + (W)dcv.y};
    const W phv[2] = {(W)ph.x, (W)ph.y};
    W out[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const W e = ef[h], e2 = e * e;
      W g = lb * (lc2 - cv[h]) * e - lc * e2 * e + ld * e2 * e2 * e + cw4 * e * (s2[h] - e2);
      if (homog) {
        W sacc = s0f + phv[h];
#pragma unroll
        for (int q = 0; q < V; ++q) sacc -= Af[q] * e2q[h][q];
        g += (W)-2 * e * sacc;
      }
      out[h] = g;
    }
    return mk((R)out[0], (R)out[1]);
  };
  R* rec = a.rec_phi ? a.rec_phi + f * N3 + z * PL : nullptr;
  // phi_f back to shared memory in real space, then one pass over the plane's pairs in
  // row order (its global loads of eta_q and dc are coalesced rows with several pairs in
  // flight per thread, which hides their L2 latency better than loading them inside the
  // register stage), then the forward from shared memory
  P::template x_stage0<false>(buf, tws, [&](int y, int n0, int dn, C* x) {
    C* rb = buf + y * P::PITCH + n0;
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) rb[r * dn] = x[r];
  });
#pragma unroll 4
  for (int i = threadIdx.x; i < N * P::LX; i += NTP) {
    const int y = i / P::LX, n = i - y * P::LX;
    const int64_t g0 = z * PL + (int64_t)y * N + 2 * n;
    C ev[V];
#pragma unroll
    for (int q = 0; q < V; ++q) ev[q] = COH ? *(const C*)(a.eta + q * N3 + g0) : __ldg((const C*)(a.eta + q * N3 + g0));
    const C dcv = COH ? *(const C*)(a.c + g0) : __ldg((const C*)(a.c + g0));
    const C ph = buf[y * P::PITCH + n];
    if (rec) ((C*)(rec + (int64_t)y * N))[n] = ph;
    if (bulk) bulk_energy(ev, dcv);
    buf[y * P::PITCH + n] = point(ev, dcv, ph);
  }
  __syncthreads();
  P::x_forward0(buf, tws, [](int, int, int, C*) {});
  if (bulk) block_reduce_store(fch, 0, a.partials + LQ_FCH * PSTRIDE + z);
  P::forward_tail(buf, tws, mp);
}
template <typename R, int N, int V, int PV, int NTP>
__global__ void __launch_bounds__(NTP, (plane_min_blocks<R, N, PV, NTP>()))
    k_lf_pb(const LanFusedArgs<R>* __restrict__ A) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  // field index fastest: the V blocks of one plane, which read the same eta and
  // dc planes, are resident together and share those reads through L2
  lf_pb_body<R, N, V, PV, NTP>(a, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------ Z2
// z FFT of g_v, TDGL update of the eta^ state, z iFFT.  The first DIF stage takes
// its butterflies straight from global memory and the last DIT stage (stage 0)
// writes straight back; the last DIF stage, the state update and the first DIT
// stage touch the same elements of one butterfly, so they run on its registers.
// With a two-stage radix plan a column makes two shared-memory round trips.
// Z2's shared memory and the resident blocks per SM it is compiled for: as many as its
// tile allows (with 2 KB for static arrays and the 1 KB runtime reserve), at most 4 (64
// registers a thread) with up to three variants in FP32, else 3
template <typename R, int N, int V, int TM>
constexpr size_t z2_smem() {
  return sizeof(cplx<R>) * (2 * (size_t)N * V * TM + N * Tw<cplx<R>>::K);
}
template <typename R, int N, int V, int TM>
constexpr int z2_min_blocks() {
  constexpr int by_smem = (int)(SM_SMEM / (z2_smem<R, N, V, TM>() + BLOCK_RESERVED + 2048));
  constexpr int cap = (sizeof(R) == 4 && V <= 3) ? 4 : 3;
  return by_smem < 1 ? 1 : (by_smem < cap ? by_smem : cap);
}

// Z2 of column tile bx of one member
template <typename R, int N, int V, int PV, int TM>
__device__ __forceinline__ void lf_z2_body(const LanFusedArgs<R>& a, const int bx) {
  using C = cplx<R>;
  constexpr int NXH = N / 2 + 1, LN = V * TM;
  constexpr int64_t PL = (int64_t)N * NXH, NK = PL * N;
  constexpr int NS = fz::rplan(N, PV).ns;
  static_assert(NS >= 2, "the column kernels need a radix plan of two stages or more");
  using S0 = fz::StageOf<N, 0, PV>;
  using SL = fz::StageOf<N, NS - 1, PV>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;  // [N][V][TM]
  C* ks = buf + N * LN;  // eta^ state tile [N][V][TM], in flight from the start
  C* tw = ks + N * LN;
  using W = R;  // working precision of the update (the state's)
  __shared__ double g[V][9];
  __shared__ int sameg;  // every variant has the gradient coefficients of variant 0
  const int64_t m0 = (int64_t)bx * TM;
  // the eta^ state was written by the previous step's Z2, which has completed once this
  // block runs (PB released it only after its own wait), and PB does not touch it: the
  // tile load overlaps PB's last blocks (L2 reads, cp.async.cg)
  tile_load<C, N, TM>(ks, LN, 0, a.Keta, NK, PL, m0, V);
  fz::cp_async_commit();
  if (threadIdx.x == 0) {
    int same = 1;
    for (int v = 0; v < V; ++v)
      for (int j = 0; j < 9; ++j) {
        g[v][j] = a.F->g[v][j];
        same &= a.F->g[v][j] == a.F->g[0][j];
      }
    sameg = same;
  }
  for (int i = threadIdx.x; i < N * Tw<C>::K; i += NT) tw[i] = a.twz[i];
  step_dep_wait();
  step_dep_release();
  __syncthreads();
  // DIF stage 0: butterflies from global memory (column-fastest: coalesced rows)
#pragma unroll 1
  for (int t = threadIdx.x; t < LN * S0::M; t += NT) {
    const int line = t % LN, j = t / LN, f = line / TM, c = line - f * TM;
    const C* src = a.M + f * NK + m0 + c;
    C x[S0::R];
#pragma unroll
    for (int r = 0; r < S0::R; ++r) x[r] = src[(int64_t)(j + r * S0::M) * PL];
    fz::dif_regs<C, N, 0, PV>(x, tw, j);
#pragma unroll
    for (int q = 0; q < S0::R; ++q) buf[(j + q * S0::M) * LN + line] = x[q];
  }
  __syncthreads();
  fz::dif_range<C, N, LN, 1, LN, NT, PV, 1, NS - 1>(buf, tw);
  fz::cp_async_wait_all();
  __syncthreads();
  const double dtld = a.F->dtl;
  const W ds = (W)dtld * (W)(1.0 / ((double)N * N * N));
  const bool one_g = sameg != 0;
  double fint = 0;
  // last DIF stage + update + first DIT stage on one butterfly (M = 1: no twiddles)
#pragma unroll 1
  for (int t = threadIdx.x; t < LN * SL::TASKS; t += NT) {
    const int line = t % LN, b = t / LN, f = line / TM, c = line - f * TM;
    const int64_t m = m0 + c;
    const int py = (int)(m / NXH), cx = (int)(m - (int64_t)py * NXH);
    const int kx = fz::kx_of_col<N, PV>(cx), ky = fz::rev<N, PV>(py);
    const double* gv = one_g ? g[0] : g[f];
    const double ax = kcomp<N>(kx), ay = kcomp<N>(ky);
    const double bx = 2 * kx == N ? 0.0 : ax, by = 2 * ky == N ? 0.0 : ay;
    // k.kappa.k = Kc + (terms in kz): constant part of this column
    const double kk0 = gv[0] * ax * ax + gv[4] * ay * ay + (gv[3] + gv[1]) * bx * by;
    const double kb0 = gv[0] * bx * bx + gv[4] * by * by + (gv[3] + gv[1]) * bx * by;
    const double kz1 = (gv[7] + gv[5]) * by + (gv[2] + gv[6]) * bx;  // times bz
    const W w = (kx == 0 || 2 * kx == N) ? (W)1 : (W)2;
    C x[SL::R];
#pragma unroll
    for (int q = 0; q < SL::R; ++q) x[q] = buf[(b * SL::R + q) * LN + line];
    Dft<SL::R, -1, C>::run(x);
    const C* kst = ks + line;
    C* kout = a.Keta_out + f * NK + m;
    W fk = 0;
#pragma unroll
    for (int q = 0; q < SL::R; ++q) {
      const int p = b * SL::R + q;
      const int kz = fz::rev<N, PV>(p);
      const double az = kcomp<N>(kz), bz = 2 * kz == N ? 0.0 : az;
      const C st = kst[p * LN];
      const W hr = (W)st.x, hi = (W)st.y;
      if (a.energy) fk += (W)(kb0 + gv[8] * bz * bz + kz1 * bz) * (hr * hr + hi * hi);
      const Damp<W> rden(recip_ge1(1.0 + dtld * (kk0 + gv[8] * az * az + kz1 * bz)));
      const C o = mk((R)rden(hr - ds * (W)x[q].x), (R)rden(hi - ds * (W)x[q].y));
      kout[(int64_t)p * PL] = o;
      x[q] = o;
    }
    Dft<SL::R, 1, C>::run(x);
#pragma unroll
    for (int q = 0; q < SL::R; ++q) buf[(b * SL::R + q) * LN + line] = x[q];
    if (a.energy) fint += (double)((W)0.5 * w * fk);
  }
  __syncthreads();
  fz::dit_range<C, N, LN, 1, LN, NT, PV, 1, NS - 2>(buf, tw);
  // DIT stage 0: butterflies straight to global memory
#pragma unroll 1
  for (int t = threadIdx.x; t < LN * S0::M; t += NT) {
    const int line = t % LN, j = t / LN, f = line / TM, c = line - f * TM;
    C x[S0::R];
#pragma unroll
    for (int q = 0; q < S0::R; ++q) x[q] = buf[(j + q * S0::M) * LN + line];
    fz::dit_regs<C, N, 0, PV>(x, tw, j);
    C* dst = a.M + f * NK + m0 + c;
#pragma unroll
    for (int r = 0; r < S0::R; ++r) dst[(int64_t)(j + r * S0::M) * PL] = x[r];
  }
  block_reduce_store(fint, 0, a.partials + Q_FINT2 * PSTRIDE + bx);
}
template <typename R, int N, int V, int PV, int TM>
__global__ void __launch_bounds__(NT, (z2_min_blocks<R, N, V, TM>())) k_lf_z2(const LanFusedArgs<R>* __restrict__ A) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  lf_z2_body<R, N, V, PV, TM>(a, blockIdx.x);
}

// ------------------------------------------------------------------ PI
// Block (z, f < V): eta_new_f -> real, eta statistics, and theta_f = eta_f^2 -> forward
// for the next step (which then starts at its column kernel).  The concentration plane
// and the end of the step are k_lf_pc's.
// PI of plane z, variant f of one member
template <typename R, int N, int PV, int NTP>
__device__ __forceinline__ void lf_pi_body(const LanFusedArgs<R>& a, const int V, const int z, const int f) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  constexpr int64_t PL = (int64_t)N * N, N3 = PL * N, NK = (int64_t)N * N * P::NXH;
  C* mp = a.M + f * NK + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  step_dep_wait();
  step_dep_release();
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  R* dst = a.eta_next + f * N3 + z * PL;
  double emax = 0.0, s2 = 0.0;
  P::template x_stage0<true>(buf, tws, [&](int y, int n0, int dn, C* x) {
    C* row = (C*)(dst + (int64_t)y * N);
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) {
      const C v = x[r];
      row[n0 + r * dn] = v;
      emax = fmax(emax, fmax((double)v.x, (double)v.y));
      s2 += (double)v.x * v.x + (double)v.y * v.y;
      x[r] = mk((R)((double)v.x * (double)v.x), (R)((double)v.y * (double)v.y));
    }
  });
  P::forward_tail(buf, tws, mp);
  // the concentration quantities of this block's partial slot hold their start values
  const int blk = z * (V + 1) + f;
  block_reduce_store(emax, 1, a.partials + LQ_PHIMAX * PSTRIDE + blk);
  block_reduce_store(s2, 0, a.partials + LQ_SOLID * PSTRIDE + blk);
  if (threadIdx.x == 0) {
    a.partials[LQ_CMIN * PSTRIDE + blk] = 1.0;
    a.partials[LQ_CMAX * PSTRIDE + blk] = 0.0;
    a.partials[LQ_CSUM * PSTRIDE + blk] = 0.0;
  }
}
template <typename R, int N, int PV, int NTP>
__global__ void __launch_bounds__(NTP, (plane_min_blocks<R, N, PV, NTP>()))
    k_lf_pi(const LanFusedArgs<R>* __restrict__ A, int V) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  lf_pi_body<R, N, PV, NTP>(a, V, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------ PC
// Block z: dc_new -> real, concentration statistics; the member's last block ends the
// step.
// PC of plane z of one member: the plane and its partial slots (not the end of the step)
template <typename R, int N, int PV, int NTP>
__device__ __forceinline__ void lf_pc_body(const LanFusedArgs<R>& a, const int V, const int z) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  C* tws = buf + P::ELEMS;
  constexpr int64_t PL = (int64_t)N * N, NK = (int64_t)N * N * P::NXH;
  C* mp = a.M + V * NK + z * (int64_t)N * P::NXH;
  P::load_tw(tws, a.twx, a.twy, a.post);
  step_dep_release();
  __syncthreads();
  P::inverse_head(buf, tws, mp, a.err);
  R* dst = a.c_next + z * PL;
  double cmin = 1.0, cmax = 0.0, csum = 0.0;
  const double cbar = a.F->cbar;
  P::template x_stage0<false>(buf, tws, [&](int y, int n0, int dn, C* x) {
    C* row = (C*)(dst + (int64_t)y * N);
#pragma unroll
    for (int r = 0; r < fz::StageOf<P::LX, 0, PV>::R; ++r) {
      const C v = x[r];
      row[n0 + r * dn] = v;
      const double c0 = cbar + (double)v.x, c1 = cbar + (double)v.y;
      cmin = fmin(cmin, fmin(c0, c1));
      cmax = fmax(cmax, fmax(c0, c1));
      csum += c0 + c1;
    }
  });
  const int blk = z * (V + 1) + V;
  if (threadIdx.x == 0) {
    a.partials[LQ_PHIMAX * PSTRIDE + blk] = 0.0;
    a.partials[LQ_SOLID * PSTRIDE + blk] = 0.0;
  }
  block_reduce_store(cmin, 2, a.partials + LQ_CMIN * PSTRIDE + blk);
  block_reduce_store(cmax, 1, a.partials + LQ_CMAX * PSTRIDE + blk);
  block_reduce_store(csum, 0, a.partials + LQ_CSUM * PSTRIDE + blk);
}

// The end of a member's step, by one block once every partial of the step is written
// and visible: every block partial in a fixed order into history row *hist_row, which
// then advances (so graph replays need no host-side row index).  Every thread loads its
// strided share of every quantity at once (all loads in flight together: one L2 round
// trip), then one block reduction of the Q_STEP_COUNT values.
template <int NTP, typename R>
__device__ __forceinline__ void lf_step_reduce(const LanFusedArgs<R>& a, const NbList& nb) {
  const int row = *(volatile const int*)a.hist_row;
  constexpr int QN = Q_STEP_COUNT, NW = NTP / 32;
  auto qop = [](int q) { return (q == Q_CMIN) ? 2 : (q == Q_CMAX || q == Q_PHIMAX) ? 1 : 0; };
  double acc[QN];
#pragma unroll
  for (int q = 0; q < QN; ++q) acc[q] = qop(q) == 0 ? 0.0 : qop(q) == 1 ? -1.0e308 : 1.0e308;
  int nmax = 0;
#pragma unroll
  for (int q = 0; q < QN; ++q) nmax = max(nmax, nb.nb[q]);
#pragma unroll 1
  for (int i = threadIdx.x; i < nmax; i += NTP) {
#pragma unroll
    for (int q = 0; q < QN; ++q) {
      if (i < nb.nb[q]) {
        const double v = __ldcg(a.partials + (int64_t)q * PSTRIDE + i);
        acc[q] = qop(q) == 0 ? acc[q] + v : qop(q) == 1 ? fmax(acc[q], v) : fmin(acc[q], v);
      }
    }
  }
  __shared__ double wred[NW][QN];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < QN; ++q) {
    const double v = qop(q) == 0 ? warp_sum(acc[q]) : qop(q) == 1 ? warp_max(acc[q]) : warp_min(acc[q]);
    if (lane == 0) wred[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < QN) {
    const int q = threadIdx.x, op = qop(q);
    double v = wred[0][q];
    for (int w = 1; w < NW; ++w) v = op == 0 ? v + wred[w][q] : op == 1 ? fmax(v, wred[w][q]) : fmin(v, wred[w][q]);
    if (row < a.hist_rows) a.hist[(int64_t)row * Q_STEP_COUNT + q] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *a.ticket = 0;
    *a.hist_row = row + 1;
  }
}

// PC reads only the dc^ spectrum (Z1's) and writes only dc and its partial slots, none
// of which PI touches, so it runs beside PI: launched right after it with programmatic
// dependent launch, its blocks take the slots PI's single wave leaves free, and only the
// member's last block waits for PI (griddepcontrol.wait) before it ends the step
// (lf_step_reduce).  That block's wait also makes PC's completion imply PI's, which the
// next step's Z1 relies on.
template <typename R, int N, int PV, int NTP>
__global__ void __launch_bounds__(NTP, (plane_min_blocks<R, N, PV, NTP>()))
    k_lf_pc(const LanFusedArgs<R>* __restrict__ A, int V, NbList nb) {
  const LanFusedArgs<R> a = A[blockIdx.z];
  lf_pc_body<R, N, PV, NTP>(a, V, blockIdx.x);
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(a.ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  step_dep_wait();  // PI complete, its partials visible
  __threadfence();
  lf_step_reduce<NTP>(a, nb);
}

// ------------------------------------------------------------------ launch sequence
struct Scope {
  LaunchHook* h;
  cudaStream_t st;
  Scope(LaunchHook* h_, const char* n, double b, cudaStream_t s) : h(h_), st(s) {
    if (h) h->begin(n, b, st);
  }
  ~Scope() {
    if (h) h->end(st);
  }
};

// launch of a per-step kernel, with programmatic dependent launch when `dep` is set
template <typename... P, typename... Args>
void launch_step_kernel(void (*k)(P...), dim3 grid, int threads, size_t smem, cudaStream_t st, bool dep,
                        Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = dep ? 1 : 0;
  MEU_CUDA(cudaLaunchKernelEx(&cfg, k, args...));
}

// Raises fn's dynamic shared-memory limit to the opt-in maximum once per (kernel,
// device) and host thread; throws if `bytes` exceeds it.
template <typename K>
void ensure_smem(K fn, size_t bytes) {
  // no shortcut below 48 KB: without the opt-in, dynamic plus static shared memory must
  // stay within 48 KB, so a 48 KB tile of a kernel with static arrays needs it too
  static thread_local std::vector<std::pair<const void*, int>> done;
  int dev = 0, optin = 0;
  MEU_CUDA(cudaGetDevice(&dev));
  for (const auto& f : done)
    if (f.first == (const void*)fn && f.second == dev) return;
  MEU_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  MEU_CUDA(cudaFuncGetAttributes(&fa, (const void*)fn));
  const int lim = optin - (int)fa.sharedSizeBytes;
  if ((int)bytes > lim) throw CudaError("fused tile exceeds shared memory", MEU_ERR_UNSUPPORTED);
  MEU_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  done.emplace_back((const void*)fn, dev);
}

template <typename R, int N, int V, int PV, int NTP, int TM>
void run_step(const LanFusedArgs<R>* dA, int members, int opts, cudaStream_t st, LaunchHook* hook, int* nb) {
  const bool energy = (opts & LS_ENERGY) != 0;
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  constexpr int NXH = N / 2 + 1;
  constexpr int tiles = N * NXH / TM;
  static_assert(N * NXH % TM == 0 && tiles <= PSTRIDE, "column tiling");
  const double mm = (double)members;
  const double n3 = (double)N * N * N * mm, nk = (double)N * N * NXH * mm;
  const size_t sp = P::smem_bytes();
  const size_t s1 = z1_smem_base<R, N, V, TM>() + (z1_prefetch<R, N, V, TM>() ? z1_smem_stage<R, N, V, TM>() : 0);
  const size_t s2 = z2_smem<R, N, V, TM>();
  const size_t spb = pb_smem<R, N, V, PV, NTP>();
  ensure_smem(k_lf_pf<R, N, PV, NTP>, sp);
  ensure_smem(k_lf_pb<R, N, V, PV, NTP>, spb);
  ensure_smem(k_lf_pi<R, N, PV, NTP>, sp);
  ensure_smem(k_lf_pc<R, N, PV, NTP>, sp);
  ensure_smem(k_lf_z1<R, N, V, PV, TM>, s1);
  ensure_smem(k_lf_z2<R, N, V, PV, TM>, s2);
  // Programmatic dependent launch of the four step kernels, except with per-kernel timing
  // (which keeps them apart).  With 256-thread plane kernels (three per SM), letting Z1
  // start in PI's last wave and PI in Z2's made deck 1 slower (171.6 -> 178.0 us per
  // step), while PB after Z1 and Z2 after PB gained; with 512-thread plane kernels all
  // four gain (180.7 -> 174.8 us, FP64 350.7 -> 339.0 us).
  const bool dep = !(hook && hook->timing());
  const bool dep_after_plane = dep && NTP >= 512;
  if (opts & LS_QCHECK) {
    Scope s(hook, "lf_qcheck", 0.0, st);
    k_lf_qcheck<R, N><<<dim3(148, 1, members), 256, 0, st>>>(dA);
    MEU_CHECK_LAUNCH();
  }
  if (!(opts & LS_THETA_READY)) {
    // theta^ of the first step after new fields (later steps get it from PI)
    Scope s(hook, "lf_plane_fwd", (double)V * nk * sizeof(C) + (double)V * n3 * sizeof(R), st);
    k_lf_pf<R, N, PV, NTP><<<dim3(N, V, members), NTP, sp, st>>>(dA, V, 0);
    MEU_CHECK_LAUNCH();
  }
  {
    Scope s(hook, "lf_z_green_ch", (2.0 * V + 3) * nk * sizeof(C), st);
    launch_step_kernel(k_lf_z1<R, N, V, PV, TM>, dim3(tiles, 1, members), NT, s1, st, dep_after_plane, dA);
  }
  {
    Scope s(hook, "lf_plane_tdgl_rhs", (2.0 * V) * nk * sizeof(C) + (V + 1.0) * n3 * sizeof(R), st);
    launch_step_kernel(k_lf_pb<R, N, V, PV, NTP>, dim3(V, N, members), NTP, spb, st, dep, dA);
  }
  {
    Scope s(hook, "lf_z_tdgl", 4.0 * V * nk * sizeof(C), st);
    launch_step_kernel(k_lf_z2<R, N, V, PV, TM>, dim3(tiles, 1, members), NT, s2, st, dep, dA);
  }
  NbList l;
  for (int q = 0; q < Q_TOTAL; ++q) l.nb[q] = 0;
  l.nb[Q_FCH] = energy ? N : 0;
  l.nb[Q_FINT] = tiles;
  l.nb[Q_ELEN] = tiles;
  l.nb[Q_FINT2] = tiles;
  l.nb[Q_CMIN] = l.nb[Q_CMAX] = l.nb[Q_PHIMAX] = l.nb[Q_SOLID] = l.nb[Q_CSUM0] = N * (V + 1);
  {
    Scope s(hook, "lf_plane_inv_stats_theta", (2.0 * V) * nk * sizeof(C) + (double)V * n3 * sizeof(R), st);
    launch_step_kernel(k_lf_pi<R, N, PV, NTP>, dim3(N, V, members), NTP, sp, st, dep_after_plane, dA, V);
  }
  {
    Scope s(hook, "lf_plane_inv_c_end", nk * sizeof(C) + n3 * sizeof(R), st);
    launch_step_kernel(k_lf_pc<R, N, PV, NTP>, dim3(N, 1, members), NTP, sp, st, dep, dA, V, l);
  }
  for (int q = 0; q < Q_TOTAL; ++q) nb[q] = l.nb[q];
}

template <typename R, int N, int V, int PV, int NTP, int TM>
void run_init(const LanFusedArgs<R>* dA, int members, cudaStream_t st, LaunchHook* hook) {
  using P = fz::Plane<R, N, NTP, PV>;
  using C = cplx<R>;
  constexpr int NXH = N / 2 + 1;
  constexpr int tiles = N * NXH / TM;
  const size_t sp = P::smem_bytes();
  const size_t s0 = sizeof(C) * ((size_t)N * (V + 1) * TM + N * Tw<C>::K);
  ensure_smem(k_lf_pf<R, N, PV, NTP>, sp);
  ensure_smem(k_lf_z0<R, N, V, PV, TM>, s0);
  const double mm = (double)members;
  const double n3 = (double)N * N * N * mm, nk = (double)N * N * NXH * mm;
  {
    Scope s(hook, "lf_plane_fwd_state", (V + 1.0) * (nk * sizeof(C) + n3 * sizeof(R)), st);
    k_lf_pf<R, N, PV, NTP><<<dim3(N, V + 1, members), NTP, sp, st>>>(dA, V, 1);
    MEU_CHECK_LAUNCH();
  }
  {
    Scope s(hook, "lf_z_state", 2.0 * (V + 1) * nk * sizeof(C), st);
    k_lf_z0<R, N, V, PV, TM><<<dim3(tiles, 1, members), NT, s0, st>>>(dA);
    MEU_CHECK_LAUNCH();
  }
  if constexpr (V == 1) {
    Scope s(hook, "lf_green_table", nk * sizeof(R), st);
    k_lf_gtab<R, N, V, PV><<<dim3(2 * 148, 1, members), 256, 0, st>>>(dA);
    MEU_CHECK_LAUNCH();
  }
}

// column tile widths instantiated: T1 (default) and T0 = T1 / 2
template <typename R> constexpr int tm_wide() { return col_tile_default<R>(); }
template <typename R> constexpr int tm_narrow() { return col_tile_default<R>() / 2; }
template <typename R, int N, int TM> constexpr bool tm_ok() { return (N * (N / 2 + 1)) % TM == 0 && N * (N / 2 + 1) / TM <= PSTRIDE; }

// Calls f.template operator()<V, PV, NTP, TM>() for the schedule s; false when
// s names no instantiated variant.
template <typename R, int N, int V, typename Fn>
bool with_sched_v(const LanSched& s, Fn&& f) {
  const int tm = s.tm ? s.tm : tm_wide<R>();
  auto pick_tm = [&](auto pv_c, auto ntp_c) -> bool {
    constexpr int PV = decltype(pv_c)::value, NTP = decltype(ntp_c)::value;
    if (tm == tm_wide<R>()) {
      if constexpr (tm_ok<R, N, tm_wide<R>()>()) { f.template operator()<V, PV, NTP, tm_wide<R>()>(); return true; }
    } else if (tm == tm_narrow<R>()) {
      if constexpr (tm_ok<R, N, tm_narrow<R>()>()) { f.template operator()<V, PV, NTP, tm_narrow<R>()>(); return true; }
    }
    return false;
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using T256 = std::integral_constant<int, 256>;
  using T512 = std::integral_constant<int, 512>;
  if (s.pv == 0 && s.ntp == 512) return pick_tm(I0{}, T512{});
  if (s.pv == 0 && s.ntp == 256) return pick_tm(I0{}, T256{});
  if (s.pv == 1 && s.ntp == 512) return pick_tm(I1{}, T512{});
  if (s.pv == 1 && s.ntp == 256) return pick_tm(I1{}, T256{});
  if (s.pv == 2 && s.ntp == 512) return pick_tm(I2{}, T512{});
  if (s.pv == 2 && s.ntp == 256) return pick_tm(I2{}, T256{});
  return false;
}
template <typename R, int N, typename Fn>
bool with_sched(int V, const LanSched& s, Fn&& f) {
  switch (V) {
    case 1: return with_sched_v<R, N, 1>(s, f);
    case 2: return with_sched_v<R, N, 2>(s, f);
    case 3: return with_sched_v<R, N, 3>(s, f);
    case 4: return with_sched_v<R, N, 4>(s, f);
    default: return false;
  }
}

}  // namespace lf

namespace lf {
template <typename R, int N>
struct StepFn {
  const LanFusedArgs<R>* dA;
  int members;
  int opts;
  cudaStream_t st;
  LaunchHook* hook;
  int* nb;
  template <int V, int PV, int NTP, int TM>
  void operator()() const {
    run_step<R, N, V, PV, NTP, TM>(dA, members, opts, st, hook, nb);
  }
};
template <typename R, int N>
struct InitFn {
  const LanFusedArgs<R>* dA;
  int members;
  cudaStream_t st;
  LaunchHook* hook;
  template <int V, int PV, int NTP, int TM>
  void operator()() const {
    run_init<R, N, V, PV, NTP, TM>(dA, members, st, hook);
  }
};
}  // namespace lf

template <typename R, int N>
bool lf_step_n(int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, int opts, cudaStream_t st,
               LaunchHook* hook, int* nb) {
  return lf::with_sched<R, N>(V, s, lf::StepFn<R, N>{dA, members, opts, st, hook, nb});
}
template <typename R, int N>
bool lf_init_n(int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, cudaStream_t st, LaunchHook* hook) {
  return lf::with_sched<R, N>(V, s, lf::InitFn<R, N>{dA, members, st, hook});
}

}  // namespace meu

// one translation unit per (R, N)
#define MEU_LF_INSTANTIATE(R, N)                                                                                    \
  template bool meu::lf_step_n<R, N>(int, const meu::LanSched&, const meu::LanFusedArgs<R>*, int, int, cudaStream_t, \
                                     meu::LaunchHook*, int*);                                                       \
  template bool meu::lf_init_n<R, N>(int, const meu::LanSched&, const meu::LanFusedArgs<R>*, int, cudaStream_t,      \
                                     meu::LaunchHook*);
