// fft.cuh -- shared-memory batched 3-D real FFT for sm_100a.
//
// Replaces the P3DFFT calls of the reference's f_trans / inv_trans
// (ModFunc.f:15-40): forward = R2C scaled by 1/(Nx Ny Nz), inverse = C2R
// unscaled.  The spectrum is stored [z][y][kx] with kx in [0, Nx/2].
//
// Each 1-D transform runs in shared memory as in-place mixed-radix stages
// (radix 8/4/2/3).  Forward = decimation in frequency (natural order in,
// digit-reversed order out); inverse = decimation in time (digit-reversed in,
// natural out).  The digit reversal is folded into the global-memory
// addressing of the load/store, so no permutation pass exists.  The x
// transform of N reals is a complex transform of length N/2 plus a split
// step; the C2R split discards Im X(0) and Im X(N/2) like FFTW's c2r.
#pragma once
#include "common.cuh"

namespace meu {

struct LinePlan {
  int L;       // transform length
  int ns;      // number of stages
  int r[12];   // radix of each DIF stage (product = L)
  const void* tw;   // cplx<R>[L], tw[n] = exp(-2 pi i n / L)
  const int* rev;   // rev[p] = frequency index held at position p after DIF
};

// ------------------------------------------------------------------ twiddles
// Twiddle tables hold exp(-2 pi i n / L) once per entry in the field precision.
template <typename C> struct Tw;
template <> struct Tw<double2> {
  static constexpr int K = 1;
  static __device__ __forceinline__ double2 mul(double2 x, const double2* t, int i, int) { return cmul(x, t[i]); }
  static __device__ __forceinline__ double2 mulc(double2 x, const double2* t, int i, int) { return cmulc(x, t[i]); }
  static __device__ __forceinline__ double2 scale(double2 x, double hi, double) { return cscale(x, hi); }
};
// FP32 twiddle tables hold the correctly rounded value only.  (A hi + lo split of
// every table twiddle was measured to change nothing once the fused step keeps its
// state spectral: config 1 after 1000 steps, eta error 1.28e-6 with, 1.30e-6 without.)
// The radix-8 / radix-3 constants keep their hi + lo form (scale).
template <> struct Tw<float2> {
  static constexpr int K = 1;
  static __device__ __forceinline__ float2 mul(float2 x, const float2* t, int i, int) { return cmul(x, t[i]); }
  static __device__ __forceinline__ float2 mulc(float2 x, const float2* t, int i, int) { return cmulc(x, t[i]); }
  static __device__ __forceinline__ float2 scale(float2 x, double hi, double lo) {
    return cadd(cscale(x, (float)hi), cscale(x, (float)lo));
  }
};

// ---------------------------------------------------------------- butterflies
// y_q = sum_r x_r exp(S * 2 pi i r q / R), in place.
template <int R, int S, typename C> struct Dft;

template <int S, typename C> struct Dft<2, S, C> {
  static __device__ __forceinline__ void run(C* x) {
    C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  }
};
template <int S, typename C> struct Dft<4, S, C> {
  static __device__ __forceinline__ void run(C* x) {
    C a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
    C c = cadd(x[1], x[3]), d = cmul_is<S>(csub(x[1], x[3]));
    x[0] = cadd(a, c);
    x[2] = csub(a, c);
    x[1] = cadd(b, d);
    x[3] = csub(b, d);
  }
};
template <int S, typename C> struct Dft<3, S, C> {
  static __device__ __forceinline__ void run(C* x) {
    using R = decltype(x[0].x);
    const R h = (R)0.5;
    // sqrt(3)/2 as hi + lo (lo = 0 for double)
    const double s3h = sizeof(R) == 4 ? (double)0.8660254f : 0.86602540378443864676;
    const double s3l = sizeof(R) == 4 ? 0.86602540378443864676 - (double)0.8660254f : 0.0;
    C t = cadd(x[1], x[2]);
    C u = cmul_is<S>(Tw<C>::scale(csub(x[1], x[2]), s3h, s3l));
    C m = csub(x[0], cscale(t, h));
    x[0] = cadd(x[0], t);
    x[1] = cadd(m, u);
    x[2] = csub(m, u);
  }
};
template <int S, typename C> struct Dft<8, S, C> {
  static __device__ __forceinline__ void run(C* x) {
    using R = decltype(x[0].x);
    // sqrt(2)/2 as hi + lo (lo = 0 for double)
    const double r2h = sizeof(R) == 4 ? (double)0.70710677f : 0.70710678118654752440;
    const double r2l = sizeof(R) == 4 ? 0.70710678118654752440 - (double)0.70710677f : 0.0;
    C a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      a[r] = cadd(x[r], x[r + 4]);
      b[r] = csub(x[r], x[r + 4]);
    }
    // b_r *= W8^r, W8 = exp(S 2 pi i / 8)
    b[1] = Tw<C>::scale(cadd(b[1], cmul_is<S>(b[1])), r2h, r2l);
    b[2] = cmul_is<S>(b[2]);
    b[3] = Tw<C>::scale(csub(cmul_is<S>(b[3]), b[3]), r2h, r2l);
    Dft<4, S, C>::run(a);
    Dft<4, S, C>::run(b);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      x[2 * q] = a[q];
      x[2 * q + 1] = b[q];
    }
  }
};

// 16 points as 4 x 4: radix-4 over a of x[4a+b], twiddle W16^(b c), radix-4 over b
// (y[c + 4d] = sum_b W4^(bd) W16^(bc) sum_a W4^(ac) x[4a+b]).  Constants in the field
// precision (the fused transforms only).
template <int S, typename C> struct Dft<16, S, C> {
  static __device__ __forceinline__ void run(C* x) {
    using R = decltype(x[0].x);
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173, r2 = (R)0.70710678118654752440;
    C t[16];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      C v[4] = {x[b], x[4 + b], x[8 + b], x[12 + b]};
      Dft<4, S, C>::run(v);
#pragma unroll
      for (int c = 0; c < 4; ++c) t[4 * b + c] = v[c];
    }
    // W16^k = (cos, S sin)(2 pi k / 16) for the exponents b*c in {1, 2, 3, 4, 6, 9}
    auto w = [&](C v, R cr, R ci) { return mk(v.x * cr - v.y * ci, v.x * ci + v.y * cr); };
    const R sg = (R)S;
    t[5] = w(t[5], c1, sg * s1);        // b=1 c=1: W^1
    t[6] = w(t[6], r2, sg * r2);        // b=1 c=2: W^2
    t[7] = w(t[7], s1, sg * c1);        // b=1 c=3: W^3
    t[9] = w(t[9], r2, sg * r2);        // b=2 c=1: W^2
    t[10] = cmul_is<S>(t[10]);          // b=2 c=2: W^4 = S i
    t[11] = w(t[11], -r2, sg * r2);     // b=2 c=3: W^6
    t[13] = w(t[13], s1, sg * c1);      // b=3 c=1: W^3
    t[14] = w(t[14], -r2, sg * r2);     // b=3 c=2: W^6
    t[15] = w(t[15], -c1, -sg * s1);    // b=3 c=3: W^9
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      C v[4] = {t[c], t[4 + c], t[8 + c], t[12 + c]};
      Dft<4, S, C>::run(v);
#pragma unroll
      for (int d = 0; d < 4; ++d) x[c + 4 * d] = v[d];
    }
  }
};

// ----------------------------------------------------------------- stages
// Lines of a batch: element e of line l sits at buf[l*ls + e*es].
template <typename C, int R>
__device__ __forceinline__ void dif_stage(C* buf, int span, int L, int nlines, int ls, int es, const C* __restrict__ tw) {
  const int m = span / R, nbf = nlines * (L / R), tws = L / span;
  for (int t = threadIdx.x; t < nbf; t += blockDim.x) {
    const int line = t % nlines, u = t / nlines, j = u % m, b = u / m;
    C* base = buf + line * ls + (b * span + j) * es;
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = base[r * m * es];
    Dft<R, -1, C>::run(x);
#pragma unroll
    for (int q = 1; q < R; ++q) x[q] = Tw<C>::mul(x[q], tw, j * q * tws, L);
#pragma unroll
    for (int q = 0; q < R; ++q) base[q * m * es] = x[q];
  }
}

template <typename C, int R>
__device__ __forceinline__ void dit_stage(C* buf, int span, int L, int nlines, int ls, int es, const C* __restrict__ tw) {
  const int m = span / R, nbf = nlines * (L / R), tws = L / span;
  for (int t = threadIdx.x; t < nbf; t += blockDim.x) {
    const int line = t % nlines, u = t / nlines, j = u % m, b = u / m;
    C* base = buf + line * ls + (b * span + j) * es;
    C x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) x[q] = base[q * m * es];
#pragma unroll
    for (int q = 1; q < R; ++q) x[q] = Tw<C>::mulc(x[q], tw, j * q * tws, L);
    Dft<R, 1, C>::run(x);
#pragma unroll
    for (int r = 0; r < R; ++r) base[r * m * es] = x[r];
  }
}

// Forward (DIF): natural -> digit reversed.  Caller syncs before; this syncs after.
template <typename C>
__device__ void fft_dif(C* buf, const LinePlan& pl, int nlines, int ls, int es) {
  const C* tw = (const C*)pl.tw;
  int span = pl.L;
  for (int s = 0; s < pl.ns; ++s) {
    switch (pl.r[s]) {
      case 8: dif_stage<C, 8>(buf, span, pl.L, nlines, ls, es, tw); break;
      case 4: dif_stage<C, 4>(buf, span, pl.L, nlines, ls, es, tw); break;
      case 3: dif_stage<C, 3>(buf, span, pl.L, nlines, ls, es, tw); break;
      default: dif_stage<C, 2>(buf, span, pl.L, nlines, ls, es, tw); break;
    }
    span /= pl.r[s];
    __syncthreads();
  }
}

// Inverse (DIT, unscaled): digit reversed -> natural.
template <typename C>
__device__ void fft_dit(C* buf, const LinePlan& pl, int nlines, int ls, int es) {
  const C* tw = (const C*)pl.tw;
  int spans[12];
  int span = pl.L;
  for (int s = 0; s < pl.ns; ++s) {
    spans[s] = span;
    span /= pl.r[s];
  }
  for (int s = pl.ns - 1; s >= 0; --s) {
    switch (pl.r[s]) {
      case 8: dit_stage<C, 8>(buf, spans[s], pl.L, nlines, ls, es, tw); break;
      case 4: dit_stage<C, 4>(buf, spans[s], pl.L, nlines, ls, es, tw); break;
      case 3: dit_stage<C, 3>(buf, spans[s], pl.L, nlines, ls, es, tw); break;
      default: dit_stage<C, 2>(buf, spans[s], pl.L, nlines, ls, es, tw); break;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ host side
struct FFTPlan3;  // defined in fft.cu

// Plan of a 3-D real transform of one grid (twiddle tables live on the device).
class FFT3 {
 public:
  // table_mem == NULL: the plan allocates its twiddle/digit tables with
  // cudaMalloc.  Otherwise the tables are copied into table_mem (device memory
  // of table_cap bytes owned by the caller) and the plan allocates nothing.
  FFT3(int nx, int ny, int nz, bool fp64, void* table_mem = nullptr, size_t table_cap = 0);
  static size_t table_bytes(int nx, int ny, int nz, bool fp64);
  ~FFT3();
  FFT3(const FFT3&) = delete;
  FFT3& operator=(const FFT3&) = delete;

  int nx, ny, nz, nxh;
  int64_t n3() const { return (int64_t)nx * ny * nz; }
  int64_t nk() const { return (int64_t)nz * ny * nxh; }

  // f_trans on nf fields: real in[f] -> spectrum out[f] (scaled by 1/n3).
  template <typename R>
  void forward(const PtrList<const R>& in, const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const;
  // inv_trans on nf fields: spectrum in[f] -> real out[f].  in[f] is used as
  // scratch and holds garbage afterwards.
  template <typename R>
  void inverse(const PtrList<cplx<R>>& in, const PtrList<R>& out, int nf, cudaStream_t st) const;
  // the y and z passes alone (forward: after the x pass, scaled; inverse: before it),
  // for callers that do the x pass themselves
  template <typename R>
  void forward_cols(const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const;
  template <typename R>
  void inverse_cols(const PtrList<cplx<R>>& in, int nf, cudaStream_t st) const;
  // single passes: x forward (real in, spectrum rows out), x inverse (spectrum rows
  // in, used as scratch; real out), y and z in place
  template <typename R>
  void forward_x(const PtrList<const R>& in, const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const;
  template <typename R>
  void inverse_x(const PtrList<cplx<R>>& in, const PtrList<R>& out, int nf, cudaStream_t st) const;
  template <typename R>
  void pass_y(const PtrList<cplx<R>>& buf, int nf, bool fwd, cudaStream_t st) const;
  template <typename R>
  void pass_z(const PtrList<cplx<R>>& buf, int nf, bool fwd, cudaStream_t st) const;

  LinePlan px, py, pz;  // px: length nx/2 (complex half-length transform)
  // radix plan of the compile-time kernels (power-of-two lengths 32..512): 0 = radix 8
  // first, 2 = radix 16 first (one shared-memory pass fewer, more registers)
  int pv = 0;
  // columns per block of the compile-time column kernels: ct = 1 about 32 KB of tile,
  // ct = 2 twice as many columns (longer contiguous runs, fewer blocks per SM)
  int ct = 1;
  LaunchHook* hook = nullptr;
  const void* post_tw;  // cplx<R>[nx/2+1]: exp(-2 pi i k / nx)
  bool fp64;

 private:
  void* dev_mem = nullptr;
  bool owns_mem = false;
};

bool fft_size_ok(int n, bool is_x);

}  // namespace meu
