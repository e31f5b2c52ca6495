// fft.cu -- batched 3-D R2C / C2R transforms (see fft.cuh).
#include <cmath>
#include <type_traits>
#include <vector>

#include "fft.cuh"
#include "fft_stages.cuh"
#include "fused.cuh"

namespace meu {

static bool factor_23(int n, std::vector<int>& r) {
  r.clear();
  while (n % 8 == 0 && n > 8) { r.push_back(8); n /= 8; }
  if (n % 8 == 0) { r.push_back(8); n /= 8; }
  if (n % 4 == 0) { r.push_back(4); n /= 4; }
  if (n % 2 == 0) { r.push_back(2); n /= 2; }
  while (n % 3 == 0) { r.push_back(3); n /= 3; }
  return n == 1;
}

bool fft_size_ok(int n, bool is_x) {
  std::vector<int> r;
  if (is_x) return n >= 4 && n % 2 == 0 && n <= 2048 && factor_23(n / 2, r);
  return n >= 2 && n <= 1024 && factor_23(n, r);
}

// digit-reversal map of the DIF stage order (position p -> frequency k)
static std::vector<int> rev_table(int L, const std::vector<int>& rad) {
  std::vector<int> out(L);
  std::vector<int> m(rad.size());
  int span = L;
  for (size_t s = 0; s < rad.size(); ++s) { span /= rad[s]; m[s] = span; }
  for (int k = 0; k < L; ++k) {
    // k = q0 + R0*(q1 + R1*(q2 + ...)) ; p = sum q_s * m_s
    int kk = k, p = 0;
    for (size_t s = 0; s < rad.size(); ++s) {
      int q = kk % rad[s];
      kk /= rad[s];
      p += q * m[s];
    }
    out[p] = k;
  }
  return out;
}

// exp(-2 pi i n / L) with long-double argument reduction; exact at multiples of L/4
static void twiddle(int n, int L, long double& c, long double& s) {
  n %= L;
  if (4 * n % L == 0) {
    int q = 4 * n / L;
    c = (q == 0) ? 1 : (q == 2) ? -1 : 0;
    s = (q == 1) ? -1 : (q == 3) ? 1 : 0;
    return;
  }
  const long double pi = 3.141592653589793238462643383279502884L;
  long double a = -2.0L * pi * (long double)n / (long double)L;
  c = cosl(a);
  s = sinl(a);
}

size_t FFT3::table_bytes(int nx, int ny, int nz, bool fp64) {
  const size_t csz = fp64 ? sizeof(double2) : sizeof(float2);
  const int K = 1;
  return ((size_t)nx / 2 + ny + nz + nx / 2 + 1) * K * csz + sizeof(int) * ((size_t)nx / 2 + ny + nz) + 256;
}

FFT3::FFT3(int nx_, int ny_, int nz_, bool fp64_, void* table_mem, size_t table_cap)
    : nx(nx_), ny(ny_), nz(nz_), nxh(nx_ / 2 + 1), fp64(fp64_) {
  std::vector<int> rx, ry, rz;
  if (!(nx % 2 == 0 && factor_23(nx / 2, rx) && factor_23(ny, ry) && factor_23(nz, rz)))
    throw CudaError("grid sizes must be 2^a 3^b (Nx even)", 100);
  const int Lx = nx / 2;
  auto rvx = rev_table(Lx, rx), rvy = rev_table(ny, ry), rvz = rev_table(nz, rz);
  const size_t csz = fp64 ? sizeof(double2) : sizeof(float2);
  const int K = 1;  // one correctly rounded entry per twiddle
  // layout: twx[Lx*K] twy[ny*K] twz[nz*K] post[nxh*K] | revx revy revz
  size_t ntw = ((size_t)Lx + ny + nz + nxh) * K;
  size_t bytes_tw = ntw * csz;
  size_t bytes = bytes_tw + sizeof(int) * ((size_t)Lx + ny + nz) + 256;
  std::vector<unsigned char> host(bytes, 0);
  auto put_table = [&](size_t base, int n_entries, int L) {
    for (int n = 0; n < n_entries; ++n) {
      long double c, s;
      twiddle(n, L, c, s);
      if (fp64) {
        double2 v = make_double2((double)c, (double)s);
        memcpy(host.data() + (base + n) * csz, &v, csz);
      } else {
        float2 v = make_float2((float)(double)c, (float)(double)s);
        memcpy(host.data() + (base + n) * csz, &v, csz);
      }
    }
  };
  const size_t ox = 0, oy = (size_t)Lx * K, oz = oy + (size_t)ny * K, op = oz + (size_t)nz * K;
  put_table(ox, Lx, Lx);
  put_table(oy, ny, ny);
  put_table(oz, nz, nz);
  put_table(op, nxh, nx);
  int* ri = (int*)(host.data() + bytes_tw);
  memcpy(ri, rvx.data(), sizeof(int) * Lx);
  memcpy(ri + Lx, rvy.data(), sizeof(int) * ny);
  memcpy(ri + Lx + ny, rvz.data(), sizeof(int) * nz);
  if (table_mem) {
    if (bytes > table_cap) throw CudaError("transform tables exceed the provided memory", 103);
    dev_mem = table_mem;
    owns_mem = false;
  } else {
    MEU_CUDA(cudaMalloc(&dev_mem, bytes));
    owns_mem = true;
  }
  MEU_CUDA(cudaMemcpy(dev_mem, host.data(), bytes, cudaMemcpyHostToDevice));
  unsigned char* d = (unsigned char*)dev_mem;
  const int* dr = (const int*)(d + bytes_tw);
  auto fill = [](LinePlan& p, int L, const std::vector<int>& r, const void* tw, const int* rev) {
    p.L = L;
    p.ns = (int)r.size();
    for (int i = 0; i < 12; ++i) p.r[i] = i < (int)r.size() ? r[i] : 1;
    p.tw = tw;
    p.rev = rev;
  };
  fill(px, Lx, rx, d + ox * csz, dr);
  fill(py, ny, ry, d + oy * csz, dr + Lx);
  fill(pz, nz, rz, d + oz * csz, dr + Lx + ny);
  post_tw = d + op * csz;
}

FFT3::~FFT3() {
  if (dev_mem && owns_mem) cudaFree(dev_mem);
}

// ------------------------------------------------------------------ kernels
__host__ __device__ inline int odd_pitch(int L) { return (L & 1) ? L : L + 1; }
__host__ __device__ inline int rows_per_block(int L) {
  int r = 2048 / L;
  return r < 1 ? 1 : (r > 64 ? 64 : r);
}

// x transform: rows of nx reals -> rows of nx/2+1 complex (unscaled)
template <typename R>
__global__ void __launch_bounds__(256) k_rows_r2c(PtrList<const R> in, PtrList<cplx<R>> out, int nx, int64_t nrows,
                                                  LinePlan pl, const cplx<R>* __restrict__ post) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int L = pl.L, pitch = odd_pitch(L), nxh = L + 1;
  const int rpb = rows_per_block(L);
  const int64_t row0 = (int64_t)blockIdx.x * rpb;
  const int nr = (int)min((int64_t)rpb, nrows - row0);
  const R* src = in.p[blockIdx.y] + row0 * nx;
  C* dst = out.p[blockIdx.y] + row0 * nxh;
  // asynchronous copies: every load of the tile is in flight at once
  for (int i = threadIdx.x; i < nr * L; i += blockDim.x) {
    int r = i / L, n = i - r * L;
    fz::cp_async_c(buf + r * pitch + n, (const C*)(src + (int64_t)r * nx) + n);
  }
  fz::cp_async_wait_all();
  __syncthreads();
  fft_dif(buf, pl, nr, pitch, 1);
  // split: X[k] = E + W^k O with E = (Z[k] + conj Z[L-k])/2, O = -i (Z[k] - conj Z[L-k])/2
  const int* rev = pl.rev;
  const int npair = L / 2 + 1;
  __shared__ int posk[1024];
  for (int i = threadIdx.x; i < L; i += blockDim.x) posk[rev[i]] = i;
  __syncthreads();
  for (int i = threadIdx.x; i < nr * npair; i += blockDim.x) {
    int r = i / npair, k = i - r * npair;
    int k2 = (L - k) % L;
    C zk = buf[r * pitch + posk[k % L]], zm = buf[r * pitch + posk[k2]];
    C* drow = dst + (int64_t)r * nxh;
    {
      C e = cscale(cadd(zk, cconj(zm)), (R)0.5);
      C o = cscale(csub(zk, cconj(zm)), (R)0.5);
      o = mk(o.y, -o.x);
      drow[k] = cadd(e, Tw<C>::mul(o, post, k, nxh));
    }
    if (k != L - k) {
      C e = cscale(cadd(zm, cconj(zk)), (R)0.5);
      C o = cscale(csub(zm, cconj(zk)), (R)0.5);
      o = mk(o.y, -o.x);
      drow[L - k] = cadd(e, Tw<C>::mul(o, post, L - k, nxh));
    }
  }
}

// x inverse: rows of nx/2+1 complex -> rows of nx reals (unscaled c2r)
template <typename R>
__global__ void __launch_bounds__(256) k_rows_c2r(PtrList<const cplx<R>> in, PtrList<R> out, int nx, int64_t nrows,
                                                  LinePlan pl, const cplx<R>* __restrict__ post) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int L = pl.L, pitch = odd_pitch(L), nxh = L + 1;
  const int rpb = rows_per_block(L);
  const int64_t row0 = (int64_t)blockIdx.x * rpb;
  const int nr = (int)min((int64_t)rpb, nrows - row0);
  const C* src = in.p[blockIdx.y] + row0 * nxh;
  R* dst = out.p[blockIdx.y] + row0 * nx;
  __shared__ int posk[1024];
  for (int i = threadIdx.x; i < L; i += blockDim.x) posk[pl.rev[i]] = i;
  __syncthreads();
  const int npair = L / 2 + 1;
#pragma unroll 4
  for (int i = threadIdx.x; i < nr * npair; i += blockDim.x) {
    int r = i / npair, k = i - r * npair;
    const C* srow = src + (int64_t)r * nxh;
    C xk = srow[k], xm = srow[L - k];
    if (k == 0) { xk.y = 0; xm.y = 0; }
    // Z[k] = (X[k] + conj X[L-k]) + i (X[k] - conj X[L-k]) W^-k
    {
      C ex = cadd(xk, cconj(xm));
      C ox = Tw<C>::mulc(csub(xk, cconj(xm)), post, k, nxh);
      buf[r * pitch + posk[k % L]] = cadd(ex, mk(-ox.y, ox.x));
    }
    if (k != 0 && k != L - k) {
      C ex = cadd(xm, cconj(xk));
      C ox = Tw<C>::mulc(csub(xm, cconj(xk)), post, L - k, nxh);
      buf[r * pitch + posk[L - k]] = cadd(ex, mk(-ox.y, ox.x));
    }
  }
  __syncthreads();
  fft_dit(buf, pl, nr, pitch, 1);
  for (int i = threadIdx.x; i < nr * L; i += blockDim.x) {
    int r = i / L, n = i - r * L;
    ((C*)(dst + (int64_t)r * nx))[n] = buf[r * pitch + n];
  }
}

// strided columns: element l of column (o, c) at base + o*ostride + l*inner + c.
// FWD: natural in -> natural out (DIF + reversed store), scaled.
// INV: natural in -> natural out (reversed load + DIT).
template <typename R, bool FWD>
__global__ void __launch_bounds__(256) k_cols(PtrList<cplx<R>> in, PtrList<cplx<R>> out, int inner, int64_t ostride,
                                              int tm, LinePlan pl, R scale) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int L = pl.L;
  const int tiles = (inner + tm - 1) / tm;
  const int o = blockIdx.x / tiles, t = blockIdx.x - o * tiles;
  const int c0 = t * tm, nc = min(tm, inner - c0);
  const C* src = in.p[blockIdx.y] + (int64_t)o * ostride + c0;
  C* dst = out.p[blockIdx.y] + (int64_t)o * ostride + c0;
  const int* rev = pl.rev;
  for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
    int l = i / nc, c = i - l * nc;
    int gl = FWD ? l : rev[l];
    fz::cp_async_c(buf + l * tm + c, src + (int64_t)gl * inner + c);
  }
  fz::cp_async_wait_all();
  __syncthreads();
  if (FWD) fft_dif(buf, pl, nc, 1, tm);
  else fft_dit(buf, pl, nc, 1, tm);
  for (int i = threadIdx.x; i < L * nc; i += blockDim.x) {
    int l = i / nc, c = i - l * nc;
    int gl = FWD ? rev[l] : l;
    C v = buf[l * tm + c];
    if (FWD) v = cscale(v, scale);
    dst[(int64_t)gl * inner + c] = v;
  }
}

// ----------------------------------------------- compile-time specialisations
// The same transforms with the length, radix plan and line count as template
// constants (stage_io of fft_stages.cuh on the radix plans of fused.cuh): index
// arithmetic folds to shifts and constant multiplies, and the digit reversal is
// computed instead of read from the table.  Lengths 32..512 (powers of two) take
// these; other lengths keep the run-time plan above.
constexpr int rows_per_block_c(int L) { return 2048 / L < 1 ? 1 : (2048 / L > 64 ? 64 : 2048 / L); }

// Rows interleaved in shared memory: element e of row r at e * ES + r with the odd
// stride ES = NR + 1, so that runs of consecutive e and runs of consecutive r both
// spread over the banks.  The global-facing stage walks consecutive elements of a
// row (JFAST); the stage next to the split step permutes between digit-reversed
// positions and natural frequency order (HOLD), so the split reads and writes
// consecutive frequencies, in shared and in global memory alike.
template <typename R, int L, int PV>
__global__ void __launch_bounds__(256) k_rows_r2c_s(PtrList<const R> in, PtrList<cplx<R>> out, int64_t nrows,
                                                    const cplx<R>* __restrict__ tw, const cplx<R>* __restrict__ post) {
  using C = cplx<R>;
  constexpr int NR = rows_per_block_c(L), ES = NR + 1, NXH = L + 1, NP = L / 2 + 1;
  constexpr int NS = fz::rplan(L, PV).ns;
  static_assert(NS >= 2, "first and last stage must differ");
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int64_t row0 = (int64_t)blockIdx.x * NR;
  const int nr = (int)min((int64_t)NR, nrows - row0);
  const C* src = (const C*)(in.p[blockIdx.y] + row0 * (2 * L));
  C* dst = out.p[blockIdx.y] + row0 * NXH;
  // a row of 2L reals is L complex pairs (rows past nr read row 0, never stored)
  stage_io<C, L, 0, NR, 256, PV, true, true>(
      tw, [&](int r, int e) { return src[(int64_t)(r < nr ? r : 0) * L + e]; },
      [&](int r, int e, C v) { buf[e * ES + r] = v; });
  __syncthreads();
  stages_smem<C, L, NR, ES, 256, PV, true, 1, NS - 1>(buf, tw);
  // last stage: position e holds frequency rev(e); store it at its frequency
  stage_io<C, L, NS - 1, NR, 256, PV, true, false, true>(
      tw, [&](int r, int e) { return buf[e * ES + r]; },
      [&](int r, int e, C v) { buf[fz::rev<L, PV>(e) * ES + r] = v; });
  __syncthreads();
  // split: X[k] = E + W^k O with E = (Z[k] + conj Z[L-k])/2, O = -i (Z[k] - conj Z[L-k])/2
  for (int i = threadIdx.x; i < NR * NP; i += 256) {
    const int r = i / NP, k = i - r * NP;
    if (r >= nr) continue;
    const int km = k == 0 ? 0 : L - k;
    const C zk = buf[k * ES + r], zm = buf[km * ES + r];
    C* drow = dst + (int64_t)r * NXH;
    {
      C e = cscale(cadd(zk, cconj(zm)), (R)0.5);
      C o = cscale(csub(zk, cconj(zm)), (R)0.5);
      o = mk(o.y, -o.x);
      drow[k] = cadd(e, Tw<C>::mul(o, post, k, NXH));
    }
    if (k != L - k) {
      C e = cscale(cadd(zm, cconj(zk)), (R)0.5);
      C o = cscale(csub(zm, cconj(zk)), (R)0.5);
      o = mk(o.y, -o.x);
      drow[L - k] = cadd(e, Tw<C>::mul(o, post, L - k, NXH));
    }
  }
}

template <typename R, int L, int PV>
__global__ void __launch_bounds__(256) k_rows_c2r_s(PtrList<const cplx<R>> in, PtrList<R> out, int64_t nrows,
                                                    const cplx<R>* __restrict__ tw, const cplx<R>* __restrict__ post) {
  using C = cplx<R>;
  constexpr int NR = rows_per_block_c(L), ES = NR + 1, NXH = L + 1, NP = L / 2 + 1;
  constexpr int NS = fz::rplan(L, PV).ns;
  static_assert(NS >= 2, "first and last stage must differ");
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int64_t row0 = (int64_t)blockIdx.x * NR;
  const int nr = (int)min((int64_t)NR, nrows - row0);
  const C* src = in.p[blockIdx.y] + row0 * NXH;
  C* dst = (C*)(out.p[blockIdx.y] + row0 * (2 * L));
  // Z[k] = (X[k] + conj X[L-k]) + i (X[k] - conj X[L-k]) W^-k, in natural order
  for (int i = threadIdx.x; i < NR * NP; i += 256) {
    const int r = i / NP, k = i - r * NP;
    if (r >= nr) continue;
    const C* srow = src + (int64_t)r * NXH;
    C xk = srow[k], xm = srow[L - k];
    if (k == 0) { xk.y = 0; xm.y = 0; }
    {
      C ex = cadd(xk, cconj(xm));
      C ox = Tw<C>::mulc(csub(xk, cconj(xm)), post, k, NXH);
      buf[k * ES + r] = cadd(ex, mk(-ox.y, ox.x));
    }
    if (k != 0 && k != L - k) {
      C ex = cadd(xm, cconj(xk));
      C ox = Tw<C>::mulc(csub(xm, cconj(xk)), post, L - k, NXH);
      buf[(L - k) * ES + r] = cadd(ex, mk(-ox.y, ox.x));
    }
  }
  __syncthreads();
  // first DIT stage: position e takes frequency rev(e)
  stage_io<C, L, NS - 1, NR, 256, PV, false, false, true>(
      tw, [&](int r, int e) { return buf[fz::rev<L, PV>(e) * ES + r]; },
      [&](int r, int e, C v) { buf[e * ES + r] = v; });
  __syncthreads();
  stages_smem<C, L, NR, ES, 256, PV, false, NS - 2, 0>(buf, tw);
  stage_io<C, L, 0, NR, 256, PV, false, true>(
      tw, [&](int r, int e) { return buf[e * ES + r]; },
      [&](int r, int e, C v) {
        if (r < nr) dst[(int64_t)r * L + e] = v;
      });
}

// TM columns of length L per block; element l of column (o, c) at o*ostride + l*inner + c.
// The first stage reads its butterflies straight from global memory and the last
// writes straight to global memory (digit reversal and forward scale folded into
// the addressing); only the stages between them go through shared memory.
template <typename R, bool FWD, int L, int TM, int PV>
__global__ void __launch_bounds__(256) k_cols_s(PtrList<cplx<R>> in, PtrList<cplx<R>> out, int inner, int64_t ostride,
                                                const cplx<R>* __restrict__ tw, R scale) {
  using C = cplx<R>;
  constexpr int NS = fz::rplan(L, PV).ns;
  static_assert(NS >= 2, "first and last stage must differ");
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int tiles = (inner + TM - 1) / TM;
  const int o = blockIdx.x / tiles, t = blockIdx.x - o * tiles;
  const int c0 = t * TM, nc = min(TM, inner - c0);
  const C* src = in.p[blockIdx.y] + (int64_t)o * ostride + c0;
  C* dst = out.p[blockIdx.y] + (int64_t)o * ostride + c0;
  // lines past nc (a partial last tile) read column 0 and are never stored
  auto gld = [&](int l, int e) {
    const int c = l < nc ? l : 0;
    return src[(int64_t)(FWD ? e : fz::rev<L, PV>(e)) * inner + c];
  };
  auto sst = [&](int l, int e, C v) { buf[e * TM + l] = v; };
  auto sld = [&](int l, int e) { return buf[e * TM + l]; };
  auto gst = [&](int l, int e, C v) {
    if (l < nc) dst[(int64_t)(FWD ? fz::rev<L, PV>(e) : e) * inner + l] = FWD ? cscale(v, scale) : v;
  };
  if constexpr (FWD) {
    stage_io<C, L, 0, TM, 256, PV, true>(tw, gld, sst);
    __syncthreads();
    stages_smem<C, L, TM, TM, 256, PV, true, 1, NS - 1>(buf, tw);
    stage_io<C, L, NS - 1, TM, 256, PV, true>(tw, sld, gst);
  } else {
    stage_io<C, L, NS - 1, TM, 256, PV, false>(tw, gld, sst);
    __syncthreads();
    stages_smem<C, L, TM, TM, 256, PV, false, NS - 2, 0>(buf, tw);
    stage_io<C, L, 0, TM, 256, PV, false>(tw, sld, gst);
  }
}

// Raise a kernel's dynamic shared-memory limit to the opt-in maximum once
// (227 KB per block on sm_100 minus the kernel's static shared memory).
template <typename R>
static void set_smem(const void* fn, size_t bytes) {
  // always: without the opt-in, dynamic plus static shared memory must stay within 48 KB
  if ((int)bytes > smem_optin(fn)) throw CudaError("transform tile exceeds shared memory", 103);
}

// columns per block of the specialised column kernels: about 32 KB of tile
template <typename R>
constexpr int col_tile_s(int L) {
  const int t = 32768 / (L * 2 * (int)sizeof(R));
  return t < 4 ? 4 : (t > 16 ? 16 : t);
}

// Call go(length, plan) as integral constants for the lengths with compile-time
// kernels; false when L has none.  Launch helpers for those kernels follow.
template <typename F>
static bool dispatch_len(int L, int pv, F&& go) {
  auto with_pv = [&](auto Lc) {
    return pv == 2 ? go(Lc, std::integral_constant<int, 2>{}) : go(Lc, std::integral_constant<int, 0>{});
  };
  switch (L) {
    case 32: return with_pv(std::integral_constant<int, 32>{});
    case 64: return with_pv(std::integral_constant<int, 64>{});
    case 128: return with_pv(std::integral_constant<int, 128>{});
    case 256: return with_pv(std::integral_constant<int, 256>{});
    case 512: return with_pv(std::integral_constant<int, 512>{});
    default: return false;
  }
}

template <typename R>
static bool rows_s(bool fwd, int L, int pv, int nf, int64_t nrows, const void* in, const void* out, const void* tw,
                   const void* post, cudaStream_t st) {
  using C = cplx<R>;
  auto go = [&](auto Lc, auto Pc) {
    constexpr int LL = decltype(Lc)::value, PV = decltype(Pc)::value;
    constexpr int NR = rows_per_block_c(LL);
    const size_t sm = (size_t)(NR + 1) * LL * sizeof(C);
    const dim3 g((unsigned)((nrows + NR - 1) / NR), nf);
    if (fwd) {
      set_smem<R>((const void*)k_rows_r2c_s<R, LL, PV>, sm);
      k_rows_r2c_s<R, LL, PV><<<g, 256, sm, st>>>(*(const PtrList<const R>*)in, *(const PtrList<C>*)out, nrows,
                                                   (const C*)tw, (const C*)post);
    } else {
      set_smem<R>((const void*)k_rows_c2r_s<R, LL, PV>, sm);
      k_rows_c2r_s<R, LL, PV><<<g, 256, sm, st>>>(*(const PtrList<const C>*)in, *(const PtrList<R>*)out, nrows,
                                                   (const C*)tw, (const C*)post);
    }
    return true;
  };
  return dispatch_len(L, pv, go);
}

template <typename R, bool FWD>
static bool cols_s(int L, int pv, int ct, int nf, int outer, int inner, int64_t ostride, const PtrList<cplx<R>>& buf,
                   const void* tw, R scale, cudaStream_t st) {
  using C = cplx<R>;
  auto go = [&](auto Lc, auto Pc) {
    constexpr int LL = decltype(Lc)::value, PV = decltype(Pc)::value;
    auto launch = [&](auto Tc) {
      constexpr int TM = decltype(Tc)::value;
      const size_t sm = (size_t)LL * TM * sizeof(C);
      set_smem<R>((const void*)k_cols_s<R, FWD, LL, TM, PV>, sm);
      const dim3 g((unsigned)(outer * ((inner + TM - 1) / TM)), nf);
      k_cols_s<R, FWD, LL, TM, PV><<<g, 256, sm, st>>>(buf, buf, inner, ostride, (const C*)tw, scale);
      return true;
    };
    constexpr int TM1 = col_tile_s<R>(LL);
    return ct == 2 ? launch(std::integral_constant<int, 2 * TM1>{}) : launch(std::integral_constant<int, TM1>{});
  };
  return dispatch_len(L, pv, go);
}

static inline int col_tile(int L, bool fp64) {
  if (fp64) return L >= 256 ? 8 : 16;
  return 16;
}

struct HookScope {
  LaunchHook* h;
  cudaStream_t st;
  HookScope(LaunchHook* h_, const char* n, double b, cudaStream_t s) : h(h_), st(s) {
    if (h) h->begin(n, b, st);
  }
  ~HookScope() {
    if (h) h->end(st);
  }
};

template <typename R>
void FFT3::forward(const PtrList<const R>& in, const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const {
  forward_x<R>(in, out, nf, st);
  forward_cols<R>(out, nf, st);
}

template <typename R>
void FFT3::forward_x(const PtrList<const R>& in, const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const {
  using C = cplx<R>;
  const int Lx = px.L;
  const int64_t nrows = (int64_t)ny * nz;
  const int rpb = rows_per_block(Lx);
  size_t sm = (size_t)rpb * odd_pitch(Lx) * sizeof(C);
  set_smem<R>((const void*)k_rows_r2c<R>, sm);
  dim3 g((unsigned)((nrows + rpb - 1) / rpb), nf);
  { HookScope hs_(hook, "fft_x_r2c", (double)nf * (n3() * sizeof(R) + nk() * sizeof(C)), st);
  if (!rows_s<R>(true, Lx, pv, nf, nrows, &in, &out, px.tw, post_tw, st))
    k_rows_r2c<R><<<g, 256, sm, st>>>(in, out, nx, nrows, px, (const C*)post_tw); }
  MEU_CHECK_LAUNCH();
}

template <typename R>
void FFT3::forward_cols(const PtrList<cplx<R>>& out, int nf, cudaStream_t st) const {
  pass_y<R>(out, nf, true, st);
  pass_z<R>(out, nf, true, st);
}

// y columns: outer = z, inner = nxh
template <typename R>
void FFT3::pass_y(const PtrList<cplx<R>>& buf, int nf, bool fwd, cudaStream_t st) const {
  using C = cplx<R>;
  const int tm = col_tile(ny, sizeof(R) == 8);
  const size_t s2 = (size_t)ny * tm * sizeof(C);
  const dim3 g2((unsigned)(nz * ((nxh + tm - 1) / tm)), nf);
  HookScope hs_(hook, fwd ? "fft_y_fwd" : "fft_y_inv", 2.0 * nf * nk() * sizeof(C), st);
  if (fwd) {
    if (!cols_s<R, true>(ny, pv, ct, nf, nz, nxh, (int64_t)ny * nxh, buf, py.tw, (R)1, st)) {
      set_smem<R>((const void*)k_cols<R, true>, s2);
      k_cols<R, true><<<g2, 256, s2, st>>>(buf, buf, nxh, (int64_t)ny * nxh, tm, py, (R)1);
    }
  } else {
    if (!cols_s<R, false>(ny, pv, ct, nf, nz, nxh, (int64_t)ny * nxh, buf, py.tw, (R)1, st)) {
      set_smem<R>((const void*)k_cols<R, false>, s2);
      k_cols<R, false><<<g2, 256, s2, st>>>(buf, buf, nxh, (int64_t)ny * nxh, tm, py, (R)1);
    }
  }
  MEU_CHECK_LAUNCH();
}

// z columns: outer = 1, inner = ny*nxh; the forward pass applies the 1/(Nx Ny Nz) scale
template <typename R>
void FFT3::pass_z(const PtrList<cplx<R>>& buf, int nf, bool fwd, cudaStream_t st) const {
  using C = cplx<R>;
  const int tm = col_tile(nz, sizeof(R) == 8);
  const size_t s3 = (size_t)nz * tm * sizeof(C);
  const int inner = ny * nxh;
  const dim3 g3((unsigned)((inner + tm - 1) / tm), nf);
  HookScope hs_(hook, fwd ? "fft_z_fwd" : "fft_z_inv", 2.0 * nf * nk() * sizeof(C), st);
  if (fwd) {
    const R scale = (R)(1.0 / ((double)nx * ny * nz));
    if (!cols_s<R, true>(nz, pv, ct, nf, 1, inner, 0, buf, pz.tw, scale, st)) {
      set_smem<R>((const void*)k_cols<R, true>, s3);
      k_cols<R, true><<<g3, 256, s3, st>>>(buf, buf, inner, 0, tm, pz, scale);
    }
  } else {
    if (!cols_s<R, false>(nz, pv, ct, nf, 1, inner, 0, buf, pz.tw, (R)1, st)) {
      set_smem<R>((const void*)k_cols<R, false>, s3);
      k_cols<R, false><<<g3, 256, s3, st>>>(buf, buf, inner, 0, tm, pz, (R)1);
    }
  }
  MEU_CHECK_LAUNCH();
}

template <typename R>
void FFT3::inverse(const PtrList<cplx<R>>& in, const PtrList<R>& out, int nf, cudaStream_t st) const {
  inverse_cols<R>(in, nf, st);
  inverse_x<R>(in, out, nf, st);
}

template <typename R>
void FFT3::inverse_cols(const PtrList<cplx<R>>& in, int nf, cudaStream_t st) const {
  pass_z<R>(in, nf, false, st);
  pass_y<R>(in, nf, false, st);
}

template <typename R>
void FFT3::inverse_x(const PtrList<cplx<R>>& in, const PtrList<R>& out, int nf, cudaStream_t st) const {
  using C = cplx<R>;
  const int Lx = px.L;
  const int64_t nrows = (int64_t)ny * nz;
  const int rpb = rows_per_block(Lx);
  size_t sm = (size_t)rpb * odd_pitch(Lx) * sizeof(C);
  set_smem<R>((const void*)k_rows_c2r<R>, sm);
  PtrList<const C> cin;
  for (int f = 0; f < MAXF; ++f) cin.p[f] = in.p[f];
  dim3 g((unsigned)((nrows + rpb - 1) / rpb), nf);
  { HookScope hs_(hook, "fft_x_c2r", (double)nf * (n3() * sizeof(R) + nk() * sizeof(C)), st);
  if (!rows_s<R>(false, Lx, pv, nf, nrows, &cin, &out, px.tw, post_tw, st))
    k_rows_c2r<R><<<g, 256, sm, st>>>(cin, out, nx, nrows, px, (const C*)post_tw); }
  MEU_CHECK_LAUNCH();
}

template void FFT3::forward<float>(const PtrList<const float>&, const PtrList<float2>&, int, cudaStream_t) const;
template void FFT3::forward<double>(const PtrList<const double>&, const PtrList<double2>&, int, cudaStream_t) const;
template void FFT3::inverse<float>(const PtrList<float2>&, const PtrList<float>&, int, cudaStream_t) const;
template void FFT3::inverse<double>(const PtrList<double2>&, const PtrList<double>&, int, cudaStream_t) const;
template void FFT3::forward_cols<float>(const PtrList<float2>&, int, cudaStream_t) const;
template void FFT3::forward_cols<double>(const PtrList<double2>&, int, cudaStream_t) const;
template void FFT3::inverse_cols<float>(const PtrList<float2>&, int, cudaStream_t) const;
template void FFT3::inverse_cols<double>(const PtrList<double2>&, int, cudaStream_t) const;
template void FFT3::forward_x<float>(const PtrList<const float>&, const PtrList<float2>&, int, cudaStream_t) const;
template void FFT3::forward_x<double>(const PtrList<const double>&, const PtrList<double2>&, int, cudaStream_t) const;
template void FFT3::inverse_x<float>(const PtrList<float2>&, const PtrList<float>&, int, cudaStream_t) const;
template void FFT3::inverse_x<double>(const PtrList<double2>&, const PtrList<double>&, int, cudaStream_t) const;
template void FFT3::pass_y<float>(const PtrList<float2>&, int, bool, cudaStream_t) const;
template void FFT3::pass_y<double>(const PtrList<double2>&, int, bool, cudaStream_t) const;
template void FFT3::pass_z<float>(const PtrList<float2>&, int, bool, cudaStream_t) const;
template void FFT3::pass_z<double>(const PtrList<double2>&, int, bool, cudaStream_t) const;

}  // namespace meu
