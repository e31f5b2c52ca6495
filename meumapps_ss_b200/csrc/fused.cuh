// fused.cuh -- compile-time shared-memory FFT building blocks for the fused
// step kernels (grids with Nx = Ny = Nz = N, N in {32, 48, 64, 96, 128}).
// Template parameter PV selects the radix plan (rplan), NT the threads of a block.
//
// Every transform length, radix plan, line count and stride is a template
// constant, so all index arithmetic folds to shifts and constant multiplies.
//
// Spectral layout of the fused path ("M-form"): a plane z of a field holds
// [p_y][c] with c in [0, N/2] (N/2+1 columns) where
//   c < N/2   holds kx = rev_x(c)   (digit-reversed order of the half-length x transform)
//   c = N/2   holds kx = N/2        (Nyquist)
//   p_y       holds ky = rev_y(p_y) (digit-reversed order of the y transform)
// The z-kernels transform columns in place and keep kz in digit-reversed order
// between their forward and inverse passes.  Nothing outside the fused step
// sees this layout.
#pragma once
#include "../../include/meu.h"
#include "common.cuh"
#include "fft.cuh"

namespace meu {
namespace fz {

struct RPlan {
  int ns;
  int r[8];
};
// Radix plans (product = L), three variants for the autotuner:
//   pv 0: radix 8 while the remainder does not end in a single factor 2
//         (128 = 8*4*4, not 8*8*2), then 4s, at most one 2, then 3s;
//   pv 1: radix 4 first (128 = 4*4*4*2), then at most one 2, then 3s;
//   pv 2: radix 16 first, then 8s, 4s, at most one 2, 3s (128 = 16*8: one
//         shared-memory pass fewer, more registers per butterfly).
__host__ __device__ constexpr int twos(int n) {
  int k = 0;
  while (n > 0 && n % 2 == 0) { n /= 2; ++k; }
  return k;
}
__host__ __device__ constexpr RPlan rplan(int L, int pv = 0) {
  RPlan p{0, {1, 1, 1, 1, 1, 1, 1, 1}};
  int n = L;
  if (pv == 2) {
    while (n % 16 == 0) { p.r[p.ns++] = 16; n /= 16; }
    while (n % 8 == 0) { p.r[p.ns++] = 8; n /= 8; }
  }
  if (pv == 0)
    while (n % 8 == 0 && twos(n / 8) != 1) { p.r[p.ns++] = 8; n /= 8; }
  while (n % 4 == 0) { p.r[p.ns++] = 4; n /= 4; }
  if (n % 2 == 0) { p.r[p.ns++] = 2; n /= 2; }
  while (n % 3 == 0) { p.r[p.ns++] = 3; n /= 3; }
  return p;
}
__host__ __device__ constexpr bool same_plan(int L, int pa, int pb) {
  const RPlan a = rplan(L, pa), b = rplan(L, pb);
  if (a.ns != b.ns) return false;
  for (int i = 0; i < a.ns; ++i)
    if (a.r[i] != b.r[i]) return false;
  return true;
}
__host__ __device__ constexpr int span_of(int L, int s, int pv) {
  int sp = L;
  for (int i = 0; i < s; ++i) sp /= rplan(L, pv).r[i];
  return sp;
}

// position after DIF -> frequency index
template <int L, int PV>
__device__ __forceinline__ int rev(int p) {
  constexpr RPlan pl = rplan(L, PV);
  int k = 0, mul = 1, span = L;
#pragma unroll
  for (int s = 0; s < pl.ns; ++s) {
    span /= pl.r[s];
    const int q = (p / span) % pl.r[s];
    k += q * mul;
    mul *= pl.r[s];
  }
  return k;
}
// frequency index -> position after DIF
template <int L, int PV>
__device__ __forceinline__ int pos(int k) {
  constexpr RPlan pl = rplan(L, PV);
  int p = 0, span = L;
#pragma unroll
  for (int s = 0; s < pl.ns; ++s) {
    span /= pl.r[s];
    p += (k % pl.r[s]) * span;
    k /= pl.r[s];
  }
  return p;
}

// One DIF stage over NL lines (element e of line l at buf[l*LS + e*ES]).
template <typename C, int L, int S, int NL, int LS, int ES, int NT, int PV>
__device__ __forceinline__ void dif_stage_s(C* buf, const C* __restrict__ tw) {
  constexpr int R = rplan(L, PV).r[S];
  constexpr int SPAN = span_of(L, S, PV);
  constexpr int M = SPAN / R, NBF = NL * (L / R), TWS = L / SPAN;
#pragma unroll 1
  for (int t = threadIdx.x; t < NBF; t += NT) {
    const int line = t % NL, u = t / NL, j = u % M, b = u / M;
    C* base = buf + line * LS + (b * SPAN + j) * ES;
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = base[r * M * ES];
    Dft<R, -1, C>::run(x);
    if (M > 1) {
#pragma unroll
      for (int q = 1; q < R; ++q) x[q] = Tw<C>::mul(x[q], tw, j * q * TWS, L);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) base[q * M * ES] = x[q];
  }
}
template <typename C, int L, int S, int NL, int LS, int ES, int NT, int PV>
__device__ __forceinline__ void dit_stage_s(C* buf, const C* __restrict__ tw) {
  constexpr int R = rplan(L, PV).r[S];
  constexpr int SPAN = span_of(L, S, PV);
  constexpr int M = SPAN / R, NBF = NL * (L / R), TWS = L / SPAN;
#pragma unroll 1
  for (int t = threadIdx.x; t < NBF; t += NT) {
    const int line = t % NL, u = t / NL, j = u % M, b = u / M;
    C* base = buf + line * LS + (b * SPAN + j) * ES;
    C x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) x[q] = base[q * M * ES];
    if (M > 1) {
#pragma unroll
      for (int q = 1; q < R; ++q) x[q] = Tw<C>::mulc(x[q], tw, j * q * TWS, L);
    }
    Dft<R, 1, C>::run(x);
#pragma unroll
    for (int r = 0; r < R; ++r) base[r * M * ES] = x[r];
  }
}

// One butterfly of DIF / DIT stage S on R elements held in registers; j is the
// butterfly's index within its span (the twiddle exponent base).  A task of
// stage S over one line is u in [0, L/R): j = u % M, b = u / M, and its elements
// sit at (b*SPAN + j) + r*M, r in [0, R).
template <int L, int S, int PV>
struct StageOf {
  static constexpr int R = rplan(L, PV).r[S];
  static constexpr int SPAN = span_of(L, S, PV);
  static constexpr int M = SPAN / R;
  static constexpr int TWS = L / SPAN;
  static constexpr int TASKS = L / R;
};
template <typename C, int L, int S, int PV>
__device__ __forceinline__ void dif_regs(C* x, const C* __restrict__ tw, int j) {
  using T = StageOf<L, S, PV>;
  Dft<T::R, -1, C>::run(x);
  if (T::M > 1) {
#pragma unroll
    for (int q = 1; q < T::R; ++q) x[q] = Tw<C>::mul(x[q], tw, j * q * T::TWS, L);
  }
}
template <typename C, int L, int S, int PV>
__device__ __forceinline__ void dit_regs(C* x, const C* __restrict__ tw, int j) {
  using T = StageOf<L, S, PV>;
  if (T::M > 1) {
#pragma unroll
    for (int q = 1; q < T::R; ++q) x[q] = Tw<C>::mulc(x[q], tw, j * q * T::TWS, L);
  }
  Dft<T::R, 1, C>::run(x);
}

// DIF stages S0 .. S1-1 (shared memory, sync after each); DIT stages S1-1 down to S0.
template <typename C, int L, int NL, int LS, int ES, int NT, int PV, int S, int S1>
__device__ __forceinline__ void dif_range(C* buf, const C* tw) {
  if constexpr (S < S1) {
    dif_stage_s<C, L, S, NL, LS, ES, NT, PV>(buf, tw);
    __syncthreads();
    dif_range<C, L, NL, LS, ES, NT, PV, S + 1, S1>(buf, tw);
  }
}
template <typename C, int L, int NL, int LS, int ES, int NT, int PV, int S0, int S>
__device__ __forceinline__ void dit_range(C* buf, const C* tw) {
  if constexpr (S >= S0) {
    dit_stage_s<C, L, S, NL, LS, ES, NT, PV>(buf, tw);
    __syncthreads();
    dit_range<C, L, NL, LS, ES, NT, PV, S0, S - 1>(buf, tw);
  }
}

// Forward DIF over all stages (natural -> digit reversed); syncs after each stage.
template <typename C, int L, int NL, int LS, int ES, int NT, int PV, int S = 0>
__device__ __forceinline__ void dif(C* buf, const C* tw) {
  if constexpr (S < rplan(L, PV).ns) {
    dif_stage_s<C, L, S, NL, LS, ES, NT, PV>(buf, tw);
    __syncthreads();
    dif<C, L, NL, LS, ES, NT, PV, S + 1>(buf, tw);
  }
}
// Inverse DIT over all stages (digit reversed -> natural), unscaled.
template <typename C, int L, int NL, int LS, int ES, int NT, int PV, int S = rplan(L, PV).ns - 1>
__device__ __forceinline__ void dit(C* buf, const C* tw) {
  if constexpr (S >= 0) {
    dit_stage_s<C, L, S, NL, LS, ES, NT, PV>(buf, tw);
    __syncthreads();
    dit<C, L, NL, LS, ES, NT, PV, S - 1>(buf, tw);
  }
}

// ------------------------------------------------------- asynchronous copies
// cp.async (global -> shared without staging through registers): every thread
// issues all of its copies before any wait, so a tile's loads are in flight together.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// copy one complex element (8 B for float2, 16 B for double2)
template <typename C>
__device__ __forceinline__ void cp_async_c(C* smem, const C* gmem) {
  if constexpr (sizeof(C) == 16) cp_async16(smem, gmem);
  else cp_async8(smem, gmem);
}
// copy n complex elements (n even, both ends 16-byte aligned) with 16-byte copies
template <typename C, int NT>
__device__ __forceinline__ void cp_async_span(C* smem, const C* gmem, int n) {
  constexpr int PER = 16 / sizeof(C);
  for (int i = threadIdx.x; i < n / PER; i += NT) cp_async16(smem + i * PER, gmem + i * PER);
}
// ------------------------------------------------------- bulk copies (TMA engine)
// One bulk copy of a contiguous span into shared memory, issued by one thread and
// completed on an mbarrier (transaction count = bytes).  No multicast: the source is
// this GPU's own global memory.  Both addresses 16-byte aligned, n a multiple of 16.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init1(uint64_t* mb) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mb)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* mb) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(mb)) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned n, uint64_t* mb) {
  // earlier generic-proxy accesses of dst are ordered before the async-proxy writes
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mb)), "r"(n) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(n), "r"(smem_u32(mb))
               : "memory");
}
// Wait for phase `parity` of mb to complete, at most `limit` polls (each try_wait
// suspends for a bounded time); false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(mb)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// polls of a bulk-copy wait before the block records MEU_ERR_TIMEOUT (far above any copy)
constexpr int BULK_WAIT_POLLS = 1 << 18;

// 16-byte vector store of n complex (n even, 16-byte aligned)
template <typename C, int NT>
__device__ __forceinline__ void store_span(C* gmem, const C* smem, int n) {
  constexpr int PER = 16 / sizeof(C);
  for (int i = threadIdx.x; i < n / PER; i += NT) *(float4*)(gmem + i * PER) = *(const float4*)(smem + i * PER);
}

// ----------------------------------------------------------- plane (x + y)
// Shared-memory image of one z-plane: NY rows of PITCH = N/2+1 complex.
template <typename R, int N, int NT, int PV>
struct Plane {
  using C = cplx<R>;
  static constexpr int LX = N / 2, NXH = LX + 1, PITCH = NXH, NY = N;
  static constexpr int ELEMS = NY * PITCH;
  // twiddles (hi then lo for float): twx[LX*K], twy[NY*K], post[NXH*K]
  static constexpr int K = Tw<C>::K;
  // rounded up to 16 bytes: PB stages its inputs with 16-byte copies right after the twiddles
  static constexpr int TW_ELEMS = (((LX + NY + NXH) * K * (int)sizeof(C) + 15) / 16) * 16 / (int)sizeof(C);
  static_assert((ELEMS * sizeof(C)) % 16 == 0, "the twiddles follow the plane image on a 16-byte boundary");
  static constexpr size_t smem_bytes() { return sizeof(C) * (size_t)(ELEMS + TW_ELEMS); }

  static __device__ __forceinline__ void load_tw(C* tws, const C* __restrict__ gx, const C* __restrict__ gy,
                                                 const C* __restrict__ gpost) {
    for (int i = threadIdx.x; i < LX * K; i += NT) tws[i] = gx[i];
    for (int i = threadIdx.x; i < NY * K; i += NT) tws[LX * K + i] = gy[i];
    for (int i = threadIdx.x; i < NXH * K; i += NT) tws[(LX + NY) * K + i] = gpost[i];
  }

  // buf rows hold (x[2n], x[2n+1]) at n in [0, LX): R2C along x, FFT along y.
  static __device__ __forceinline__ void forward(C* buf, const C* tws) {
    const C* twx = tws;
    const C* twy = tws + LX * K;
    const C* post = tws + (LX + NY) * K;
    dif<C, LX, NY, PITCH, 1, NT, PV>(buf, twx);
    // split in place, in digit-reversed column order (Nyquist into column LX)
    constexpr int NP = LX / 2 + 1;
#pragma unroll 1
    for (int i = threadIdx.x; i < NY * NP; i += NT) {
      const int row = i % NY, k = i / NY;
      C* rb = buf + row * PITCH;
      const int pk = pos<LX, PV>(k % LX), pm = pos<LX, PV>((LX - k) % LX);
      const C zk = rb[pk], zm = rb[pm];
      C e = cscale(cadd(zk, cconj(zm)), (R)0.5);
      C o = cscale(csub(zk, cconj(zm)), (R)0.5);
      o = mk(o.y, -o.x);
      const C xk = cadd(e, Tw<C>::mul(o, post, k, NXH));
      if (k == 0) {
        // X[0] = E + O and X[LX] = E - O are real: packed as X[0] + i X[LX] into
        // column 0, so the y transform runs over LX columns instead of LX + 1
        rb[0] = mk(xk.x, csub(e, o).x);
      } else {
        rb[pk] = xk;
        if (k != LX - k) {
          C e2 = cscale(cadd(zm, cconj(zk)), (R)0.5);
          C o2 = cscale(csub(zm, cconj(zk)), (R)0.5);
          o2 = mk(o2.y, -o2.x);
          rb[pm] = cadd(e2, Tw<C>::mul(o2, post, LX - k, NXH));
        }
      }
    }
    __syncthreads();
    dif<C, NY, LX, 1, PITCH, NT, PV>(buf, twy);
    // unpack column 0: Z = Y0 + i YN  ->  Y0(ky) = (Z(ky) + conj Z(-ky)) / 2 into column 0,
    // YN(ky) = -i (Z(ky) - conj Z(-ky)) / 2 into column LX (rows in digit-reversed order)
    for (int ky = threadIdx.x; ky <= NY / 2; ky += NT) {
      const int p1 = pos<NY, PV>(ky), p2 = pos<NY, PV>((NY - ky) % NY);
      const C z1 = buf[p1 * PITCH], z2 = buf[p2 * PITCH];
      const C y0 = cscale(cadd(z1, cconj(z2)), (R)0.5);
      const C d = cscale(csub(z1, cconj(z2)), (R)0.5);
      const C yn = mk(d.y, -d.x);
      buf[p1 * PITCH] = y0;
      buf[p1 * PITCH + LX] = yn;
      buf[p2 * PITCH] = cconj(y0);
      buf[p2 * PITCH + LX] = cconj(yn);
    }
    __syncthreads();
  }

  // inverse of forward(): M-form plane -> rows of (x[2n], x[2n+1]), unscaled.
  static __device__ __forceinline__ void inverse(C* buf, const C* tws) {
    const C* twx = tws;
    const C* twy = tws + LX * K;
    const C* post = tws + (LX + NY) * K;
    // columns 0 and LX (Hermitian in ky) packed as X0 + i XN, so the inverse y
    // transform runs over LX columns; its column 0 then holds x0 + i xN, both real
    for (int y = threadIdx.x; y < NY; y += NT) {
      const C x0 = buf[y * PITCH], xn = buf[y * PITCH + LX];
      buf[y * PITCH] = mk(x0.x - xn.y, x0.y + xn.x);
    }
    __syncthreads();
    dit<C, NY, LX, 1, PITCH, NT, PV>(buf, twy);
    constexpr int NP = LX / 2 + 1;
#pragma unroll 1
    for (int i = threadIdx.x; i < NY * NP; i += NT) {
      const int row = i % NY, k = i / NY;
      C* rb = buf + row * PITCH;
      const int pk = (k == 0) ? 0 : pos<LX, PV>(k);
      const int pm = (k == 0) ? LX : pos<LX, PV>(LX - k);
      C xk, xm;
      if (k == 0) {
        const C z = rb[0];
        xk = mk(z.x, (R)0);
        xm = mk(z.y, (R)0);
      } else {
        xk = rb[pk];
        xm = rb[pm];
      }
      {
        const C ex = cadd(xk, cconj(xm));
        const C ox = Tw<C>::mulc(csub(xk, cconj(xm)), post, k, NXH);
        rb[pk] = cadd(ex, mk(-ox.y, ox.x));
      }
      if (k != 0 && k != LX - k) {
        const C ex = cadd(xm, cconj(xk));
        const C ox = Tw<C>::mulc(csub(xm, cconj(xk)), post, LX - k, NXH);
        rb[pm] = cadd(ex, mk(-ox.y, ox.x));
      }
    }
    __syncthreads();
    dit<C, LX, NY, PITCH, 1, NT, PV>(buf, twx);
  }

  // ---- streaming form: the plane's first inverse stage reads global memory, its last
  // forward stage writes it, and the x transform's stage 0 of the inverse and of the
  // forward run on one butterfly's registers with the caller's pointwise work in
  // between (x_stage0), so a plane makes about half the shared-memory round trips
  // of inverse() + pointwise pass + forward().
  static constexpr int NSX = rplan(LX, PV).ns, NSY = rplan(NY, PV).ns;

  // Inverse of an M-form plane in global memory (src) into shared memory, every
  // stage except the x transform's stage 0.  Ends with a barrier.  Once per block: the
  // plane arrives by one bulk copy on the block's mbarrier; a wait that runs out records
  // MEU_ERR_TIMEOUT in *err.
  static __device__ __forceinline__ void inverse_head(C* buf, const C* tws, const C* __restrict__ src, int* err) {
    const C* twx = tws;
    const C* twy = tws + LX * K;
    const C* post = tws + (LX + NY) * K;
    static_assert(NSY >= 2, "the streaming plane needs a y plan of two stages or more");
    using SY = StageOf<NY, NSY - 1, PV>;  // first executed y stage (M = 1: no twiddles)
    // the whole plane in one bulk copy, then the first stage in place; columns 0 and LX
    // (Hermitian in ky) are packed as X0 + i XN, so the y transform runs over LX
    // columns; its column 0 then holds x0 + i xN, both real
    static_assert((ELEMS * sizeof(C)) % 16 == 0, "bulk copy size");
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) mbar_init1(&mb);
    __syncthreads();
    if (threadIdx.x == 0) bulk_load(buf, src, (unsigned)(ELEMS * sizeof(C)), &mb);
    if (!mbar_wait(&mb, 0, BULK_WAIT_POLLS)) {
      if (err) atomicMax(err, MEU_ERR_TIMEOUT);
      mbar_wait(&mb, 0, BULK_WAIT_POLLS);  // the copy's own completion, bounded too
    }
    __syncthreads();
    // every thread is past its wait: the mbarrier is invalidated, so a block that runs
    // several planes (the persistent ensemble kernel) initialises it afresh for the next
    if (threadIdx.x == 0) mbar_inval(&mb);
#pragma unroll 1
    for (int t = threadIdx.x; t < LX * SY::TASKS; t += NT) {
      const int c = t % LX, b = t / LX;
      C x[SY::R];
#pragma unroll
      for (int q = 0; q < SY::R; ++q) {
        const C* row = buf + (b * SY::R + q) * PITCH;
        x[q] = row[c];
        if (c == 0) {
          const C xn = row[LX];
          x[q] = mk(x[q].x - xn.y, x[q].y + xn.x);
        }
      }
      Dft<SY::R, 1, C>::run(x);
#pragma unroll
      for (int q = 0; q < SY::R; ++q) buf[(b * SY::R + q) * PITCH + c] = x[q];
    }
    __syncthreads();
    dit_range<C, NY, LX, 1, PITCH, NT, PV, 0, NSY - 2>(buf, twy);
    constexpr int NP = LX / 2 + 1;
#pragma unroll 1
    for (int i = threadIdx.x; i < NY * NP; i += NT) {
      const int row = i % NY, k = i / NY;
      C* rb = buf + row * PITCH;
      const int pk = (k == 0) ? 0 : pos<LX, PV>(k);
      const int pm = (k == 0) ? LX : pos<LX, PV>(LX - k);
      C xk, xm;
      if (k == 0) {
        const C z = rb[0];
        xk = mk(z.x, (R)0);
        xm = mk(z.y, (R)0);
      } else {
        xk = rb[pk];
        xm = rb[pm];
      }
      {
        const C ex = cadd(xk, cconj(xm));
        const C ox = Tw<C>::mulc(csub(xk, cconj(xm)), post, k, NXH);
        rb[pk] = cadd(ex, mk(-ox.y, ox.x));
      }
      if (k != 0 && k != LX - k) {
        const C ex = cadd(xm, cconj(xk));
        const C ox = Tw<C>::mulc(csub(xm, cconj(xk)), post, LX - k, NXH);
        rb[pm] = cadd(ex, mk(-ox.y, ox.x));
      }
    }
    __syncthreads();
    dit_range<C, LX, NY, PITCH, 1, NT, PV, 1, NSX - 1>(buf, twx);
  }

  // Task t of the x transform's stage 0 -> (row y, butterfly j in [0, M)).  A shared-
  // memory wavefront serves G = 128 B / sizeof(C) lanes; the pitch is odd, so the lanes'
  // banks are distinct when (y + j) mod G is.  When M divides G (M < G), a group of G
  // lanes takes rows spaced by M (y = y0 + h + M i) and all M butterflies of each, which
  // also gives every row M consecutive pairs in global memory (full 32-byte sectors for
  // the pointwise loads and stores); otherwise butterflies run fastest within a row.
  static __device__ __forceinline__ void x_task(int t, int& y, int& j) {
    constexpr int M = StageOf<LX, 0, PV>::M, G = 128 / (int)sizeof(C);
    if constexpr (M >= G || G % M != 0) {
      j = t % M;
      y = t / M;
    } else {
      static_assert(NY % G == 0, "rows in groups of G");
      const int grp = t / (G * M), rem = t - grp * (G * M), h = rem / G, l = rem - h * G;
      j = l % M;
      y = grp * G + h + M * (l / M);
    }
  }

  // The x transform's stage 0 of the inverse on one butterfly's registers, then
  // fn(y, n0, dn, x): x[r] holds the pair (x[2n], x[2n+1]) of row y at n = n0 + r*dn.
  // With FWD the butterfly then runs the forward's stage 0 on what fn left in x and
  // writes it back.  Ends with a barrier.
  template <bool FWD, typename Fn>
  static __device__ __forceinline__ void x_stage0(C* buf, const C* tws, Fn&& fn) {
    using SX = StageOf<LX, 0, PV>;
    const C* twx = tws;
#pragma unroll 1
    for (int t = threadIdx.x; t < NY * SX::M; t += NT) {
      int y, j;
      x_task(t, y, j);
      C* rb = buf + y * PITCH + j;
      C x[SX::R];
#pragma unroll
      for (int q = 0; q < SX::R; ++q) x[q] = rb[q * SX::M];
      dit_regs<C, LX, 0, PV>(x, twx, j);
      fn(y, j, SX::M, x);
      if constexpr (FWD) {
        dif_regs<C, LX, 0, PV>(x, twx, j);
#pragma unroll
        for (int q = 0; q < SX::R; ++q) rb[q * SX::M] = x[q];
      }
    }
    __syncthreads();
  }

  // Rows of (x[2n], x[2n+1]) already in shared memory (load_real): fn(y, n0, dn, x) on
  // the butterfly's pairs, then the x transform's forward stage 0 on its registers --
  // the same arithmetic as x_stage0<true> after its inverse stage.  Ends with a barrier.
  template <typename Fn>
  static __device__ __forceinline__ void x_forward0(C* buf, const C* tws, Fn&& fn) {
    using SX = StageOf<LX, 0, PV>;
    const C* twx = tws;
#pragma unroll 1
    for (int t = threadIdx.x; t < NY * SX::M; t += NT) {
      int y, j;
      x_task(t, y, j);
      C* rb = buf + y * PITCH + j;
      C x[SX::R];
#pragma unroll
      for (int q = 0; q < SX::R; ++q) x[q] = rb[q * SX::M];
      fn(y, j, SX::M, x);
      dif_regs<C, LX, 0, PV>(x, twx, j);
#pragma unroll
      for (int q = 0; q < SX::R; ++q) rb[q * SX::M] = x[q];
    }
    __syncthreads();
  }

  // Forward from rows whose x transform has run stage 0 (x_stage0<true>) to an M-form
  // plane in global memory (dst).  buf is scratch afterwards.
  static __device__ __forceinline__ void forward_tail(C* buf, const C* tws, C* __restrict__ dst) {
    const C* twx = tws;
    const C* twy = tws + LX * K;
    const C* post = tws + (LX + NY) * K;
    dif_range<C, LX, NY, PITCH, 1, NT, PV, 1, NSX>(buf, twx);
    constexpr int NP = LX / 2 + 1;
#pragma unroll 1
    for (int i = threadIdx.x; i < NY * NP; i += NT) {
      const int row = i % NY, k = i / NY;
      C* rb = buf + row * PITCH;
      const int pk = pos<LX, PV>(k % LX), pm = pos<LX, PV>((LX - k) % LX);
      const C zk = rb[pk], zm = rb[pm];
      C e = cscale(cadd(zk, cconj(zm)), (R)0.5);
      C o = cscale(csub(zk, cconj(zm)), (R)0.5);
      o = mk(o.y, -o.x);
      const C xk = cadd(e, Tw<C>::mul(o, post, k, NXH));
      if (k == 0) {
        rb[0] = mk(xk.x, csub(e, o).x);  // X[0] + i X[LX], both real
      } else {
        rb[pk] = xk;
        if (k != LX - k) {
          C e2 = cscale(cadd(zm, cconj(zk)), (R)0.5);
          C o2 = cscale(csub(zm, cconj(zk)), (R)0.5);
          o2 = mk(o2.y, -o2.x);
          rb[pm] = cadd(e2, Tw<C>::mul(o2, post, LX - k, NXH));
        }
      }
    }
    __syncthreads();
    dif_range<C, NY, LX, 1, PITCH, NT, PV, 0, NSY - 1>(buf, twy);
    using SY = StageOf<NY, NSY - 1, PV>;  // last y stage (M = 1): straight to global memory
#pragma unroll 1
    for (int t = threadIdx.x; t < LX * SY::TASKS; t += NT) {
      const int c = t % LX, b = t / LX;
      C x[SY::R];
#pragma unroll
      for (int q = 0; q < SY::R; ++q) x[q] = buf[(b * SY::R + q) * PITCH + c];
      Dft<SY::R, -1, C>::run(x);
      if (c != 0) {
#pragma unroll
        for (int q = 0; q < SY::R; ++q) dst[(b * SY::R + q) * NXH + c] = x[q];
      } else {
#pragma unroll
        for (int q = 0; q < SY::R; ++q) buf[(b * SY::R + q) * PITCH] = x[q];
      }
    }
    __syncthreads();
    // column 0 holds Z = Y0 + i YN: Y0(ky) = (Z(ky) + conj Z(-ky)) / 2 -> column 0,
    // YN(ky) = -i (Z(ky) - conj Z(-ky)) / 2 -> column LX (rows in digit-reversed order)
    for (int ky = threadIdx.x; ky <= NY / 2; ky += NT) {
      const int p1 = pos<NY, PV>(ky), p2 = pos<NY, PV>((NY - ky) % NY);
      const C z1 = buf[p1 * PITCH], z2 = buf[p2 * PITCH];
      const C y0 = cscale(cadd(z1, cconj(z2)), (R)0.5);
      const C d = cscale(csub(z1, cconj(z2)), (R)0.5);
      const C yn = mk(d.y, -d.x);
      dst[p1 * NXH] = y0;
      dst[p1 * NXH + LX] = yn;
      dst[p2 * NXH] = cconj(y0);
      dst[p2 * NXH + LX] = cconj(yn);
    }
  }

  // M-form plane <-> shared memory (rows of NXH complex, contiguous in both).
  // load_m only issues the copies; the caller waits (cp_async_wait_all + sync).
  static __device__ __forceinline__ void load_m(C* buf, const C* __restrict__ src) {
    cp_async_span<C, NT>(buf, src, ELEMS);
  }
  static __device__ __forceinline__ void store_m(const C* buf, C* __restrict__ dst) {
    store_span<C, NT>(dst, buf, ELEMS);
  }
  // real plane (NY rows of N reals) into rows of (x[2n], x[2n+1]); issue only
  static __device__ __forceinline__ void load_real(C* buf, const R* __restrict__ src) {
    for (int i = threadIdx.x; i < NY * LX; i += NT) {
      const int y = i / LX, n = i - y * LX;
      cp_async_c(buf + y * PITCH + n, (const C*)(src + (int64_t)y * N) + n);
    }
  }
};

// kx of M-form column c
template <int N, int PV>
__device__ __forceinline__ int kx_of_col(int c) {
  return c == N / 2 ? N / 2 : rev<N / 2, PV>(c);
}

}  // namespace fz
}  // namespace meu
