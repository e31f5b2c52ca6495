// fft_stages.cuh -- compile-time radix stages with caller-supplied element access,
// shared by the generic transforms (fft.cu) and the fused elastic row kernel
// (el_rows.cu).
#pragma once
#include "fft.cuh"
#include "fused.cuh"

namespace meu {


// One radix stage over NL lines with caller-supplied element access: ld(line, e)
// and st(line, e, v) address element e of a line in whatever memory the stage
// reads or writes.  FWD: DIF butterfly then twiddle; else twiddle then DIT butterfly.
// JFAST: consecutive threads take consecutive butterflies of one line (consecutive
// elements, for row-contiguous global memory) instead of the same butterfly of
// consecutive lines.  HOLD: every thread loads and transforms all of its
// butterflies, the block synchronises, then all store -- for a stage whose
// stores land on other threads' inputs (a permuting, in-place stage).
template <typename C, int L, int S, int NL, int NT, int PV, bool FWD, bool JFAST = false, bool HOLD = false,
          typename LD, typename ST>
__device__ __forceinline__ void stage_io(const C* __restrict__ tw, LD&& ld, ST&& st) {
  constexpr int R = fz::rplan(L, PV).r[S];
  constexpr int SPAN = fz::span_of(L, S, PV);
  constexpr int M = SPAN / R, NBF = NL * (L / R), TWS = L / SPAN;
  auto map = [](int t, int& line, int& j, int& e0) {
    int b;
    if constexpr (JFAST) {
      j = t % M;
      const int u = t / M;
      line = u % NL;
      b = u / NL;
    } else {
      line = t % NL;
      const int u = t / NL;
      j = u % M;
      b = u / M;
    }
    e0 = b * SPAN + j;
  };
  auto butterfly = [&](C* x, int j) {
    if constexpr (FWD) {
      Dft<R, -1, C>::run(x);
      if (M > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) x[q] = Tw<C>::mul(x[q], tw, j * q * TWS, L);
      }
    } else {
      if (M > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) x[q] = Tw<C>::mulc(x[q], tw, j * q * TWS, L);
      }
      Dft<R, 1, C>::run(x);
    }
  };
  if constexpr (HOLD) {
    constexpr int IT = (NBF + NT - 1) / NT;
    C x[IT][R];
    int ln[IT], ee[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int t = threadIdx.x + it * NT;
      if (t < NBF) {
        int j;
        map(t, ln[it], j, ee[it]);
#pragma unroll
        for (int r = 0; r < R; ++r) x[it][r] = ld(ln[it], ee[it] + r * M);
        butterfly(x[it], j);
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; ++it)
      if (threadIdx.x + it * NT < NBF) {
#pragma unroll
        for (int q = 0; q < R; ++q) st(ln[it], ee[it] + q * M, x[it][q]);
      }
  } else {
#pragma unroll 1
    for (int t = threadIdx.x; t < NBF; t += NT) {
      int line, j, e0;
      map(t, line, j, e0);
      C x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = ld(line, e0 + r * M);
      butterfly(x, j);
#pragma unroll
      for (int q = 0; q < R; ++q) st(line, e0 + q * M, x[q]);
    }
  }
}

// Stages S, S+1, .. (FWD) or S, S-1, .. (inverse), up to but excluding SEND, in
// shared memory (element e of line l at buf[e * ES + l]); each ends with a barrier.
template <typename C, int L, int NL, int ES, int NT, int PV, bool FWD, int S, int SEND>
__device__ __forceinline__ void stages_smem(C* buf, const C* tw) {
  if constexpr (FWD ? (S < SEND) : (S > SEND)) {
    stage_io<C, L, S, NL, NT, PV, FWD>(
        tw, [&](int l, int e) { return buf[e * ES + l]; }, [&](int l, int e, C v) { buf[e * ES + l] = v; });
    __syncthreads();
    stages_smem<C, L, NL, ES, NT, PV, FWD, FWD ? S + 1 : S - 1, SEND>(buf, tw);
  }
}

}  // namespace meu
