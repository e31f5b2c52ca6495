// el_rows.cu -- the x-direction work of one elastic fixed-point iteration in one
// pass (proportional moduli: the polarisation of ModElastic.f:248-327 between the
// strain's inverse transforms, ModElastic.f:396-411, and the forward transforms of
// x, ModElastic.f:329-334).  For a block of rows of the six strain spectra (after
// their z and y inverse passes) the kernel runs the x C2R transform, forms the
// polarisation x of every voxel pair from the strain and the order parameters,
// and runs the x R2C transform of x back into the same spectral rows, which the
// y and z forward passes then finish.  The real strain and polarisation fields
// never reach global memory: per cell 6 complex in, V reals in, 6 complex out,
// against three separate passes that also write and re-read 12 real fields.
#include "engine.cuh"
#include "fft_stages.cuh"
#include "step_kernels.cuh"

namespace meu {

// rows per block: 6 * NR lines of L complex in shared memory
constexpr int el_rows_per_block(int L) { return 512 / L < 1 ? 1 : (512 / L > 16 ? 16 : 512 / L); }
// order parameters prefetched into shared memory up to this many variants
constexpr int EL_ROWS_PF_VAR = 4;

// polarisation of one voxel from its engineering strain g[6] (k_el_x_prop's formula,
// in the field precision R: FP64 for the plain path, FP32 for the FP32-bulk path;
// order parameters at pp[v * n3])
template <typename R, bool ORTHO, int NVMAX = MEU_MAX_VAR>
__device__ __forceinline__ void elx_voxel(const ElxCoef<R>& E, R cfac, const R* g, const R* pp, int64_t pstride, R* x,
                                          int* err) {
  const int V = E.nvar;
  R e0[6] = {0, 0, 0, 0, 0, 0}, psum = 0, sc = 0;
#pragma unroll
  for (int v = 0; v < NVMAX; ++v) {
    if (v >= V) break;
    const R q = pp[(int64_t)v * pstride];
    psum += E.inc[v] * q;
    sc += E.av[v] * q;
#pragma unroll
    for (int m = 0; m < 6; ++m) e0[m] += q * E.ep[v][m];
  }
  if (psum < (R)1) sc += (R)1 - psum;
  if (!(sc != (R)0)) set_err(err, MEU_ERR_C_SINGULAR);
  const R r = (R)1 / sc;
  R gam[6], d[6], a0[6], a1[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    gam[m] = g[m] + E.ebar[m];
    d[m] = e0[m] - cfac * gam[m];
  }
  mv6<ORTHO>(E.c0, gam, a0);
  mv6<ORTHO>(E.c1, d, a1);
#pragma unroll
  for (int i = 0; i < 6; ++i) x[i] = cfac * a0[i] + r * a1[i];
}

// Shared memory: element e of line l = m * NR + r (component m of row r) at
// buf[e * ES + l], ES = 6 NR + 1.  sp.p[m] holds component m's spectrum, rows of
// L + 1 complex, in place (read whole before written).  PF: the block's order
// parameters (V <= EL_ROWS_PF_VAR rows of 2L reals each) follow buf, copied with
// cp.async at the start so that they arrive during the inverse transform.
template <typename R, int L, int PV, bool ORTHO, bool PF>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 2 : 4) k_el_rows(PtrList<cplx<R>> sp, const R* __restrict__ pphi, int64_t nrows,
                                                 const cplx<R>* __restrict__ tw, const cplx<R>* __restrict__ post,
                                                 const __grid_constant__ ElxCoef<R> E, int64_t n3, R cfac, int* err) {
  using C = cplx<R>;
  constexpr int NR = el_rows_per_block(L), NL = 6 * NR, ES = NL + 1, NXH = L + 1, NP = L / 2 + 1;
  constexpr int NS = fz::rplan(L, PV).ns;
  static_assert(NS >= 2, "first and last stage must differ");
  extern __shared__ __align__(16) unsigned char smraw[];
  C* buf = (C*)smraw;
  const int64_t row0 = (int64_t)blockIdx.x * NR;
  const int nr = (int)min((int64_t)NR, nrows - row0);
  R* pbuf = (R*)(buf + ES * L);
  if constexpr (PF) {
    // rows row0 .. row0 + nr - 1 of each order parameter: 16-byte pieces (2L reals
    // per row, a multiple of 16 bytes; n3 a multiple of 2L)
    constexpr int PER = 16 / (int)sizeof(R), CPR = 2 * L / PER;
    const int nchunk = E.nvar * nr * CPR;
    for (int c = threadIdx.x; c < nchunk; c += 256) {
      const int v = c / (nr * CPR), rem = c - v * nr * CPR, r = rem / CPR, j = (rem - r * CPR) * PER;
      fz::cp_async16(pbuf + (v * NR + r) * (2 * L) + j, pphi + (int64_t)v * n3 + (row0 + r) * (2 * L) + j);
    }
    fz::cp_async_commit();
  }

  // ---- x C2R of the six strain components: split into natural order ...
  for (int i = threadIdx.x; i < NL * NP; i += 256) {
    const int l = i / NP, k = i - l * NP, m = l / NR, r = l - m * NR;
    if (r >= nr) continue;
    const C* srow = sp.p[m] + (row0 + r) * NXH;
    C xk = srow[k], xm = srow[L - k];
    if (k == 0) { xk.y = 0; xm.y = 0; }
    {
      C ex = cadd(xk, cconj(xm));
      C ox = Tw<C>::mulc(csub(xk, cconj(xm)), post, k, NXH);
      buf[k * ES + l] = cadd(ex, mk(-ox.y, ox.x));
    }
    if (k != 0 && k != L - k) {
      C ex = cadd(xm, cconj(xk));
      C ox = Tw<C>::mulc(csub(xm, cconj(xk)), post, L - k, NXH);
      buf[(L - k) * ES + l] = cadd(ex, mk(-ox.y, ox.x));
    }
  }
  __syncthreads();
  // ... then the DIT stages (the first permutes natural order into positions)
  stage_io<C, L, NS - 1, NL, 256, PV, false, false, true>(
      tw, [&](int l, int e) { return buf[fz::rev<L, PV>(e) * ES + l]; },
      [&](int l, int e, C v) { buf[e * ES + l] = v; });
  __syncthreads();
  stages_smem<C, L, NL, ES, 256, PV, false, NS - 2, 0>(buf, tw);
  stage_io<C, L, 0, NL, 256, PV, false>(
      tw, [&](int l, int e) { return buf[e * ES + l]; }, [&](int l, int e, C v) { buf[e * ES + l] = v; });
  if constexpr (PF) fz::cp_async_wait_all();
  __syncthreads();

  // ---- polarisation: element e of row r holds voxels 2e and 2e+1
  for (int i = threadIdx.x; i < NR * L; i += 256) {
    const int r = i / L, e = i - r * L;
    if (r >= nr) continue;
    const int64_t id = (row0 + r) * (2 * L) + 2 * e;
    R g[6], x0[6], x1[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) g[m] = buf[e * ES + m * NR + r].x;
    if constexpr (PF) {
      // the pair's order parameters as one 2-element load per variant
      R q0[EL_ROWS_PF_VAR], q1[EL_ROWS_PF_VAR];
      const C* pq = (const C*)(pbuf + r * (2 * L)) + e;
#pragma unroll
      for (int v = 0; v < EL_ROWS_PF_VAR; ++v) {
        const C q = v < E.nvar ? pq[v * NR * L] : mk((R)0, (R)0);
        q0[v] = q.x;
        q1[v] = q.y;
      }
      elx_voxel<R, ORTHO, EL_ROWS_PF_VAR>(E, cfac, g, q0, 1, x0, err);
#pragma unroll
      for (int m = 0; m < 6; ++m) g[m] = buf[e * ES + m * NR + r].y;
      elx_voxel<R, ORTHO, EL_ROWS_PF_VAR>(E, cfac, g, q1, 1, x1, err);
    } else {
      elx_voxel<R, ORTHO>(E, cfac, g, pphi + id, n3, x0, err);
#pragma unroll
      for (int m = 0; m < 6; ++m) g[m] = buf[e * ES + m * NR + r].y;
      elx_voxel<R, ORTHO>(E, cfac, g, pphi + id + 1, n3, x1, err);
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) buf[e * ES + m * NR + r] = mk((R)x0[m], (R)x1[m]);
  }
  __syncthreads();

  // ---- x R2C of the six polarisation components back into the spectral rows
  stage_io<C, L, 0, NL, 256, PV, true>(
      tw, [&](int l, int e) { return buf[e * ES + l]; }, [&](int l, int e, C v) { buf[e * ES + l] = v; });
  __syncthreads();
  stages_smem<C, L, NL, ES, 256, PV, true, 1, NS - 1>(buf, tw);
  stage_io<C, L, NS - 1, NL, 256, PV, true, false, true>(
      tw, [&](int l, int e) { return buf[e * ES + l]; },
      [&](int l, int e, C v) { buf[fz::rev<L, PV>(e) * ES + l] = v; });
  __syncthreads();
  for (int i = threadIdx.x; i < NL * NP; i += 256) {
    const int l = i / NP, k = i - l * NP, m = l / NR, r = l - m * NR;
    if (r >= nr) continue;
    const int km = k == 0 ? 0 : L - k;
    const C zk = buf[k * ES + l], zm = buf[km * ES + l];
    C* drow = sp.p[m] + (row0 + r) * NXH;
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

bool el_rows_ok(int nx) {
  const int L = nx / 2;
  return nx % 2 == 0 && (L == 32 || L == 64 || L == 128 || L == 256 || L == 512);
}

template <typename R>
void el_rows_launch(const FFT3& f, const PtrList<cplx<R>>& sp, const R* pphi, const ElxCoef<R>& E, bool ortho,
                    double cfac, int* err, cudaStream_t st) {
  using C = cplx<R>;
  const int64_t nrows = (int64_t)f.ny * f.nz, n3 = f.n3();
  const bool pf = E.nvar <= EL_ROWS_PF_VAR;
  auto go = [&](auto Lc, auto Pc, auto Oc) {
    constexpr int L = decltype(Lc)::value, PV = decltype(Pc)::value;
    constexpr bool O = decltype(Oc)::value;
    constexpr int NR = el_rows_per_block(L);
    auto fn = pf ? k_el_rows<R, L, PV, O, true> : k_el_rows<R, L, PV, O, false>;
    const size_t sm = (size_t)(6 * NR + 1) * L * sizeof(C) + (pf ? (size_t)E.nvar * NR * 2 * L * sizeof(R) : 0);
    if ((int)sm > smem_optin((const void*)fn))  // dynamic + static above 48 KB needs the opt-in
      throw CudaError("fused elastic rows exceed shared memory", MEU_ERR_UNSUPPORTED);
    fn<<<(unsigned)((nrows + NR - 1) / NR), 256, sm, st>>>(sp, pphi, nrows, (const C*)f.px.tw, (const C*)f.post_tw, E,
                                                          n3, (R)cfac, err);
  };
  auto with_o = [&](auto Lc, auto Pc) {
    if (ortho) go(Lc, Pc, std::true_type{});
    else go(Lc, Pc, std::false_type{});
  };
  // The kernel's radix plan is its own (the twiddle table is plan-independent and the
  // spectral rows are in natural order): radix 16 first, whatever plan the transform
  // passes run.  Deck 2 at 512^3 (L = 256, 16 x 16 against 8 x 8 x 4): 4.16 -> 3.50 ms
  // per launch on one B200, the same FP32 error against FP64.
  auto with_pv = [&](auto Lc) { with_o(Lc, std::integral_constant<int, 2>{}); };
  switch (f.nx / 2) {
    case 32: with_pv(std::integral_constant<int, 32>{}); break;
    case 64: with_pv(std::integral_constant<int, 64>{}); break;
    case 128: with_pv(std::integral_constant<int, 128>{}); break;
    case 256: with_pv(std::integral_constant<int, 256>{}); break;
    case 512: with_pv(std::integral_constant<int, 512>{}); break;
    default: throw CudaError("internal: fused elastic rows for an unsupported length", MEU_ERR_UNSUPPORTED);
  }
}

template void el_rows_launch<float>(const FFT3&, const PtrList<float2>&, const float*, const ElxCoef<float>&, bool,
                                    double, int*, cudaStream_t);
template void el_rows_launch<double>(const FFT3&, const PtrList<double2>&, const double*, const ElxCoef<double>&, bool,
                                     double, int*, cudaStream_t);

}  // namespace meu
