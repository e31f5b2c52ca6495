// engine.cu -- the step engine behind include/meu.h.
//
// One Engine owns the device state of one grid: fields, spectra, the elastic
// state (u^ and the engineering strain), reduction buffers and a CUDA stream.
// Engine<R>::run() executes the reference time loop body
// (Multi_MEUMAPPS.f:548-1106) for the KKS model, or the Landau step, as a
// sequence of kernels on that stream.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <thread>
#include <memory>
#include <string>
#include <vector>

#include "engine.cuh"
#include "step_kernels.cuh"

namespace meu {

// A 6x6 stiffness or compliance with decoupled normal / shear parts and independent
// shears (the zero pattern mv6<true> skips).
static bool ortho6(const double* c) {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j)
      if (!((i < 3 && j < 3) || i == j) && c[i + j * 6] != 0.0) return false;
  return true;
}

// Fixed-order finalisation: block q reduces partials[q*PSTRIDE .. + nb[q]) with ops[q].
__global__ void k_finalize(const double* __restrict__ partials, NbList nb, const int* __restrict__ ops, double* out) {
  const int q = blockIdx.x, op = ops[q];
  double acc = op == 0 ? 0.0 : op == 1 ? -1.0e308 : 1.0e308;
  for (int i = threadIdx.x; i < nb.nb[q]; i += blockDim.x) {
    const double v = partials[(int64_t)q * PSTRIDE + i];
    acc = op == 0 ? acc + v : op == 1 ? fmax(acc, v) : fmin(acc, v);
  }
  block_reduce_store(acc, op, out + q);
}

// per-component sums of an AoS chunk (block partials; component e at out[e*PSTRIDE + b])
__global__ void __launch_bounds__(RED_THREADS) k_aos_colsum(const double* __restrict__ src, int ncomp, int64_t nv,
                                                            double* out) {
  for (int e = 0; e < ncomp; ++e) {
    double acc = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x)
      acc += src[i * ncomp + e];
    block_reduce_store(acc, 0, out + (int64_t)e * PSTRIDE + blockIdx.x);
  }
}
__global__ void k_accumulate(const double* __restrict__ r, double* acc, int n) {
  if (threadIdx.x < n) acc[threadIdx.x] += r[threadIdx.x];
}
__global__ void k_set_cmean(DevConst* K, LanFusedConst* F, const double* __restrict__ acc, int n, double inv_n3) {
  if (threadIdx.x < n) K->c_mean[threadIdx.x] = acc[threadIdx.x] * inv_n3;
  if (F && threadIdx.x == 0) F->cbar = acc[0] * inv_n3;
}
// gradient energy of eta (Parseval on natural-order spectra), block partials
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_grad_energy(const DevConst* __restrict__ Kp, PtrList<cplx<R>> sp, int V,
                                                             double* out) {
  const DevConst& K = *Kp;
  double acc = 0;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    double f = 0;
    for (int v = 0; v < V; ++v) {
      const double re = (double)sp.p[v][id].x, im = (double)sp.p[v][id].y;
      f += kkappak_b(K.p.grad_coeff[v], b) * (re * re + im * im);
    }
    acc += 0.5 * hweight(K, kx) * f;
  }
  block_reduce_store(acc, 0, out + blockIdx.x);
}

// the fluctuation spectrum has no k = 0 mode
template <typename R>
__global__ void k_zero_k0(cplx<R>* kc) {
  if (threadIdx.x == 0) kc[0] = mk((R)0, (R)0);
}

// AoS (component fastest, double) <-> SoA (R)
// offs: NULL or per-component offsets subtracted on the way in (added on the way out)
template <typename R>
__global__ void k_aos_to_soa(const double* __restrict__ src, R* __restrict__ dst, int ncomp, int64_t v0, int64_t nv,
                             int64_t n3, int add, const double* offs) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv * ncomp; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t vox = i / ncomp;
    const int c = (int)(i - vox * ncomp);
    R* d = dst + (int64_t)c * n3 + v0 + vox;
    const double v = offs ? src[i] - offs[c] : src[i];
    if (add) *d = (R)((double)*d + v);
    else *d = (R)v;
  }
}
template <typename R>
__global__ void k_soa_to_aos(const R* __restrict__ src, double* __restrict__ dst, int ncomp, int64_t v0, int64_t nv,
                             int64_t n3, const double* offs) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv * ncomp; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t vox = i / ncomp;
    const int c = (int)(i - vox * ncomp);
    dst[i] = (double)src[(int64_t)c * n3 + v0 + vox] + (offs ? offs[c] : 0.0);
  }
}
template <typename R>
__global__ void k_convert(const R* __restrict__ src, double* __restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
template <typename R>
__global__ void k_convert_in(const double* __restrict__ src, R* __restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (R)src[i];
}
// engineering strain from the 9 gradients grad_j_ui (data_save order (j-1)*3+(i-1))
// gu holds nv voxels of each gradient back to back; strain is offset to the chunk
template <typename R>
__global__ void k_grads_to_strain(const double* __restrict__ gu, R* __restrict__ strain, int64_t nv, int64_t n3) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    auto G = [&](int ui, int dj) { return gu[(int64_t)((dj - 1) * 3 + (ui - 1)) * nv + i]; };
    strain[0 * n3 + i] = (R)G(1, 1);
    strain[1 * n3 + i] = (R)G(2, 2);
    strain[2 * n3 + i] = (R)G(3, 3);
    strain[3 * n3 + i] = (R)(G(3, 2) + G(2, 3));
    strain[4 * n3 + i] = (R)(G(3, 1) + G(1, 3));
    strain[5 * n3 + i] = (R)(G(2, 1) + G(1, 2));
  }
}
// u^ -> [u_i^ (3), kf_j u_i^ (9)] in data_save order
template <typename R>
__global__ void k_u_spectra(const DevConst* __restrict__ Kp, const cplx<R>* __restrict__ uk, PtrList<cplx<R>> out) {
  const DevConst& K = *Kp;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < K.nk; id += (int64_t)gridDim.x * blockDim.x) {
    int kx, ky, kz;
    kdecode(K, id, kx, ky, kz);
    double a[3], b[3];
    kvec(K, kx, ky, kz, a, b);
    for (int i = 0; i < 3; ++i) {
      double re, im;
      ld2(uk[(int64_t)i * K.nk + id], re, im);
      out.p[i][id] = mk((R)re, (R)im);
      for (int j = 0; j < 3; ++j) out.p[3 + j * 3 + i][id] = mk((R)(-b[j] * im), (R)(b[j] * re));
    }
  }
}

template <typename R>
Engine<R>::Engine(const meu_params& p) : P(p) {
  V = p.nvar;
  E = p.numel;
  if (p.nx < 4 || p.ny < 2 || p.nz < 2 || V < 1 || V > MEU_MAX_VAR || E < 1 || E > MEU_MAX_EL || p.numph < 2 ||
      p.numph > MEU_MAX_PH || p.numph * p.numel > 12)
    throw CudaError("parameters out of range", MEU_ERR_BADARG);
  if (p.model == MEU_MODEL_LANDAU && (E != 1 || p.numph != 2))
    throw CudaError("Landau decks have one solute and two phases", MEU_ERR_BADARG);
  if (!fft_size_ok(p.nx, true) || !fft_size_ok(p.ny, false) || !fft_size_ok(p.nz, false))
    throw CudaError("grid sizes must be 2^a 3^b with Nx even", MEU_ERR_UNSUPPORTED);
  int sum = 0;
  for (int n = 0; n < p.numph; ++n) sum += p.nvar_ph[n];
  if (V + 1 - sum != 0) throw CudaError("variant numbers (initerr 1)", MEU_ERR_BADARG);
  step = p.step;
  MEU_CUDA(cudaStreamCreateWithFlags(&own_st, cudaStreamNonBlocking));
  st = own_st;
  fft.reset(new FFT3(p.nx, p.ny, p.nz, sizeof(R) == 8));
  fft->hook = &prof;
  n3 = fft->n3();
  nk = fft->nk();
  // ---- device constants
  memset(&hK, 0, sizeof(hK));
  hK.p = p;
  hK.nx = p.nx; hK.ny = p.ny; hK.nz = p.nz; hK.nxh = p.nx / 2 + 1;
  hK.n3 = n3; hK.nk = nk;
  {
    int ivn = 0;
    for (int n = 2; n <= p.numph; ++n) {
      ivn += p.nvar_ph[n - 2];
      int fvn = ivn + p.nvar_ph[n - 1] - 1;
      hK.ph_lo[n] = ivn - 1;
      hK.ph_hi[n] = fvn;
      for (int v = ivn - 1; v < fvn; ++v) hK.var_phase[v] = n;
    }
  }
  hK.zdim = p.numph * p.numel;
  hK.c_shift = (p.model == MEU_MODEL_LANDAU) ? 1 : 0;
  if (p.model == MEU_MODEL_KKS) {
    const int numel = p.numel, numph = p.numph, zdim = hK.zdim;
    for (int e = 1; e <= numel; ++e) {
      const int i1 = e + numel + 1;
      for (int n = 1; n <= numph - 1; ++n) {
        const int i0 = (numph - 1) * (e - 1) + n, j0 = numph * (e - 1) + n;
        hK.zconst[(i0 - 1) + (j0 - 1) * zdim] = p.gparams[n - 1][e - 1];
        hK.zconst[(i0 - 1) + j0 * zdim] = -p.gparams[n][e - 1];
        hK.zr_const[i0 - 1] = p.gparams[n - 1][e - 1] * p.gparams[n - 1][i1 - 1] - p.gparams[n][e - 1] * p.gparams[n][i1 - 1];
      }
    }
  }
  for (int i = 0; i < 36; ++i) hK.c0m[i] = p.cela[1][i];
  {
    // Q_il = -sum_{j,k} C0(voigt(i,j), voigt(k,l)) K_kj, K_kk = a_k^2, K_kj = b_k b_j (k != j)
    auto vq = [](int i, int j) { return i == j ? i : 9 - i - j; };
    const int mi[6] = {1, 2, 3, 2, 1, 1}, ml[6] = {1, 2, 3, 3, 3, 2};
    auto kidx = [](int k, int j) { return k == j ? k - 1 : (k + j == 5 ? 3 : (k + j == 4 ? 4 : 5)); };
    for (int m = 0; m < 6; ++m)
      for (int j = 1; j <= 3; ++j)
        for (int k = 1; k <= 3; ++k)
          hK.qcoef[m][kidx(k, j)] -= p.cela[1][(vq(mi[m], j) - 1) + (vq(k, ml[m]) - 1) * 6];
  }
  // proportional compliances: S_n = alpha_n S_1 for every phase (and a non-zero matrix)
  {
    bool prop = p.cela[0][0] > 0;
    hK.alpha[0] = 1.0;
    for (int n = 1; n < p.numph && prop; ++n) {
      const double al = p.sela[n][0] / p.sela[0][0];
      for (int i = 0; i < 36; ++i) {
        const double d = p.sela[n][i] - al * p.sela[0][i];
        if (std::fabs(d) > 1e-12 * (std::fabs(p.sela[n][i]) + std::fabs(al * p.sela[0][i])) + 1e-300) prop = false;
      }
      hK.alpha[n] = al;
    }
    // C_1 must be the inverse of S_1 for C = C_1 / s to hold
    if (prop) {
      for (int i = 0; i < 6 && prop; ++i)
        for (int j = 0; j < 6; ++j) {
          double acc = 0;
          for (int k = 0; k < 6; ++k) acc += p.cela[0][i + k * 6] * p.sela[0][k + j * 6];
          if (std::fabs(acc - (i == j ? 1.0 : 0.0)) > 1e-10) { prop = false; break; }
        }
    }
    hK.prop_moduli = prop ? 1 : 0;
  }
  auto vg = [](int i, int j) { return i == j ? i : 9 - i - j; };
  for (int v = 0; v < V; ++v) {
    const int n = hK.var_phase[v];
    for (int ij = 1; ij <= 6; ++ij) {
      double acc = 0;
      for (int k = 1; k <= 3; ++k)
        for (int l = 1; l <= 3; ++l) acc += p.trans_ppt[v][vg(k, l) - 1] * p.cela[n - 1][(ij - 1) + (vg(k, l) - 1) * 6];
      hK.sig0[v][ij - 1] = acc;
    }
    for (int m = 0; m < 6; ++m) hK.eps_eng[v][m] = (m < 3 ? 1.0 : 2.0) * p.trans_ppt[v][m];
    double ts = 0;
    for (int m = 0; m < 6; ++m) ts += p.trans_ppt[v][m];
    hK.use_var[v] = (p.model == MEU_MODEL_LANDAU) ? 1 : (ts > (double)1.e-9f ? 1 : 0);
    double se = 0;
    for (int m = 0; m < 6; ++m) se += (m < 3 ? 1.0 : 2.0) * hK.sig0[v][m] * p.e_mean[m];
    hK.sig0_ebar[v] = se;
  }
  for (int v = 0; v < V; ++v)
    for (int q = 0; q < V; ++q) {
      double acc = 0;
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) acc += hK.eps_eng[v][i] * p.cela[1][i + j * 6] * hK.eps_eng[q][j];
      hK.A[v][q] = acc;
    }
  for (int m = 0; m < 6; ++m) hK.ebar_eng[m] = (m < 3 ? 1.0 : 2.0) * p.e_mean[m];
  if (p.model == MEU_MODEL_LANDAU && p.elastic == MEU_ELAST_HOMOG) {
    for (int i = 0; i < 36; ++i)
      if (std::fabs(p.cela[0][i] - p.cela[1][i]) > 1e-12 * (std::fabs(p.cela[1][i]) + 1e-300))
        throw CudaError("MEU_ELAST_HOMOG needs equal matrix and precipitate moduli", MEU_ERR_BADARG);
  }
  // ---- buffers
  c = dalloc<R>(E * n3);
  c2 = dalloc<R>(E * n3);
  phi = dalloc<R>(V * n3);
  pphi = dalloc<R>(V * n3);
  fd = dalloc<R>(V * n3);
  el_en = dalloc<R>(n3);
  const bool elast = p.elastic != MEU_ELAST_NONE;
  const bool het = (p.model == MEU_MODEL_KKS) || p.elastic == MEU_ELAST_HETERO;
  if (p.model == MEU_MODEL_KKS) {
    noise = dalloc<R>(V * n3);
    fc = dalloc<R>(3 * E * n3);
    NWR = 4 * V;
    NS = std::max(5 * V, 4 * E);
  } else {
    NWR = 2 * V + 1;
    NS = 2 * V + 2;
  }
  if (elast && het) {
    strain = dalloc<R>(6 * n3);
    xs = dalloc<R>(6 * n3);
    uk = dalloc<C>(3 * nk);
    NS = std::max(NS, V + 6);
  }
  NS = std::max(NS, 12);  // u_state download uses 12 spectra
  NWR = std::max(NWR, 1);
  wr = dalloc<R>((int64_t)NWR * n3);
  sp = dalloc<C>((int64_t)NS * nk);
  partials = dalloc<double>((int64_t)Q_TOTAL * PSTRIDE);
  results = dalloc<double>(Q_TOTAL);
  hist = dalloc<double>((int64_t)HIST_MAX * Q_STEP_COUNT);
  cmean_acc = dalloc<double>(MEU_MAX_EL);
  d_ops = dalloc<int>(Q_TOTAL);
  d_err = dalloc<int>(1);
  dK = dalloc<DevConst>(1);
  MEU_CUDA(cudaHostAlloc((void**)&h_results, sizeof(double) * Q_TOTAL, cudaHostAllocDefault));
  MEU_CUDA(cudaHostAlloc((void**)&h_err, sizeof(int), cudaHostAllocDefault));
  int ops[Q_TOTAL];
  for (int q = 0; q < Q_TOTAL; ++q) ops[q] = 0;
  ops[Q_CMIN] = 2;
  ops[Q_CMAX] = 1;
  ops[Q_PHIMAX] = 1;
  MEU_CUDA(cudaMemcpy(d_ops, ops, sizeof(ops), cudaMemcpyHostToDevice));
  MEU_CUDA(cudaMemcpy(dK, &hK, sizeof(DevConst), cudaMemcpyHostToDevice));
  if (p.model == MEU_MODEL_LANDAU) {
    // spectral state eta^ and dc^ of the Landau step (layout of the path in use)
    keta = dalloc<C>((int64_t)V * nk);
    kc = dalloc<C>(nk);
    MEU_CUDA(cudaMemset(keta, 0, sizeof(C) * V * nk));
    MEU_CUDA(cudaMemset(kc, 0, sizeof(C) * nk));
  }
  fused = lan_fused_supported(p) && !(p.flags & MEU_FLAG_GENERIC);
  if (fused) {
    LanFusedConst F;
    memset(&F, 0, sizeof(F));
    memcpy(F.qcoef, hK.qcoef, sizeof(F.qcoef));
    {
      // cubic pattern of qcoef (exact comparisons: the constants are copied, not refit)
      const auto& q = hK.qcoef;
      bool cub = true;
      for (int m = 0; m < 3 && cub; ++m)
        for (int n = 0; n < 6; ++n) {
          const double want = n >= 3 ? 0.0 : (n == m ? q[0][0] : q[0][1]);
          if (q[m][n] != want) cub = false;
        }
      for (int m = 3; m < 6 && cub; ++m)
        for (int n = 0; n < 6; ++n)
          if (q[m][n] != (n == m ? q[3][3] : 0.0)) cub = false;
      F.q_cubic = cub ? 1.0 : 0.0;
      F.q_own = q[0][0];
      F.q_other = q[0][1];
      F.q_off = q[3][3];
    }
    for (int v = 0; v < V; ++v) {
      for (int m = 0; m < 6; ++m) {
        F.sig0[v][m] = hK.sig0[v][m];
        F.eps_eng[v][m] = hK.eps_eng[v][m];
      }
      for (int i = 0; i < 9; ++i) F.g[v][i] = p.grad_coeff[v][i];
      for (int q = 0; q < V; ++q) F.A[v][q] = hK.A[v][q];
      F.sig0_ebar[v] = hK.sig0_ebar[v];
    }
    for (int i = 0; i < 36; ++i) F.c0m[i] = p.cela[1][i];
    F.elastic_on = p.elastic != MEU_ELAST_NONE ? 1.0 : 0.0;
    for (int m = 0; m < 6; ++m) F.ebar_eng[m] = hK.ebar_eng[m];
    F.lan_a = p.lan_a; F.lan_b = p.lan_b; F.lan_c = p.lan_c; F.lan_d = p.lan_d;
    F.lan_c1 = p.lan_c1; F.lan_c2 = p.lan_c2; F.cross_w = p.cross_w; F.kappa_c = p.kappa_c;
    F.dm = p.dt * p.cmobs[0];
    F.dtl = p.dt * p.b_mob;
    dF = dalloc<LanFusedConst>(1);
    MEU_CUDA(cudaMemcpy(dF, &F, sizeof(F), cudaMemcpyHostToDevice));
    dA = dalloc<LanFusedArgs<R>>(1);
    d_row = dalloc<int>(2);
    d_ticket = d_row + 1;
    MEU_CUDA(cudaMemset(d_row, 0, 2 * sizeof(int)));
    if (p.elastic != MEU_ELAST_NONE && V == 1) {
      gtab = dalloc<R>(nk);
      MEU_CUDA(cudaMemset(gtab, 0, sizeof(R) * nk));
    }
  }
  MEU_CUDA(cudaMemset(d_err, 0, sizeof(int)));
  MEU_CUDA(cudaMemset(c, 0, sizeof(R) * E * n3));
  MEU_CUDA(cudaMemset(phi, 0, sizeof(R) * V * n3));
  if (noise) MEU_CUDA(cudaMemset(noise, 0, sizeof(R) * V * n3));
  MEU_CUDA(cudaMemset(el_en, 0, sizeof(R) * n3));
  if (strain) MEU_CUDA(cudaMemset(strain, 0, sizeof(R) * 6 * n3));
  if (uk) MEU_CUDA(cudaMemset(uk, 0, sizeof(C) * 3 * nk));
  stage_elems = std::min<int64_t>(n3 * std::max(std::max(V, E), 1), (int64_t)32 << 20);
  stage = dalloc<double>(stage_elems);
  {
    int dev = 0, sms = 0;
    MEU_CUDA(cudaGetDevice(&dev));
    MEU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    auto resident = [&](const void* fn) {
      int nb = 0;
      MEU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, RED_THREADS, 0));
      return std::max(1, std::min(RED_BLOCKS, nb * sms));
    };
    g_el_k = resident((const void*)k_el_k<R>);
    g_lan_k1 = resident((const void*)k_lan_k1<R>);
    el_ortho_gen = ortho6(hK.c0m);
    for (int n = 0; n < p.numph; ++n) el_ortho_gen = el_ortho_gen && ortho6(p.sela[n]);
    g_elener = resident(el_ortho_gen ? (const void*)k_elener<R, true> : (const void*)k_elener<R>);
    if (hK.prop_moduli) {
      ElxProp& X = el_prop;
      for (int i = 0; i < 36; ++i) {
        X.c0[i] = hK.c0m[i];
        X.c1[i] = p.cela[0][i];
      }
      for (int m = 0; m < 6; ++m) X.ebar[m] = hK.ebar_eng[m];
      for (int v = 0; v < V; ++v) {
        const int n = hK.var_phase[v];
        for (int m = 0; m < 6; ++m) X.ep[v][m] = hK.eps_eng[v][m];
        X.av[v] = n >= 2 ? hK.alpha[n - 1] : 0.0;
        X.inc[v] = n >= 2 ? 1.0 : 0.0;
      }
      X.nvar = V;
      el_prop_r.assign(X);
      ElenProp& Y = en_prop;
      for (int i = 0; i < 36; ++i) {
        Y.c1[i] = p.cela[0][i];
        Y.s1[i] = p.sela[0][i];
      }
      for (int m = 0; m < 6; ++m) Y.emean[m] = p.e_mean[m];
      for (int v = 0; v < V; ++v) {
        const int n = hK.var_phase[v];
        for (int m = 0; m < 6; ++m) Y.tp[v][m] = p.trans_ppt[v][m];
        Y.av[v] = n >= 2 ? hK.alpha[n - 1] : 0.0;
        Y.use[v] = (n >= 2 && hK.use_var[v]) ? 1 : 0;
      }
      Y.nvar = V;
      const bool ortho = ortho6(hK.c0m) && ortho6(p.cela[0]) && ortho6(p.sela[0]);
      el_ortho = ortho;
      el_fused_rows = el_rows_ok(p.nx);
      // 16-byte tile copies when every field starts on a 16-byte boundary
      const bool vec = n3 % (16 / (int64_t)sizeof(R)) == 0;
      fn_el_x = ortho ? (vec ? k_el_x_prop<R, true, true> : k_el_x_prop<R, true, false>)
                      : (vec ? k_el_x_prop<R, false, true> : k_el_x_prop<R, false, false>);
      fn_elener = ortho ? (vec ? k_elener_prop<R, true, true> : k_elener_prop<R, true, false>)
                        : (vec ? k_elener_prop<R, false, true> : k_elener_prop<R, false, false>);
      sm_el_x = (size_t)2 * (6 + V) * PF_TILE * sizeof(R);
      sm_elener = (size_t)2 * (6 + 2 * V) * PF_TILE * sizeof(R);
      const int64_t ntiles = (n3 + PF_TILE - 1) / PF_TILE;
      // grid: the blocks that fit at once (each loops over tiles), at most one per tile
      auto fit = [&](const void* fn, size_t smem) {
        if ((int)smem > smem_optin(fn))  // dynamic + static above 48 KB needs the opt-in
          throw CudaError("elastic prefetch tiles exceed shared memory", MEU_ERR_UNSUPPORTED);
        int nb = 0;
        MEU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, PF_TILE, smem));
        return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(nb, 1) * sms, ntiles));
      };
      g_el_x = fit((const void*)fn_el_x, sm_el_x);
      g_elener = std::min(fit((const void*)fn_elener, sm_elener), RED_BLOCKS);
    }
  }
  if (fused) {
    MEU_CUDA(cudaMemset(sp, 0, sizeof(C) * (size_t)NS * nk));
    if (p.flags & MEU_FLAG_AUTOTUNE) {
      sync_args();
      sched = lan_autotune<R>(p.nx, V, dA, 1, p.diag_energy != 0, st, nullptr);
      reset_fused_state();
    }
  } else if (p.flags & MEU_FLAG_AUTOTUNE) {
    tune_transforms();
  }
}

// Generic path: time the radix plans and column tiles of the compile-time transforms
// (forward and inverse of V fields, the batch of the driving-force transforms) and
// keep the fastest.
template <typename R>
void Engine<R>::tune_transforms() {
  const int nf = std::min(V, NS);
  MEU_CUDA(cudaMemsetAsync(pphi, 0, sizeof(R) * V * n3, st));
  std::vector<const R*> in;
  std::vector<R*> out;
  for (int v = 0; v < nf; ++v) {
    in.push_back(field(pphi, v));
    out.push_back(field(fd, v));
  }
  cudaEvent_t e0, e1;
  MEU_CUDA(cudaEventCreate(&e0));
  MEU_CUDA(cudaEventCreate(&e1));
  float best = 0;
  int best_pv = 0, best_ct = 1;
  for (int cand = 0; cand < 4; ++cand) {
    const int pv = (cand & 1) ? 2 : 0, ct = (cand & 2) ? 2 : 1;
    fft->pv = pv;
    fft->ct = ct;
    for (int i = 0; i < 2; ++i) {
      fwd_list(in, 0);
      inv_list(0, out);
    }
    MEU_CUDA(cudaEventRecord(e0, st));
    for (int i = 0; i < 4; ++i) {
      fwd_list(in, 0);
      inv_list(0, out);
    }
    MEU_CUDA(cudaEventRecord(e1, st));
    MEU_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MEU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (cand == 0 || ms < best) {
      best = ms;
      best_pv = pv;
      best_ct = ct;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fft->pv = best_pv;
  fft->ct = best_ct;
  MEU_CUDA(cudaMemsetAsync(sp, 0, sizeof(C) * (size_t)NS * nk, st));
  MEU_CUDA(cudaMemsetAsync(fd, 0, sizeof(R) * V * n3, st));
  MEU_CUDA(cudaStreamSynchronize(st));
}

template <typename R>
void Engine<R>::set_schedule(const int32_t* in3) {
  if (!fused) {
    // the transforms keep no state between calls, so the plan may change at any time
    if ((in3[0] != 0 && in3[0] != 2) || in3[1] != 0 || (in3[2] != 1 && in3[2] != 2))
      throw CudaError("generic path: the schedule is (radix plan 0 or 2, 0, column-tile factor 1 or 2)",
                      MEU_ERR_UNSUPPORTED);
    fft->pv = in3[0];
    fft->ct = in3[2];
    return;
  }
  if (fields_set) throw CudaError("set the schedule before the first meu_set_fields", MEU_ERR_BADARG);
  for (const LanSched& c : lan_sched_candidates(P.nx, sizeof(R) == 8)) {
    if (c.pv == in3[0] && c.ntp == in3[1] && c.tm == in3[2]) {
      sched = c;
      drop_graphs();
      fused_warm = false;
      return;
    }
  }
  throw CudaError("no such schedule for this grid and precision", MEU_ERR_UNSUPPORTED);
}

// zero fields, spectral state and history after the autotuner ran steps on them
template <typename R>
void Engine<R>::reset_fused_state() {
  MEU_CUDA(cudaMemsetAsync(c, 0, sizeof(R) * E * n3, st));
  MEU_CUDA(cudaMemsetAsync(phi, 0, sizeof(R) * V * n3, st));
  MEU_CUDA(cudaMemsetAsync(sp, 0, sizeof(C) * (size_t)NS * nk, st));
  MEU_CUDA(cudaMemsetAsync(keta, 0, sizeof(C) * V * nk, st));
  MEU_CUDA(cudaMemsetAsync(kc, 0, sizeof(C) * nk, st));
  MEU_CUDA(cudaMemsetAsync(hist, 0, sizeof(double) * HIST_MAX * Q_STEP_COUNT, st));
  MEU_CUDA(cudaMemsetAsync(d_row, 0, 2 * sizeof(int), st));
  MEU_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  MEU_CUDA(cudaStreamSynchronize(st));
  theta_ready = false;
}

template <typename R>
Engine<R>::~Engine() {
  if (st) cudaStreamSynchronize(st);
  if (own_st) cudaStreamSynchronize(own_st);
  drop_graphs();
  prof.reset();
  for (void* q : allocs) cudaFree(q);
  if (h_results) cudaFreeHost(h_results);
  if (h_err) cudaFreeHost(h_err);
  for (int b = 0; b < 2; ++b) {
    if (noise_host[b]) cudaFreeHost(noise_host[b]);
    if (noise_ev[b]) cudaEventDestroy(noise_ev[b]);
  }
  fft.reset();
  if (own_st) cudaStreamDestroy(own_st);
}

template <typename R>
void Engine<R>::check_err() {
  MEU_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MEU_CUDA(cudaStreamSynchronize(st));
  if (*h_err) {
    int code = *h_err;
    MEU_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    if (code == MEU_ERR_TIMEOUT) throw CudaError("a bounded device-side wait ran out in the step", code);
    throw CudaError("singular matrix in the step (reference err_flag " + std::to_string(code) + ")", code);
  }
}

template <typename R>
void Engine<R>::finalize(int q0, int nq, double* out, const int* nbs) {
  NbList nb;
  for (int q = 0; q < nq; ++q) nb.nb[q] = nbs ? nbs[q] : RED_BLOCKS;
  KLAUNCH("finalize", 8.0 * nq * RED_BLOCKS,
          k_finalize<<<nq, 256, 0, st>>>(partials + (int64_t)q0 * PSTRIDE, nb, d_ops + q0, out ? out : results + q0));
}

// ---- host-side AoS conversion in chunks through the staging buffer
template <typename R>
void Engine<R>::set_fields(const double* cons, const double* phi_in, const double* ustate) {
  auto up = [&](const double* src, R* dst, int ncomp, int add) {
    const int64_t chunk = std::max<int64_t>(stage_elems / ncomp, 1);
    for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
      const int64_t nv = std::min(chunk, n3 - v0);
      MEU_CUDA(cudaMemcpyAsync(stage, src + v0 * ncomp, sizeof(double) * nv * ncomp, cudaMemcpyHostToDevice, st));
      KLAUNCH("aos_to_soa", (double)nv * ncomp * (8 + sizeof(R)), k_aos_to_soa<R><<<grid_for(nv * ncomp, 256), 256, 0, st>>>(stage, dst, ncomp, v0, nv, n3, add, nullptr));
    }
  };
  if (cons) {
    // upload + conserved FP64 mean of each solute (the k = 0 mode), summed from
    // the double input in a fixed order: per chunk, block partials -> finalize -> accumulate
    MEU_CUDA(cudaMemsetAsync(cmean_acc, 0, sizeof(double) * MEU_MAX_EL, st));
    const int64_t chunk = std::max<int64_t>(stage_elems / E, 1);
    const bool one_chunk = chunk >= n3;
    for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
      const int64_t nv = std::min(chunk, n3 - v0);
      MEU_CUDA(cudaMemcpyAsync(stage, cons + v0 * E, sizeof(double) * nv * E, cudaMemcpyHostToDevice, st));
      KLAUNCH("aos_colsum", (double)nv * E * 8,
              k_aos_colsum<<<RED_BLOCKS, RED_THREADS, 0, st>>>(stage, E, nv, partials + (int64_t)Q_CSUM0 * PSTRIDE));
      finalize(Q_CSUM0, E);
      KLAUNCH("accumulate", 16.0 * E, k_accumulate<<<1, 32, 0, st>>>(results + Q_CSUM0, cmean_acc, E));
    }
    KLAUNCH("set_cmean", 16.0 * E, k_set_cmean<<<1, 32, 0, st>>>(dK, dF, cmean_acc, E, 1.0 / (double)n3));
    const double* offs = hK.c_shift ? dK->c_mean : nullptr;
    for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
      const int64_t nv = std::min(chunk, n3 - v0);
      if (!one_chunk)
        MEU_CUDA(cudaMemcpyAsync(stage, cons + v0 * E, sizeof(double) * nv * E, cudaMemcpyHostToDevice, st));
      KLAUNCH("aos_to_soa", (double)nv * E * (8 + sizeof(R)),
              k_aos_to_soa<R><<<grid_for(nv * E, 256), 256, 0, st>>>(stage, c, E, v0, nv, n3, 0, offs));
    }
  }
  if (phi_in) up(phi_in, phi, V, 0);
  if (cons || phi_in) {
    fields_set = true;
    theta_ready = false;
  }
  if (P.model == MEU_MODEL_LANDAU && (cons || phi_in)) {
    // spectral state of the step from the uploaded real fields
    if (fused) {
      sync_args();
      if (!lan_fused_init<R>(P.nx, V, sched, dA, 1, st, &prof))
        throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
    } else {
      PtrList<const R> a{};
      PtrList<C> b{};
      a.p[0] = c;
      b.p[0] = kc;
      for (int v = 0; v < V; ++v) {
        a.p[1 + v] = field(phi, v);
        b.p[1 + v] = keta + (int64_t)v * nk;
      }
      fft->forward<R>(a, b, 1 + V, st);
      KLAUNCH("zero_k0", 16.0, k_zero_k0<R><<<1, 32, 0, st>>>(kc));
    }
  }
  if (strain) {
    if (ustate) {
      // u (3 x n3) -> u^ ; grads (9 x n3) -> engineering strain
      for (int i = 0; i < 3; ++i) {
        const int64_t chunk = stage_elems;
        for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
          const int64_t nv = std::min(chunk, n3 - v0);
          MEU_CUDA(cudaMemcpyAsync(stage, ustate + i * n3 + v0, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
          KLAUNCH("convert_in", (double)nv * (8 + sizeof(R)), k_convert_in<R><<<grid_for(nv, 256), 256, 0, st>>>(stage, wr + v0, nv));
        }
        PtrList<const R> a{};
        PtrList<C> b{};
        a.p[0] = wr;
        b.p[0] = uk + (int64_t)i * nk;
        fft->forward<R>(a, b, 1, st);
      }
      // the 9 gradients, chunked through the staging buffer
      const int64_t chunk = std::max<int64_t>(stage_elems / 9, 1);
      for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
        const int64_t nv = std::min(chunk, n3 - v0);
        for (int g = 0; g < 9; ++g)
          MEU_CUDA(cudaMemcpyAsync(stage + (int64_t)g * nv, ustate + (int64_t)(3 + g) * n3 + v0, sizeof(double) * nv,
                                   cudaMemcpyHostToDevice, st));
        KLAUNCH("grads_to_strain", (double)nv * (9 * 8 + 6 * sizeof(R)), k_grads_to_strain<R><<<grid_for(nv, 256), 256, 0, st>>>(stage, strain + v0, nv, n3));
      }
      el_ready = true;
    } else {
      MEU_CUDA(cudaMemsetAsync(strain, 0, sizeof(R) * 6 * n3, st));
      MEU_CUDA(cudaMemsetAsync(uk, 0, sizeof(C) * 3 * nk, st));
      el_ready = false;
    }
  }
  MEU_CUDA(cudaStreamSynchronize(st));
}

template <typename R>
void Engine<R>::add_noise(const double* incr) {
  if (!noise) return;
  const int64_t chunk = std::max<int64_t>(stage_elems / V, 1);
  for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
    const int64_t nv = std::min(chunk, n3 - v0);
    MEU_CUDA(cudaMemcpyAsync(stage, incr + v0 * V, sizeof(double) * nv * V, cudaMemcpyHostToDevice, st));
    KLAUNCH("aos_to_soa", (double)nv * V * (8 + 2 * sizeof(R)), k_aos_to_soa<R><<<grid_for(nv * V, 256), 256, 0, st>>>(stage, noise, V, v0, nv, n3, 1, nullptr));
  }
  MEU_CUDA(cudaStreamSynchronize(st));
}

// phi_noise += one step's increments already in device memory (Fortran layout)
template <typename R>
void Engine<R>::upload_noise(const double* dev_incr) {
  KLAUNCH("aos_to_soa", (double)n3 * V * (8 + 2 * sizeof(R)),
          k_aos_to_soa<R><<<grid_for(n3 * V, 256), 256, 0, st>>>(dev_incr, noise, V, 0, n3, n3, 1, nullptr));
}

// The noise of Multi_MEUMAPPS.f:552-571: while step <= noise_step, every step first
// adds V*n3 langevin draws (ran_2.f via ModFunc.f:77-100) to phi_noise, in the loop
// order of the reference (variant index fastest, then x, y, z).  ran_2 is one serial
// chain (each draw picks its shuffle-table slot from the previous one), so the draws
// stay on the host; a host thread generates step s+1's increments into one pinned
// buffer while step s runs, and each buffer goes up with one asynchronous copy.  The
// caller's rng state ends exactly where the same number of serial draws leaves it.
template <typename R>
void Engine<R>::run_noise(int nsteps, meu_ran2_state* rng, double sd, meu_diag* diag) {
  if (P.model != MEU_MODEL_KKS || !noise)
    throw CudaError("run_noise: the Langevin noise belongs to the KKS model", MEU_ERR_UNSUPPORTED);
  if (!rng) throw CudaError("run_noise: NULL ran_2 state", MEU_ERR_BADARG);
  const int64_t cnt = (int64_t)V * n3;
  int noisy = 0;  // the first `noisy` steps of the call draw noise (step <= noise_step)
  while (noisy < nsteps && step + noisy <= P.noise_step) ++noisy;
  if (noisy > 0 && !noise_dev) {
    for (int b = 0; b < 2; ++b) {
      void* hp = nullptr;
      MEU_CUDA(cudaMallocHost(&hp, sizeof(double) * cnt));
      noise_host[b] = (double*)hp;
      MEU_CUDA(cudaEventCreateWithFlags(&noise_ev[b], cudaEventDisableTiming));
    }
    noise_dev = dalloc<double>(cnt);
  }
  // the chain on the drawing thread, the transcendental part of its accepted pairs on the
  // other host threads (meu_langevin_fill: the numbers of cnt meu_langevin calls)
  const unsigned hc = std::thread::hardware_concurrency();  // 0 when unknown
  const int32_t fill_threads = (int32_t)(hc > 1 ? hc - 1 : 1);
  auto generate = [rng, sd, cnt, fill_threads](double* dst, cudaEvent_t free_ev) {
    cudaEventSynchronize(free_ev);  // the buffer's previous copy has run
    meu_langevin_fill(rng, sd, cnt, dst, fill_threads);
  };
  std::future<void> next;
  if (noisy > 0) next = std::async(std::launch::async, generate, noise_host[0], noise_ev[0]);
  int done = 0;
  hist_n = 0;
  while (done < nsteps) {
    const int chunk = std::min(nsteps - done, HIST_MAX);
    for (int i = 0; i < chunk; ++i) {
      const int s = done + i;
      if (s < noisy) {
        const int b = s & 1;
        next.get();
        MEU_CUDA(cudaMemcpyAsync(noise_dev, noise_host[b], sizeof(double) * cnt, cudaMemcpyHostToDevice, st));
        MEU_CUDA(cudaEventRecord(noise_ev[b], st));
        upload_noise(noise_dev);
        if (s + 1 < noisy) next = std::async(std::launch::async, generate, noise_host[b ^ 1], noise_ev[b ^ 1]);
      }
      kks_step(nullptr);
    }
    check_err();
    flush_hist(diag ? diag + done : nullptr);
    done += chunk;
  }
}

template <typename R>
void Engine<R>::get_fields(double* cons, double* phi_out, double* el_out, double* ustate) {
  auto down = [&](const R* src, double* dst, int ncomp, const double* offs = nullptr) {
    const int64_t chunk = std::max<int64_t>(stage_elems / ncomp, 1);
    for (int64_t v0 = 0; v0 < n3; v0 += chunk) {
      const int64_t nv = std::min(chunk, n3 - v0);
      KLAUNCH("soa_to_aos", (double)nv * ncomp * (8 + sizeof(R)), k_soa_to_aos<R><<<grid_for(nv * ncomp, 256), 256, 0, st>>>(src, stage, ncomp, v0, nv, n3, offs));
      MEU_CUDA(cudaMemcpyAsync(dst + v0 * ncomp, stage, sizeof(double) * nv * ncomp, cudaMemcpyDeviceToHost, st));
    }
  };
  if (cons) down(c, cons, E, hK.c_shift ? dK->c_mean : nullptr);
  if (phi_out) down(phi, phi_out, V);
  if (el_out) down(el_en, el_out, 1);
  if (ustate) {
    if (uk) {
      KLAUNCH("u_spectra", 15.0 * nk * sizeof(C), k_u_spectra<R><<<gridk(), 256, 0, st>>>(dK, uk, specs(0, 12)));
      for (int f = 0; f < 12; ++f) {
        PtrList<C> a{};
        PtrList<R> b{};
        a.p[0] = spec(f);
        b.p[0] = wr;
        fft->inverse<R>(a, b, 1, st);
        down(wr, ustate + (int64_t)f * n3, 1);
      }
    } else {
      memset(ustate, 0, sizeof(double) * 12 * n3);
    }
  }
  MEU_CUDA(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------- elasticity
// eldis (ModElastic.f:11-489) + elener (:493-691).  P_phi in pphi.
template <typename R>
void Engine<R>::elastic(const R* ph_for_ppr, R* elg, int mode, bool zeroth_only) {
  const bool first = zeroth_only || step == P.elastep0 || !el_ready;
  // the reference computes the zeroth order only at step == elastep0; a run that
  // enters later without an uploaded state starts from u = 0 like the reference.
  const bool do_zeroth = zeroth_only || step == P.elastep0;
  (void)first;
  if (do_zeroth) {
    std::vector<const R*> in;
    for (int v = 0; v < V; ++v) in.push_back(field(pphi, v));
    fwd_list(in, 0);
    KLAUNCH("el_zeroth", (double)(V + 9) * nk * sizeof(C), k_el_zeroth<R><<<gridk(), 256, 0, st>>>(dK, specs(0, V), V, uk, specs(V, 6), d_err));
    std::vector<R*> out;
    for (int m = 0; m < 6; ++m) out.push_back(field(strain, m));
    inv_list(V, out);
  }
  el_ready = true;
  int total = 0;
  if (!zeroth_only) {
    double newfac = 0.5, cfac = 1.0, err_old[6] = {0, 0, 0, 0, 0, 0};
    int niter = 0;
    bool converged = false;
    std::vector<R*> out;
    for (int m = 0; m < 6; ++m) out.push_back(field(strain, m));
    // spec(0..5) holds the strain spectrum of the last el_k and the real strain is not
    // formed yet: the next iteration runs its x passes and el_x as one kernel
    bool spec_pending = false;
    for (;;) {
      niter += 1;
      total += 1;
      if (total > 100000) throw CudaError("elastic iteration runaway", MEU_ERR_NOT_CONVERGED);
      if (spec_pending) {
        fft->inverse_cols<R>(specs(0, 6), 6, st);
        KLAUNCH("el_rows", 6.0 * 2 * nk * sizeof(C) + (double)V * n3 * sizeof(R),
                el_rows_launch<R>(*fft, specs(0, 6), pphi, el_prop_r, el_ortho, cfac, d_err, st));
        fft->forward_cols<R>(specs(0, 6), 6, st);
        spec_pending = false;
      } else {
        if (hK.prop_moduli) {
          KLAUNCH("el_x", (double)(V + 12) * n3 * sizeof(R),
                  fn_el_x<<<g_el_x, PF_TILE, sm_el_x, st>>>(el_prop, (int64_t)n3, pphi, strain, xs, cfac, d_err));
        } else
          KLAUNCH("el_x", (double)(V + 12) * n3 * sizeof(R),
                  (el_ortho_gen ? k_el_x<R, true> : k_el_x<R>)<<<gridr(), 256, 0, st>>>(dK, pphi, strain, xs, cfac, d_err));
        std::vector<const R*> in;
        for (int m = 0; m < 6; ++m) in.push_back(field(xs, m));
        fwd_list(in, 0);
      }
      KLAUNCH("el_k", 18.0 * nk * sizeof(C), k_el_k<R><<<g_el_k, RED_THREADS, 0, st>>>(dK, specs(0, 6), uk, partials, d_err));
      if (el_fused_rows) spec_pending = true;
      else inv_list(0, out);
      finalize(Q_ERR0, 6);
      MEU_CUDA(cudaMemcpyAsync(h_results + Q_ERR0, results + Q_ERR0, sizeof(double) * 6, cudaMemcpyDeviceToHost, st));
      check_err();  // synchronises
      double err[6];
      for (int q = 0; q < 6; ++q) err[q] = h_results[Q_ERR0 + q] * (double)n3;
      const double tol = P.el_tol;
      if (err[0] / err[1] < tol && err[2] / err[3] < tol && err[4] / err[5] < tol) converged = true;
      if (niter > 1 && !converged) {
        if (err[0] / err[1] > err_old[0] / err_old[1] || err[2] / err[3] > err_old[2] / err_old[3] ||
            err[4] / err[5] > err_old[4] / err_old[5]) {
          cfac = cfac * newfac;
          newfac = newfac * 0.5;
          if (newfac < 1e-7) throw CudaError("newfac is too small ... trouble converging", MEU_ERR_NOT_CONVERGED);
          niter = 0;
          converged = false;
          continue;
        }
      }
      memcpy(err_old, err, sizeof(err));
      if (niter == P.el_max_iter) converged = true;
      if (!converged || niter < P.el_min_iter) continue;
      if (cfac < 1.0 - 1e-6) {
        cfac = cfac + 0.1;
        if (cfac > 1.0) cfac = 1.0;
        niter = 0;
        converged = false;
        continue;
      }
      break;
    }
    if (spec_pending) inv_list(0, out);
  }
  last_iters = total;
  const int eta2 = (P.model == MEU_MODEL_LANDAU && P.eig_coupling == MEU_EIG_ETA2) ? 1 : 0;
  if (hK.prop_moduli) {
    KLAUNCH("elener", (double)(2 * V + 6 + 1 + V) * n3 * sizeof(R),
            fn_elener<<<g_elener, PF_TILE, sm_elener, st>>>(en_prop, (int64_t)n3, ph_for_ppr, pphi, strain, el_en, elg,
                                                            mode, eta2, partials, d_err));
  } else
    KLAUNCH("elener", (double)(2 * V + 6 + 1 + V) * n3 * sizeof(R),
            (el_ortho_gen ? k_elener<R, true> : k_elener<R>)<<<g_elener, RED_THREADS, 0, st>>>(dK, ph_for_ppr, pphi, strain, el_en, elg, mode,
                                                  (P.model == MEU_MODEL_LANDAU && P.eig_coupling == MEU_EIG_ETA2) ? 1 : 0,
                                                  partials, d_err));
}

// ------------------------------------------------------------------- KKS step
template <typename R>
void Engine<R>::kks_step(meu_diag* d) {
  MEU_CUDA(cudaMemsetAsync(partials, 0, sizeof(double) * Q_TOTAL * PSTRIDE, st));
  if (!(step <= P.noise_step)) MEU_CUDA(cudaMemsetAsync(noise, 0, sizeof(R) * V * n3, st));
  // spectral gradients (:575-615)
  {
    std::vector<const R*> in;
    for (int v = 0; v < V; ++v) in.push_back(field(phi, v));
    fwd_list(in, 0);
    KLAUNCH("kks_grad", (double)5 * V * nk * sizeof(C), k_kks_grad<R><<<gridk(), 256, 0, st>>>(dK, spec(0), spec(V), V));
    std::vector<R*> out;
    for (int f = 0; f < 4 * V; ++f) out.push_back(field(wr, f));
    inv_list(V, out);
  }
  // local driving force (:619-845)
  {
    // compile-time phase and solute counts for the common decks (composition solve in registers)
    auto kp = k_kks_point<R>;
    if (P.numph == 2 && P.numel == 1) kp = k_kks_point<R, 2, 1>;
    else if (P.numph == 3 && P.numel == 1) kp = k_kks_point<R, 3, 1>;
    else if (P.numph == 2 && P.numel == 2) kp = k_kks_point<R, 2, 2>;
    KLAUNCH("kks_point", (double)(7 * V + 4 * E) * n3 * sizeof(R),
            kp<<<RED_BLOCKS, RED_THREADS, 0, st>>>(dK, phi, c, wr, pphi, fd, fc, partials, d_err));
  }
  // elasticity (:851-880)
  last_iters = 0;
  if (step >= P.elastep0 && P.elastic != MEU_ELAST_NONE) {
    elastic(phi, fd, 0, false);
  } else {
    MEU_CUDA(cudaMemsetAsync(el_en, 0, sizeof(R) * n3, st));
  }
  // diffusion (:910-949)
  for (int e = 0; e < E; ++e) {
    fwd({field(c, e), field(fc, 3 * e), field(fc, 3 * e + 1), field(fc, 3 * e + 2)}, 0);
    KLAUNCH("kks_ch", 5.0 * nk * sizeof(C), k_kks_ch<R><<<gridk(), 256, 0, st>>>(dK, spec(0), spec(1), spec(2), spec(3), P.dt * P.cmobs[e]));
    inv_list(0, {field(c, e)});
  }
  // TDGL (:955-1001)
  KLAUNCH("tdgl_pre", 4.0 * V * n3 * sizeof(R), k_tdgl_pre<R><<<grid_for((int64_t)V * n3, 256), 256, 0, st>>>(phi, fd, noise, wr, (int64_t)V * n3, P.dt * P.b_mob, P.dt));
  {
    std::vector<const R*> in;
    for (int v = 0; v < V; ++v) in.push_back(field(wr, v));
    fwd_list(in, 0);
    KLAUNCH("tdgl", 2.0 * V * nk * sizeof(C), k_tdgl<R><<<gridk(), 256, 0, st>>>(dK, specs(0, V), V, P.dt * P.b_mob));
    std::vector<R*> out;
    for (int v = 0; v < V; ++v) out.push_back(field(phi, v));
    inv_list(0, out);
  }
  end_step(d, 1);
}

// ---------------------------------------------------------------- Landau step
template <typename R>
LanFusedArgs<R> Engine<R>::fused_args() const {
  LanFusedArgs<R> a;
  memset(&a, 0, sizeof(a));
  a.F = dF;
  a.eta = phi;
  a.c = c;
  a.M = sp;
  a.Keta = keta;
  a.Kc = kc;
  a.partials = partials;
  a.err = d_err;
  a.homog = (P.elastic != MEU_ELAST_NONE && step >= P.elastep0) ? 1 : 0;
  a.energy = P.diag_energy;
  a.twx = (const C*)fft->px.tw;
  a.twy = (const C*)fft->py.tw;
  a.twz = (const C*)fft->pz.tw;
  a.post = (const C*)fft->post_tw;
  a.hist = hist;
  a.hist_row = d_row;
  a.ticket = d_ticket;
  a.hist_rows = HIST_MAX;
  a.eta_next = phi;
  a.c_next = c;
  a.Keta_out = keta;
  a.Kc_out = kc;
  a.gtab = gtab;
  return a;
}

template <typename R>
void Engine<R>::sync_args() {
  const LanFusedArgs<R> a = fused_args();
  if (hA_valid && memcmp(&a, &hA, sizeof(a)) == 0) return;
  hA = a;
  hA_valid = true;
  // pageable source: the call returns once hA has been staged, so hA may change afterwards
  MEU_CUDA(cudaMemcpyAsync(dA, &hA, sizeof(hA), cudaMemcpyHostToDevice, st));
}

template <typename R>
void Engine<R>::fused_step_launches() {
  const int opts = (P.diag_energy ? LS_ENERGY : 0) | (theta_ready ? LS_THETA_READY : 0) | (q_checked ? 0 : LS_QCHECK);
  q_checked = true;  // the first step is never captured (fused_warm is false until it has run)
  if (!lan_fused_step<R>(P.nx, V, sched, dA, 1, opts, st, &prof, fnb))
    throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
  theta_ready = true;
}

template <typename R>
void Engine<R>::landau_step_fused() { fused_steps(1); }

// Captures 2^slot fused steps into gexec[slot] without running them.
template <typename R>
void Engine<R>::capture_graph(int slot) {
  const int k = 1 << slot;
  const int64_t l0 = prof.launches;
  cudaGraph_t g = nullptr;
  MEU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    for (int i = 0; i < k; ++i) fused_step_launches();
  } catch (...) {
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  MEU_CUDA(cudaStreamEndCapture(st, &g));
  const cudaError_t e = cudaGraphInstantiate(&gexec[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    gexec[slot] = nullptr;
    throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e), MEU_ERR_CUDA);
  }
  graph_launches[slot] = prof.launches - l0;
  prof.launches = l0;  // captured, not run
}

template <typename R>
void Engine<R>::drop_graphs() {
  for (auto& g : gexec) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

// n fused steps into history rows hist_n .. hist_n + n - 1 (d_row == hist_n on entry).
// Once the step is warm, every run of steps with one elastic state (homog flag) replays
// CUDA graphs of 8, 4, 2 and 1 steps (largest first) when the per-kernel timer is off
// and the stream can be captured.  The graphs are captured at the end of the first call
// that leaves the step able to replay them, so a later call of any length only replays
// (capture and instantiation stay out of the caller's next timed run).
template <typename R>
void Engine<R>::fused_steps(int n) {
  int done = 0;
  while (done < n) {
    sync_args();
    const bool can = fused_warm && theta_ready && !prof.on && st != nullptr;
    int slot = -1;
    if (can) {
      const bool homog_now = hA.homog != 0;
      for (int sl = GRAPH_SLOTS - 1; sl >= 0; --sl) {
        const int k = 1 << sl;
        const bool homog_later = P.elastic != MEU_ELAST_NONE && step + k - 1 >= P.elastep0;
        if (n - done >= k && homog_now == homog_later) {
          slot = sl;
          break;
        }
      }
    }
    if (slot >= 0) {
      const int k = 1 << slot;
      if (!gexec[slot]) capture_graph(slot);
      MEU_CUDA(cudaGraphLaunch(gexec[slot], st));
      prof.launches += graph_launches[slot];
      for (int i = 0; i < k; ++i) {
        hist_step[hist_n] = step;
        hist_iters[hist_n] = 0;
        hist_n += 1;
        step += 1;
      }
      done += k;
    } else {
      fused_step_launches();
      fused_warm = true;  // kernel attributes are set; capture is possible from here
      hist_step[hist_n] = step;
      hist_iters[hist_n] = 0;
      hist_n += 1;
      step += 1;
      done += 1;
    }
  }
  if (fused_warm && theta_ready && !prof.on && st != nullptr)
    for (int sl = 0; sl < GRAPH_SLOTS; ++sl)
      if (!gexec[sl]) capture_graph(sl);
  last_iters = 0;
}

template <typename R>
void Engine<R>::landau_step(meu_diag* d) {
  if (fused) {
    landau_step_fused();
    return;
  }
  // generic path: eta^ and dc^ are spectral state (keta, kc); the real fields
  // are re-derived each step for the nonlinear terms
  MEU_CUDA(cudaMemsetAsync(partials, 0, sizeof(double) * Q_TOTAL * PSTRIDE, st));
  const bool elast = P.elastic != MEU_ELAST_NONE && step >= P.elastep0;
  const bool homog = elast && P.elastic == MEU_ELAST_HOMOG;
  const bool het = elast && P.elastic == MEU_ELAST_HETERO;
  R* mu = field(wr, 0);
  KLAUNCH("lan_a", (double)(2 * V + 2) * n3 * sizeof(R), k_lan_a<R><<<RED_BLOCKS, RED_THREADS, 0, st>>>(dK, c, phi, pphi, mu, partials));
  {
    std::vector<const R*> in;
    for (int v = 0; v < V; ++v) in.push_back(field(pphi, v));
    in.push_back(mu);
    fwd_list(in, 0);
  }
  KLAUNCH("lan_k1", (double)(homog ? 3 * V + 4 : 2 * V + 4) * nk * sizeof(C),
          k_lan_k1<R><<<g_lan_k1, RED_THREADS, 0, st>>>(dK, specs(0, V + 1), V, kc, keta, homog ? 1 : 0,
                                                          P.diag_energy, partials, d_err));
  R* phel = field(wr, 1);  // V fields: strain interaction (homog) or el_grad (hetero)
  {
    std::vector<R*> out;
    if (homog) {
      for (int v = 0; v < V; ++v) out.push_back(field(phel, v));
      out.push_back(c2);
      inv_list(0, out);
    } else {
      inv_list(V, {c2});
    }
  }
  last_iters = 0;
  if (het) {
    // P_phi = theta (already in pphi), elener gives el_grad into phel
    elastic(phi, phel, 1, false);
  } else if (!homog) {
    MEU_CUDA(cudaMemsetAsync(el_en, 0, sizeof(R) * n3, st));
  }
  KLAUNCH("lan_b", (double)(3 * V + 1) * n3 * sizeof(R), k_lan_b<R><<<gridr(), 256, 0, st>>>(dK, c, phi, elast ? phel : nullptr, homog ? 1 : 0, pphi));
  {
    std::vector<const R*> in;
    for (int v = 0; v < V; ++v) in.push_back(field(pphi, v));
    fwd_list(in, 0);
    KLAUNCH("tdgl", 4.0 * V * nk * sizeof(C), k_tdgl_state<R><<<gridk(), 256, 0, st>>>(dK, specs(0, V), V, keta, P.dt * P.b_mob));
    std::vector<R*> out;
    for (int v = 0; v < V; ++v) out.push_back(field(phi, v));
    inv_list(0, out);
  }
  std::swap(c, c2);
  end_step(d, P.clip_phi);
}

template <typename R>
void Engine<R>::end_step(meu_diag* d, int clip) {
  KLAUNCH("stats", (double)(E + V * (clip ? 2 : 1)) * n3 * sizeof(R),
          k_stats<R><<<RED_BLOCKS, RED_THREADS, 0, st>>>(dK, c, phi, clip, partials));
  // this step's reductions go straight into the device history, read once per meu_run
  finalize(0, Q_STEP_COUNT, hist + (int64_t)hist_n * Q_STEP_COUNT);
  hist_step[hist_n] = step;
  hist_iters[hist_n] = last_iters;
  hist_n += 1;
  (void)d;
  step += 1;
}

// Turn the device history of reductions into fort.98 / fort.99 rows.
template <typename R>
void Engine<R>::flush_hist(meu_diag* diag) {
  if (hist_n == 0) return;
  std::vector<double> h((size_t)hist_n * Q_STEP_COUNT);
  MEU_CUDA(cudaMemcpyAsync(h.data(), hist, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  MEU_CUDA(cudaStreamSynchronize(st));
  const double sn3 = (double)n3;
  const bool lan = P.model == MEU_MODEL_LANDAU;
  for (int i = 0; i < hist_n; ++i) {
    const double* r = h.data() + (size_t)i * Q_STEP_COUNT;
    if (diag) {
      meu_diag* d = diag + i;
      d->step = hist_step[i];
      d->el_iters = hist_iters[i];
      d->status = 0;
      d->fint = lan ? (r[Q_FINT] + r[Q_FINT2]) * sn3 : r[Q_FINT];
      d->fw = r[Q_FW];
      d->fch = r[Q_FCH];
      d->elen = (lan && P.elastic == MEU_ELAST_HOMOG) ? r[Q_ELEN] * sn3 : r[Q_ELEN];
      d->etot = d->fint + d->fch + d->elen + d->fw;
      d->glob_min = prev_min;
      d->glob_max = prev_max;
      d->phi_max = prev_phimax;
      d->solid = prev_solid / sn3;
      d->cmin = r[Q_CMIN];
      d->cmax = r[Q_CMAX];
      d->phimax = r[Q_PHIMAX];
      d->solid_now = r[Q_SOLID] / sn3;
      for (int e = 0; e < MEU_MAX_EL; ++e) d->cavg[e] = e < E ? r[Q_CSUM0 + e] / sn3 : 0.0;
    }
    prev_min = r[Q_CMIN];
    prev_max = r[Q_CMAX];
    prev_phimax = r[Q_PHIMAX];
    prev_solid = r[Q_SOLID];
    const double et = r[Q_FINT] + r[Q_FCH] + r[Q_ELEN] + r[Q_FW];
    if (!std::isfinite(et) || !std::isfinite(r[Q_CSUM0]) || !std::isfinite(r[Q_SOLID])) {
      hist_n = 0;
      throw CudaError("non-finite field values at step " + std::to_string(hist_step[i]), MEU_ERR_NOT_FINITE);
    }
  }
  hist_n = 0;
}

template <typename R>
void Engine<R>::run(int nsteps, meu_diag* diag) {
  int done = 0;
  hist_n = 0;
  while (done < nsteps) {
    const int chunk = std::min(nsteps - done, HIST_MAX);
    if (fused) {
      MEU_CUDA(cudaMemsetAsync(d_row, 0, 2 * sizeof(int), st));
      fused_steps(chunk);
    } else {
      for (int i = 0; i < chunk; ++i) {
        if (P.model == MEU_MODEL_KKS) kks_step(nullptr);
        else landau_step(nullptr);
      }
    }
    check_err();
    flush_hist(diag ? diag + done : nullptr);
    done += chunk;
  }
}

template class Engine<double>;
template class Engine<float>;

}  // namespace meu

// =============================================================== C-ABI
struct meu_handle {
  std::unique_ptr<meu::EngineBase> eng;
  std::string err;
};

static int fail(meu_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define MEU_TRY(h, body)                                              \
  try {                                                               \
    body;                                                             \
  } catch (const meu::CudaError& e) {                                 \
    return fail(h, e.code, e.what());                                 \
  } catch (const std::bad_alloc&) {                                   \
    return fail(h, MEU_ERR_NOMEM, "host allocation failed");          \
  } catch (const std::exception& e) {                                 \
    return fail(h, MEU_ERR_CUDA, e.what());                           \
  }

static thread_local std::string g_create_err;
namespace meu {
// message returned by meu_last_error(NULL) for calls that have no handle
void set_thread_error(const std::string& msg) { g_create_err = msg; }
}  // namespace meu

extern "C" {

int meu_create(const meu_params* params, meu_handle** out) {
  if (!params || !out) return MEU_ERR_BADARG;
  *out = nullptr;
  meu_handle* h = new (std::nothrow) meu_handle();
  if (!h) return MEU_ERR_NOMEM;
  try {
    if (params->precision == MEU_PREC_F64) h->eng.reset(new meu::Engine<double>(*params));
    else if (params->precision == MEU_PREC_F32) h->eng.reset(new meu::Engine<float>(*params));
    else throw meu::CudaError("unknown precision", MEU_ERR_BADARG);
  } catch (const meu::CudaError& e) {
    g_create_err = e.what();
    delete h;
    return e.code;
  } catch (const std::exception& e) {
    g_create_err = e.what();
    delete h;
    return MEU_ERR_CUDA;
  }
  *out = h;
  return MEU_OK;
}

int meu_set_fields(meu_handle* h, const double* cons, const double* phi, const double* u_state) {
  if (!h) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->set_fields(cons, phi, u_state));
  return MEU_OK;
}

int meu_run_noise(meu_handle* h, int32_t nsteps, meu_ran2_state* rng, double sd, meu_diag* diag) {
  if (!h || nsteps < 0) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->run_noise(nsteps, rng, sd, diag));
  return MEU_OK;
}

int meu_add_noise(meu_handle* h, const double* incr) {
  if (!h || !incr) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->add_noise(incr));
  return MEU_OK;
}

int meu_run(meu_handle* h, int32_t nsteps, meu_diag* diag) {
  if (!h || nsteps < 0) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->run(nsteps, diag));
  return MEU_OK;
}

int meu_get_fields(meu_handle* h, double* cons, double* phi, double* el_en, double* u_state) {
  if (!h) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->get_fields(cons, phi, el_en, u_state));
  return MEU_OK;
}

int64_t meu_get_step(const meu_handle* h) { return h ? h->eng->step : -1; }

const char* meu_last_error(const meu_handle* h) {
  if (!h) return g_create_err.c_str();
  return h->err.c_str();
}

int meu_set_stream(meu_handle* h, void* cuda_stream) {
  if (!h) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->set_stream((cudaStream_t)cuda_stream));
  return MEU_OK;
}

int meu_timing(meu_handle* h, int32_t enable) {
  if (!h) return MEU_ERR_BADARG;
  MEU_TRY(h, {
    h->eng->prof.reset();
    h->eng->prof.on = enable != 0;
  });
  return MEU_OK;
}

int32_t meu_timing_report(meu_handle* h, int32_t max, char* names, int64_t* counts, double* total_ms, double* bytes) {
  if (!h || max < 0) return -MEU_ERR_BADARG;
  try {
    meu::Profiler& pr = h->eng->prof;
    pr.resolve();
    const int n = (int)pr.names.size();
    for (int i = 0; i < n && i < max; ++i) {
      if (names) {
        memset(names + 32 * i, 0, 32);
        strncpy(names + 32 * i, pr.names[i].c_str(), 31);
      }
      if (counts) counts[i] = pr.stats[i].n;
      if (total_ms) total_ms[i] = pr.stats[i].ms;
      if (bytes) bytes[i] = pr.stats[i].bytes;
    }
    return n;
  } catch (const meu::CudaError& e) {
    h->err = e.what();
    return -e.code;
  }
}

int64_t meu_launch_count(const meu_handle* h) { return h ? h->eng->prof.launches : -1; }

int meu_adjoint(meu_handle* h, int32_t nsteps, int32_t checkpoint_every, const double* cons_target,
                const double* phi_target, double* loss, double* dparams, double* dphi0) {
  if (!h) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->adjoint(nsteps, checkpoint_every, cons_target, phi_target, loss, dparams, dphi0));
  return MEU_OK;
}

int meu_set_schedule(meu_handle* h, const int32_t* in3) {
  if (!h || !in3) return MEU_ERR_BADARG;
  MEU_TRY(h, h->eng->set_schedule(in3));
  return MEU_OK;
}

int meu_schedule(meu_handle* h, int32_t* out3) {
  if (!h || !out3) return MEU_ERR_BADARG;
  if (!h->eng->schedule(out3)) return fail(h, MEU_ERR_UNSUPPORTED, "the handle has no schedule");
  return MEU_OK;
}

int meu_destroy(meu_handle* h) {
  if (!h) return MEU_ERR_BADARG;
  delete h;
  return MEU_OK;
}

}  // extern "C"

// ---------------------------------------------------------- diagnostics
namespace {
// device buffer freed when the call returns, on success and on every error path
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

extern "C" int meu_fft_roundtrip(int32_t nx, int32_t ny, int32_t nz, int32_t precision, const double* in,
                                 double* spec_out, double* back_out) {
  using namespace meu;
  try {
    if (!in || !spec_out || !back_out) {
      set_thread_error("meu_fft_roundtrip: NULL array");
      return MEU_ERR_BADARG;
    }
    if (!fft_size_ok(nx, true) || !fft_size_ok(ny, false) || !fft_size_ok(nz, false)) {
      set_thread_error("meu_fft_roundtrip: grid sizes must be 2^a 3^b with Nx even");
      return MEU_ERR_UNSUPPORTED;
    }
    const bool f64 = precision == MEU_PREC_F64;
    if (!f64 && precision != MEU_PREC_F32) {
      set_thread_error("meu_fft_roundtrip: unknown precision");
      return MEU_ERR_BADARG;
    }
    FFT3 f(nx, ny, nz, f64);
    const int64_t n3 = f.n3(), nk = f.nk();
    DevBuf b_in, b_spec, b_fin, b_fsp;
    MEU_CUDA(cudaMalloc(&b_in.p, sizeof(double) * n3));
    MEU_CUDA(cudaMalloc(&b_spec.p, sizeof(double) * 2 * nk));
    double* d_in = (double*)b_in.p;
    double* d_spec = (double*)b_spec.p;
    MEU_CUDA(cudaMemcpy(d_in, in, sizeof(double) * n3, cudaMemcpyHostToDevice));
    cudaStream_t st = 0;
    if (f64) {
      PtrList<const double> a{};
      PtrList<double2> b{};
      a.p[0] = d_in;
      b.p[0] = (double2*)d_spec;
      f.forward<double>(a, b, 1, st);
      MEU_CUDA(cudaMemcpy(spec_out, d_spec, sizeof(double) * 2 * nk, cudaMemcpyDeviceToHost));
      PtrList<double2> c{};
      PtrList<double> d{};
      c.p[0] = (double2*)d_spec;
      d.p[0] = d_in;
      f.inverse<double>(c, d, 1, st);
      MEU_CUDA(cudaMemcpy(back_out, d_in, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    } else {
      MEU_CUDA(cudaMalloc(&b_fin.p, sizeof(float) * n3));
      MEU_CUDA(cudaMalloc(&b_fsp.p, sizeof(float2) * nk));
      float* fin = (float*)b_fin.p;
      float2* fsp = (float2*)b_fsp.p;
      k_convert_in<float><<<grid_for(n3, 256), 256>>>(d_in, fin, n3);
      MEU_CHECK_LAUNCH();
      PtrList<const float> a{};
      PtrList<float2> b{};
      a.p[0] = fin;
      b.p[0] = fsp;
      f.forward<float>(a, b, 1, st);
      k_convert<float><<<grid_for(2 * nk, 256), 256>>>((const float*)fsp, d_spec, 2 * nk);
      MEU_CHECK_LAUNCH();
      MEU_CUDA(cudaMemcpy(spec_out, d_spec, sizeof(double) * 2 * nk, cudaMemcpyDeviceToHost));
      PtrList<float2> c{};
      PtrList<float> d{};
      c.p[0] = fsp;
      d.p[0] = fin;
      f.inverse<float>(c, d, 1, st);
      k_convert<float><<<grid_for(n3, 256), 256>>>(fin, d_in, n3);
      MEU_CHECK_LAUNCH();
      MEU_CUDA(cudaMemcpy(back_out, d_in, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    }
    MEU_CUDA(cudaDeviceSynchronize());
  } catch (const CudaError& e) {
    set_thread_error(std::string("meu_fft_roundtrip: ") + e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_thread_error("meu_fft_roundtrip: host allocation failed");
    return MEU_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_thread_error(std::string("meu_fft_roundtrip: ") + e.what());
    return MEU_ERR_CUDA;
  }
  return MEU_OK;
}
