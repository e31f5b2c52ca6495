// adjoint.cu -- the adjoint of the fused Landau step: launch sequence, and the
// gradient driver Engine<R>::adjoint (forward with checkpoints, then per segment
// a recomputation that records the step's states followed by the adjoint steps
// in reverse).  Kernels: adjoint_kernels.cuh.
#include <algorithm>
#include <vector>

#include "adjoint_kernels.cuh"
#include "engine.cuh"

namespace meu {

namespace {

template <typename R>
__global__ void __launch_bounds__(256) k_ad_seed(const R* __restrict__ eta, const R* __restrict__ dc,
                                                 const LanFusedConst* __restrict__ F, const double* __restrict__ te,
                                                 const double* __restrict__ tc, R* lamT, R* nuT, int64_t n3, int V,
                                                 double* part) {
  const double cbar = F->cbar, inv = 1.0 / (double)n3;
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
    for (int v = 0; v < V; ++v) {
      const double d1 = (double)eta[v * n3 + i] - te[v * n3 + i];
      lamT[v * n3 + i] = (R)(d1 * inv);
      acc += d1 * d1;
    }
    const double d2 = cbar + (double)dc[i] - tc[i];
    nuT[i] = (R)(d2 * inv);
    acc += d2 * d2;
  }
  block_reduce_store(acc, 0, part + blockIdx.x);
}

// acc[q] += fixed-order sum of partials[q][0 .. nb[q])
__global__ void __launch_bounds__(256) k_ad_acc(const double* __restrict__ partials, NbList nb, double* acc) {
  const int q = blockIdx.x;
  double s = 0;
  for (int i = threadIdx.x; i < nb.nb[q]; i += blockDim.x) s += partials[(int64_t)q * PSTRIDE + i];
  const double x = block_reduce_value(s, 0);
  if (threadIdx.x == 0) acc[q] += x;
}

template <typename R>
__global__ void k_to_double(const R* __restrict__ src, double* dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

template <typename R, int N>
void adj_step_n(const AdjArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb) {
  using C = cplx<R>;
  using P = fz::Plane<R, N, adj::NTP, adj::PV>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1, tiles = N * NXH / TM;
  const double n3 = (double)N * N * N, nk = (double)N * N * NXH;
  const size_t sc = sizeof(C) * ((size_t)N * TM + N * Tw<C>::K);
  const size_t sp = P::smem_bytes();
  lf::ensure_smem(adj::k_ad_ea<R, N>, sc);
  lf::ensure_smem(adj::k_ad_c<R, N>, sc);
  lf::ensure_smem(adj::k_ad_b<R, N>, sp);
  lf::ensure_smem(adj::k_ad_d<R, N>, sp);
  {
    lf::Scope s(hook, "adj_z_lambda", 6.0 * nk * sizeof(C), st);
    adj::k_ad_ea<R, N><<<tiles, lf::NT, sc, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_plane_pointwise", 2.0 * nk * sizeof(C) + 4.0 * n3 * sizeof(R), st);
    adj::k_ad_b<R, N><<<N, adj::NTP, sp, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_z_nu", 4.0 * nk * sizeof(C), st);
    adj::k_ad_c<R, N><<<tiles, lf::NT, sc, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_plane_lambda", (a.lam_out ? 1.0 : 2.0) * nk * sizeof(C) + 3.0 * n3 * sizeof(R), st);
    adj::k_ad_d<R, N><<<N, adj::NTP, sp, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  for (int q = 0; q < Q_TOTAL; ++q) nb[q] = 0;
  nb[AQ_X] = nb[AQ_Y] = nb[AQ_Z] = tiles;
  nb[AQ_WG] = nb[AQ_EA] = N;
}

// one adjoint step of V >= 2 variants (adjoint.cuh: EA_v, B1_v, B2_v, B3_v, C_v, D_v)
template <typename R, int N, int V>
void adj_step_nv(const AdjArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb) {
  using C = cplx<R>;
  using P = fz::Plane<R, N, adj::NTP, adj::PV>;
  constexpr int TM = lf::col_tile_default<R>(), NXH = N / 2 + 1, tiles = N * NXH / TM;
  const double n3 = (double)N * N * N, nk = (double)N * N * NXH;
  const size_t sc = sizeof(C) * ((size_t)N * V * TM + N * Tw<C>::K);
  const size_t sp = P::smem_bytes();
  lf::ensure_smem(adj::k_ad_ea_v<R, N, V>, sc);
  lf::ensure_smem(adj::k_ad_c_v<R, N, V>, sc);
  lf::ensure_smem(adj::k_ad_b1_v<R, N>, sp);
  lf::ensure_smem(adj::k_ad_b3_v<R, N>, sp);
  lf::ensure_smem(adj::k_ad_d_v<R, N>, sp);
  {
    lf::Scope s(hook, "adj_z_lambda", (3.0 + 2.0) * V * nk * sizeof(C) + 2.0 * nk * sizeof(C), st);
    adj::k_ad_ea_v<R, N, V><<<tiles, lf::NT, sc, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_plane_w", V * (nk * sizeof(C) + n3 * sizeof(R)), st);
    adj::k_ad_b1_v<R, N><<<dim3(N, V), adj::NTP, sp, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_pointwise", (5.0 * V + 1.0) * n3 * sizeof(R), st);
    adj::k_ad_b2_v<R, V><<<RED_BLOCKS, RED_THREADS, 0, st>>>(a, (int64_t)n3);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_plane_h", V * (nk * sizeof(C) + n3 * sizeof(R)), st);
    adj::k_ad_b3_v<R, N><<<dim3(N, V), adj::NTP, sp, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_z_nu", 2.0 * V * nk * sizeof(C) + 2.0 * nk * sizeof(C), st);
    adj::k_ad_c_v<R, N, V><<<tiles, lf::NT, sc, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  {
    lf::Scope s(hook, "adj_plane_lambda", V * ((a.lam_out ? 1.0 : 2.0) * nk * sizeof(C) + 3.0 * n3 * sizeof(R)), st);
    adj::k_ad_d_v<R, N><<<dim3(N, V), adj::NTP, sp, st>>>(a);
    MEU_CHECK_LAUNCH();
  }
  for (int q = 0; q < Q_TOTAL; ++q) nb[q] = 0;
  nb[AQ_X] = nb[AQ_Y] = nb[AQ_Z] = tiles;
  nb[AQ_WG] = nb[AQ_EA] = RED_BLOCKS;
}

template <typename R, int N>
void adj_step_any(const AdjArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb) {
  switch (a.V) {
    case 1: adj_step_n<R, N>(a, st, hook, nb); break;
    case 2: adj_step_nv<R, N, 2>(a, st, hook, nb); break;
    case 3: adj_step_nv<R, N, 3>(a, st, hook, nb); break;
    case 4: adj_step_nv<R, N, 4>(a, st, hook, nb); break;
    default: throw CudaError("adjoint: 1 to 4 variants", MEU_ERR_UNSUPPORTED);
  }
}

}  // namespace

template <typename R>
bool adj_step(int N, const AdjArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb) {
  switch (N) {
    case 32: adj_step_any<R, 32>(a, st, hook, nb); return true;
    case 48: adj_step_any<R, 48>(a, st, hook, nb); return true;
    case 64: adj_step_any<R, 64>(a, st, hook, nb); return true;
    case 96: adj_step_any<R, 96>(a, st, hook, nb); return true;
    case 128: adj_step_any<R, 128>(a, st, hook, nb); return true;
    default: return false;
  }
}

// device memory of the gradient driver, kept by the engine between calls
template <typename R>
struct AdjBuffers {
  using C = cplx<R>;
  std::vector<void*> allocs;
  int K = 0, nck = 0;
  std::vector<R*> ck_eta, ck_c, s_eta, s_c, s_phi;
  std::vector<C*> ck_keta, ck_kc, ck_theta, s_keta, s_kc, s_theta;
  std::vector<int> ck_has_theta;  // the checkpoint holds the forward's theta^ of its fields
  int V = 0;
  C *nu = nullptr, *lam_seed = nullptr, *M = nullptr;  // M: the adjoint's own M-form field (the
                                                       // recomputation uses the engine's)
  R *aw = nullptr, *lamT = nullptr, *nuT = nullptr, *lam0 = nullptr, *wv = nullptr, *hv = nullptr;
  double *tgt_eta = nullptr, *tgt_c = nullptr, *partials = nullptr, *acc = nullptr, *loss_part = nullptr;
  double* d_out = nullptr;
  LanFusedArgs<R>* dRec = nullptr;  // recomputation records, one per step of a segment
  LanFusedArgs<R>* hRec = nullptr;  // pinned staging of dRec
  LanFusedArgs<R>* dFwd = nullptr;  // forward (in place) and seed-transform records
  LanFusedArgs<R>* dSeed = nullptr;
  template <typename T> T* alloc(int64_t n) {
    void* p = nullptr;
    MEU_CUDA(cudaMalloc(&p, sizeof(T) * (size_t)std::max<int64_t>(n, 1)));
    allocs.push_back(p);
    return (T*)p;
  }
  ~AdjBuffers() {
    for (void* p : allocs) cudaFree(p);
    if (hRec) cudaFreeHost(hRec);
  }
};
template <typename R>
void adj_buffers_free(AdjBuffers<R>* b) { delete b; }

template <typename R>
void Engine<R>::adjoint(int T, int K, const double* cons_tgt, const double* phi_tgt, double* loss, double* dparams,
                        double* dphi0) {
  if (!fused || V < 1 || V > 4)
    throw CudaError("the adjoint covers the fused Landau step with 1 to 4 order parameters", MEU_ERR_UNSUPPORTED);
  const int tm_def = sizeof(R) == 4 ? 16 : 8;
  if (sched.pv != 0 || sched.ntp != 512 || (sched.tm != 0 && sched.tm != tm_def))
    throw CudaError("the adjoint runs on the default schedule", MEU_ERR_UNSUPPORTED);
  if (T < 1 || K < 1 || !cons_tgt || !phi_tgt) throw CudaError("adjoint: bad arguments", MEU_ERR_BADARG);
  if (!fields_set) throw CudaError("adjoint: set the initial fields first", MEU_ERR_BADARG);
  K = std::min(K, T);
  const int nck = (T + K - 1) / K;
  const int N = P.nx;
  // ---- buffers
  if (!adjb || adjb->K < K || adjb->nck < nck || adjb->V != V) {
    adjb.reset();
    AdjBuffers<R>* b = new AdjBuffers<R>();
    adjb = std::unique_ptr<AdjBuffers<R>, void (*)(AdjBuffers<R>*)>(b, adj_buffers_free<R>);
    b->K = K;
    b->nck = nck;
    b->V = V;
    const int64_t vn3 = (int64_t)V * n3, vnk = (int64_t)V * nk;
    for (int i = 0; i < nck; ++i) {
      b->ck_eta.push_back(b->template alloc<R>(vn3));
      b->ck_c.push_back(b->template alloc<R>(n3));
      b->ck_keta.push_back(b->template alloc<C>(vnk));
      b->ck_kc.push_back(b->template alloc<C>(nk));
      b->ck_theta.push_back(b->template alloc<C>(vnk));  // theta^_v: the first V M-form fields
    }
    b->ck_has_theta.assign(nck, 0);
    for (int j = 0; j <= K; ++j) {
      b->s_eta.push_back(b->template alloc<R>(vn3));
      b->s_c.push_back(b->template alloc<R>(n3));
      b->s_keta.push_back(b->template alloc<C>(vnk));
      b->s_kc.push_back(b->template alloc<C>(nk));
      b->s_phi.push_back(b->template alloc<R>(vn3));
      b->s_theta.push_back(b->template alloc<C>(vnk));
    }
    b->nu = b->template alloc<C>(nk);
    b->lam_seed = b->template alloc<C>(vnk);
    b->M = b->template alloc<C>(vnk);
    b->aw = b->template alloc<R>(vn3);
    if (V > 1) {
      b->wv = b->template alloc<R>(vn3);
      b->hv = b->template alloc<R>(vn3);
    }
    b->lamT = b->template alloc<R>(vn3);
    b->nuT = b->template alloc<R>(n3);
    b->lam0 = b->template alloc<R>(vn3);
    b->tgt_eta = b->template alloc<double>(vn3);
    b->tgt_c = b->template alloc<double>(n3);
    b->partials = b->template alloc<double>((int64_t)ADJ_Q * PSTRIDE);
    b->loss_part = b->template alloc<double>(PSTRIDE);
    b->acc = b->template alloc<double>(8);
    b->d_out = b->template alloc<double>(vn3);
    b->dRec = b->template alloc<LanFusedArgs<R>>(K);
    b->dFwd = b->template alloc<LanFusedArgs<R>>(1);
    b->dSeed = b->template alloc<LanFusedArgs<R>>(1);
    MEU_CUDA(cudaHostAlloc((void**)&b->hRec, sizeof(LanFusedArgs<R>) * K, cudaHostAllocDefault));
  }
  AdjBuffers<R>& B = *adjb;
  MEU_CUDA(cudaMemcpyAsync(B.tgt_c, cons_tgt, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
  // the target eta in the meu_set_fields layout phi(vartot,Nx,Ny,Nz) -> one field per variant
  std::vector<double> tgt_soa;
  const double* te_src = phi_tgt;
  if (V > 1) {
    tgt_soa.resize((size_t)V * n3);
    for (int64_t i = 0; i < n3; ++i)
      for (int v = 0; v < V; ++v) tgt_soa[(size_t)v * n3 + i] = phi_tgt[i * V + v];
    te_src = tgt_soa.data();
  }
  MEU_CUDA(cudaMemcpyAsync(B.tgt_eta, te_src, sizeof(double) * V * n3, cudaMemcpyHostToDevice, st));
  int nb[Q_TOTAL];
  const int64_t step0 = step;
  auto homog_at = [&](int64_t s) { return (P.elastic != MEU_ELAST_NONE && s >= P.elastep0) ? 1 : 0; };
  // ---- forward, in place, with checkpoints every K steps
  LanFusedArgs<R> fa = fused_args();
  fa.energy = 0;
  int up_homog = -1;
  for (int i = 0; i < T; ++i) {
    if (i % K == 0) {
      const int s = i / K;
      MEU_CUDA(cudaMemcpyAsync(B.ck_eta[s], phi, sizeof(R) * V * n3, cudaMemcpyDeviceToDevice, st));
      MEU_CUDA(cudaMemcpyAsync(B.ck_c[s], c, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st));
      MEU_CUDA(cudaMemcpyAsync(B.ck_keta[s], keta, sizeof(C) * V * nk, cudaMemcpyDeviceToDevice, st));
      MEU_CUDA(cudaMemcpyAsync(B.ck_kc[s], kc, sizeof(C) * nk, cudaMemcpyDeviceToDevice, st));
      // theta^ of these fields, as the previous forward step's PI wrote it: the recomputed
      // segment then starts from the same numbers instead of transforming theta afresh
      B.ck_has_theta[s] = theta_ready ? 1 : 0;
      if (theta_ready) MEU_CUDA(cudaMemcpyAsync(B.ck_theta[s], sp, sizeof(C) * V * nk, cudaMemcpyDeviceToDevice, st));
    }
    const int hg = homog_at(step0 + i);
    if (hg != up_homog) {
      fa.homog = hg;
      MEU_CUDA(cudaMemcpyAsync(B.dFwd, &fa, sizeof(fa), cudaMemcpyHostToDevice, st));
      up_homog = hg;
    }
    if (!lan_fused_step<R>(N, V, sched, B.dFwd, 1, theta_ready ? LS_THETA_READY : 0, st, &prof, nb))
      throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
    theta_ready = true;
  }
  step = step0 + T;
  // ---- loss and seed lam_T, nu_T (real) -> spectra
  KLAUNCH("adj_seed", (double)n3 * (2 * sizeof(R) + 16 + 2 * sizeof(R)),
          k_ad_seed<R><<<RED_BLOCKS, RED_THREADS, 0, st>>>(phi, c, dF, B.tgt_eta, B.tgt_c, B.lamT, B.nuT, n3, V, B.loss_part));
  MEU_CUDA(cudaMemsetAsync(B.acc, 0, sizeof(double) * 8, st));
  {
    NbList l;
    for (int q = 0; q < Q_TOTAL; ++q) l.nb[q] = 0;
    l.nb[0] = RED_BLOCKS;
    KLAUNCH("adj_acc", 8.0 * RED_BLOCKS, k_ad_acc<<<1, 256, 0, st>>>(B.loss_part, l, B.acc + ADJ_Q));
  }
  LanFusedArgs<R> sa = fa;
  sa.eta = B.lamT;
  sa.c = B.nuT;
  sa.Keta = B.lam_seed;
  sa.Kc = B.nu;
  MEU_CUDA(cudaMemcpyAsync(B.dSeed, &sa, sizeof(sa), cudaMemcpyHostToDevice, st));
  if (!lan_fused_init<R>(N, V, sched, B.dSeed, 1, st, &prof))
    throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
  // ---- reverse sweep, one checkpoint segment at a time
  for (int seg = nck - 1; seg >= 0; --seg) {
    const int i0 = seg * K, S = std::min(K, T - i0);
    auto eta_p = [&](int j) { return j == 0 ? B.ck_eta[seg] : B.s_eta[j]; };
    auto c_p = [&](int j) { return j == 0 ? B.ck_c[seg] : B.s_c[j]; };
    auto keta_p = [&](int j) { return j == 0 ? B.ck_keta[seg] : B.s_keta[j]; };
    auto kc_p = [&](int j) { return j == 0 ? B.ck_kc[seg] : B.s_kc[j]; };
    MEU_CUDA(cudaStreamSynchronize(st));  // hRec is about to be rewritten
    for (int j = 0; j < S; ++j) {
      LanFusedArgs<R> r = fa;
      r.homog = homog_at(step0 + i0 + j);
      r.eta = eta_p(j);
      r.c = c_p(j);
      r.Keta = keta_p(j);
      r.Kc = kc_p(j);
      r.eta_next = B.s_eta[j + 1];
      r.c_next = B.s_c[j + 1];
      r.Keta_out = B.s_keta[j + 1];
      r.Kc_out = B.s_kc[j + 1];
      r.rec_phi = B.s_phi[j];
      r.rec_theta = B.s_theta[j];
      B.hRec[j] = r;
    }
    MEU_CUDA(cudaMemcpyAsync(B.dRec, B.hRec, sizeof(LanFusedArgs<R>) * S, cudaMemcpyHostToDevice, st));
    // the segment starts from a checkpoint with the forward's theta^ (or, at the very first
    // step, transforms theta itself as the forward did), so it repeats the forward exactly
    const bool ck_theta = B.ck_has_theta[seg] != 0;
    if (ck_theta) MEU_CUDA(cudaMemcpyAsync(sp, B.ck_theta[seg], sizeof(C) * V * nk, cudaMemcpyDeviceToDevice, st));
    for (int j = 0; j < S; ++j)
      if (!lan_fused_step<R>(N, V, sched, B.dRec + j, 1, (j || ck_theta) ? LS_THETA_READY : 0, st, &prof, nb))
        throw CudaError("fused step not instantiated", MEU_ERR_UNSUPPORTED);
    theta_ready = false;  // the engine's M now holds a recomputed step's theta^
    for (int m = S - 1; m >= 0; --m) {
      const int g = i0 + m;
      AdjArgs<R> a;
      memset(&a, 0, sizeof(a));
      a.F = dF;
      a.M = B.M;
      a.nu = B.nu;
      a.lam_seed = B.lam_seed;
      a.eta_k1 = keta_p(m + 1);
      a.c_k1 = kc_p(m + 1);
      a.c_k0 = kc_p(m);
      a.theta_k0 = B.s_theta[m];
      a.eta = eta_p(m);
      a.c = c_p(m);
      a.phi = B.s_phi[m];
      a.aw = B.aw;
      a.lam_out = g == 0 ? B.lam0 : nullptr;
      a.wv = B.wv;
      a.hv = B.hv;
      a.V = V;
      a.partials = B.partials;
      a.homog = homog_at(step0 + g);
      a.from_seed = g == T - 1 ? 1 : 0;
      a.twx = (const C*)fft->px.tw;
      a.twy = (const C*)fft->py.tw;
      a.twz = (const C*)fft->pz.tw;
      a.post = (const C*)fft->post_tw;
      a.err = d_err;
      int nbq[Q_TOTAL];
      if (!adj_step<R>(N, a, st, &prof, nbq)) throw CudaError("adjoint not instantiated", MEU_ERR_UNSUPPORTED);
      NbList l;
      for (int q = 0; q < Q_TOTAL; ++q) l.nb[q] = nbq[q];
      KLAUNCH("adj_acc", 8.0 * (3 * nbq[AQ_X] + 2 * nbq[AQ_WG]), k_ad_acc<<<ADJ_Q, 256, 0, st>>>(B.partials, l, B.acc));
    }
  }
  // ---- results
  double h[8];
  MEU_CUDA(cudaMemcpyAsync(h, B.acc, sizeof(h), cudaMemcpyDeviceToHost, st));
  if (dphi0) {
    KLAUNCH("adj_out", (double)V * n3 * (sizeof(R) + 8),
            k_to_double<R><<<gridr(), 256, 0, st>>>(B.lam0, B.d_out, (int64_t)V * n3));
    if (V == 1) {
      MEU_CUDA(cudaMemcpyAsync(dphi0, B.d_out, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    } else {
      // back to the meu_set_fields layout phi(vartot,Nx,Ny,Nz)
      std::vector<double> soa((size_t)V * n3);
      MEU_CUDA(cudaMemcpyAsync(soa.data(), B.d_out, sizeof(double) * V * n3, cudaMemcpyDeviceToHost, st));
      MEU_CUDA(cudaStreamSynchronize(st));
      for (int64_t i = 0; i < n3; ++i)
        for (int v = 0; v < V; ++v) dphi0[i * V + v] = soa[(size_t)v * n3 + i];
    }
  }
  MEU_CUDA(cudaStreamSynchronize(st));
  check_err();
  const double n3d = (double)n3, dtl = P.dt * P.b_mob, dm = P.dt * P.cmobs[0];
  const double SX = h[AQ_X] * n3d, SY = h[AQ_Y] * n3d, SZ = h[AQ_Z] * n3d;
  const double d_dtl = -SX - h[AQ_WG];
  const double d_dm = -P.kappa_c * SY - SZ;
  if (loss) *loss = 0.5 * h[ADJ_Q] / n3d;
  if (dparams) {
    dparams[0] = -dtl * SX;      // d/d(beta): kappa_eta -> beta kappa_eta at beta = 1
    dparams[1] = -dm * SY;       // d/d(kappa_c)
    dparams[2] = P.dt * d_dtl;   // d/d(L)
    dparams[3] = P.dt * d_dm;    // d/d(M)
    dparams[4] = h[AQ_EA];       // d/d(alpha): eigenstrains -> alpha eigenstrains at alpha = 1
  }
}

template bool adj_step<float>(int, const AdjArgs<float>&, cudaStream_t, LaunchHook*, int*);
template bool adj_step<double>(int, const AdjArgs<double>&, cudaStream_t, LaunchHook*, int*);
template void Engine<float>::adjoint(int, int, const double*, const double*, double*, double*, double*);
template void Engine<double>::adjoint(int, int, const double*, const double*, double*, double*, double*);
template void adj_buffers_free<float>(AdjBuffers<float>*);
template void adj_buffers_free<double>(AdjBuffers<double>*);

}  // namespace meu
