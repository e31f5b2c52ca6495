/*
 * meu_oracle.c -- CPU FP64 restatement of the MEUMAPPS-SS time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the CUDA library is
 * checked against it, and bench.py times it as the CPU baseline.  Nothing in
 * the product library links, loads or calls it.
 *
 * Parity status: UNPINNED by reference artefacts.  The reference ships no test,
 * golden vector or example input, and its Fortran/MPI/P3DFFT/LINPACK build cannot
 * be compiled here (no Fortran compiler, no P3DFFT/FFTW/LINPACK).  The oracle is
 * pinned instead, on the CPU, by:
 *   tests/test_oracle_fft.py  f_trans / inv_trans against numpy.fft (incl. the
 *                             c2r convention) and invert with its condition flag;
 *   tests/test_oracle_kat.py  single Fourier-mode decay (Landau eta and c, KKS c),
 *                             uniform fields (uniformity and the k = 0 recurrence),
 *                             mass conservation (Landau and KKS), Khachaturyan's
 *                             closed-form elastic energy of a dilatational inclusion
 *                             in a cubic medium (Landau) and of a tetragonal one in
 *                             the KKS model (eldis + elener with equal matrix and
 *                             precipitate moduli), and a numpy restatement of one
 *                             Landau step (1 to 3 variants, eta^2 and h(eta)
 *                             coupling, with and without elasticity) to 1e-12;
 *   tests/test_oracle_kks_mirror.py  a numpy restatement of one KKS step of the
 *                             reference (gradients, composition solve, driving forces,
 *                             n_tilda projection, both updates, clip; and at the first
 *                             elastic step eldis and elener with heterogeneous moduli),
 *                             1 and 3 variants, 1 and 2 solutes, to 1e-12;
 *   tests/test_host.py        ran_2 / langevin against two other restatements.
 *
 * It follows the reference statement by statement:
 *   KKS step              Multi_MEUMAPPS.f:548-1106
 *   spectral gradients    Multi_MEUMAPPS.f:575-615
 *   KKS driving force     Multi_MEUMAPPS.f:634-845
 *   eldis                 ModElastic.f:11-489
 *   elener                ModElastic.f:493-691
 *   CH (diffusion) update Multi_MEUMAPPS.f:910-949
 *   TDGL update           Multi_MEUMAPPS.f:955-1001
 *   clip + reductions     Multi_MEUMAPPS.f:1008-1065, :885-908
 *   k-vectors             ModInitials.f:348-409
 *   f_trans / inv_trans   ModFunc.f:15-40 (forward scaled by 1/NxNyNz, inverse unscaled)
 *   invert                ModFunc.f:44-72 (inverse + reciprocal condition check)
 *   ran_2, langevin       ran_2.f:1-42, ModFunc.f:77-100
 * The Landau model (the configuration decks' free energy) has no counterpart in
 * the reference; it reuses the same spectral skeleton and eldis/elener.
 *
 * Internal layout: structure of arrays, x fastest: a[f][z][y][x]; spectra
 * a[f][z][y][kx] with kx in [0, Nx/2].
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/meu.h"

typedef double complex cplx;

/* ------------------------------------------------------------------ FFT -- */
/* Mixed-radix recursive decimation-in-time FFT on one line (natural order). */
typedef struct {
  int n, nr, r[40];
  cplx* tw; /* tw[k] = exp(-2 pi i k / n) */
} line_plan;

static int line_plan_init(line_plan* p, int n) {
  p->n = n;
  p->nr = 0;
  int m = n;
  while (m > 1) {
    int r = (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : m;
    p->r[p->nr++] = r;
    m /= r;
  }
  p->tw = (cplx*)malloc(sizeof(cplx) * (size_t)n);
  if (!p->tw) return -1;
  for (int k = 0; k < n; ++k) {
    long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
    p->tw[k] = (double)cosl(a) + I * (double)sinl(a);
  }
  return 0;
}

static void line_plan_free(line_plan* p) { free(p->tw); p->tw = NULL; }

/* out[0..n) = DFT of in[0], in[stride], ... ; depth = index into radix list */
static void fft_rec(const line_plan* p, int depth, const cplx* in, int stride, cplx* out, int n) {
  if (n == 1) { out[0] = in[0]; return; }
  int R = p->r[depth], m = n / R, N = p->n, s = N / n;
  for (int r = 0; r < R; ++r) fft_rec(p, depth + 1, in + (size_t)r * stride, stride * R, out + (size_t)r * m, m);
  cplx a[16];
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < R; ++r) a[r] = out[r * m + k] * p->tw[(size_t)(r * k) * s % N];
    for (int q = 0; q < R; ++q) {
      cplx acc = 0;
      for (int r = 0; r < R; ++r) acc += a[r] * p->tw[(size_t)((r * q) % R) * (N / R)];
      out[k + q * m] = acc;
    }
  }
}

/* in-place on buf (natural order); dir = -1 forward, +1 inverse (unscaled) */
static void fft_line(const line_plan* p, cplx* buf, cplx* tmp, int dir) {
  int n = p->n;
  if (dir > 0) for (int i = 0; i < n; ++i) buf[i] = conj(buf[i]);
  fft_rec(p, 0, buf, 1, tmp, n);
  if (dir > 0) for (int i = 0; i < n; ++i) buf[i] = conj(tmp[i]);
  else memcpy(buf, tmp, sizeof(cplx) * (size_t)n);
}

typedef struct {
  int nx, ny, nz, nxh;
  line_plan px, py, pz;
} fft3;

static int fft3_init(fft3* f, int nx, int ny, int nz) {
  f->nx = nx; f->ny = ny; f->nz = nz; f->nxh = nx / 2 + 1;
  if (line_plan_init(&f->px, nx) || line_plan_init(&f->py, ny) || line_plan_init(&f->pz, nz)) return -1;
  return 0;
}
static void fft3_free(fft3* f) { line_plan_free(&f->px); line_plan_free(&f->py); line_plan_free(&f->pz); }

/* f_trans (ModFunc.f:15-26): 3-D real-to-complex DFT scaled by 1/(Nx Ny Nz). */
static void f_trans(const fft3* f, const double* in, cplx* out) {
  const int nx = f->nx, ny = f->ny, nz = f->nz, nxh = f->nxh;
  const double sc = 1.0 / ((double)nx * ny * nz);
  int nmax = nx > ny ? nx : ny; if (nz > nmax) nmax = nz;
#pragma omp parallel
  {
    cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    cplx* t = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
    for (int64_t row = 0; row < (int64_t)ny * nz; ++row) {
      const double* src = in + row * nx;
      for (int x = 0; x < nx; ++x) b[x] = src[x];
      fft_line(&f->px, b, t, -1);
      cplx* dst = out + row * nxh;
      for (int k = 0; k < nxh; ++k) dst[k] = b[k];
    }
#pragma omp for schedule(static)
    for (int64_t col = 0; col < (int64_t)nz * nxh; ++col) {
      int z = (int)(col / nxh), kx = (int)(col % nxh);
      cplx* base = out + (size_t)z * ny * nxh + kx;
      for (int y = 0; y < ny; ++y) b[y] = base[(size_t)y * nxh];
      fft_line(&f->py, b, t, -1);
      for (int y = 0; y < ny; ++y) base[(size_t)y * nxh] = b[y];
    }
#pragma omp for schedule(static)
    for (int64_t col = 0; col < (int64_t)ny * nxh; ++col) {
      cplx* base = out + col;
      for (int z = 0; z < nz; ++z) b[z] = base[(size_t)z * ny * nxh];
      fft_line(&f->pz, b, t, -1);
      for (int z = 0; z < nz; ++z) base[(size_t)z * ny * nxh] = b[z] * sc;
    }
    free(b); free(t);
  }
}

/* inv_trans (ModFunc.f:30-40): unscaled complex-to-real DFT.  The input is
 * left untouched.  The x transform uses the Hermitian extension of each row,
 * whose real part discards Im X(0) and Im X(Nx/2) as FFTW's c2r does. */
static void inv_trans(const fft3* f, const cplx* in, double* out, cplx* work) {
  const int nx = f->nx, ny = f->ny, nz = f->nz, nxh = f->nxh;
  const int64_t nk = (int64_t)nz * ny * nxh;
  int nmax = nx > ny ? nx : ny; if (nz > nmax) nmax = nz;
#pragma omp parallel
  {
    cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
    cplx* t = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
    for (int64_t col = 0; col < (int64_t)ny * nxh; ++col) {
      for (int z = 0; z < nz; ++z) b[z] = in[col + (size_t)z * ny * nxh];
      fft_line(&f->pz, b, t, +1);
      for (int z = 0; z < nz; ++z) work[col + (size_t)z * ny * nxh] = b[z];
    }
#pragma omp for schedule(static)
    for (int64_t col = 0; col < (int64_t)nz * nxh; ++col) {
      int z = (int)(col / nxh), kx = (int)(col % nxh);
      cplx* base = work + (size_t)z * ny * nxh + kx;
      for (int y = 0; y < ny; ++y) b[y] = base[(size_t)y * nxh];
      fft_line(&f->py, b, t, +1);
      for (int y = 0; y < ny; ++y) base[(size_t)y * nxh] = b[y];
    }
#pragma omp for schedule(static)
    for (int64_t row = 0; row < (int64_t)ny * nz; ++row) {
      const cplx* src = work + row * nxh;
      for (int k = 0; k < nxh; ++k) b[k] = src[k];
      for (int k = nxh; k < nx; ++k) b[k] = conj(src[nx - k]);
      fft_line(&f->px, b, t, +1);
      double* dst = out + row * nx;
      for (int x = 0; x < nx; ++x) dst[x] = creal(b[x]);
    }
    free(b); free(t);
  }
  (void)nk;
}

/* --------------------------------------------------------------- invert -- */
/* invert (ModFunc.f:44-72): a <- a^-1 for an n x n column-major matrix by
 * Gauss-Jordan elimination with partial pivoting.  Returns 0, or flag when
 * the reciprocal 1-norm condition number is <= 1e-16 (the reference's
 * rcond test after dgeco) or a pivot vanishes. */
static int invert(double* a, int n, int flag) {
  double anorm = 0;
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += fabs(a[i + j * n]);
    if (s > anorm) anorm = s;
  }
  int piv[16];
  double w[256];
  memcpy(w, a, sizeof(double) * (size_t)n * n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  /* in-place Gauss-Jordan with row pivoting, recording the permutation */
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(w[k + k * n]);
    for (int i = k + 1; i < n; ++i)
      if (fabs(w[i + k * n]) > best) { best = fabs(w[i + k * n]); p = i; }
    if (best == 0.0) return flag;
    if (p != k) {
      for (int j = 0; j < n; ++j) { double t = w[k + j * n]; w[k + j * n] = w[p + j * n]; w[p + j * n] = t; }
      int t = piv[k]; piv[k] = piv[p]; piv[p] = t;
    }
    double d = 1.0 / w[k + k * n];
    w[k + k * n] = 1.0;
    for (int j = 0; j < n; ++j) w[k + j * n] *= d;
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      double f = w[i + k * n];
      if (f == 0.0) continue;
      w[i + k * n] = 0.0;
      for (int j = 0; j < n; ++j) w[i + j * n] -= f * w[k + j * n];
    }
  }
  /* undo the row permutation as a column permutation of the inverse */
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + piv[j] * n] = w[i + j * n];
  double inorm = 0;
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += fabs(a[i + j * n]);
    if (s > inorm) inorm = s;
  }
  double rcond = 1.0 / (anorm * inorm);
  if (!(rcond > 1e-16)) return flag;
  return 0;
}

/* ---------------------------------------------------------------- ran_2 -- */
/* ran_2.f:1-42.  am = 1./im1 is a REAL*4 expression: float(2147483563)
 * rounds to 2^31 - 128 and the quotient is rounded to REAL*4 before it widens
 * to the REAL*8 parameter; rnmx = 1.-eps is evaluated in double. */
#define R2_IM1 2147483563
#define R2_IM2 2147483399
#define R2_IMM1 (R2_IM1 - 1)
#define R2_IA1 40014
#define R2_IA2 40692
#define R2_IQ1 53668
#define R2_IQ2 52774
#define R2_IR1 12211
#define R2_IR2 3791
#define R2_NTAB 32
#define R2_NDIV (1 + R2_IMM1 / R2_NTAB)

double orc_ran2(meu_ran2_state* s) {
  const double am = (double)(1.0f / (float)R2_IM1);
  const double rnmx = 1.0 - 1.2e-7;
  int32_t k;
  if (s->idum <= 0) {
    s->idum = (-s->idum > 1) ? -s->idum : 1;
    s->idum2 = s->idum;
    for (int j = R2_NTAB + 8; j >= 1; --j) {
      k = s->idum / R2_IQ1;
      s->idum = R2_IA1 * (s->idum - k * R2_IQ1) - k * R2_IR1;
      if (s->idum < 0) s->idum += R2_IM1;
      if (j <= R2_NTAB) s->iv[j - 1] = s->idum;
    }
    s->iy = s->iv[0];
  }
  k = s->idum / R2_IQ1;
  s->idum = R2_IA1 * (s->idum - k * R2_IQ1) - k * R2_IR1;
  if (s->idum < 0) s->idum += R2_IM1;
  k = s->idum2 / R2_IQ2;
  s->idum2 = R2_IA2 * (s->idum2 - k * R2_IQ2) - k * R2_IR2;
  if (s->idum2 < 0) s->idum2 += R2_IM2;
  int j = 1 + s->iy / R2_NDIV;
  s->iy = s->iv[j - 1] - s->idum2;
  s->iv[j - 1] = s->idum;
  if (s->iy < 1) s->iy += R2_IMM1;
  double v = am * (double)s->iy;
  return v < rnmx ? v : rnmx;
}

void orc_ran2_init(meu_ran2_state* s, int32_t iseed) {
  memset(s, 0, sizeof(*s));
  s->idum = iseed;
  s->idum2 = 123456789; /* DATA idum2 /123456789/ */
}

/* Uniform-noise initial fields of the Landau decks: per voxel in Fortran
 * order, c = c0 + c_amp*(2u-1), then eta_v = eta_amp*(2u-1) for v = 1..nvar,
 * u from ran_2.  cons is (Nx,Ny,Nz); phi is phi(nvar,Nx,Ny,Nz), component fastest. */
void orc_init_uniform(meu_ran2_state* s, int nx, int ny, int nz, int nvar, double c0, double c_amp, double eta_amp,
                      double* cons, double* phi) {
  const int64_t n3 = (int64_t)nx * ny * nz;
  for (int64_t i = 0; i < n3; ++i) {
    cons[i] = c0 + c_amp * (2.0 * orc_ran2(s) - 1.0);
    for (int v = 0; v < nvar; ++v) phi[i * nvar + v] = eta_amp * (2.0 * orc_ran2(s) - 1.0);
  }
}

/* langevin (ModFunc.f:77-100) */
double orc_langevin(meu_ran2_state* s, double sd) {
  for (;;) {
    double v1 = orc_ran2(s), v2 = orc_ran2(s);
    v1 = 2.0 * v1 - 1.0;
    v2 = 2.0 * v2 - 1.0;
    double rsq = v1 * v1 + v2 * v2;
    if (rsq > 0.0 && rsq < 1.0) {
      rsq = sqrt(-2.0 * log(rsq) / rsq);
      return v2 * rsq * sd;
    }
  }
}

/* ------------------------------------------------------------ simulation -- */
typedef struct orc_sim {
  meu_params p;
  fft3 f;
  int nx, ny, nz, nxh, V, E;
  int64_t n3, nk;
  int64_t step;
  /* fields (SoA) */
  double *cons, *phi, *phi_noise, *pphi, *el_en;
  double *u;     /* 3 * n3: u1,u2,u3 */
  double *gu;    /* 9 * n3 in data_save order: grad_1_u1,grad_1_u2,grad_1_u3,grad_2_u1,... */
  /* work */
  double *gx, *gy, *gz, *kds, *fgrad, *fdiff, *elgrad, *fcx, *fcy, *fcz, *rtmp;
  double *xs;    /* 6 * n3 polarization x_1..x_6 */
  double *uold;  /* 3 * n3 */
  cplx *ck, *ck2, *ck3, *work, *pk /* V*nk */, *uk /* 12*nk */, *xk /* 6*nk */;
  /* reference's quirks: values written on the next fort.98 line */
  double glob_min, glob_max, phi_max, solid_frac;
  /* elastic control state */
  int el_visit;
  /* Z-matrix constant rows (Multi_MEUMAPPS.f:426-448) */
  double zconst[256], zr_const[16];
  int last_iters;
} orc_sim;

#define IDX3(x, y, z, nx, ny) ((size_t)(x) + (size_t)(nx) * ((size_t)(y) + (size_t)(ny) * (size_t)(z)))

/* kf / kf_sq of k_space (ModInitials.f:348-409) for one half-spectrum point.
 * kf = i*b (b zeroed at the Nyquist index), kf_sq = -a^2 (Nyquist kept). */
static inline void kvec(const orc_sim* s, int kx, int ky, int kz, double a[3], double b[3]) {
  const double pi = atan(1.0) * 4.0;
  int n[3] = {s->nx, s->ny, s->nz}, m[3] = {kx, ky, kz};
  for (int d = 0; d < 3; ++d) {
    double unit = 2.0 * pi / (double)n[d];
    int mm = (m[d] <= n[d] / 2) ? m[d] : m[d] - n[d];
    a[d] = (double)mm * unit;
    b[d] = (2 * m[d] == n[d]) ? 0.0 : a[d];
  }
}

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

void orc_destroy(orc_sim* s);

orc_sim* orc_create(const meu_params* p) {
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  if (!s) return NULL;
  s->p = *p;
  s->nx = p->nx; s->ny = p->ny; s->nz = p->nz; s->nxh = p->nx / 2 + 1;
  s->V = p->nvar; s->E = p->numel;
  s->n3 = (int64_t)p->nx * p->ny * p->nz;
  s->nk = (int64_t)p->nz * p->ny * s->nxh;
  s->step = p->step;
  if (fft3_init(&s->f, p->nx, p->ny, p->nz)) { orc_destroy(s); return NULL; }
  size_t n3 = (size_t)s->n3, nk = (size_t)s->nk, V = (size_t)s->V, E = (size_t)(s->E > 0 ? s->E : 1);
  s->cons = xcalloc(E * n3, 8); s->phi = xcalloc(V * n3, 8); s->phi_noise = xcalloc(V * n3, 8);
  s->pphi = xcalloc(V * n3, 8); s->el_en = xcalloc(n3, 8);
  s->u = xcalloc(3 * n3, 8); s->gu = xcalloc(9 * n3, 8); s->uold = xcalloc(3 * n3, 8);
  s->gx = xcalloc(V * n3, 8); s->gy = xcalloc(V * n3, 8); s->gz = xcalloc(V * n3, 8);
  s->kds = xcalloc(V * n3, 8); s->fgrad = xcalloc(V * n3, 8); s->fdiff = xcalloc(V * n3, 8);
  s->elgrad = xcalloc(V * n3, 8);
  s->fcx = xcalloc(E * n3, 8); s->fcy = xcalloc(E * n3, 8); s->fcz = xcalloc(E * n3, 8);
  s->rtmp = xcalloc(n3, 8); s->xs = xcalloc(6 * n3, 8);
  s->ck = xcalloc(nk, sizeof(cplx)); s->ck2 = xcalloc(nk, sizeof(cplx)); s->ck3 = xcalloc(nk, sizeof(cplx));
  s->work = xcalloc(nk, sizeof(cplx));
  s->pk = xcalloc(V * nk, sizeof(cplx)); s->uk = xcalloc(12 * nk, sizeof(cplx)); s->xk = xcalloc(6 * nk, sizeof(cplx));
  if (!s->work || !s->uk || !s->xk || !s->gu) { orc_destroy(s); return NULL; }
  /* fort.98 values before the first step: glob_min = 1.d0 (:420); the others
   * are never assigned before the first write and are reported as 0. */
  s->glob_min = 1.0; s->glob_max = 0.0; s->phi_max = 0.0; s->solid_frac = 0.0;
  /* constant rows of the Z matrix (Multi_MEUMAPPS.f:426-448) */
  if (p->model == MEU_MODEL_KKS) {
    int numel = p->numel, numph = p->numph, zdim = numph * numel;
    memset(s->zconst, 0, sizeof(s->zconst));
    memset(s->zr_const, 0, sizeof(s->zr_const));
#define GP(j, n) p->gparams[(n) - 1][(j) - 1]
    for (int nelc = 1; nelc <= numel; ++nelc) {
      int i1 = nelc + numel + 1;
      for (int nphc = 1; nphc <= numph - 1; ++nphc) {
        int i0 = (numph - 1) * (nelc - 1) + nphc;
        int j0 = numph * (nelc - 1) + nphc;
        int nphc1 = nphc + 1;
        s->zconst[(i0 - 1) + (j0 - 1) * zdim] = GP(nelc, nphc);
        s->zconst[(i0 - 1) + (j0) * zdim] = -GP(nelc, nphc1);
        s->zr_const[i0 - 1] = GP(nelc, nphc) * GP(i1, nphc) - GP(nelc, nphc1) * GP(i1, nphc1);
      }
    }
#undef GP
  }
  return s;
}

void orc_destroy(orc_sim* s) {
  if (!s) return;
  fft3_free(&s->f);
  void* ptrs[] = {s->cons, s->phi, s->phi_noise, s->pphi, s->el_en, s->u, s->gu, s->uold, s->gx, s->gy,
                  s->gz, s->kds, s->fgrad, s->fdiff, s->elgrad, s->fcx, s->fcy, s->fcz, s->rtmp, s->xs,
                  s->ck, s->ck2, s->ck3, s->work, s->pk, s->uk, s->xk};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(s);
}

/* SoA in: cons[E][n3], phi[V][n3], ustate[12][n3] or NULL */
int orc_set_fields(orc_sim* s, const double* cons, const double* phi, const double* ustate) {
  size_t n3 = (size_t)s->n3;
  if (cons) memcpy(s->cons, cons, sizeof(double) * (size_t)s->E * n3);
  if (phi) memcpy(s->phi, phi, sizeof(double) * (size_t)s->V * n3);
  if (ustate) {
    memcpy(s->u, ustate, sizeof(double) * 3 * n3);
    memcpy(s->gu, ustate + 3 * n3, sizeof(double) * 9 * n3);
  } else {
    memset(s->u, 0, sizeof(double) * 3 * n3);
    memset(s->gu, 0, sizeof(double) * 9 * n3);
  }
  return 0;
}

int orc_get_fields(orc_sim* s, double* cons, double* phi, double* el_en, double* ustate) {
  size_t n3 = (size_t)s->n3;
  if (cons) memcpy(cons, s->cons, sizeof(double) * (size_t)s->E * n3);
  if (phi) memcpy(phi, s->phi, sizeof(double) * (size_t)s->V * n3);
  if (el_en) memcpy(el_en, s->el_en, sizeof(double) * n3);
  if (ustate) {
    memcpy(ustate, s->u, sizeof(double) * 3 * n3);
    memcpy(ustate + 3 * n3, s->gu, sizeof(double) * 9 * n3);
  }
  return 0;
}

int orc_add_noise(orc_sim* s, const double* incr) {
  size_t n = (size_t)s->V * (size_t)s->n3;
  for (size_t i = 0; i < n; ++i) s->phi_noise[i] += incr[i];
  return 0;
}

int64_t orc_get_step(const orc_sim* s) { return s->step; }
int orc_last_iters(const orc_sim* s) { return s->last_iters; }

/* variant range of phase nphc (2..numph): the reference's ivn/fvn bookkeeping
 * (Multi_MEUMAPPS.f:643-648).  Returns 0-based [lo, hi). */
static void phase_range(const meu_params* p, int nphc, int* lo, int* hi) {
  int ivn = 0;
  for (int n = 2; n <= nphc; ++n) ivn += p->nvar_ph[n - 2];
  int fvn = ivn + p->nvar_ph[nphc - 1] - 1;
  *lo = ivn - 1;
  *hi = fvn;
}
static int phase_of_var(const meu_params* p, int v) {
  for (int n = 2; n <= p->numph; ++n) {
    int lo, hi;
    phase_range(p, n, &lo, &hi);
    if (v >= lo && v < hi) return n;
  }
  return 2;
}

/* Voigt index of (i,j), 1-based (ModElastic.f:124-126) */
static inline int voigt(int i, int j) { return i == j ? i : 9 - i - j; }
#define CE(p, n, a, b) ((p)->cela[(n) - 1][((b) - 1) * 6 + ((a) - 1)])
#define SE(p, n, a, b) ((p)->sela[(n) - 1][((b) - 1) * 6 + ((a) - 1)])

/* Q(k) of ModElastic.f:119-158 (with C0 = CEla(:,:,2)); column-major 3x3. */
static void build_q(const meu_params* p, const double a[3], const double b[3], double Q[9]) {
  for (int i = 0; i < 9; ++i) Q[i] = 0;
  for (int i = 1; i <= 3; ++i)
    for (int j = 1; j <= 3; ++j) {
      int ij = voigt(i, j);
      for (int k = 1; k <= 3; ++k)
        for (int l = 1; l <= 3; ++l) {
          int kl = voigt(k, l);
          /* kpr = kf(k)*kf(j), or kf_sq(k) when k == j */
          double kpr = (k == j) ? -(a[k - 1] * a[k - 1]) : -(b[k - 1] * b[j - 1]);
          Q[(i - 1) + (l - 1) * 3] += CE(p, 2, ij, kl) * kpr;
        }
    }
}

/* gradient of u in the data_save order index: grad_j_ui -> (j-1)*3 + (i-1) */
#define GU(s, i, j) ((s)->gu + (size_t)(((j) - 1) * 3 + ((i) - 1)) * (size_t)(s)->n3)

/* eldis (ModElastic.f:11-489) followed by elener (:493-691).
 * pp = P_phi (interpolated phase), ppr = its derivative used by elener.
 * zeroth_only: compute only the zeroth-order solution (homogeneous moduli). */
static int eldis(orc_sim* s, const double* ppr, int zeroth_only) {
  const meu_params* p = &s->p;
  const int nx = s->nx, ny = s->ny, nz = s->nz, nxh = s->nxh, V = s->V;
  const size_t n3 = (size_t)s->n3, nk = (size_t)s->nk;
  double newfac = 0.5, cfac = 1.0;
  int niter = 0, converged = 0, total_iters = 0;
  double err[6], err_old[6] = {0};
  int status = 0;
  const int first = zeroth_only || (s->step == p->elastep0);

  for (int v = 0; v < V; ++v) f_trans(&s->f, s->pphi + v * n3, s->pk + v * nk);

  /* zeroth order (ModElastic.f:115-236).  sig0[v][ij] = sum_kl trans_ppt(kl,v) *
   * CEla(ij,kl,phase(v)) is the reference's inner sum (:129-155) with the
   * variant-independent factor taken out of the k loop. */
  if (first) {
    double sig0[MEU_MAX_VAR][6];
    for (int v = 0; v < V; ++v) {
      int n = phase_of_var(p, v);
      for (int ij = 1; ij <= 6; ++ij) {
        double acc = 0;
        for (int k = 1; k <= 3; ++k)
          for (int l = 1; l <= 3; ++l) {
            int kl = voigt(k, l);
            acc += p->trans_ppt[v][kl - 1] * CE(p, n, ij, kl);
          }
        sig0[v][ij - 1] = acc;
      }
    }
#pragma omp parallel for schedule(static) reduction(max : status)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      cplx R[3] = {0, 0, 0};
      for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) {
          int ij = voigt(i, j);
          cplx sum0 = 0;
          for (int v = 0; v < V; ++v) sum0 += s->pk[v * nk + id] * sig0[v][ij - 1];
          R[i - 1] += sum0 * (I * b[j - 1]);
        }
      cplx uu[3] = {0, 0, 0};
      if (id != 0) {
        double Q[9];
        build_q(p, a, b, Q);
        int st = invert(Q, 3, MEU_ERR_Q_SINGULAR);
        if (st) status = st;
        for (int i = 0; i < 3; ++i) uu[i] = Q[i] * R[0] + Q[i + 3] * R[1] + Q[i + 6] * R[2];
      }
      for (int i = 0; i < 3; ++i) {
        s->uk[i * nk + id] = uu[i];
        for (int j = 0; j < 3; ++j) s->uk[(3 + j * 3 + i) * nk + id] = (I * b[j]) * uu[i];
      }
    }
    if (status) return status;
    for (int c = 0; c < 3; ++c) inv_trans(&s->f, s->uk + c * nk, s->u + c * n3, s->work);
    for (int c = 0; c < 9; ++c) inv_trans(&s->f, s->uk + (3 + c) * nk, s->gu + c * n3, s->work);
  }

  if (!zeroth_only) {
  iterate: /* label 2 (ModElastic.f:241) */
    memcpy(s->uold, s->u, sizeof(double) * 3 * n3);
    niter += 1;
    total_iters += 1;
    if (total_iters > 100000) return MEU_ERR_NOT_CONVERGED;
#pragma omp parallel for schedule(static) reduction(max : status)
    for (int64_t id = 0; id < (int64_t)n3; ++id) {
      double C[36], Cp[36], gradu[9];
      double psum = 0;
      for (int i = 0; i < 36; ++i) C[i] = 0;
      for (int n = 2; n <= p->numph; ++n) {
        int lo, hi;
        phase_range(p, n, &lo, &hi);
        for (int v = lo; v < hi; ++v) {
          double pv = s->pphi[v * n3 + id];
          psum += pv;
          for (int i = 0; i < 36; ++i) C[i] += pv * p->sela[n - 1][i];
        }
      }
      if (psum < 1.0)
        for (int i = 0; i < 36; ++i) C[i] += (1.0 - psum) * p->sela[0][i];
      int st = invert(C, 6, MEU_ERR_C_SINGULAR);
      if (st) status = st;
      for (int i = 0; i < 36; ++i) Cp[i] = p->cela[1][i] - C[i];
      /* gradu(i,j) = grad_j_ui */
      for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) gradu[(i - 1) + (j - 1) * 3] = GU(s, i, j)[id];
      for (int i = 1; i <= 3; ++i)
        for (int j = i; j <= 3; ++j) {
          int ij = voigt(i, j);
          double sum0 = 0;
          for (int k = 1; k <= 3; ++k)
            for (int l = 1; l <= 3; ++l) {
              int kl = voigt(k, l);
              sum0 += cfac * Cp[(ij - 1) + (kl - 1) * 6] * (gradu[(k - 1) + (l - 1) * 3] + p->e_mean[kl - 1]);
              for (int v = 0; v < V; ++v)
                sum0 += C[(ij - 1) + (kl - 1) * 6] * s->pphi[v * n3 + id] * p->trans_ppt[v][kl - 1];
            }
          s->xs[(size_t)(ij - 1) * n3 + id] = sum0;
        }
    }
    if (status) return status;
    for (int c = 0; c < 6; ++c) f_trans(&s->f, s->xs + c * n3, s->xk + c * nk);
#pragma omp parallel for schedule(static) reduction(max : status)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      cplx k1 = I * b[0], k2 = I * b[1], k3 = I * b[2];
      cplx x1 = s->xk[0 * nk + id], x2 = s->xk[1 * nk + id], x3 = s->xk[2 * nk + id];
      cplx x4 = s->xk[3 * nk + id], x5 = s->xk[4 * nk + id], x6 = s->xk[5 * nk + id];
      cplx R[3];
      R[0] = x1 * k1 + x6 * k2 + x5 * k3;
      R[1] = x6 * k1 + x2 * k2 + x4 * k3;
      R[2] = x5 * k1 + x4 * k2 + x3 * k3;
      cplx uu[3] = {0, 0, 0};
      if (id != 0) {
        double Q[9];
        build_q(p, a, b, Q);
        int st = invert(Q, 3, MEU_ERR_Q_SINGULAR);
        if (st) status = st;
        for (int i = 0; i < 3; ++i) uu[i] = Q[i] * R[0] + Q[i + 3] * R[1] + Q[i + 6] * R[2];
      }
      for (int i = 0; i < 3; ++i) {
        s->uk[i * nk + id] = uu[i];
        for (int j = 0; j < 3; ++j) s->uk[(3 + j * 3 + i) * nk + id] = (I * b[j]) * uu[i];
      }
    }
    if (status) return status;
    for (int c = 0; c < 3; ++c) inv_trans(&s->f, s->uk + c * nk, s->u + c * n3, s->work);
    for (int c = 0; c < 9; ++c) inv_trans(&s->f, s->uk + (3 + c) * nk, s->gu + c * n3, s->work);
    /* convergence test (ModElastic.f:413-436) */
    double e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
#pragma omp parallel for schedule(static) reduction(+ : e0, e1, e2, e3, e4, e5)
    for (int64_t id = 0; id < (int64_t)n3; ++id) {
      double d;
      d = s->u[id] - s->uold[id]; e0 += d * d; e1 += s->uold[id] * s->uold[id];
      d = s->u[n3 + id] - s->uold[n3 + id]; e2 += d * d; e3 += s->uold[n3 + id] * s->uold[n3 + id];
      d = s->u[2 * n3 + id] - s->uold[2 * n3 + id]; e4 += d * d; e5 += s->uold[2 * n3 + id] * s->uold[2 * n3 + id];
    }
    err[0] = e0; err[1] = e1; err[2] = e2; err[3] = e3; err[4] = e4; err[5] = e5;
    const double tol = p->el_tol;
    if (err[0] / err[1] < tol && err[2] / err[3] < tol && err[4] / err[5] < tol) converged = 1;
    if (niter > 1 && !converged) {
      if (err[0] / err[1] > err_old[0] / err_old[1] || err[2] / err[3] > err_old[2] / err_old[3] ||
          err[4] / err[5] > err_old[4] / err_old[5]) {
        cfac = cfac * newfac;
        newfac = newfac * 0.5;
        if (newfac < 1e-7) return MEU_ERR_NOT_CONVERGED;
        niter = 0;
        converged = 0;
        goto iterate;
      }
    }
    memcpy(err_old, err, sizeof(err));
    if (niter == p->el_max_iter) converged = 1;
    if (!converged || niter < p->el_min_iter) goto iterate;
    if (cfac < 1.0 - 1e-6) {
      cfac = cfac + 0.1;
      if (cfac > 1.0) cfac = 1.0;
      niter = 0;
      converged = 0;
      goto iterate;
    }
  }
  s->last_iters = total_iters;

  /* elener (ModElastic.f:493-691) */
  double transsum[MEU_MAX_VAR];
  for (int v = 0; v < V; ++v) {
    transsum[v] = 0;
    for (int i = 0; i < 6; ++i) transsum[v] += p->trans_ppt[v][i];
  }
  const double tiny = (double)1.e-9f; /* REAL*4 literal 1.e-9 (ModElastic.f:653) */
#pragma omp parallel for schedule(static) reduction(max : status)
  for (int64_t id = 0; id < (int64_t)n3; ++id) {
    double te[6] = {0, 0, 0, 0, 0, 0}, psum = 0, eps[6], C[36], sig[6];
    for (int v = 0; v < V; ++v) {
      double pl = s->pphi[v * n3 + id];
      psum += pl;
      for (int i = 0; i < 6; ++i) te[i] += pl * p->trans_ppt[v][i];
    }
    eps[0] = p->e_mean[0] + GU(s, 1, 1)[id] - te[0];
    eps[1] = p->e_mean[1] + GU(s, 2, 2)[id] - te[1];
    eps[2] = p->e_mean[2] + GU(s, 3, 3)[id] - te[2];
    eps[3] = 2.0 * p->e_mean[3] + GU(s, 3, 2)[id] + GU(s, 2, 3)[id] - 2.0 * te[3];
    eps[4] = 2.0 * p->e_mean[4] + GU(s, 3, 1)[id] + GU(s, 1, 3)[id] - 2.0 * te[4];
    eps[5] = 2.0 * p->e_mean[5] + GU(s, 1, 2)[id] + GU(s, 2, 1)[id] - 2.0 * te[5];
    for (int i = 0; i < 36; ++i) C[i] = 0;
    for (int n = 2; n <= p->numph; ++n) {
      int lo, hi;
      phase_range(p, n, &lo, &hi);
      for (int v = lo; v < hi; ++v)
        for (int i = 0; i < 36; ++i) C[i] += s->pphi[v * n3 + id] * p->sela[n - 1][i];
    }
    for (int i = 0; i < 36; ++i) C[i] += (1.0 - psum) * p->sela[0][i];
    int st = invert(C, 6, MEU_ERR_C_ELENER_SINGULAR);
    if (st) status = st;
    for (int i = 0; i < 6; ++i) {
      sig[i] = 0;
      for (int j = 0; j < 6; ++j) sig[i] += C[i + j * 6] * eps[j];
    }
    double elmat = 0;
    for (int i = 0; i < 6; ++i) {
      double em = 0;
      for (int j = 0; j < 6; ++j) em += SE(p, 1, i + 1, j + 1) * sig[j];
      elmat += sig[i] * em;
    }
    elmat *= 0.5;
    double en = (1.0 - psum) * elmat;
    for (int n = 2; n <= p->numph; ++n) {
      int lo, hi;
      phase_range(p, n, &lo, &hi);
      for (int v = lo; v < hi; ++v) {
        if (transsum[v] > tiny) {
          double elp = 0;
          for (int i = 0; i < 6; ++i) {
            double ep = 0;
            for (int j = 0; j < 6; ++j) ep += SE(p, n, i + 1, j + 1) * sig[j];
            elp += sig[i] * ep;
          }
          elp *= 0.5;
          en += elp * s->pphi[v * n3 + id];
          const double* t = p->trans_ppt[v];
          double g = sig[0] * t[0] + sig[1] * t[1] + sig[2] * t[2] + 2.0 * (sig[3] * t[3] + sig[4] * t[4] + sig[5] * t[5]);
          double pr = ppr[v * n3 + id];
          s->elgrad[v * n3 + id] = pr * (elmat - elp) - g * pr;
        }
      }
    }
    s->el_en[id] = en;
  }
  (void)nx; (void)nz;
  return status;
}

/* half-spectrum Parseval weight */
static inline double hweight(const orc_sim* s, int kx) {
  return (kx == 0 || 2 * kx == s->nx) ? 1.0 : 2.0;
}

/* fills the per-step reductions of the clip loop (Multi_MEUMAPPS.f:1008-1065) */
static void end_of_step(orc_sim* s, meu_diag* d, int clip) {
  const size_t n3 = (size_t)s->n3;
  const int V = s->V, E = s->E;
  double con_min = 1.0, con_max = 0.0, max_phi = 0.0, solid = 0.0;
  double cloc[MEU_MAX_EL] = {0};
  for (size_t id = 0; id < n3; ++id) {
    for (int e = 0; e < E; ++e) {
      double c = s->cons[e * n3 + id];
      if (c < con_min) con_min = c;
      if (c > con_max) con_max = c;
      cloc[e] += c;
    }
    for (int v = 0; v < V; ++v) {
      double* ph = &s->phi[v * n3 + id];
      if (clip) {
        if (*ph < 0.0) *ph = 0.0;
        if (*ph > 1.0) *ph = 1.0;
      }
      if (*ph > max_phi) max_phi = *ph;
      if (clip) {
        if (*ph > 0.0) solid += *ph;
      } else {
        solid += (*ph) * (*ph);
      }
    }
  }
  double oo = 1.0 / (double)s->n3;
  if (d) {
    d->cmin = con_min; d->cmax = con_max; d->phimax = max_phi; d->solid_now = solid / (double)s->n3;
    for (int e = 0; e < MEU_MAX_EL; ++e) d->cavg[e] = (e < E) ? cloc[e] * oo : 0.0;
  }
  s->glob_min = con_min; s->glob_max = con_max; s->phi_max = max_phi; s->solid_frac = solid;
}

/* One KKS step: Multi_MEUMAPPS.f:548-1106 */
static int kks_step(orc_sim* s, meu_diag* d) {
  const meu_params* p = &s->p;
  const int nx = s->nx, ny = s->ny, nz = s->nz, nxh = s->nxh, V = s->V, E = s->E;
  const int numph = p->numph, numel = p->numel, zdim = numph * numel;
  const size_t n3 = (size_t)s->n3, nk = (size_t)s->nk;
  int status = 0;
  (void)nx; (void)nz;

  /* noise (:552-571): increments arrive through orc_add_noise */
  if (!(s->step <= p->noise_step)) memset(s->phi_noise, 0, sizeof(double) * V * n3);

  /* spectral gradients and gradient-energy Laplacian (:575-615) */
  for (int v = 0; v < V; ++v) {
    f_trans(&s->f, s->phi + v * n3, s->ck);
    const double* g = p->grad_coeff[v];
#define GC(i, j) g[((j) - 1) * 3 + ((i) - 1)]
    for (int comp = 0; comp < 4; ++comp) {
#pragma omp parallel for schedule(static)
      for (int64_t id = 0; id < (int64_t)nk; ++id) {
        int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
        double a[3], b[3];
        kvec(s, kx, ky, kz, a, b);
        cplx val = s->ck[id];
        if (comp < 3) s->ck2[id] = val * (I * b[comp]);
        else {
          double k1s = -a[0] * a[0], k2s = -a[1] * a[1], k3s = -a[2] * a[2];
          double k12 = -b[0] * b[1], k23 = -b[1] * b[2], k31 = -b[2] * b[0];
          s->ck2[id] = val * (GC(1, 1) * k1s + GC(2, 2) * k2s + GC(3, 3) * k3s + (GC(1, 2) + GC(2, 1)) * k12 +
                              (GC(2, 3) + GC(3, 2)) * k23 + (GC(3, 1) + GC(1, 3)) * k31);
        }
      }
      double* dst = comp == 0 ? s->gx : comp == 1 ? s->gy : comp == 2 ? s->gz : s->kds;
      inv_trans(&s->f, s->ck2, dst + v * n3, s->work);
    }
  }

  /* per-voxel KKS driving force (:619-845) */
  double fch = 0, fw = 0, f_int = 0;
  memset(s->fcx, 0, sizeof(double) * E * n3);
  memset(s->fcy, 0, sizeof(double) * E * n3);
  memset(s->fcz, 0, sizeof(double) * E * n3);
#pragma omp parallel for schedule(static) reduction(+ : fch, fw, f_int) reduction(max : status)
  for (int64_t id = 0; id < (int64_t)n3; ++id) {
    double Pph[MEU_MAX_PH] = {0}, Gph[MEU_MAX_PH] = {0}, Ppr[MEU_MAX_VAR];
    double Z[256], Zr[16], X[MEU_MAX_EL][MEU_MAX_PH], Gib[MEU_MAX_PH] = {0}, MuC[MEU_MAX_EL] = {0};
    for (int n = 2; n <= numph; ++n) {
      int lo, hi;
      phase_range(p, n, &lo, &hi);
      for (int v = lo; v < hi; ++v) {
        double fi = s->phi[v * n3 + id], fi_sq = fi * fi;
        double pl = fi_sq * fi * (6.0 * fi_sq - 15.0 * fi + 10.0);
        s->pphi[v * n3 + id] = pl;
        Ppr[v] = 30.0 * fi_sq * (fi_sq - 2.0 * fi + 1.0);
        Pph[0] += pl;
        Pph[n - 1] += pl;
        Gph[n - 1] += fi_sq * (1.0 - fi) * (1.0 - fi);
        for (int u = 0; u < V; ++u)
          if (u != v) { double pu = s->phi[u * n3 + id]; Gph[0] += fi_sq * pu * pu; }
      }
    }
    Pph[0] = 1.0 - Pph[0];
    /* interface compositions (:677-710) */
    memcpy(Z, s->zconst, sizeof(double) * zdim * zdim);
    memcpy(Zr, s->zr_const, sizeof(double) * zdim);
    for (int e = 1; e <= numel; ++e) {
      int i0 = zdim - numel + e;
      Zr[i0 - 1] = s->cons[(e - 1) * n3 + id];
      for (int n = 1; n <= numph; ++n) {
        int j0 = numph * (e - 1) + n;
        Z[(i0 - 1) + (j0 - 1) * zdim] = Pph[n - 1];
      }
    }
    int st = invert(Z, zdim, MEU_ERR_Z_SINGULAR);
    if (st) status = st;
    for (int n = 1; n <= numph; ++n)
      for (int e = 1; e <= numel; ++e) {
        int i0 = numph * (e - 1) + n;
        double acc = 0;
        for (int j0 = 1; j0 <= zdim; ++j0) acc += Z[(i0 - 1) + (j0 - 1) * zdim] * Zr[j0 - 1];
        X[e - 1][n - 1] = acc;
      }
#define GP(j, n) p->gparams[(n) - 1][(j) - 1]
    for (int n = 1; n <= numph; ++n) {
      double gsum = 0;
      for (int e = 1; e <= numel; ++e) {
        int i1 = e + numel + 1;
        double dx = X[e - 1][n - 1] - GP(i1, n);
        gsum += GP(e, n) * dx * dx;
      }
      gsum += GP(numel + 1, n);
      Gib[n - 1] = gsum;
    }
    for (int e = 1; e <= numel; ++e) {
      int i1 = e + numel + 1;
      MuC[e - 1] = 2.0 * GP(e, 1) * (X[e - 1][0] - GP(i1, 1));
    }
    double fchloc = Pph[0] * Gib[0];
    double fwloc = p->wellph[0] * Gph[0];
    double fint_loc = 0;
    for (int n = 2; n <= numph; ++n) {
      int lo, hi;
      phase_range(p, n, &lo, &hi);
      for (int v = lo; v < hi; ++v) {
        const double* g = p->grad_coeff[v];
        double gxv = s->gx[v * n3 + id], gyv = s->gy[v * n3 + id], gzv = s->gz[v * n3 + id];
        double term = GC(1, 1) * gxv * gxv + GC(2, 2) * gyv * gyv + GC(3, 3) * gzv * gzv +
                      (GC(1, 2) + GC(2, 1)) * gxv * gyv + (GC(1, 3) + GC(3, 1)) * gxv * gzv +
                      (GC(2, 3) + GC(3, 2)) * gyv * gzv;
        fint_loc += 0.5 * term;
        double fi = s->phi[v * n3 + id];
        double termch = Gib[n - 1] - Gib[0];
        for (int e = 1; e <= numel; ++e) {
          double xdiff = X[e - 1][0] - X[e - 1][n - 1];
          termch += MuC[e - 1] * xdiff;
          double tprc = Ppr[v] * xdiff;
          s->fcx[(e - 1) * n3 + id] += tprc * gxv;
          s->fcy[(e - 1) * n3 + id] += tprc * gyv;
          s->fcz[(e - 1) * n3 + id] += tprc * gzv;
        }
        double well = 2.0 * p->wellph[n - 1] * fi * (1.0 - fi) * (1.0 - 2.0 * fi);
        for (int u = 0; u < V; ++u)
          if (u != v) { double pu = s->phi[u * n3 + id]; well += 4.0 * p->wellph[0] * fi * pu * pu; }
        s->fgrad[v * n3 + id] = termch * Ppr[v] + well;
      }
      fchloc += Pph[n - 1] * Gib[n - 1];
      fwloc += p->wellph[n - 1] * Gph[n - 1];
    }
#undef GP
    fch += fchloc;
    fw += fwloc;
    f_int += fint_loc;
    /* n_tilda projection (:824-841) */
    for (int jv = 0; jv < V; ++jv) {
      double term11 = 0;
      int ntil = 1;
      if (s->phi[jv * n3 + id] > 0.0) {
        for (int iv = 0; iv < V; ++iv)
          if (s->phi[iv * n3 + id] > 0.0 && iv != jv) {
            term11 += s->fgrad[iv * n3 + id] - s->kds[iv * n3 + id];
            ntil += 1;
          }
      }
      s->fdiff[jv * n3 + id] = s->fgrad[jv * n3 + id] - term11 / (double)ntil;
    }
  }
#undef GC
  if (status) return status;

  /* elasticity (:851-880) */
  double el_sum = 0;
  s->last_iters = 0;
  memset(s->elgrad, 0, sizeof(double) * V * n3);
  if (s->step >= p->elastep0 && p->elastic != MEU_ELAST_NONE) {
    memset(s->el_en, 0, sizeof(double) * n3);
    /* elener recomputes Ppr from phi (ModElastic.f:557); kds is free by now */
    double* pprall = s->kds;
    for (size_t i = 0; i < (size_t)V * n3; ++i) {
      double fi = s->phi[i], fi_sq = fi * fi;
      pprall[i] = 30.0 * fi_sq * (fi_sq - 2.0 * fi + 1.0);
    }
    status = eldis(s, pprall, 0);
    if (status) return status;
  } else {
    memset(s->el_en, 0, sizeof(double) * n3);
  }
  for (size_t i = 0; i < (size_t)V * n3; ++i) s->fdiff[i] += s->elgrad[i];
  for (size_t i = 0; i < n3; ++i) el_sum += s->el_en[i];

  if (d) {
    d->step = s->step;
    d->el_iters = s->last_iters;
    d->status = 0;
    d->fint = f_int; d->fw = fw; d->fch = fch; d->elen = el_sum;
    d->etot = f_int + fch + el_sum + fw;
    d->glob_min = s->glob_min; d->glob_max = s->glob_max; d->phi_max = s->phi_max;
    d->solid = s->solid_frac / (double)s->n3;
  }

  /* diffusion update (:910-949) */
  for (int e = 0; e < E; ++e) {
    f_trans(&s->f, s->cons + e * n3, s->ck);
    f_trans(&s->f, s->fcx + e * n3, s->ck2);
    f_trans(&s->f, s->fcy + e * n3, s->ck3);
    f_trans(&s->f, s->fcz + e * n3, s->work);
    const double dm = p->dt * p->cmobs[e];
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      double ksq = -a[0] * a[0] - a[1] * a[1] - a[2] * a[2];
      cplx term1 = (I * b[0]) * s->ck2[id] + (I * b[1]) * s->ck3[id] + (I * b[2]) * s->work[id];
      double term2 = 1.0 - dm * ksq;
      s->ck[id] = (s->ck[id] + dm * term1) / term2;
    }
    inv_trans(&s->f, s->ck, s->cons + e * n3, s->work);
  }

  /* TDGL update (:955-1001) */
  for (int v = 0; v < V; ++v) {
    f_trans(&s->f, s->phi + v * n3, s->ck);
    f_trans(&s->f, s->fdiff + v * n3, s->ck2);
    f_trans(&s->f, s->phi_noise + v * n3, s->ck3);
    const double* g = p->grad_coeff[v];
#define GC(i, j) g[((j) - 1) * 3 + ((i) - 1)]
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      double k1s = -a[0] * a[0], k2s = -a[1] * a[1], k3s = -a[2] * a[2];
      double k12 = -b[0] * b[1], k23 = -b[1] * b[2], k31 = -b[2] * b[0];
      cplx term1 = p->dt * p->b_mob * s->ck2[id];
      double term2 = 1.0 - p->dt * p->b_mob *
                               (GC(1, 1) * k1s + GC(2, 2) * k2s + GC(3, 3) * k3s + (GC(1, 2) + GC(2, 1)) * k12 +
                                (GC(2, 3) + GC(3, 2)) * k23 + (GC(3, 1) + GC(1, 3)) * k31);
      cplx term3 = s->ck3[id] * p->dt;
      s->ck[id] = (s->ck[id] - term1 + term3) / term2;
    }
#undef GC
    inv_trans(&s->f, s->ck, s->phi + v * n3, s->work);
  }

  end_of_step(s, d, p->clip_phi);
  s->step += 1;
  return 0;
}

/* One Landau step (configuration decks).  Same explicit coupling as the
 * reference: every force is evaluated on the fields at the start of the step. */
static int landau_step(orc_sim* s, meu_diag* d) {
  const meu_params* p = &s->p;
  const int ny = s->ny, nxh = s->nxh, V = s->V;
  const size_t n3 = (size_t)s->n3, nk = (size_t)s->nk;
  const double A = p->lan_a, B = p->lan_b, Cc = p->lan_c, D = p->lan_d, c1 = p->lan_c1, c2 = p->lan_c2;
  const double w = p->cross_w;
  int status = 0;
  double* c = s->cons;
  double* theta_pr = s->fgrad; /* V*n3 */
  double fch = 0;
  /* theta, theta', mu_c, bulk energy */
#pragma omp parallel for schedule(static) reduction(+ : fch)
  for (int64_t id = 0; id < (int64_t)n3; ++id) {
    double cv = c[id], s2 = 0, s4 = 0, s6 = 0, cross = 0;
    for (int v = 0; v < V; ++v) {
      double e = s->phi[v * n3 + id], e2 = e * e;
      s2 += e2; s4 += e2 * e2; s6 += e2 * e2 * e2;
      if (p->eig_coupling == MEU_EIG_H) {
        s->pphi[v * n3 + id] = e2 * e * (6.0 * e2 - 15.0 * e + 10.0);
        theta_pr[v * n3 + id] = 30.0 * e2 * (e2 - 2.0 * e + 1.0);
      } else {
        s->pphi[v * n3 + id] = e2;
        theta_pr[v * n3 + id] = 2.0 * e;
      }
    }
    for (int v = 0; v < V; ++v)
      for (int u = 0; u < V; ++u)
        if (u != v) cross += s->phi[v * n3 + id] * s->phi[v * n3 + id] * s->phi[u * n3 + id] * s->phi[u * n3 + id];
    fch += 0.5 * A * (cv - c1) * (cv - c1) + 0.5 * B * (c2 - cv) * s2 - 0.25 * Cc * s4 + D / 6.0 * s6 + w * cross;
    s->rtmp[id] = A * (cv - c1) - 0.5 * B * s2; /* mu_c */
  }
  /* elasticity */
  double el_sum = 0;
  s->last_iters = 0;
  memset(s->elgrad, 0, sizeof(double) * V * n3);
  memset(s->el_en, 0, sizeof(double) * n3);
  if (p->elastic != MEU_ELAST_NONE && s->step >= p->elastep0) {
    status = eldis(s, theta_pr, p->elastic == MEU_ELAST_HOMOG);
    if (status) return status;
    for (size_t i = 0; i < n3; ++i) el_sum += s->el_en[i];
  }
  /* gradient energy by Parseval on the start-of-step fields (reference f_int
   * form: Nyquist-zeroed derivative vectors) */
  double fint = 0;
  f_trans(&s->f, c, s->ck);
  if (p->diag_energy) {
    double acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      double bb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
      double cc = creal(s->ck[id]) * creal(s->ck[id]) + cimag(s->ck[id]) * cimag(s->ck[id]);
      acc += hweight(s, kx) * 0.5 * p->kappa_c * bb * cc;
    }
    fint += acc * (double)s->n3;
  }
  /* Cahn-Hilliard: c^ <- (c^ - dt M k^2 mu^) / (1 + dt M kappa_c k^4) */
  f_trans(&s->f, s->rtmp, s->ck2);
  const double dm = p->dt * p->cmobs[0];
#pragma omp parallel for schedule(static)
  for (int64_t id = 0; id < (int64_t)nk; ++id) {
    int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
    double a[3], b[3];
    kvec(s, kx, ky, kz, a, b);
    double k2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    s->ck[id] = (s->ck[id] - dm * k2 * s->ck2[id]) / (1.0 + dm * p->kappa_c * k2 * k2);
  }
  /* TDGL */
  for (int v = 0; v < V; ++v) {
    const double* g = p->grad_coeff[v];
#define GC(i, j) g[((j) - 1) * 3 + ((i) - 1)]
    f_trans(&s->f, s->phi + v * n3, s->ck3);
    if (p->diag_energy) {
      double acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
      for (int64_t id = 0; id < (int64_t)nk; ++id) {
        int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
        double a[3], b[3];
        kvec(s, kx, ky, kz, a, b);
        double q = GC(1, 1) * b[0] * b[0] + GC(2, 2) * b[1] * b[1] + GC(3, 3) * b[2] * b[2] +
                   (GC(1, 2) + GC(2, 1)) * b[0] * b[1] + (GC(1, 3) + GC(3, 1)) * b[0] * b[2] +
                   (GC(2, 3) + GC(3, 2)) * b[1] * b[2];
        double cc = creal(s->ck3[id]) * creal(s->ck3[id]) + cimag(s->ck3[id]) * cimag(s->ck3[id]);
        acc += hweight(s, kx) * 0.5 * q * cc;
      }
      fint += acc * (double)s->n3;
    }
    /* local driving force g_v = df/deta_v + el_grad_v */
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < (int64_t)n3; ++id) {
      double e = s->phi[v * n3 + id], others = 0;
      for (int u = 0; u < V; ++u)
        if (u != v) others += s->phi[u * n3 + id] * s->phi[u * n3 + id];
      double gv = B * (c2 - c[id]) * e - Cc * e * e * e + D * e * e * e * e * e + 4.0 * w * e * others;
      s->fdiff[v * n3 + id] = gv + s->elgrad[v * n3 + id];
    }
    f_trans(&s->f, s->fdiff + v * n3, s->ck2);
#pragma omp parallel for schedule(static)
    for (int64_t id = 0; id < (int64_t)nk; ++id) {
      int kx = (int)(id % nxh), ky = (int)((id / nxh) % ny), kz = (int)(id / ((int64_t)nxh * ny));
      double a[3], b[3];
      kvec(s, kx, ky, kz, a, b);
      double k1s = -a[0] * a[0], k2s = -a[1] * a[1], k3s = -a[2] * a[2];
      double k12 = -b[0] * b[1], k23 = -b[1] * b[2], k31 = -b[2] * b[0];
      double term2 = 1.0 - p->dt * p->b_mob *
                               (GC(1, 1) * k1s + GC(2, 2) * k2s + GC(3, 3) * k3s + (GC(1, 2) + GC(2, 1)) * k12 +
                                (GC(2, 3) + GC(3, 2)) * k23 + (GC(3, 1) + GC(1, 3)) * k31);
      s->ck3[id] = (s->ck3[id] - p->dt * p->b_mob * s->ck2[id]) / term2;
    }
#undef GC
    /* the new eta is staged in gx: every variant's force must see the old eta */
    inv_trans(&s->f, s->ck3, s->gx + v * n3, s->work);
  }
  memcpy(s->phi, s->gx, sizeof(double) * V * n3);
  inv_trans(&s->f, s->ck, c, s->work);

  if (d) {
    d->step = s->step;
    d->el_iters = s->last_iters;
    d->status = 0;
    d->fint = fint; d->fw = 0.0; d->fch = fch; d->elen = el_sum;
    d->etot = fint + fch + el_sum;
    d->glob_min = s->glob_min; d->glob_max = s->glob_max; d->phi_max = s->phi_max;
    d->solid = s->solid_frac / (double)s->n3;
  }
  end_of_step(s, d, p->clip_phi);
  s->step += 1;
  return 0;
}

int orc_run(orc_sim* s, int nsteps, meu_diag* diag) {
  for (int i = 0; i < nsteps; ++i) {
    meu_diag* d = diag ? diag + i : NULL;
    int st = (s->p.model == MEU_MODEL_KKS) ? kks_step(s, d) : landau_step(s, d);
    if (st) return st;
  }
  return 0;
}

/* --------------------------------------------------- exported test hooks -- */
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* f_trans / inv_trans on caller arrays; spectra are interleaved re,im doubles */
int orc_rfft3(int nx, int ny, int nz, const double* in, double* out_ri) {
  fft3 f;
  if (fft3_init(&f, nx, ny, nz)) return -1;
  f_trans(&f, in, (cplx*)out_ri);
  fft3_free(&f);
  return 0;
}
int orc_irfft3(int nx, int ny, int nz, const double* in_ri, double* out) {
  fft3 f;
  if (fft3_init(&f, nx, ny, nz)) return -1;
  size_t nk = (size_t)nz * ny * (nx / 2 + 1);
  cplx* work = (cplx*)malloc(sizeof(cplx) * nk);
  inv_trans(&f, (const cplx*)in_ri, out, work);
  free(work);
  fft3_free(&f);
  return 0;
}
int orc_invert(double* a, int n) { return invert(a, n, 1); }
