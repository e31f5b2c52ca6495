// host.cu -- host-side helpers of the C-ABI (no GPU work): the reference's
// ran_2 generator (ran_2.f:1-42) with its SAVE state made explicit, the
// langevin draw (ModFunc.f:77-100) and the uniform-noise initialiser of the
// Landau decks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/meu.h"

namespace {
constexpr int32_t kIm1 = 2147483563, kIm2 = 2147483399, kImm1 = kIm1 - 1;
constexpr int32_t kIa1 = 40014, kIa2 = 40692, kIq1 = 53668, kIq2 = 52774, kIr1 = 12211, kIr2 = 3791;
constexpr int32_t kNtab = 32, kNdiv = 1 + kImm1 / kNtab;

// One Schrage step of a multiplicative congruential generator (a*x mod m
// without overflow): x <- a*(x - k*q) - k*r, then wrap into [0, m).
inline int32_t schrage(int32_t x, int32_t a, int32_t q, int32_t r, int32_t m) {
  const int32_t k = x / q;
  const int32_t y = a * (x - k * q) - k * r;
  return y + (m & (y >> 31));  // + m when y < 0, without a branch (its sign is random)
}

// the shuffle-table set-up ran_2 makes on a call with idum <= 0 (ran_2.f:14-24)
inline void ran2_seed(meu_ran2_state* s) {
  if (s->idum <= 0) {
    s->idum = (-s->idum > 1) ? -s->idum : 1;
    s->idum2 = s->idum;
    for (int j = kNtab + 8; j >= 1; --j) {
      s->idum = schrage(s->idum, kIa1, kIq1, kIr1, kIm1);
      if (j <= kNtab) s->iv[j - 1] = s->idum;
    }
    s->iy = s->iv[0];
  }
}

// ran_2 on a state held in locals (registers and a stack table) for a run of draws;
// the same steps as meu_ran2 after its initialisation
struct Ran2Local {
  int32_t idum, idum2, iy, iv[kNtab];
  explicit Ran2Local(const meu_ran2_state& s) : idum(s.idum), idum2(s.idum2), iy(s.iy) {
    for (int j = 0; j < kNtab; ++j) iv[j] = s.iv[j];
  }
  void store(meu_ran2_state& s) const {
    s.idum = idum;
    s.idum2 = idum2;
    s.iy = iy;
    for (int j = 0; j < kNtab; ++j) s.iv[j] = iv[j];
  }
  inline double next() {
    const double am = (double)(1.0f / (float)kIm1);
    const double rnmx = 1.0 - 1.2e-7;
    idum = schrage(idum, kIa1, kIq1, kIr1, kIm1);
    idum2 = schrage(idum2, kIa2, kIq2, kIr2, kIm2);
    const int j = iy / kNdiv;
    iy = iv[j] - idum2;
    iv[j] = idum;
    iy += (iy < 1) ? kImm1 : 0;
    const double v = am * (double)iy;
    return v < rnmx ? v : rnmx;
  }
};
}  // namespace

extern "C" {

void meu_ran2_init(meu_ran2_state* s, int32_t iseed) {
  std::memset(s, 0, sizeof(*s));
  s->idum = iseed;
  s->idum2 = 123456789;
}

double meu_ran2(meu_ran2_state* s) {
  // am = 1./im1 is single precision in the reference: float(im1) rounds to
  // 2^31 - 128 and the quotient is rounded to single before widening
  const double am = (double)(1.0f / (float)kIm1);
  const double rnmx = 1.0 - 1.2e-7;
  ran2_seed(s);
  s->idum = schrage(s->idum, kIa1, kIq1, kIr1, kIm1);
  s->idum2 = schrage(s->idum2, kIa2, kIq2, kIr2, kIm2);
  const int j = s->iy / kNdiv;  // 0-based slot of the shuffle table
  s->iy = s->iv[j] - s->idum2;
  s->iv[j] = s->idum;
  if (s->iy < 1) s->iy += kImm1;
  const double v = am * (double)s->iy;
  return v < rnmx ? v : rnmx;
}

double meu_langevin(meu_ran2_state* s, double sd) {
  for (;;) {
    const double v1 = 2.0 * meu_ran2(s) - 1.0;
    const double v2 = 2.0 * meu_ran2(s) - 1.0;
    double rsq = v1 * v1 + v2 * v2;
    if (rsq > 0.0 && rsq < 1.0) {
      rsq = std::sqrt(-2.0 * std::log(rsq) / rsq);
      return v2 * rsq * sd;
    }
  }
}

// n langevin draws, the numbers of n meu_langevin calls: the serial ran_2 chain and the
// polar method's accept test run on the calling thread (the state in locals), which
// keeps v2 and rsq of every accepted pair; the transcendental part,
// v2 * sqrt(-2 log(rsq) / rsq) * sd, then runs on up to `threads` host threads.
int meu_langevin_fill(meu_ran2_state* s, double sd, int64_t n, double* out, int32_t threads) {
  if (!s || (!out && n > 0) || n < 0) return MEU_ERR_BADARG;
  if (n == 0) return MEU_OK;
  std::vector<double> rsqv;
  try {
    rsqv.resize((size_t)n);
  } catch (...) {
    return MEU_ERR_NOMEM;
  }
  ran2_seed(s);
  {
    // every attempt is stored at slot i, which advances only when the pair is accepted
    // (a rejected attempt is overwritten by the next): no branch on the random test
    Ran2Local r(*s);
    int64_t i = 0;
    while (i < n) {
      const double v1 = 2.0 * r.next() - 1.0;
      const double v2 = 2.0 * r.next() - 1.0;
      const double rsq = v1 * v1 + v2 * v2;
      out[i] = v2;
      rsqv[(size_t)i] = rsq;
      i += (rsq > 0.0) & (rsq < 1.0);
    }
    r.store(*s);
  }
  auto finish = [&](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; ++i) {
      const double rsq = std::sqrt(-2.0 * std::log(rsqv[(size_t)i]) / rsqv[(size_t)i]);
      out[i] = out[i] * rsq * sd;
    }
  };
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(threads > 0 ? threads : 1, n / 65536 + 1));
  const int64_t per = (n + nt - 1) / nt;
  auto part = [&](int64_t t) { finish(std::min(n, t * per), std::min(n, (t + 1) * per)); };
  std::vector<std::thread> pool;
  try {
    for (int64_t t = 1; t < nt; ++t) pool.emplace_back(part, t);
  } catch (...) {
    // fewer threads than asked (the system refused one): this thread takes the rest
  }
  part(0);
  for (int64_t t = 1 + (int64_t)pool.size(); t < nt; ++t) part(t);
  for (auto& th : pool) th.join();
  return MEU_OK;
}

void meu_init_uniform(meu_ran2_state* s, int32_t nx, int32_t ny, int32_t nz, int32_t nvar, double c0, double c_amp,
                      double eta_amp, double* cons, double* phi) {
  const int64_t n3 = (int64_t)nx * ny * nz;
  for (int64_t i = 0; i < n3; ++i) {
    cons[i] = c0 + c_amp * (2.0 * meu_ran2(s) - 1.0);
    for (int v = 0; v < nvar; ++v) phi[i * nvar + v] = eta_amp * (2.0 * meu_ran2(s) - 1.0);
  }
}

int meu_params_from_gparams(int32_t nx, int32_t ny, int32_t nz, int32_t vartot, int32_t numel, int32_t numph,
                            const int32_t* nvar_ph, int64_t step, int64_t elastep0, int64_t noise_step,
                            double t_step, double b_mob, const double* cmobs, const double* e_mean,
                            const double* grad_coeff, const double* trans_ppt, const double* cela,
                            const double* sela, const double* gparams, const double* wellph, meu_params* out) {
  if (!out || !nvar_ph || !cmobs || !e_mean || !grad_coeff || !trans_ppt || !cela || !sela || !gparams || !wellph)
    return MEU_ERR_BADARG;
  if (vartot < 1 || vartot > MEU_MAX_VAR || numel < 1 || numel > MEU_MAX_EL || numph < 1 || numph > MEU_MAX_PH ||
      nx < 1 || ny < 1 || nz < 1)
    return MEU_ERR_BADARG;
  meu_params p;
  std::memset(&p, 0, sizeof(p));
  p.step = step;
  p.elastep0 = elastep0;
  p.noise_step = noise_step;
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.model = MEU_MODEL_KKS;
  p.precision = MEU_PREC_F64;
  p.nvar = vartot;
  p.numel = numel;
  p.numph = numph;
  for (int n = 0; n < numph; ++n) p.nvar_ph[n] = nvar_ph[n];
  p.elastic = MEU_ELAST_HETERO;
  p.el_min_iter = 4;   // ModElastic.f:469
  p.el_max_iter = 10;  // ModElastic.f:462
  p.clip_phi = 1;      // Multi_MEUMAPPS.f:1034-1035
  p.diag_energy = 1;
  p.dt = t_step;
  p.b_mob = b_mob;
  for (int e = 0; e < numel; ++e) p.cmobs[e] = cmobs[e];
  p.el_tol = 1e-7;  // ModElastic.f:435
  for (int i = 0; i < 6; ++i) p.e_mean[i] = e_mean[i];
  // the Fortran arrays are column-major with the leading index fastest: element
  // (i, j, v) of grad_coeff(3,3,vartot) sits at (i-1) + 3 (j-1) + 9 (v-1), which is
  // the row-major [v][(j-1)*3 + (i-1)] of meu_params
  for (int v = 0; v < vartot; ++v) {
    for (int i = 0; i < 9; ++i) p.grad_coeff[v][i] = grad_coeff[9 * v + i];
    for (int i = 0; i < 6; ++i) p.trans_ppt[v][i] = trans_ppt[6 * v + i];
  }
  const int ngp = 2 * numel + 1;
  for (int n = 0; n < numph; ++n) {
    for (int i = 0; i < 36; ++i) {
      p.cela[n][i] = cela[36 * n + i];
      p.sela[n][i] = sela[36 * n + i];
    }
    for (int j = 0; j < ngp; ++j) p.gparams[n][j] = gparams[ngp * n + j];
    p.wellph[n] = wellph[n];
  }
  *out = p;
  return MEU_OK;
}

}  // extern "C"
