// adjoint.cuh -- hand-written adjoint of the fused Landau step, on the default
// schedule (radix plan 0, 512-thread planes, default column tile).  The formulas
// below are written for one order parameter; V variants (V >= 2, kernels *_v)
// generalise them as set out after them.
//
// Forward step n (real fields eta, dc; spectra normalised, x = F^-1 x^):
//   theta = eta^2
//   dc^_{n+1}  = P [ (1 - dm A k^2) dc^_n + dm k^2 (B/2) theta^ ],   P = 1/(1 + dm kc k^4)  (k != 0)
//   phi        = F^-1 [ g(k) theta^ ],   g(k) = -(sig0 b)^T Omega(k) (sig0 b)
//   G          = B(c2 - c)eta - C eta^3 + D eta^5 - 2 eta (s0 + phi - A11 eta^2),  c = cbar + dc
//   eta^_{n+1} = H [ eta^_n - dtL G^ ],   H = 1/(1 + dtL k.kappa.k)
// With lam = dJ/deta_n, nu = dJ/ddc_n (real fields, spectra as above), every
// operator F^-1 D(k) F with real even D is symmetric, so one adjoint step is
//   w  = F^-1 [H lam^_{n+1}],   z = -dtL w,   h = -eta z
//   a  = w + z dG/deta
//   r  = F^-1 [ 2 g h^ + P dm k^2 (B/2) nu^_{n+1} ]
//   lam_n = a + 2 eta r,        nu^_n = P (1 - dm A k^2) nu^_{n+1} + B h^
// and the parameter derivatives of the step are (<x,y> the real-space sum)
//   d/d(dtL):  -<lam_{n+1}, F^-1[kk H eta^_{n+1}]> - <w, G>
//   d/d(beta): -dtL <lam_{n+1}, F^-1[kk H eta^_{n+1}]>      (kappa_eta -> beta kappa_eta)
//   d/d(kc):   -dm <nu_{n+1}, F^-1[k^4 P dc^_{n+1}]>
//   d/d(dm):   -kc <nu_{n+1}, F^-1[k^4 P dc^_{n+1}]> - <nu_{n+1}, F^-1[P k^2 mu^_n]>,
//              mu^_n = A dc^_n - (B/2) theta^_n
//   d/d(alpha): <z, -2 eta (s0 + 2 phi - 2 A11 eta^2)>       (eigenstrain -> alpha eigenstrain)
// Four launches per adjoint step, the same plane / column split as the forward:
//   EA column: z FFT of lam_{n+1} -> lam^ -> w^ = H lam^ (+ d/d(dtL), beta, kc, dm sums) -> z iFFT
//   B  plane:  xy iFFT of w -> a (real), h -> xy FFT (+ <w,G>, d/d(alpha) sums)
//   C  column: z FFT of h -> nu^ update, r^ -> z iFFT
//   D  plane:  xy iFFT of r -> lam_n = a + 2 eta r -> xy FFT (or lam_0 out)
//
// V variants (forward: theta_v = eta_v^2, phi_v = F^-1 [sum_q g_vq theta^_q] with the
// symmetric g_vq(k) = -(sig0_v b)^T Q^-1 (sig0_q b), mu^ = A dc^ - (B/2) sum_v theta^_v,
//   G_v = B(c2 - c) eta_v - C eta_v^3 + D eta_v^5 + 4 w eta_v sum_{q != v} eta_q^2
//         - 2 eta_v (s0_v + phi_v - sum_q A_vq eta_q^2),   A_vq = eps0_v.C0.eps0_q,
// H_v from variant v's gradient tensor):
//   w_v = F^-1 [H_v lam^_v],  z_v = -dtL w_v,  h_v = -eta_v z_v
//   a_u = w_u + sum_v z_v dG_v/deta_u, with
//     dG_v/deta_v = B(c2 - c) - 3C eta_v^2 + 5D eta_v^4 + 4w sum_{q != v} eta_q^2
//                   - 2 (s0_v + phi_v - sum_q A_vq eta_q^2) + 4 A_vv eta_v^2,
//     dG_v/deta_u = 8 w eta_v eta_u + 4 A_vu eta_v eta_u   (u != v)
//   r^_q = -2 (sig0_q b)^T Q^-1 sum_v (sig0_v b) h^_v + P dm k^2 (B/2) nu^_{n+1}
//   lam_q = a_q + 2 eta_q r_q,   nu^_n = P (1 - dm A k^2) nu^_{n+1} + B sum_v h^_v
// and the parameter sums add over the variants.  Six launches per adjoint step:
//   EA_v column (V fields), B1_v plane (xy iFFT of w_v), B2_v pointwise (a_v, h_v, <w,G>,
//   d/d(alpha)), B3_v plane (xy FFT of h_v), C_v column (V fields), D_v plane (per q).
#pragma once
#include "landau_fused_kernels.cuh"

namespace meu {

template <typename R>
struct AdjArgs {
  const LanFusedConst* F;
  cplx<R>* M;                 // one M-form field of scratch
  cplx<R>* nu;                // adjoint state nu^ (column layout)
  const cplx<R>* lam_seed;    // lam^_T (column layout) for the first adjoint step
  const cplx<R>* eta_k1;      // eta^_{n+1}
  const cplx<R>* c_k1;        // dc^_{n+1}
  const cplx<R>* c_k0;        // dc^_n
  const cplx<R>* theta_k0;    // theta^_n
  const R* eta;               // eta_n
  const R* c;                 // dc_n
  const R* phi;               // phi_n
  R* aw;                      // a of the step (real scratch; V fields)
  R* wv;                      // w_v (V real fields; V >= 2 only)
  R* hv;                      // h_v (V real fields; V >= 2 only)
  int V;                      // variants
  R* lam_out;                 // lam_0 (last adjoint step), else NULL
  double* partials;           // [ADJ_Q][PSTRIDE]
  int homog;
  int from_seed;              // EA: lam^ from lam_seed instead of the M field
  const cplx<R>* twx;
  const cplx<R>* twy;
  const cplx<R>* twz;
  const cplx<R>* post;
  int* err;                   // the handle's error word (bounded waits that ran out)
};

enum AdjQ : int { AQ_X = 0, AQ_Y, AQ_Z, AQ_WG, AQ_EA, ADJ_Q };

// launches of one adjoint step and of the loss seed (adjoint.cu)
template <typename R>
bool adj_step(int N, const AdjArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb);

}  // namespace meu
