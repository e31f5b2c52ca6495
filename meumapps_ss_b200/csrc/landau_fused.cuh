// landau_fused.cuh -- the fused Landau time step (cubic grids N in
// {32, 48, 64, 96, 128}, 1..4 variants, theta = eta^2 coupling, homogeneous
// elasticity or none).
//
// The state of the step is spectral: eta^_v and the fluctuation dc^ are kept
// in device memory in the column kernels' layout ([kz position][column]) and
// every step only adds its increment to them.  The real-space eta and dc are
// re-derived each step for the nonlinear terms and the output.  (Re-transforming
// the real fields every step instead makes an FP32 forward/inverse pair act on
// slowly varying data each step, whose rounding errors then add up coherently.)
// Five launches per step:
//
//   PF  plane:  theta_v = eta_v^2 -> x R2C + y FFT                         (+ bulk energy)
//   Z1  column: z FFT of theta -> Green operator phi_v; Cahn-Hilliard update of
//              the dc^ state (mu^ = A dc^ - B/2 sum theta^_v) -> z iFFT of phi_v, dc_new
//   PB  plane:  y iFFT + x C2R of phi_v -> g_v = df/deta_v + el_grad_v -> x R2C + y FFT;
//              plane of dc_new -> real
//   Z2  column: z FFT of g -> eta^ state <- (eta^ - dt L g^) / (1 + dt L k.kappa.k) -> z iFFT
//   PI  plane:  y iFFT + x C2R of eta_new -> real eta (+ end-of-step statistics)
//
// Set-up (after new fields are uploaded): PF in raw mode transforms eta_v and dc,
// Z0 finishes the z transform into the spectral state.
#pragma once
#include "fused.cuh"
#include "kernels.cuh"

namespace meu {

// Per-engine constants of the fused Landau step (device memory, copied to
// shared memory by the column kernels).
struct LanFusedConst {
  double qcoef[6][6];     // Q_m = sum_n qcoef[m][n] Kv_n, m in (11,22,33,23,13,12), Kv = (a1^2,a2^2,a3^2,b2b3,b1b3,b1b2)
  double sig0[4][6];      // eigenstress (tensor Voigt)
  double eps_eng[4][6];   // eigenstrain (engineering Voigt)
  double c0m[36];         // C0 (column-major 6x6)
  double ebar_eng[6];
  double g[4][9];         // grad_coeff (kappa_eta) per variant
  double A[4][4], sig0_ebar[4];
  double lan_a, lan_b, lan_c, lan_d, lan_c1, lan_c2, cross_w, kappa_c, dm, dtl, cbar;
};

template <typename R>
struct LanFusedArgs {
  const LanFusedConst* F;
  R* eta;     // V real fields
  R* c;       // dc (start of step)
  R* c2;      // dc (end of step)
  cplx<R>* M; // V+1 M-form spectra
  cplx<R>* Keta;  // spectral state eta^_v (V spectra, normalised, column-kernel layout)
  cplx<R>* Kc;    // spectral state dc^ (normalised, column-kernel layout)
  double* partials;
  int pstride;
  int* err;
  int homog, energy;
  const cplx<R>* twx;
  const cplx<R>* twy;
  const cplx<R>* twz;
  const cplx<R>* post;
};

enum LanQ : int {
  LQ_FCH = Q_FCH, LQ_FINT = Q_FINT, LQ_ELEN = Q_ELEN, LQ_CMIN = Q_CMIN, LQ_CMAX = Q_CMAX, LQ_PHIMAX = Q_PHIMAX,
  LQ_SOLID = Q_SOLID, LQ_CSUM = Q_CSUM0
};

// host launch entry (landau_fused.cu): returns false if (N, V) has no instantiation
template <typename R>
bool lan_fused_step(int N, int V, const LanFusedArgs<R>& a, cudaStream_t st, LaunchHook* hook, int* nb_out);
// spectral state from the real fields eta and dc (after an upload)
template <typename R>
bool lan_fused_init(int N, int V, const LanFusedArgs<R>& a, cudaStream_t st, LaunchHook* hook);
bool lan_fused_supported(const meu_params& p);

}  // namespace meu
