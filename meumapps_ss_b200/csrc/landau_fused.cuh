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
// Four launches per step (five on the first step after new fields):
//
//   PF  plane:  theta_v = eta_v^2 -> x R2C + y FFT   (first step after new fields only)
//   Z1  column: z FFT of theta -> Green operator phi_v; Cahn-Hilliard update of
//              the dc^ state (mu^ = A dc^ - B/2 sum theta^_v) -> z iFFT of phi_v, dc_new
//   PB  plane:  y iFFT + x C2R of phi_v -> g_v = df/deta_v + el_grad_v -> x R2C + y FFT
//              (+ bulk free energy of the start-of-step fields)
//   Z2  column: z FFT of g -> eta^ state <- (eta^ - dt L g^) / (1 + dt L k.kappa.k) -> z iFFT
//   PI  plane:  y iFFT + x C2R of eta_new, dc_new -> real eta, dc in place
//              (+ end-of-step statistics; theta_v = eta_v^2 -> x R2C + y FFT for the
//              next step; the last block reduces the step's partials into its history row)
//
// Set-up (after new fields are uploaded): PF in raw mode transforms eta_v and dc,
// Z0 finishes the z transform into the spectral state.
//
// The real-field inputs of the step (eta and dc) are read by PF and PB and
// rewritten only by PI, the last launch, so both are updated in place.
#pragma once
#include <vector>

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
  double elastic_on;  // 1: the deck has elasticity (Q(k) is checked once, LS_QCHECK)
  // 1 when qcoef has the cubic pattern Q_ii = q_own a_i^2 + q_other (|a|^2 - a_i^2),
  // Q_ij = q_off b_i b_j (i != j), which Z1 then evaluates with these three constants
  double q_cubic, q_own, q_other, q_off;
};

// Device-side arguments of one simulation ("member").  Kernels read them from a
// device array indexed by blockIdx.z, so one launch covers every member of an
// ensemble bucket (same N, V and precision); a single simulation is a bucket of one.
template <typename R>
struct LanFusedArgs {
  const LanFusedConst* F;
  R* eta;     // V real fields (updated in place)
  R* c;       // dc (updated in place)
  cplx<R>* M; // V+1 M-form spectra
  cplx<R>* Keta;  // spectral state eta^_v (V spectra, normalised, column-kernel layout)
  cplx<R>* Kc;    // spectral state dc^ (normalised, column-kernel layout)
  double* partials;  // per-block reductions [quantity][PSTRIDE]
  int* err;
  int homog, energy;
  const cplx<R>* twx;
  const cplx<R>* twy;
  const cplx<R>* twz;
  const cplx<R>* post;
  double* hist;   // per-step reduction rows [hist_rows][Q_STEP_COUNT]
  int* hist_row;  // row of the current step (advanced at the end of the step)
  int* ticket;    // completion counter of the step's last kernel
  int hist_rows;
  // where the step writes the new state (equal to eta, c, Keta, Kc for an in-place step)
  R* eta_next;
  R* c_next;
  cplx<R>* Keta_out;
  cplx<R>* Kc_out;
  // Green-operator table of homogeneous elasticity for one variant: one real plane in
  // the dc^ state layout (k_lf_gtab); NULL without elasticity or with several variants
  R* gtab;
  // optional records of the step for the adjoint (NULL: off): the real elastic
  // potential phi_v (V fields) and the normalised spectra theta^_v (V spectra)
  R* rec_phi;
  cplx<R>* rec_theta;
};

// Schedule of the fused kernels: radix plan variant (fz::rplan), threads of the
// plane kernels, column tile width (complex columns per column-kernel block).
struct LanSched {
  int pv = 0, ntp = 512, tm = 0;  // tm = 0: 16 columns (FP32) / 8 columns (FP64)
};

enum LanQ : int {
  LQ_FCH = Q_FCH, LQ_FINT = Q_FINT, LQ_ELEN = Q_ELEN, LQ_CMIN = Q_CMIN, LQ_CMAX = Q_CMAX, LQ_PHIMAX = Q_PHIMAX,
  LQ_SOLID = Q_SOLID, LQ_CSUM = Q_CSUM0
};

// options of lan_fused_step
enum LanStepOpt : int {
  LS_ENERGY = 1,       // fort.98 energies of the step
  LS_THETA_READY = 2,  // M holds theta^ of the current fields (written by the previous step's PI)
  LS_QCHECK = 4,       // first step: test Q(k) of every k with the reference's rcond rule
};

// Host launch entries (landau_fused.cu).  dA: device array of `members`
// argument records.  Return false if (N, V, schedule) has no instantiation.
// lan_fused_step writes the per-block reduction counts of the step into nb.
template <typename R>
bool lan_fused_step(int N, int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, int opts,
                    cudaStream_t st, LaunchHook* hook, int* nb);
// spectral state from the real fields eta and dc (after an upload)
template <typename R>
bool lan_fused_init(int N, int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, cudaStream_t st,
                    LaunchHook* hook);
// the schedules instantiated for (N, precision)
std::vector<LanSched> lan_sched_candidates(int N, bool f64);
// Times every candidate schedule on the members' buffers (a few steps each, the
// fields must not hold a simulation yet: tuning advances them) and returns the
// fastest.  Results are cached per (precision, N, V, members, energy) for the
// process and, when the environment names a file in MEU_AUTOTUNE_CACHE, in that file.
template <typename R>
LanSched lan_autotune(int N, int V, const LanFusedArgs<R>* dA, int members, bool energy, cudaStream_t st,
                      double* best_ms);
bool lan_fused_supported(const meu_params& p);

// per-(R, N) entries, one translation unit each (lf_inst_*.cu)
template <typename R, int N>
bool lf_step_n(int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, int opts, cudaStream_t st,
               LaunchHook* hook, int* nb);
template <typename R, int N>
bool lf_init_n(int V, const LanSched& s, const LanFusedArgs<R>* dA, int members, cudaStream_t st, LaunchHook* hook);

}  // namespace meu
