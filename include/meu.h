/*
 * meu.h -- C-ABI of the B200 (sm_100a) time step of MEUMAPPS-SS.
 *
 * One call of meu_run() replaces the body of the reference time loop
 *   Multi_MEUMAPPS.f:548-1106  ("4 continue ... if(step.lt.Nt) go to 4"),
 * i.e. the spectral gradients (:575-615), the KKS driving force (:634-845),
 * the elasticity solve `eldis`/`elener` (ModElastic.f:11-691), the
 * semi-implicit Cahn-Hilliard/diffusion update (:910-949), the TDGL update
 * (:955-1001) and the post-step clip and reductions (:1008-1065, :885-908).
 * The data_save I/O (:1074-1100) stays with the caller.
 *
 * All entry points take plain C types, return an int status (never exit the
 * process) and are synchronous on return.  A handle owns its device memory and
 * its CUDA stream; one handle must not be used by two host threads at once.
 *
 * Array layout at the boundary is the reference's Fortran layout, component
 * index fastest:  Cons(numel,Nx,Ny,Nz), phi(vartot,Nx,Ny,Nz)
 * (Multi_MEUMAPPS.f:260,267), el_en(Nx,Ny,Nz) and each displacement field
 * u1..u3 / grad_j_ui as (Nx,Ny,Nz) (:279-293).  The library converts to its
 * own structure-of-arrays layout on upload and back on download.
 */
#ifndef MEU_H
#define MEU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MEU_MAX_VAR 16 /* variants (vartot) */
#define MEU_MAX_PH 4   /* phases including the matrix (numph) */
#define MEU_MAX_EL 3   /* solutes (numel after Multi_MEUMAPPS.f:153) */
#define MEU_MAX_GP (2 * MEU_MAX_EL + 1) /* rows of Gparams (pmax, :155) */

/* model */
#define MEU_MODEL_KKS 0    /* the reference's KKS model, Multi_MEUMAPPS.f:634-845 */
#define MEU_MODEL_LANDAU 1 /* Landau polynomial in c and eta (configuration decks) */

/* arithmetic of the bulk fields and transforms */
#define MEU_PREC_F64 0 /* plain FP64 everywhere */
#define MEU_PREC_F32 1 /* FP32 fields/FFTs; FP64 for Omega(k), k=0, reductions */

/* elasticity */
#define MEU_ELAST_NONE 0
#define MEU_ELAST_HOMOG 1  /* Landau only: homogeneous moduli, Green operator */
#define MEU_ELAST_HETERO 2 /* eldis fixed-point iteration (KKS always uses it) */

/* flags */
#define MEU_FLAG_GENERIC 1  /* use the generic kernels even where the fused Landau step applies */
#define MEU_FLAG_AUTOTUNE 2 /* time the schedule variants in meu_create and keep the fastest (fused Landau
                             * step; on the generic path the transforms' radix plan and column tile) */

/* Landau eigenstrain coupling theta(eta) */
#define MEU_EIG_ETA2 0 /* theta = eta^2 */
#define MEU_EIG_H 1    /* theta = eta^3 (6 eta^2 - 15 eta + 10) */

/* status codes; 2,3,4,6,20 are the reference's err_flag values (ModFunc.f:55-67,
 * set at Multi_MEUMAPPS.f:690, ModElastic.f:187,270,599, ModInitials.f:98) and 7
 * is the elastic "newfac is too small" stop (ModElastic.f:446-450). */
#define MEU_OK 0
#define MEU_ERR_Z_SINGULAR 2
#define MEU_ERR_Q_SINGULAR 3
#define MEU_ERR_C_SINGULAR 4
#define MEU_ERR_C_ELENER_SINGULAR 6
#define MEU_ERR_NOT_CONVERGED 7
#define MEU_ERR_SETUP_SINGULAR 20
#define MEU_ERR_BADARG 100
#define MEU_ERR_CUDA 101
#define MEU_ERR_NOMEM 102
#define MEU_ERR_UNSUPPORTED 103
#define MEU_ERR_NOT_FINITE 104
#define MEU_ERR_TIMEOUT 105 /* a bounded device-side wait ran out; the call's results are not valid */

/*
 * Parameters consumed by the step (ModGparams.f:59-90 after the setup of
 * Multi_MEUMAPPS.f:153-156,218-236,354-405).  Matrices are stored exactly as
 * the Fortran module holds them (column-major), so a bind(C) copy is a flat
 * assignment:
 *   grad_coeff[v][(j-1)*3+(i-1)] = grad_coeff(i,j,v+1)   (already / del_N**2)
 *   trans_ppt[v][i-1]            = trans_ppt(i,v+1)
 *   cela[n][(j-1)*6+(i-1)]       = CEla(i,j,n+1), sela likewise (SEla)
 *   gparams[n][j-1]              = Gparams(j,n+1)         (after / 1.055e-5)
 */
typedef struct meu_params {
  int64_t step;       /* `step` at entry; incremented once per time step */
  int64_t elastep0;   /* first elastic step (KKS; Landau uses it too) */
  int64_t noise_step; /* phi_noise is kept while step <= noise_step */
  int32_t nx, ny, nz;
  int32_t model;      /* MEU_MODEL_* */
  int32_t precision;  /* MEU_PREC_* */
  int32_t nvar;       /* vartot */
  int32_t numel;      /* solutes E */
  int32_t numph;      /* phases (matrix = 1) */
  int32_t nvar_ph[MEU_MAX_PH]; /* Nvar(1..numph); Nvar(1) = 1 */
  int32_t elastic;      /* MEU_ELAST_* */
  int32_t eig_coupling; /* MEU_EIG_* (Landau) */
  int32_t el_min_iter;  /* 4 in the reference (ModElastic.f:469) */
  int32_t el_max_iter;  /* 10 in the reference (ModElastic.f:462) */
  int32_t clip_phi;     /* 1: clip phi to [0,1] after each step (:1034-1035) */
  int32_t diag_energy;  /* 1: compute the fort.98 energies every step */
  int32_t flags;        /* MEU_FLAG_* */
  double dt;            /* t_step */
  double b_mob;         /* L */
  double cmobs[MEU_MAX_EL]; /* Cmobs = diff_coeff/del_N**2 (M for Landau) */
  double el_tol;        /* 1e-7 in the reference (ModElastic.f:435) */
  double e_mean[6];     /* applied mean strain */
  double grad_coeff[MEU_MAX_VAR][9];
  double trans_ppt[MEU_MAX_VAR][6];
  double cela[MEU_MAX_PH][36];
  double sela[MEU_MAX_PH][36];
  double gparams[MEU_MAX_PH][MEU_MAX_GP];
  double wellph[MEU_MAX_PH];
  /* Landau free energy f = A/2 (c-c1)^2 + B/2 (c2-c) sum eta^2 - C/4 sum eta^4
   * + D/6 sum eta^6 + cross_w sum_{u!=v} eta_u^2 eta_v^2, gradient kappa_c/2 |grad c|^2
   * (kappa_eta enters through grad_coeff, L through b_mob, M through cmobs[0]). */
  double lan_a, lan_b, lan_c, lan_d, lan_c1, lan_c2, kappa_c, cross_w;
} meu_params;

/*
 * One row of per-step diagnostics: the fort.98 line (Multi_MEUMAPPS.f:903-906,
 * format :1113) and the fort.99 line (:1064).  glob_min, glob_max, phi_max and
 * solid are reported as the reference writes them, i.e. the values reduced at
 * the end of the PREVIOUS step (:1057-1062, :891 precede the next write);
 * cmin..solid_now are this step's end-of-step values.
 */
typedef struct meu_diag {
  int64_t step;      /* value of `step` on this fort.98 line */
  int32_t el_iters;  /* elastic fixed-point iterations run in this step */
  int32_t status;
  double fint, fw, fch, elen, etot;
  double glob_min, glob_max, phi_max, solid;
  double cmin, cmax, phimax, solid_now;
  double cavg[MEU_MAX_EL];
} meu_diag;

/* State of the reference's ran_2 (ran_2.f:1-42), whose SAVE variables
 * iv, iy, idum2 become explicit fields.  Initialise with meu_ran2_init. */
typedef struct meu_ran2_state {
  int32_t idum, idum2, iy, iv[32];
} meu_ran2_state;

typedef struct meu_handle meu_handle;

/* Create a step engine on the current CUDA device.  Replaces the per-step
 * state allocation of Multi_MEUMAPPS.f:254-332 and k_space (ModInitials.f:348). */
int meu_create(const meu_params* params, meu_handle** out);

/* Upload fields.  cons: Cons(numel,Nx,Ny,Nz); phi: phi(vartot,Nx,Ny,Nz);
 * u_state: NULL (zero) or 12 consecutive (Nx,Ny,Nz) arrays in the data_save
 * record order u1,u2,u3, grad_1_u1,grad_1_u2,grad_1_u3, grad_2_u1,..,
 * grad_3_u3 (Multi_MEUMAPPS.f:474-480).  Landau: cons holds c, phi holds eta. */
int meu_set_fields(meu_handle* h, const double* cons, const double* phi, const double* u_state);

/* Add a host-generated Langevin increment phi(vartot,Nx,Ny,Nz) to phi_noise
 * (Multi_MEUMAPPS.f:552-566; the generator ran_2/langevin stays on the host). */
int meu_add_noise(meu_handle* h, const double* incr);

/* Run nsteps time steps.  diag: NULL or nsteps rows. */
int meu_run(meu_handle* h, int32_t nsteps, meu_diag* diag);

/* meu_run with the reference's Langevin noise (Multi_MEUMAPPS.f:552-571): every
 * step with step <= noise_step first adds vartot*Nx*Ny*Nz draws langevin(rng, sd)
 * (ModFunc.f:77-100, ran_2.f) to phi_noise, in the reference's loop order
 * (variant index fastest, then x, y, z) -- the same numbers as calling meu_langevin
 * serially and passing them to meu_add_noise before each meu_run(h, 1, ..).  A host
 * thread draws step s+1's increments while step s runs on the GPU; rng ends where
 * the serial draws would leave it.  KKS model only (MEU_ERR_UNSUPPORTED otherwise). */
int meu_run_noise(meu_handle* h, int32_t nsteps, meu_ran2_state* rng, double sd, meu_diag* diag);

/* Download fields (any pointer may be NULL).  u_state as in meu_set_fields. */
int meu_get_fields(meu_handle* h, double* cons, double* phi, double* el_en, double* u_state);

/* Current `step` counter. */
int64_t meu_get_step(const meu_handle* h);

/* Message of the last failing call on this handle (static storage). */
const char* meu_last_error(const meu_handle* h);

int meu_destroy(meu_handle* h);

/* Schedule of a fused Landau handle: out3 = radix plan variant (0: radix 8
 * first, 1: radix 4 first, 2: radix 16 first), threads of the plane kernels,
 * complex columns per column-kernel block.  Handles on the generic path (KKS,
 * heterogeneous or non-cubic Landau) report (radix plan of their power-of-two
 * transforms, 0, column-tile factor 1 or 2); MEU_FLAG_AUTOTUNE picks both by
 * timing at meu_create. */
int meu_schedule(meu_handle* h, int32_t* out3);
/* Choose the schedule (same three values) of a fused Landau handle before its
 * first meu_set_fields; MEU_ERR_UNSUPPORTED if the grid and precision have no
 * such variant (the variants: radix plan 0, 1 or 2, 512 or 256 plane threads,
 * column tile 16 or 8 in FP32, 8 or 4 in FP64 where the tiles fit).  A generic
 * handle takes (0 or 2, 0, 1 or 2) at any time. */
int meu_set_schedule(meu_handle* h, const int32_t* in3);

/* Adjoint. ---------------------------------------------------------------
 * Loss and gradient of the Landau step for calibration.  From the handle's
 * current fields (eta_0, c_0) the call runs nsteps steps (the handle ends at
 * the final state, step counter advanced) and returns
 *   loss = 1/(2 Nx Ny Nz) sum_x [ (eta_T - eta*)^2 + (c_T - c*)^2 ]
 * with its derivatives computed by the hand-written adjoint of the step
 * (checkpoints of the state every checkpoint_every steps, recomputation of
 * each segment in the reverse sweep):
 *   dparams[0] = dJ/dbeta   (grad_coeff of eta scaled by beta, at beta = 1)
 *   dparams[1] = dJ/dkappa_c
 *   dparams[2] = dJ/db_mob  (L)
 *   dparams[3] = dJ/dcmobs[0] (M)
 *   dparams[4] = dJ/dalpha  (every eigenstrain scaled by alpha, at alpha = 1)
 *   dphi0      = dJ/deta_0 (layout as phi; may be NULL)
 * cons_target and phi_target hold c* and eta* (layouts as meu_set_fields).
 * With several order parameters the loss sums (eta_v - eta_v*)^2 over them.
 * Fused Landau handles with 1 to 4 order parameters on the default schedule only
 * (MEU_ERR_UNSUPPORTED otherwise).  The reference has no adjoint. */
int meu_adjoint(meu_handle* h, int32_t nsteps, int32_t checkpoint_every, const double* cons_target,
                const double* phi_target, double* loss, double* dparams, double* dphi0);

/* Ensembles. -------------------------------------------------------------
 * Many independent fused Landau simulations ("members", each a meu_params
 * deck on a cubic grid N in {32,48,64,96,128}, 1-4 variants, eta^2 coupling,
 * homogeneous or no elasticity, one shared precision and start step) advanced
 * together: members of equal (N, nvar, diag_energy) share every kernel launch
 * of a step, the size buckets run concurrently, and runs of whole-ensemble
 * steps replay one CUDA graph.  This batching has no counterpart in the
 * reference, which runs one simulation per MPI job; each member's step is the
 * single-handle step (same results as meu_run on its own handle). */
typedef struct meu_ensemble meu_ensemble;

/* flags for meu_ensemble_create */
#define MEU_ENS_AUTOTUNE 1 /* time the schedule variants of each bucket before any field is set */
/* One persistent launch per run of up to 64 steps: every pass of every member, whatever
 * its grid size, is a work item that the launch's blocks claim in order, each member's
 * passes ordered by a device counter (no grid-wide barrier; every wait is bounded and
 * ends in MEU_ERR_TIMEOUT).  One order parameter per member (MEU_ERR_UNSUPPORTED
 * otherwise); every member runs the schedule (2, 256, 16 FP32 / 8 FP64) and gives the
 * results of a single handle on that schedule.  Overrides MEU_ENS_AUTOTUNE.  The first
 * step after new fields runs as per-bucket launches. */
#define MEU_ENS_PERSISTENT 2

int meu_ensemble_create(int32_t n_members, const meu_params* params, int32_t flags, meu_ensemble** out);
/* fields of one member, layouts as meu_set_fields (no u_state: no heterogeneous elasticity) */
int meu_ensemble_set_fields(meu_ensemble* e, int32_t member, const double* cons, const double* phi);
/* nsteps steps of every member; diag: NULL or n_members * nsteps rows, member-major */
int meu_ensemble_run(meu_ensemble* e, int32_t nsteps, meu_diag* diag);
int meu_ensemble_get_fields(meu_ensemble* e, int32_t member, double* cons, double* phi, double* el_en);
int64_t meu_ensemble_get_step(const meu_ensemble* e);
/* out4 = the member's bucket schedule as meu_schedule, then its bucket index */
int meu_ensemble_schedule(meu_ensemble* e, int32_t member, int32_t* out4);
int meu_ensemble_set_stream(meu_ensemble* e, void* cuda_stream);
int meu_ensemble_timing(meu_ensemble* e, int32_t enable);
int32_t meu_ensemble_timing_report(meu_ensemble* e, int32_t max, char* names, int64_t* counts, double* total_ms,
                                   double* bytes);
int64_t meu_ensemble_launch_count(const meu_ensemble* e);
/* message of the last failing call (e = NULL: of the last failed meu_ensemble_create) */
const char* meu_ensemble_last_error(const meu_ensemble* e);
int meu_ensemble_destroy(meu_ensemble* e);

/* Host-side helpers (no GPU work). ------------------------------------- */

/* ran_2 with the state meu_ran2_state (declared above). */
void meu_ran2_init(meu_ran2_state* s, int32_t iseed);
double meu_ran2(meu_ran2_state* s);
/* langevin (ModFunc.f:77-100): one N(0,sd) draw by the polar method. */
double meu_langevin(meu_ran2_state* s, double sd);
/* n langevin draws into out[0..n-1] (the noise loop of Multi_MEUMAPPS.f:552-566 over
 * ModFunc.f:77-100): the numbers, and the final state of *s, of n meu_langevin calls.  The ran_2 chain and the accept test run on the calling thread;
 * the logarithm and square root of the accepted pairs on up to `threads` host threads. */
int meu_langevin_fill(meu_ran2_state* s, double sd, int64_t n, double* out, int32_t threads);

/* Uniform-noise initial fields for the Landau decks: per voxel in Fortran
 * order (x fastest), c = c0 + c_amp*(2u-1), then for each variant
 * eta_v = eta_amp*(2u-1), u = ran_2 draws.  Layout as meu_set_fields. */
void meu_init_uniform(meu_ran2_state* s, int32_t nx, int32_t ny, int32_t nz, int32_t nvar,
                      double c0, double c_amp, double eta_amp, double* cons, double* phi);

/* Fills *out from the ModGparams state after the set-up of
 * Multi_MEUMAPPS.f:153-417 (the reference's module variables, in their Fortran
 * layout and units: grad_coeff(3,3,vartot) already divided by del_N**2,
 * trans_ppt(6,vartot), CEla/SEla(6,6,numph), Gparams(2*numel+1,numph) after the
 * molar-volume division, Wellph(numph), Cmobs(numel), e_mean(6), Nvar(numph)).
 * The C twin of meu_fill_params in fortran/meu_iface.f90, for drivers written in
 * C or C++: KKS model, plain FP64, heterogeneous elasticity, the reference's
 * iteration controls (4..10 iterations, 1e-7), clipping and energies on.
 * Returns MEU_ERR_BADARG when a size exceeds the MEU_MAX_* limits or a pointer
 * is NULL.  No GPU work. */
int meu_params_from_gparams(int32_t nx, int32_t ny, int32_t nz, int32_t vartot, int32_t numel, int32_t numph,
                            const int32_t* nvar_ph, int64_t step, int64_t elastep0, int64_t noise_step,
                            double t_step, double b_mob, const double* cmobs, const double* e_mean,
                            const double* grad_coeff, const double* trans_ppt, const double* cela,
                            const double* sela, const double* gparams, const double* wellph, meu_params* out);

/* Diagnostics. --------------------------------------------------------- */

/* Launch the handle's work on a caller-owned CUDA stream (cudaStream_t passed
 * as void*; NULL returns to the handle's own stream).  The stream must outlive
 * its use by the handle. */
int meu_set_stream(meu_handle* h, void* cuda_stream);

/* Per-kernel CUDA-event timing: enable = 1 clears and starts it, 0 stops it. */
int meu_timing(meu_handle* h, int32_t enable);

/* Per-kernel timing table: up to max rows of (name[32], launches, total ms,
 * algorithmic bytes = compulsory reads + writes summed over the launches).
 * Returns the number of kernel names (or -status). */
int32_t meu_timing_report(meu_handle* h, int32_t max, char* names, int64_t* counts, double* total_ms,
                          double* bytes);

/* Number of kernels this handle has launched since creation. */
int64_t meu_launch_count(const meu_handle* h);

/* One f_trans / inv_trans pair (ModFunc.f:15-40) of a real (Nx,Ny,Nz) field on
 * the GPU, for transform tests: spec_out receives the scaled half spectrum
 * [z][y][kx] as interleaved re,im doubles (Nz*Ny*(Nx/2+1) complex), back_out
 * the unscaled inverse of that spectrum (equal to the input up to round-off). */
int meu_fft_roundtrip(int32_t nx, int32_t ny, int32_t nz, int32_t precision, const double* in, double* spec_out,
                      double* back_out);

/* Slab-decomposed f_trans / inv_trans over P GPUs, one process per GPU, for grids
 * larger than one GPU holds.  Replaces the P3DFFT decomposition of the reference
 * (Multi_MEUMAPPS.f:124-128 process grid, :241-248 plan; ModFunc.f:15-40 calls) with
 * one all-to-all per transform, which the caller issues (NCCL all-to-all of P equal
 * chunks; meumapps_ss_b200/slab_fft.py does it with torch.distributed).  Rank r holds
 * the real z-planes [r*Nz/P, (r+1)*Nz/P) as [z][y][x] and the spectrum of the ky rows
 * [r*Ny/P, (r+1)*Ny/P) as the "k-slab" [kz][ky][kx] (kx in [0, Nx/2]), in the field
 * precision (float / float2 for MEU_PREC_F32, double / double2 for MEU_PREC_F64).
 * Forward: forward_planes (real slab -> send buffer of P chunks, chunk d for rank d),
 * all-to-all (chunk q from rank q into slot q of the receive buffer, which is the
 * k-slab), forward_columns (in place; the result is scaled by 1/(Nx Ny Nz) like
 * f_trans).  Inverse: inverse_columns (k-slab in place, unscaled; chunk q of it is
 * rank q's), all-to-all, inverse_planes (receive buffer -> real slab).  Device arrays
 * are 16-byte aligned; work is queued on `stream` (a cudaStream_t, NULL = legacy
 * default) and not synchronised.  Ny and Nz are multiples of P; Nx, Ny, Nz, Ny/P and
 * Nz/P are 2^a 3^b (Nx even); otherwise MEU_ERR_UNSUPPORTED / MEU_ERR_BADARG. */
typedef struct meu_slab_fft meu_slab_fft;
int meu_slab_fft_create(int32_t nx, int32_t ny, int32_t nz, int32_t nranks, int32_t rank, int32_t precision,
                        meu_slab_fft** out);
/* out4: real slab elements, complex elements of one chunk, complex elements of the
 * send / receive / k-slab buffers (P chunks), P */
int meu_slab_fft_sizes(const meu_slab_fft* h, int64_t* out4);
int meu_slab_fft_forward_planes(meu_slab_fft* h, const void* real_dev, void* send_dev, void* stream);
int meu_slab_fft_forward_columns(meu_slab_fft* h, void* kslab_dev, void* stream);
int meu_slab_fft_inverse_columns(meu_slab_fft* h, void* kslab_dev, void* stream);
int meu_slab_fft_inverse_planes(meu_slab_fft* h, const void* recv_dev, void* real_dev, void* stream);
int64_t meu_slab_fft_launch_count(const meu_slab_fft* h);
const char* meu_slab_fft_last_error(const meu_slab_fft* h);
int meu_slab_fft_destroy(meu_slab_fft* h);

/* Allocation-free variant of meu_fft_roundtrip.  It has no counterpart in the
 * reference.  For callers that cannot call cudaMalloc: a driver whose device
 * memory belongs to its OpenACC / managed-memory runtime, a framework whose
 * allocator has already reserved the GPU, or code that must not add the device
 * synchronisation of cudaMalloc/cudaFree.  in_dev, spec_dev and back_dev are
 * device-accessible arrays of the caller (device or managed memory), each
 * 16-byte aligned for MEU_PREC_F64 and 8-byte aligned for MEU_PREC_F32 (an
 * array section or an offset into a pool may not be; misaligned arrays return
 * MEU_ERR_BADARG before any work is issued): in_dev holds Nx*Ny*Nz doubles, spec_dev receives 2*Nz*Ny*(Nx/2+1) doubles (the scaled
 * half spectrum, re,im interleaved), back_dev the unscaled inverse (Nx*Ny*Nz
 * doubles).  The library's own working memory is a fixed static device array of
 * about 3.3 MB that every GPU loading the library keeps until exit, so the grid
 * may hold at most MEU_NOALLOC_MAX_POINTS points; larger grids return
 * MEU_ERR_UNSUPPORTED (message in meu_last_error(NULL)).  The first call on a
 * device looks up that array's device address; make that first call before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents (nothing in it needs to start at zero): calls that overlap on the GPU
 * -- from several host threads at once -- race.  Runs on the default stream and
 * is synchronous on return. */
#define MEU_NOALLOC_MAX_POINTS 262144 /* 64^3 */
int meu_fft_roundtrip_noalloc(int32_t nx, int32_t ny, int32_t nz, int32_t precision, const double* in_dev,
                              double* spec_dev, double* back_dev);

#ifdef __cplusplus
}
#endif
#endif /* MEU_H */
