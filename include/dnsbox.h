/* dnsbox.h -- C ABI of libdnsbox_gpu.so, the B200 (sm_100a) pseudospectral
 * Navier-Stokes time step of dnsbox.
 *
 * The reference (DavetheSlayer/dnsbox) exposes its hot path as Fortran module
 * subroutines without arguments acting on module globals.  Each entry point
 * below replaces one of them; the reference routine is cited beside it
 * (file:line in the reference tree).  All pointers named ``*_dev`` are device
 * pointers; ``*_host`` are host pointers.  Every call returns an int status
 * (DNSBOX_OK = 0, negative = DNSBOX_ERR_*); nothing throws across the ABI.
 *
 * Layouts in device memory (the library's own):
 *   spectral field : [nz][ny][nx/2+1] complex, kx fastest; complex double for
 *                    DNSBOX_FP64, complex float for DNSBOX_FP32.
 *   vector field   : three spectral fields back to back (u, v, w).
 *   physical field : [nz][ny][nx] real, x fastest (the reference's (x, y, z)).
 * Transforms are unnormalised both ways, as p3dfft's ftran_r2c / btran_c2r.
 * Host layouts of the upload/download calls are the reference's: complex(8)
 * (kz, ky, kx) with kz fastest (p3dfft STRIDE1) and real(8) (x, y, z).
 *
 * Threading: one context per host thread; calls are asynchronous on the
 * context's stream unless they return host values.
 */
#ifndef DNSBOX_H
#define DNSBOX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DNSBOX_ABI_VERSION 1

enum {
  DNSBOX_OK = 0,
  DNSBOX_ERR_ARG = -1,          /* null pointer or invalid parameter        */
  DNSBOX_ERR_SIZE = -2,         /* grid size not supported                  */
  DNSBOX_ERR_CUDA = -3,         /* CUDA runtime error (see dnsbox_last_error) */
  DNSBOX_ERR_OOM = -4,          /* device allocation failed                 */
  DNSBOX_ERR_NONFINITE = -5,    /* NaN/Inf found by a fused reduction       */
  DNSBOX_ERR_TIMEOUT = -6,      /* a bounded device wait gave up            */
  DNSBOX_ERR_STATE = -7,        /* call order (e.g. no time step set)       */
  DNSBOX_ERR_UNSUPPORTED = -8   /* option not available in this build       */
};

enum dnsbox_precision { DNSBOX_FP64 = 0, DNSBOX_FP32 = 1, DNSBOX_TC_SPLIT = 2 };
/* DNSBOX_SEMI_IMPLICIT: the fixed-point semi-implicit step of
 * dnsboximplicit.f90:88-181 (implicitness implicit_c, parameters.f90:47) */
enum dnsbox_stepper { DNSBOX_HEUN = 0, DNSBOX_AB2 = 1, DNSBOX_SEMI_IMPLICIT = 2 };
/* dnsbox.f90:150-161 literal coefficients (quirk Q2) or standard IF-AB2 */
enum dnsbox_ab2_mode { DNSBOX_AB2_REFERENCE = 0, DNSBOX_AB2_STANDARD = 1 };
/* state.f90:350-411 (MPI build) or single/state.f90:191-230 (quirk Q4) */
enum dnsbox_spectrum_mode { DNSBOX_SPECTRUM_MPI = 0, DNSBOX_SPECTRUM_SINGLE = 1 };
/* rhsAdj.f90:343-348: phatadj := phat (intent) or 0 (literal, quirk Q6) */
enum dnsbox_adj_phat { DNSBOX_ADJ_PHAT_INTENT = 0, DNSBOX_ADJ_PHAT_LITERAL = 1 };

/* Runtime form of the compile-time parameters of parameters.f90:11-50. */
typedef struct dnsbox_params {
  int32_t nx, ny, nz;            /* parameters.f90:12-14                     */
  int32_t precision;             /* enum dnsbox_precision                    */
  int32_t stepper;               /* enum dnsbox_stepper (parameters.f90:44)  */
  int32_t ab2_mode;              /* enum dnsbox_ab2_mode                     */
  int32_t bandlim;               /* parameters.f90:50                        */
  int32_t spherical;             /* parameters.f90:48                        */
  int32_t tstep_fix;             /* parameters.f90:38                        */
  int32_t hminone;               /* parameters.f90:43                        */
  int32_t spectrum_mode;         /* enum dnsbox_spectrum_mode                */
  int32_t adj_phat;              /* enum dnsbox_adj_phat                     */
  int32_t device;                /* CUDA device ordinal                      */
  int32_t nbatch;                /* boxes of this size advanced together (0 or 1: one box) */
  int32_t no_prune;              /* 1: dnsbox_step never prunes the 2/3-rule zeros (default 0: it
                                    prunes when the state vanishes on the cut set; bit-identical) */
  int32_t implicit_max_iter;     /* DNSBOX_SEMI_IMPLICIT: fixed-point iterations per step at most */
  double alpha_x, alpha_y, alpha_z; /* parameters.f90:18-20                  */
  double nu;                     /* parameters.f90:21                        */
  double Q;                      /* parameters.f90:22                        */
  double kCutOff;                /* parameters.f90:23                        */
  double Pin;                    /* parameters.f90:24                        */
  double Deltak;                 /* parameters.f90:27                        */
  double courant_min, courant_max; /* parameters.f90:33-34                   */
  double dt_max;                 /* parameters.f90:35 (tStepMax)             */
  double dt;                     /* initial time step (variables.f90:9)      */
  double implicit_c;             /* parameters.f90:47 (implicitness, 0.5)    */
  double implicit_tol;           /* parameters.f90:26 (tol: sum of the component max |change|
                                    of the spectral iterate, unnormalised)   */
  double reserved_d[2];
} dnsbox_params;

/* Per-step diagnostics (the quantities io_save_stats writes to Ekin.dat,
 * io.f90:628-661, computed on the device every step). */
typedef struct dnsbox_diag {
  double t;                      /* time after the step                      */
  double dt;                     /* step size used                           */
  double ekin;                   /* state_kinetic of the new state           */
  double dissipation;            /* nu <|grad u|^2> of the new state (Parseval) */
  double production_literal;     /* 2 Q Ekin, as io.f90:644                  */
  double injected_power;         /* Pin (band forcing) + 2 Q Ekin            */
  double courant;                /* io_Courant of the step's initial state   */
  double umax[3];                /* max |u_i| of the step's initial state    */
  double eband;                  /* rhs_Eband of the step's initial state    */
  int32_t nonfinite;             /* 1 if a NaN/Inf was seen                  */
  int32_t step;                  /* step counter after the step              */
} dnsbox_diag;

typedef struct dnsbox_ctx dnsbox_ctx;
typedef struct dnsbox_ensemble dnsbox_ensemble;

/* ---- context (replaces var_init, variables.f90:99-280) ------------------ */
void dnsbox_default_params(dnsbox_params *p);
int dnsbox_create(const dnsbox_params *p, dnsbox_ctx **out);
int dnsbox_destroy(dnsbox_ctx *ctx);
int dnsbox_set_stream(dnsbox_ctx *ctx, void *cuda_stream);
const char *dnsbox_last_error(void);
int dnsbox_supported_size(int n);
int dnsbox_abi_version(void);
int dnsbox_field_bytes(const dnsbox_ctx *ctx, size_t *spectral_bytes, size_t *physical_bytes);
int dnsbox_nspec(const dnsbox_ctx *ctx);

/* ---- time step (rhs_int_fact, rhs.f90:8-16; set_time_step,
 *      dnsboxheun.f90:227-246).  The integrating factor is evaluated on the
 *      fly, so setting dt stores it only. -------------------------------- */
int dnsbox_set_dt(dnsbox_ctx *ctx, double dt);
int dnsbox_get_dt(dnsbox_ctx *ctx, double *dt);
int dnsbox_set_time(dnsbox_ctx *ctx, double t);
int dnsbox_get_time(dnsbox_ctx *ctx, double *t);
/* AB2: the next dnsbox_step starts with a predictor-corrector step
 * (dnsbox.f90:87-141). */
int dnsbox_reset_history(dnsbox_ctx *ctx);

/* ---- operators ----------------------------------------------------------- */
/* rhs_nonlinear, rhs.f90:18-135 (+ rhs_Eband, rhs.f90:137-168).
 * uhat3_dev -> nonlin3_dev (may not alias); eband_host may be NULL. */
int dnsbox_rhs_nonlinear(dnsbox_ctx *ctx, const void *uhat3_dev, void *nonlin3_dev,
                         double *eband_host);
/* Integrating-factor Heun (dnsboxheun.f90:85-126), IF-AB2 with a
 * predictor-corrector first step (dnsbox.f90:87-218) or the semi-implicit
 * fixed-point step (dnsboximplicit.f90:88-181), nsteps in place, with CFL
 * control (dnsboxheun.f90:153-157 + io_Courant, io.f90:664-676) unless
 * tstep_fix.  diag_host (nsteps records) may be NULL; when given, the call
 * synchronises the stream before returning.  The semi-implicit step reads the
 * change of every fixed-point iteration back to the host (one
 * synchronisation per iteration); dnsbox_implicit_iterations reports the
 * iterations of the last step. */
int dnsbox_step(dnsbox_ctx *ctx, void *uhat3_dev, int nsteps, dnsbox_diag *diag_host);
/* Fixed-point iterations of the last semi-implicit step (the `iter` counter of
 * dnsboximplicit.f90:127-131), -1 for a null context. */
int dnsbox_implicit_iterations(const dnsbox_ctx *ctx);
/* 1 if the last dnsbox_step call ran the pruned passes (the state vanished on
 * the 2/3-rule cut set, so loads of those zeros and transforms of modes the
 * mask discards were skipped, bit-identically), 0 if it ran the full passes,
 * -1 for a null context.  No reference counterpart. */
int dnsbox_step_pruned(const dnsbox_ctx *ctx);
/* state_project, state.f90:120-179 (in place) */
int dnsbox_project(dnsbox_ctx *ctx, void *uhat3_dev);
/* state_dealias, state.f90:181-209 (in place) */
int dnsbox_dealias(dnsbox_ctx *ctx, void *uhat3_dev);
/* state_spectrum, state.f90:350-411: espec_host has dnsbox_nspec() entries */
int dnsbox_spectrum(dnsbox_ctx *ctx, const void *uhat3_dev, double *espec_host,
                    double *ezero, double *eone, double *esqrt2);
/* state_kinetic, state.f90:429-454 */
int dnsbox_kinetic(dnsbox_ctx *ctx, const void *uhat3_dev, double *ekin);
/* state_dissipation, state.f90:517-544, in its Parseval form */
int dnsbox_dissipation(dnsbox_ctx *ctx, const void *uhat3_dev, double *disp);
/* io_Courant, io.f90:664-676, from the current velocity; umax3 may be NULL */
int dnsbox_courant(dnsbox_ctx *ctx, const void *uhat3_dev, double dt, double *courant,
                   double *umax3);
/* state_divergence, state.f90:413-427 (signed maximum on the grid) */
int dnsbox_divergence(dnsbox_ctx *ctx, const void *uhat3_dev, double *divmax);
/* rhs_Eband, rhs.f90:137-168 */
int dnsbox_eband(dnsbox_ctx *ctx, const void *uhat3_dev, double *eband);

/* ---- transforms: p3dfft_ftran_r2c / p3dfft_btran_c2r (state.f90:58-72),
 *      unnormalised, input not destroyed ------------------------------------ */
int dnsbox_r2c(dnsbox_ctx *ctx, const void *phys_dev, void *spec_dev);
int dnsbox_c2r(dnsbox_ctx *ctx, const void *spec_dev, void *phys_dev);
/* No counterpart in the reference.  dnsbox_c2r for callers that cannot
 * allocate device memory (their memory belongs to a pool they must not bypass,
 * or they run where allocating is not allowed) and so cannot create a context.
 * No context; allocates nothing: the two intermediate fields live in a static
 * 8 MiB device array, so 2 * nz*ny*(nx/2+1) * (16 for DNSBOX_FP64, 8 for
 * DNSBOX_FP32) bytes must fit in 8 MiB (64^3 FP64, 96^3 FP32), else
 * DNSBOX_ERR_SIZE.  Runs on the current device and the given stream.  The first
 * call on a device sets that device up (resolves the arrays' addresses, fills
 * the twiddle tables): make it before any stream capture, and likewise the
 * first call after a cudaDeviceReset, which repeats the set-up.  All calls
 * share the scratch array, so calls that overlap on the GPU race. */
int dnsbox_c2r_noalloc(int nx, int ny, int nz, int precision, const void *spec_dev, void *phys_dev,
                       void *cuda_stream);

/* ---- slab-decomposed 3D FFT over ranks --------------------------------- */
/* p3dfft's one-dimensional decomposition (variables.f90:131-157, processor
 * grid 1 x nranks; p3dfft_ftran_r2c / p3dfft_btran_c2r, dnsbox.f90:44-46,
 * 229-231), one GPU per rank.  Physical slab: (nz/P, ny, nx) reals, z-planes
 * [rank nz/P, (rank+1) nz/P); spectral slab: (nz, ny/P, nx/2+1) complex, ky
 * rows [rank ny/P, (rank+1) ny/P); P = nranks must divide ny and nz.  Each
 * transform is a local half, an all-to-all of P equal blocks that the CALLER
 * runs (block q of every rank's send buffer to rank q, arriving as block r of
 * its recv buffer for sender r; NCCL through torch.distributed in the Python
 * binding), and a finishing half; the library does no communication.  send /
 * recv: P * block_elems complex elements of the precision, device memory.
 * Transforms are unnormalised (as dnsbox_r2c / dnsbox_c2r).  Work runs on
 * `stream` (NULL: the default stream) on the slab's device.
 * Replaces p3dfft_setup / p3dfft_get_dims / p3dfft_ftran_r2c /
 * p3dfft_btran_c2r of the reference's distributed runs. */
typedef struct dnsbox_slab dnsbox_slab;
int dnsbox_slab_create(int nx, int ny, int nz, int nranks, int rank, int precision, int device,
                       dnsbox_slab **out);
void dnsbox_slab_destroy(dnsbox_slab *slab);
/* (z, y, x)-ordered starts and sizes of this rank's physical and spectral
 * slabs (0-based), and the complex elements of one exchange block */
int dnsbox_slab_dims(const dnsbox_slab *slab, int phys_start[3], int phys_size[3], int spec_start[3],
                     int spec_size[3], size_t *block_elems);
/* forward: x R2C and y FFT of the physical slab, packed by destination rank */
int dnsbox_slab_ftran_local(dnsbox_slab *slab, const void *phys_dev, void *send_dev, void *cuda_stream);
/* forward: z FFT of the received blocks into the spectral slab */
int dnsbox_slab_ftran_finish(dnsbox_slab *slab, const void *recv_dev, void *spec_dev, void *cuda_stream);
/* inverse: z FFT of the spectral slab into the send buffer (block q: planes of rank q) */
int dnsbox_slab_btran_local(dnsbox_slab *slab, const void *spec_dev, void *send_dev, void *cuda_stream);
/* inverse: unpack the received ky rows, y FFT and x C2R into the physical slab */
int dnsbox_slab_btran_finish(dnsbox_slab *slab, const void *recv_dev, void *phys_dev, void *cuda_stream);

/* rhs_nonlinear over the slabs (rhs.f90:18-135 with rhs_Eband :137-168): the
 * single-box right-hand side's passes (unpruned) with the exchanges between
 * them, which the caller runs.  uh / out: the spectral ky-slab state and
 * nonlinear term, 3 components of nz * ny/P * (nx/2+1) each.
 *   rhs_begin   band-energy partial (one device double; the caller sums it
 *               over the ranks) and the inverse z pass into send5 (5 fields,
 *               each P blocks as for dnsbox_slab_btran_local);
 *   (one all-to-all per field: 5)
 *   rhs_middle  inverse y, the fused x pass (CFL maxima max|u_i| of the local
 *               planes into umax_dev, 3 device doubles; the caller reduces them
 *               by max) and forward y, packed into send3 (3 fields);
 *   (one all-to-all per field: 3)
 *   rhs_finish  forward z and the finish (2/3 mask, projection, band forcing
 *               with the summed band energy eband_dev) into out.
 * dnsbox_slab_rhs_setup takes the physics from params (nx, ny, nz must be
 * the slab's; precision, stepper and the step-control fields are ignored). */
int dnsbox_slab_rhs_setup(dnsbox_slab *slab, const dnsbox_params *params);
int dnsbox_slab_rhs_begin(dnsbox_slab *slab, const void *uh_dev, double *eband_dev, void *send5_dev,
                          void *cuda_stream);
int dnsbox_slab_rhs_middle(dnsbox_slab *slab, const void *recv5_dev, double *umax_dev, void *send3_dev,
                           void *cuda_stream);
int dnsbox_slab_rhs_finish(dnsbox_slab *slab, const void *recv3_dev, const void *uh_dev, const double *eband_dev,
                           void *out_dev, void *cuda_stream);
/* IF-Heun over the slabs (dnsboxheun.f90:88-126; the caller picks dt, e.g.
 * by set_time_step on the reduced CFL maxima): after rhs_begin / rhs_middle
 * and the exchanges, the finish of the predictor (corrector = 0: out_dev <-
 * u* = IF (u + dt N(u)), uin_dev = u) or of the corrector (corrector = 1:
 * out_dev = u, updated in place to (IF u + u*) / 2 + dt/2 N(u*), uin_dev =
 * u*) replaces rhs_finish.  ed_dev (corrector, or NULL): 2 device doubles,
 * the rank's unscaled (E, D) sums of the new state; summed over the ranks,
 * Ekin = s^2 E and the dissipation nu s^2 D with s = 1/(nx ny nz). */
int dnsbox_slab_heun_finish(dnsbox_slab *slab, const void *recv3_dev, const void *uin_dev, const double *eband_dev,
                            int corrector, double dt, void *out_dev, double *ed_dev, void *cuda_stream);

/* ---- initial conditions on the device ---------------------------------- */
/* state_init_rand, state.f90:211-285 (Yoffe 2012, s. 2.2.5): a random physical
 * field, R2C, state_dealias, state_project, state_spectrum (in the context's
 * spectrum mode) and a rescale of every mode by
 * sqrt(C1 (nk dk)^C2 exp(-C3 (nk dk)^C4) / E(nk)) with C1..C4 of
 * state.f90:218-221 and nk the nearest shell (modes with nk = 0 or
 * nk >= Nspec zeroed).  noise3_dev: the physical random field, [3][nz][ny][nx]
 * reals of the context precision, or NULL to draw it on the device from seed
 * (uniform in [-0.5, 0.5) for all three components; the reference's draw
 * leaves w undrawn, quirk Q7).  Writes the spectral state (the reference then
 * transforms it to physical space, state_uhat2u). */
int dnsbox_init_yoffe(dnsbox_ctx *ctx, const void *noise3_dev, uint64_t seed, void *uhat3_dev);
/* state_init_analytic, state.f90:287-307: the Beltrami (Shapiro) solution at
 * time t, transformed to the spectral state. */
int dnsbox_init_beltrami(dnsbox_ctx *ctx, double t, void *uhat3_dev);
/* dnsboxband.f90:142-143: when on, every step ends with state_project and
 * state_dealias of the new state (the step records then describe the
 * projected state). */
int dnsbox_set_step_projection(dnsbox_ctx *ctx, int on);

/* Device storage for one spectral state (3 fields) in the context's precision,
 * for callers without a CUDA allocator of their own (the Fortran driver's
 * uhat/vhat/what, variables.f90:193-213).  Freed with dnsbox_state_free. */
int dnsbox_state_alloc(dnsbox_ctx *ctx, void **uhat3_dev);
int dnsbox_state_free(dnsbox_ctx *ctx, void *uhat3_dev);

/* ---- host <-> device state (replaces the module arrays uhat/vhat/what and
 *      u/v/w; io.f90:100-278 / 455-626 read and write the physical form) --- */
/* complex(8) (kz, ky, kx), kz fastest, 3 components -> device state */
int dnsbox_upload_state(dnsbox_ctx *ctx, const double *uhat3_host, void *uhat3_dev);
int dnsbox_download_state(dnsbox_ctx *ctx, const void *uhat3_dev, double *uhat3_host);
/* real(8) (x, y, z), 3 components: R2C on upload (state_u2uhat,
 * state.f90:74-80), C2R * scalemodes on download (state_uhat2u, state.f90:82-96) */
int dnsbox_upload_physical(dnsbox_ctx *ctx, const double *u3_host, void *uhat3_dev);
int dnsbox_download_physical(dnsbox_ctx *ctx, const void *uhat3_dev, double *u3_host);

/* ---- adjoint (rhsAdj.f90) --------------------------------------------------- */
/* rhsAdj, rhsAdj.f90:356-381: r~ (rhsupptilde, :177-213) and rhsadj. */
int dnsbox_rhs_adj(dnsbox_ctx *ctx, const void *uhat3_dev, void *rtilde3_dev,
                   void *rhsadj3_dev);
/* Fixed spectral forcing f (3 fields, kept by the caller; NULL clears) added to
 * the nonlinear term of rhs_nonlinear and of every step.  An ensemble keeps
 * the forcing in effect when it was created; the adjoint descent recaptures
 * its graphs when the forcing changes.  No reference
 * counterpart (the reference forces only through Q and the band term); used for
 * the Kolmogorov flow f = (F sin(4y), 0, 0). */
int dnsbox_set_forcing(dnsbox_ctx *ctx, const void *f3_dev);
/* Exact transpose of the linearised rhs_nonlinear at uhat, applied to g
 * (Euclidean inner product on the Re/Im parts of the half spectrum).  No
 * reference counterpart: the reference's rhsNonlinearAdj (rhsAdj.f90:261-354)
 * is its continuous-adjoint analogue. */
int dnsbox_rhs_nonlinear_vjp(dnsbox_ctx *ctx, const void *uhat3_dev, const void *g3_dev,
                             void *out3_dev);
/* J(u) = 1/2 <r, H^-1 r> with r = (nu k.k + Q) uhat + N(uhat) (+ forcing), the
 * residual of rhsupptilde (rhsAdj.f90:177-213) in the physical L2 norm
 * (H^-1 = 1/(1+|k|^2) when hminone, else 1), accumulated in FP64. */
int dnsbox_residual(dnsbox_ctx *ctx, const void *uhat3_dev, double *J);
/* J and its gradient (Euclidean on Re/Im of the half spectrum) through the
 * exact adjoint; the reference's counterpart is the descent direction of
 * dnsboxAdj.f90:76-117. */
int dnsbox_residual_grad(dnsbox_ctx *ctx, const void *uhat3_dev, void *grad3_dev, double *J);
/* niter steepest-descent iterations on J in place (direction -P D W^-1 grad,
 * FP64 Armijo backtracking line search); replaces the pseudo-time Heun loop of
 * dnsboxAdj.f90:76-199.  J_host (niter+1 values) and alpha_io (initial/final
 * step length) may be NULL. */
int dnsbox_adjoint_descent(dnsbox_ctx *ctx, void *uhat3_dev, int niter, double *J_host, double *alpha_io);

/* ---- time-horizon gradients (the periodic-orbit variant of the adjoint
 *      configuration; no reference counterpart: the reference's adjoint
 *      (dnsboxAdj.f90) descends on the instantaneous residual only).  All
 *      three need one box, the Heun stepper and a fixed time step (tstep_fix);
 *      they advance states with dnsbox_step, so the context's clock moves. -- */
/* out = S'(u)^T g for one IF-Heun step S of the current dt (dnsboxheun.f90:85-126
 * linearised at uhat), Euclidean on Re/Im of the half spectrum; out may not
 * alias an input. */
int dnsbox_heun_step_vjp(dnsbox_ctx *ctx, const void *uhat3_dev, const void *g3_dev, void *out3_dev);
/* g0 = (S^nsteps)'(u0)^T gT, with the states recomputed per segment from
 * checkpoints taken every `every` steps (device memory: nsteps/every + every + 2
 * states, held by the context).  uT3_dev (may be NULL) receives u(T). */
int dnsbox_heun_steps_vjp(dnsbox_ctx *ctx, const void *u0_3_dev, int nsteps, int every, const void *gT3_dev,
                          void *g0_3_dev, void *uT3_dev);
/* J = 1/2 <|u(T) - u0|^2> (mean square over the physical grid, FP64) with
 * T = nsteps dt, and, when grad3_dev is not NULL, its gradient
 * ((S^nsteps)'^T - I)(s^2 W r), checkpointed every `every` steps. */
int dnsbox_orbit_residual(dnsbox_ctx *ctx, const void *u0_3_dev, int nsteps, int every, void *grad3_dev,
                          double *J);

/* ---- batched boxes and ensembles (independent boxes of mixed N and nu,
 *      e.g. 96 boxes of 32^3, 64^3 and 96^3; no reference counterpart -- the
 *      reference runs one box per MPI job).  A context created with nbatch > 1 holds nbatch boxes of
 *      one size; its states are component-major, [3][nbatch][nz][ny][nx/2+1],
 *      and dnsbox_step / dnsbox_rhs_nonlinear advance all boxes in the same
 *      launches (box index on the grid's y dimension), each box with its own
 *      dt, clock, band energy, CFL control, diagnostics and viscosity.  The
 *      single-box operators (project, spectrum, transforms, upload/download,
 *      adjoint) return DNSBOX_ERR_UNSUPPORTED on batched contexts. -------- */
int dnsbox_batch_size(const dnsbox_ctx *ctx);
int dnsbox_set_batch_nu(dnsbox_ctx *ctx, const double *nu_host);
/* Step records of the last nrecent steps (nrecent * nbatch records, step
 * major); the device keeps the last 1024 steps. */
int dnsbox_diag_read(dnsbox_ctx *ctx, int nrecent, dnsbox_diag *diag_host);
/* Captures one step of every (context, state) pair into a CUDA graph on the
 * first context's stream (all contexts are switched to it), each context's
 * step an independent branch of the graph (the branches may run
 * concurrently).  Every state is first advanced by one step eagerly, so the
 * captured step is a steady one.  When every state vanishes on its 2/3-rule
 * cut set, a second graph of the pruned passes (as dnsbox_step uses them) is
 * captured beside the full one. */
int dnsbox_ensemble_create(dnsbox_ctx *const *ctxs, void *const *states_dev, int n, dnsbox_ensemble **out);
/* Replays the captured step nsteps times: the pruned graph when it exists and
 * every state still vanishes on its cut set (checked once per call, which
 * waits for the work queued before it on the first context's stream), else
 * the full graph.  The replays themselves are asynchronous. */
int dnsbox_ensemble_run(dnsbox_ensemble *ens, int nsteps);
/* 1 when the last dnsbox_ensemble_run replayed the pruned graph. */
int dnsbox_ensemble_pruned(const dnsbox_ensemble *ens);
int dnsbox_ensemble_destroy(dnsbox_ensemble *ens);

/* ---- kernel schedule and its autotuner ---------------------------------------
 * No reference counterpart as code: the reference leaves transform planning to
 * p3dfft / FFTW (variables.f90:154).  The schedule picks, per tensor-core
 * strided pass of the right-hand side of the tensor-core form, the TMA-staged
 * or the cp.async-fed tensor-core kernel or the FP32 SIMT kernel, and for the
 * fused x pass the block or the warp kernel. */
typedef struct dnsbox_schedule {
  int32_t tc_kernel[4];   /* passes A (inverse z), B (inverse y), D (forward y): 0 TMA-staged tensor-core
                             kernel, 1 cp.async-fed one (the default), 2 FP32 SIMT kernel; [3] pass E1
                             (forward z): 0 SIMT (the default), 1 TMA-staged tensor-core kernel */
  int32_t x_kernel;       /* fused x pass: 0 default for the size, 1 block kernel, 2 warp kernel,
                             3 (N = 256, FP32) warp kernel with each line's fields in registers,
                             4 the same held to 128 registers (four blocks per SM); 3 and 4 run the
                             warp kernel at other sizes */
  int32_t tuned;          /* 1 when chosen by dnsbox_autotune */
  double ms_default;      /* step time of the default schedule in the tuning run (ms) */
  double ms_tuned;        /* step time of the chosen schedule (ms) */
} dnsbox_schedule;
int dnsbox_get_schedule(const dnsbox_ctx *ctx, dnsbox_schedule *out);
int dnsbox_set_schedule(dnsbox_ctx *ctx, const dnsbox_schedule *s);
/* Times every candidate kernel of every pass on nsteps steps of a copy of the
 * state (uhat3_dev is not modified; the context's clock, dt and history are
 * restored; the pass-timing counters are reset), keeps the fastest per pass
 * (never a schedule slower than the default as measured), and caches the
 * choice per device and shape: contexts created later with the same device,
 * precision, grid and box count start with it.  out may be NULL. */
int dnsbox_autotune(dnsbox_ctx *ctx, const void *uhat3_dev, int nsteps, dnsbox_schedule *out);

/* ---- measurement ------------------------------------------------------------
 * No reference counterpart (the reference times nothing; Makefile:3 passes
 * -DMEASURE to p3dfft only).  When enabled, CUDA events are recorded on the
 * context's stream around every kernel launch of the library and summed per
 * pass; the launch counter always runs. */
enum dnsbox_pass {
  DNSBOX_PASS_Z_INV = 0,     /* pass A: inverse z FFT + curl terms           */
  DNSBOX_PASS_Y_INV = 1,     /* pass B: inverse y FFT, vorticity assembly    */
  DNSBOX_PASS_X_NL = 2,      /* pass C: C2R x, u x omega, CFL max, R2C x     */
  DNSBOX_PASS_Y_FWD = 3,     /* pass D: forward y FFT                        */
  DNSBOX_PASS_Z_FIN = 4,     /* pass E2: projection, forcing, stepper, E/D   */
  DNSBOX_PASS_SMALL = 5,     /* band energy, CFL, step bookkeeping           */
  DNSBOX_PASS_OTHER = 6,     /* standalone transforms and diagnostics        */
  DNSBOX_PASS_Z_FWD = 7,     /* pass E1: forward z FFT of the nonlinear term */
  DNSBOX_NPASS = 8
};
typedef struct dnsbox_profile {
  double ms[DNSBOX_NPASS];          /* summed event time per pass (ms)       */
  int64_t launches[DNSBOX_NPASS];   /* kernel launches per pass              */
  int64_t total_launches;           /* all kernel launches since reset       */
} dnsbox_profile;
int dnsbox_profile_enable(dnsbox_ctx *ctx, int on);
/* Waits for the context's stream and reports a device-side failure of the
 * work queued so far: DNSBOX_ERR_TIMEOUT when a tensor-core pass gave up
 * waiting for its MMAs (its output is then invalid).  Entry points that return
 * host values make this check themselves; asynchronous ones (transforms,
 * rhs_nonlinear without eband, step without diagnostics, VJPs) leave it to the
 * next such call or to this one.  No reference counterpart (the reference has
 * no error channel). */
int dnsbox_sync(dnsbox_ctx *ctx);
int dnsbox_profile_read(dnsbox_ctx *ctx, dnsbox_profile *out, int reset);

#ifdef __cplusplus
}
#endif
#endif /* DNSBOX_H */
