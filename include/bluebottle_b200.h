/* bluebottle_b200.h -- C ABI of libbbb200.so.
 *
 * Part 1 is the drop-in boundary: the extern "C" GPU entry points that
 * bluebottle's time loop (src/bluebottle.c:415-450 init, 528-543 pre-loop,
 * 603-708 step) calls.  They take no arguments (or the reference's
 * arguments) and work on the reference's global state, declared in part 2,
 * exactly like the reference's src/cuda_*.cu implementations.  Each comment
 * names the reference prototype it replaces.
 *
 * Part 3 is this library's own extension API: host-side set-up (config files
 * in the reference's format), build-side options that the reference lacks
 * (fixed dt, Taylor-Green start, seeded particle packs, precision mode,
 * learned initial guess), a whole-step driver and solver statistics.
 *
 * Error convention: the reference exits the process when a Krylov solve fails
 * to converge (src/cuda_bicgstab.cu:293-296, 1029-1032).  Here every entry
 * point records a status instead; bbb_last_status() returns it, and the
 * process exits only if bbb_set_exit_on_failure(1) was called (the default
 * matches the reference: 1).
 */
#ifndef BLUEBOTTLE_B200_H
#define BLUEBOTTLE_B200_H

#include "bluebottle_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ===== Part 1: drop-in GPU entry points ================================ */

/* lifecycle -- src/bluebottle.h:2373-2484, src/particle.h:1097-1149 */
void cuda_dom_malloc(void);            /* src/cuda_bluebottle.cu:36   */
void cuda_part_malloc(void);           /* src/cuda_particle.cu:28     */
void cuda_dom_push(void);              /* src/cuda_bluebottle.cu:299  */
void cuda_part_push(void);             /* src/cuda_particle.cu:170    */
void cuda_dom_pull(void);              /* src/cuda_bluebottle.cu:794  */
void cuda_part_pull(void);             /* src/cuda_particle.cu:234    */
void cuda_dom_free(void);              /* src/cuda_bluebottle.cu:1441 */
void cuda_part_free(void);             /* src/cuda_particle.cu        */

/* per-step -- src/bluebottle.h:2492-2943, src/cuda_bicgstab.h:55-141 */
void cuda_compute_forcing(real *pid_int, real *pid_back, real Kp, real Ki,
  real Kd);                            /* src/cuda_bluebottle.cu:3674 */
void cuda_build_cages(void);           /* src/cuda_particle.cu:357    */
void cuda_U_star_2(void);              /* src/cuda_bluebottle.cu:2930 */
void cuda_ustar_helmholtz(int rank);   /* src/cuda_bicgstab.cu:44     */
void cuda_vstar_helmholtz(int rank);   /* src/cuda_bicgstab.cu:319    */
void cuda_wstar_helmholtz(int rank);   /* src/cuda_bicgstab.cu:517    */
void cuda_ustar_rhs(int dev);          /* src/cuda_bicgstab.cu:1091   */
void cuda_vstar_rhs(int dev);          /* src/cuda_bicgstab.cu:1119   */
void cuda_wstar_rhs(int dev);          /* src/cuda_bicgstab.cu:1147   */
void cuda_PP_rhs(int dev);             /* src/cuda_bicgstab.cu:1178   */
void cuda_part_BC(void);               /* src/cuda_particle.cu:899    */
void cuda_part_BC_star(void);          /* src/cuda_particle.cu:947    */
void cuda_part_BC_p(int dev);          /* src/cuda_particle.cu:996    */
void cuda_part_p_fill(void);           /* src/cuda_particle.cu:1019   */
void cuda_dom_BC(void);                /* src/cuda_bluebottle.cu:1549 */
void cuda_dom_BC_star(void);           /* src/cuda_bluebottle.cu:2302 */
void cuda_dom_BC_phi(void);            /* src/cuda_bluebottle.cu:3030 */
void cuda_dom_BC_p(void);              /* src/cuda_bluebottle.cu:3226 */
void cuda_solvability(void);           /* src/cuda_bluebottle.cu:4122 */
void cuda_PP_bicgstab(int rank);       /* src/cuda_bicgstab.cu:715    */
void cuda_project(void);               /* src/cuda_bluebottle.cu:3422 */
void cuda_update_p(void);              /* src/cuda_bluebottle.cu:3616 */
void cuda_move_parts_sub(void);        /* src/cuda_bluebottle.cu:4317 */
void cuda_move_parts(void);            /* src/cuda_bluebottle.cu:4435 */
void cuda_Lamb(void);                  /* src/cuda_quadrature.cu:64   */
real cuda_lamb_err(void);              /* src/cuda_quadrature.cu:316  */
void cuda_parts_internal(void);        /* src/cuda_bluebottle.cu:4822 */
void cuda_store_u(void);               /* src/cuda_bluebottle.cu:3580 */
void cuda_store_coeffs(void);          /* src/cuda_particle.cu:1046   */
real cuda_find_dt(void);               /* src/cuda_bluebottle.cu:3500 */
real cuda_compute_energy(void);        /* src/cuda_bluebottle.cu:3944 */
void cuda_div_U(void);                 /* src/bluebottle.h:2717       */

/* precursor-only symbols that bluebottle.c references; the two-rank
 * turbulence precursor is out of scope, so these are link stubs that record
 * BBB_ERR_UNSUPPORTED -- src/bluebottle.h:2411, 2447, 2877, 2926 */
void cuda_dom_turb_planes_push(int *bc_configs);
void cuda_dom_turb_planes_pull(int *bc_configs);
void cuda_compute_turb_forcing(void);
void cuda_yank_turb_planes(int *bc_flow_configs, real *bc_plane_pos,
  real *vel);

/* ===== Part 2: the reference's global state ============================ */
/* Defined (weakly) inside libbbb200.so; when linked under the reference's
 * bluebottle.c, that file's definitions take precedence.  Names and types
 * follow src/bluebottle.h:364-3329 and src/particle.h. */
extern int dev_start, dev_end, nsubdom;
extern dom_struct *dom;
extern dom_struct Dom;
extern real *p0, *p, *phi;
extern real *u, *u0, *v, *v0, *w, *w0;
extern real *f_x, *f_y, *f_z;
extern real *diff0_u, *diff0_v, *diff0_w;
extern real *conv0_u, *conv0_v, *conv0_w;
extern real *diff_u, *diff_v, *diff_w;
extern real *conv_u, *conv_v, *conv_w;
extern real *u_star, *v_star, *w_star;
extern real duration, ttime, vel_tDelay, p_tDelay, g_tDelay;
extern real dt, dt0, CFL;
extern int pp_max_iter;
extern real pp_residual;
extern int lamb_max_iter;
extern real lamb_residual, lamb_relax, lamb_cut;
extern int out_plane, stepnum, init_cond;
extern g_struct g;
extern real rho_f, mu, nu;
extern BC bc;
extern gradP_struct gradP;
extern long int cpumem, gpumem;
extern real pid_int, pid_back, Kp, Ki, Kd;
/* recorder clocks and precursor plane positions that the restart file
 * carries (src/bluebottle.c:127-182) */
extern int rec_paraview_stepnum_out;
extern real rec_flow_field_ttime_out, rec_paraview_ttime_out,
  rec_particle_ttime_out, rec_restart_ttime_out, rec_prec_ttime_out;
extern real bc_plane_pos[9];
extern int *phase, *phase_shell, *flag_u, *flag_v, *flag_w;
extern int nparts;
extern real interactionLengthRatio;
extern dom_struct binDom;
extern part_struct *parts;
extern int coeff_stride;
extern real *pnm_re, *pnm_im, *phinm_re, *phinm_im, *chinm_re, *chinm_im;
extern real *pnm_re0, *pnm_im0, *phinm_re0, *phinm_im0, *chinm_re0,
  *chinm_im0;
extern real *pnm_re00, *pnm_im00, *phinm_re00, *phinm_im00, *chinm_re00,
  *chinm_im00;

/* ===== Part 3: extension API =========================================== */

/* status codes */
#define BBB_OK 0
#define BBB_ERR_CUDA 1            /* a CUDA call failed                    */
#define BBB_ERR_NOT_CONVERGED 2   /* Krylov solve hit its iteration cap    */
#define BBB_ERR_CONFIG 3          /* bad or missing input file             */
#define BBB_ERR_UNSUPPORTED 4     /* feature outside this library's scope  */
#define BBB_ERR_STATE 5           /* called in the wrong order             */
#define BBB_ERR_DIVERGED 6        /* dt left [1e-10, 1e10] (bluebottle.c:801) */
#define BBB_ERR_TOO_LARGE 7       /* request exceeds a stated size limit   */
#define BBB_ERR_NONFINITE 8       /* NaN/Inf met in a solver residual      */

/* precision forms of the Krylov solves */
#define BBB_PREC_FP64 0           /* plain FP64 BiCGSTAB / CG              */
#define BBB_PREC_MIXED 1          /* FP32 inner solves inside FP64 defect
                                     correction (FP64 outer residual,
                                     dots, norms and accumulation)        */

/* Build-side options.  The reference compiles some of these in (IMPLICIT)
 * and lacks the rest; they live here so the reference's input files stay
 * readable by the reference's own parser. */
typedef struct bbb_options {
  int implicit;            /* 1: Crank-Nicolson + Helmholtz CG (-DIMPLICIT);
                              0: explicit AB2 (cuda_U_star_2)              */
  real fixed_dt;           /* >0: use this dt every step instead of CFL    */
  int precision;           /* BBB_PREC_FP64 or BBB_PREC_MIXED              */
  real inner_tol;          /* mixed form: relative tolerance of each FP32
                              inner solve                                  */
  int max_outer;           /* mixed form: defect-correction sweep cap      */
  int learned_guess;       /* conv-net initial guess of the first Poisson
                              solve of each step, a bit mask: 1 record
                              training crops, 2 use the (gated) guess;
                              applied by bbb_prepare via bbb_learn_enable */
  int record;              /* 1: append solver_expd.rec like the reference */
  int gravity_balance;     /* 1: set gradP.z so the box's net weight is 0  */
  int lamb_max_iter_override; /* >0: replaces lamb_max_iter               */
  int verbose;
  int reliable;            /* mixed form: 1 carries the FP32 BiCGSTAB's
                              Krylov state across the FP64 residual
                              replacements (reliable updates, falling back
                              to a restart on breakdown); 0 restarts it at
                              every sweep                                  */
  int contact_overrun;     /* 1: the sphere/wall contact-list searches run
                              one slot past iSt / St as the reference's
                              collision kernels do (reading and writing the
                              part_struct bytes after those arrays: the low
                              word of e_dry, iSt[0..1]), for byte-for-byte
                              comparison with them; 0 (default): the
                              searches stop at the list's end and a contact
                              that finds no free slot uses its current
                              Stokes number unstored                       */
  real lamb_pp_tol;        /* >0: relative tolerance of the pressure solves
                              of every Lamb sub-iteration but the last
                              (0, the default: pp_residual, as the
                              reference).  A loosened sub-iteration whose
                              coefficient error meets lamb_residual is
                              followed by one more at pp_residual, so a
                              step always ends on a solve to pp_residual  */
} bbb_options;

void bbb_default_options(bbb_options *opt);
void bbb_set_options(const bbb_options *opt);
void bbb_get_options(bbb_options *opt);

/* Host set-up in the reference's input format (restates domain_read_input
 * src/domain.c:30, parts_read_input src/particle.c:79, domain_init
 * src/domain.c:1591, parts_init src/particle.c:295). `dir` holds
 * flow.config and part.config. Return BBB_OK or BBB_ERR_CONFIG. */
int bbb_read_input(const char *dir);
int bbb_domain_init(void);
int bbb_parts_init(void);
/* Replace the particle list by a seeded random pack (the reference's
 * seeder, src/seeder.c:220, made reproducible): n spheres of radius a at
 * uniform non-overlapping centres with surface gap >= min_gap*a (periodic
 * images along the periodic axes included), inside the domain less its
 * screens bc.dsW .. bc.dsT and at least a + min_gap*a/2 from a non-periodic
 * wall; density rho, Lamb order `order`, rs/r = rsr.  Returns BBB_OK or
 * BBB_ERR_CONFIG when the pack cannot be placed. */
int bbb_seed_particles(int n, real a, real min_gap, real rho, int order,
  real rsr, unsigned long long seed);
/* The particle list as the reference's part.config (src/seeder.c:786-815
 * layout, read by src/particle.c:79), numbers to 17 digits; path NULL:
 * ./input/part_seeder.config.  BBB_OK or BBB_ERR_CONFIG. */
int bbb_write_part_config(const char *path);
/* 3-D Taylor-Green start: u = U sin x cos y cos z, v = -U cos x sin y cos z,
 * w = 0 on the staggered faces (domain assumed [0, 2pi)^3 scaled). */
void bbb_init_taylor_green(real U);
void bbb_host_free(void);

/* The reference's restart file (out_restart / in_restart,
 * src/domain.c:3223, :3318): the same bytes from and into the host copies
 * of the state.  path NULL or "" means ./input/restart.config, the
 * reference's fixed name.  The diffusion histories are in the file only
 * when the step is explicit (option implicit = 0), as in a reference built
 * without -DIMPLICIT.  Pull the device state before writing and push it
 * after reading.  Return BBB_OK, BBB_ERR_STATE (no domain set up) or
 * BBB_ERR_CONFIG (the file cannot be opened, is short, or holds another
 * coefficient stride). */
int bbb_out_restart(const char *path);
int bbb_in_restart(const char *path);

/* Device set-up after the host initialisation, in the order of
 * src/bluebottle.c:415-543: cuda_dom_malloc, cuda_part_malloc, the pushes,
 * cuda_build_cages, cuda_part_pull, the initial cuda_find_dt (replaced by
 * the fixed dt when one is set), particle and domain boundary conditions
 * and the rigid-body fill.  bbb_release frees the device state. */
int bbb_prepare(void);
void bbb_release(void);
/* directory that receives solver_expd.rec when options.record is set */
void bbb_set_record_dir(const char *dir);

/* one whole time step of src/bluebottle.c:603-708 (compute_forcing,
 * vel BC ramps, cage build, Lamb sub-iterations, particle update, history
 * store, next dt).  Returns BBB_OK or an error code. */
int bbb_step(void);
/* ttime/dt/stepnum bookkeeping before the step, as bluebottle.c:603-609 */
void bbb_advance_clock(void);

/* solver statistics of the most recent step */
typedef struct bbb_stats {
  int pp_solves;           /* Poisson solves in the step (Lamb iterations) */
  int pp_iters_total;      /* BiCGSTAB iterations summed over those solves */
  int pp_iters_last;       /* iterations of the latest solve               */
  real pp_resid_last;      /* final residual (normalised) of latest solve  */
  int pp_outer_last;       /* defect-correction sweeps of latest solve     */
  int helm_iters_total;    /* CG iterations summed over Helmholtz solves   */
  int lamb_iters;          /* Lamb sub-iterations in the step              */
  real lamb_err;           /* final Lamb coefficient error                 */
  int guess_used;          /* learned guess accepted (1) / rejected (0)    */
  real guess_r0;           /* initial residual norm from the chosen guess  */
  real extrap_r0;          /* initial residual norm of the extrapolation   */
  int guess_evaluated;     /* the guess was computed for this step (1/0)   */
  real guess_cost_ms;      /* device time of that evaluation               */
  real guess_benefit_ms;   /* estimated solve time it saved (cost gate)    */
  real step_dt;            /* dt the step advanced by                      */
  real cfl_adv;            /* step_dt * (max u / dx + max v / dy + max w /
                              dz) of the velocity the step ended with: the
                              advective CFL number cuda_find_dt bounds     */
  int helm_solves;         /* Helmholtz (CG) solves in the step            */
  int pp_iters_max;        /* most iterations of one Poisson solve         */
  int pp_iters_first;      /* iterations of the step's first Poisson solve
                              (the one the learned guess may start)        */
} bbb_stats;
void bbb_get_stats(bbb_stats *st);

int bbb_last_status(void);
const char *bbb_status_string(int status);
void bbb_clear_status(void);
void bbb_set_exit_on_failure(int on);

/* device diagnostics */
int bbb_device_count(void);
/* divergence of (u, v, w) over the interior cells: max |div| and the
 * L2 norm; computed on the device from the current fields */
void bbb_divergence(real *max_abs, real *l2);

/* kernel launch counter (this library's kernels only), for benchmarks */
long long bbb_kernel_launches(void);
void bbb_reset_kernel_launches(void);

/* Live timing of the solver and right-hand-side kernels, by CUDA events
 * on the library's stream around each launch, over the launches that did
 * work while enabled (launches that returned at once after a solve had
 * converged are left out).  bbb_profile_get: the BiCGSTAB iterations'
 * total milliseconds, iteration count and algorithmic bytes (15 vector
 * words + 2 mask bytes per unknown and iteration; 14 words in the passes
 * staged by tensor-map copies, whose pass B stores no s).  bbb_profile_get_pass:
 * milliseconds, launches and algorithmic bytes of one kernel kind --
 * 0: BiCGSTAB pass A (the p/v update and first stencil), 1: pass B (the
 * s/t update and second stencil), 2: the FP64 outer residual of the mixed
 * form, 3: the Helmholtz CG stencil pass, 4: its pointwise pass, 5: the
 * momentum right-hand side. */
void bbb_profile_enable(int on);
void bbb_profile_reset(void);
void bbb_profile_get(double *ms, long long *iters, double *bytes);
void bbb_profile_get_pass(int pass, double *ms, long long *launches,
  double *bytes);

/* Shared-memory stage layout of one tensor-map-staged solver pass as
 * compiled (no counterpart in the reference; a diagnostic for host-side
 * checks of the copies and reads, no GPU needed).  fp64: 0 or 1; pass: 0
 * BiCGSTAB pass A, 1 pass B, 2 the FP64 outer residual (fp64 = 1 only), 3
 * the Helmholtz CG stencil pass.  Writes BBB_STAGE_LAYOUT_N ints, in
 * bytes unless named otherwise: element size, 16-byte chunk in elements,
 * halo arrays, own arrays, rows per warp, tile rows, warps, threads, box
 * width (elements), box rows, box row pitch, own row bytes, wrap-row
 * offset, halo array region, mask row pitch, mask wrap-row offset, mask
 * region, mask offset, own-array offset, x-wrap offset, x-wrap bytes per
 * array, stage, stages, dynamic shared memory per block, armed bytes of
 * the boxes, of one x side, of one y side, resident blocks the register
 * budget targets.  Returns BBB_STAGE_LAYOUT_N, or -1 for an unknown pass
 * or a short buffer. */
#define BBB_STAGE_LAYOUT_N 28
int bbb_stage_layout(int fp64, int pass, int *out, int nout);

/* Copy only the particle records (part_struct array) between the host
 * `parts` and the device: the per-step exchange of a caller that moves
 * particle state, without the phase/flag arrays cuda_part_push/pull also
 * carry. */
void bbb_part_state_push(void);
void bbb_part_state_pull(void);

/* Asynchronous output snapshot of the fields the reference's writers read
 * (out_VTK, src/vtk.c:48; cgns_flow_field / cgns_particles,
 * src/recorder.c:487-1890): u, v, w, p, phase and parts.  The reference
 * pulls them with a blocking cuda_dom_pull / cuda_part_pull before every
 * output (src/bluebottle.c:717-760).  bbb_snapshot_start copies them on the
 * device after the step and moves the copy to pinned host staging on a
 * stream of its own while the following steps run; bbb_snapshot_finish
 * waits for that transfer and writes the snapshot into the host arrays
 * (the state at the start call, whatever steps ran since).  One snapshot
 * at a time: a second start before the finish, or a finish without a
 * start, returns BBB_ERR_STATE.  The first start allocates the device copy
 * and the pinned staging (about twice the six fields); cuda_dom_free
 * releases them.  bbb_snapshot_busy: 1 between start and finish. */
int bbb_snapshot_start(void);
int bbb_snapshot_finish(void);
int bbb_snapshot_busy(void);

/* CUDA-event time marks (0..7) on the library's stream; elapsed waits for
 * mark b and returns milliseconds between marks a and b (-1 on error) */
void bbb_mark(int i);
double bbb_mark_elapsed(int a, int b);

/* Learned initial guess of the pressure-Poisson solve.  No counterpart in
 * the reference, which starts each solve from the previous correction phi
 * (src/cuda_bicgstab.cu:971-979).  A 4-layer 3x3x3 convolutional net (16
 * channels, GELU, BF16 tensor-core convolutions with FP32 accumulation)
 * predicts a correction to that extrapolation from (b, phi_prev, p0, solid
 * mask); the first solve of each step starts from it when its FP64
 * residual is below the extrapolation's (counted in bbb_stats.guess_used,
 * with both initial residuals in guess_r0 / extrap_r0).
 *   bbb_learn_enable(mode): bit 1 record crops of (features, converged
 *     correction) at the first solve of each step; bit 2 use the guess;
 *     bit 4 gate the evaluation on its cost: the evaluation and the solve
 *     after it are timed on the device, and while the guess's estimated
 *     saving (bbb_stats.guess_benefit_ms) stays below its cost
 *     (guess_cost_ms) it is evaluated only every 8, 16, .. 256 steps.
 *   bbb_learn_gate_decide: that decision as a pure host function (steps
 *     to skip; *fails counts consecutive evaluations that did not pay).
 *   bbb_learn_train(iters, lr): Adam steps on batches of 8 recorded crops;
 *     returns the relative MSE of the last batch (-1 without crops).
 *   bbb_learn_get/set_params: FP32 weights [layer][tap][cout][cin] then
 *     biases [layer][cout], bbb_learn_param_count() floats.
 *   bbb_learn_forward: the net on a caller's device box of features
 *     (channels-last BF16, 16 channels) into FP32 out; ref = 1 runs the
 *     FP32 CUDA-core convolution instead of the tensor cores.
 *   bbb_learn_use_reference_conv(on): route every convolution (inference
 *     and training) through the FP32 CUDA-core kernels. */
int bbb_learn_enable(int mode);
int bbb_learn_gate_decide(double t_guess_ms, double t_solve_ms, double r_ext,
  double r_start, double r_final, int *fails, double *benefit_ms);
double bbb_learn_train(int iters, double lr);
int bbb_learn_crops(void);
int bbb_learn_param_count(void);
int bbb_learn_get_params(float *host, int n);
int bbb_learn_set_params(const float *host, int n);
int bbb_learn_forward(int nx, int ny, int nz, int px, int py, int pz,
  const void *feat_d, float *out_d, int ref);
/* loss and gradient (no update) on a caller's device batch of nb crops of
 * cx*cy*cz cells stacked along z (features as above, FP32 targets), MSE
 * over cells at least `margin` from crop faces; grad_host receives
 * bbb_learn_param_count() floats.  Returns the MSE, -1 on failure. */
double bbb_learn_grad(int cx, int cy, int cz, int nb, int margin,
  const void *feat_d, const float *tgt_d, float *grad_host);
void bbb_learn_use_reference_conv(int on);
/* crops (128 x 32 x 32 cells, or the box where smaller) recorded at each
 * recorded solve, 1..64 (8 by default); BBB_ERR_CONFIG outside that */
int bbb_learn_set_crops_per_step(int n);

/* Allocation-free pressure-Poisson solve.  No counterpart in the
 * reference: it is the FP64 solve of cuda_PP_bicgstab for callers that
 * cannot allocate device memory (a host application whose pool allocator
 * owns all GPU memory, or a time-critical loop that cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree).  It calls no
 * cudaMalloc, cudaFree or allocating library routine.
 *   - Inputs and output are device pointers in the reference's ghosted
 *     layouts: u_star/v_star/w_star (Gfx/Gfy/Gfz), phase and flag_u/v/w,
 *     and phi, read as the initial guess and overwritten on the interior
 *     with the mean-free solution (its ghosts are left to the caller's
 *     boundary-condition pass, as with cuda_PP_bicgstab).
 *   - Scratch lives in one file-scope device array of about 22 MB, held by
 *     every GPU that loads the library until the process exits; it limits
 *     the grid to nx*ny*nz <= 64^3 cells, and larger requests return
 *     BBB_ERR_TOO_LARGE.
 *   - The first call on a device looks up that array's device address
 *     (with that device current; host threads calling for the first time
 *     together take one look-up); make that first call before any stream
 *     capture.
 *   - Every call shares the array and it keeps the last call's contents:
 *     calls that overlap on the GPU (other streams, other host threads)
 *     race and must be serialised by the caller.
 * perx/pery/perz select periodic wrap per axis; tol is the relative
 * residual ||b - A x|| <= tol ||b||.  Returns BBB_OK,
 * BBB_ERR_NOT_CONVERGED, BBB_ERR_NONFINITE, BBB_ERR_TOO_LARGE,
 * BBB_ERR_CONFIG or BBB_ERR_CUDA; iters/resid (may be NULL) receive the
 * iteration count and the final relative residual.  `stream` is a
 * cudaStream_t (NULL for the default stream); the call returns after the
 * solve has finished on it. */
int bbb_PP_bicgstab_static(int nx, int ny, int nz, double dx, double dy,
  double dz, int perx, int pery, int perz, const double *u_star,
  const double *v_star, const double *w_star, const int *phase,
  const int *flag_u, const int *flag_v, const int *flag_w, double rho_f,
  double dt, double tol, int maxit, double *phi, int *iters, double *resid,
  void *stream);

#ifdef __cplusplus
}
#endif
#endif
