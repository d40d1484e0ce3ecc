/* orc.h -- CPU FP64 oracle for the bluebottle per-time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C99 + OpenMP restatement of the
 * reference's algorithm, used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg as the result to check against.  The product library
 * (libbbb200.so) never links, loads or calls it.
 *
 * Every routine names the reference file:line it restates.  The arrays use
 * the reference's host layouts: ghost-padded, x fastest, C = i + j*s1b +
 * k*s2b with DOM_BUF = 1 (src/domain.c:1612-1725).  The Krylov solvers hold
 * the operator as the reference's 13-diagonal DIA matrix
 * (src/cuda_bicgstab.cu:729-806, src/bicgstab_kernel.cu:643-1856), built the
 * way the reference builds it, so that the GPU's matrix-free operator is
 * checked against an independent representation.
 *
 * The CUSP solvers the reference calls (krylov::bicgstab, krylov::cg,
 * precond::diagonal, monitor) are not vendored in the reference; they are
 * restated here from the published algorithms (van der Vorst's BiCGSTAB in
 * the right-preconditioned form CUSP uses, and preconditioned CG) with CUSP's
 * stopping rule ||r|| <= tol*||b|| on the ||b||-normalised system
 * (src/cuda_bicgstab.cu:996-1018).
 */
#ifndef ORC_H
#define ORC_H

#include "../include/bluebottle_b200_types.h"

typedef struct orc_params {
  real rho_f, nu, mu;
  real dt, dt0, ttime, CFL;
  int pp_max_iter;
  real pp_residual;
  int lamb_max_iter;
  real lamb_residual, lamb_relax, lamb_cut;
  int out_plane;
  int implicit;               /* 1: CN + Helmholtz CG, 0: explicit AB2 */
  real fixed_dt;              /* >0: constant dt                       */
  real vel_tDelay, p_tDelay, g_tDelay;
  real Kp, Ki, Kd, pid_int, pid_back;
  real interactionLengthRatio;
  BC bc;
  g_struct g;
  gradP_struct gradP;
  int stepnum;
  int contact_overrun;        /* 1: contact-list searches reach slot 12 as
                                 the reference's kernels do (option
                                 contact_overrun of the library)          */
} orc_params;

typedef struct orc_state {
  dom_struct dom;
  orc_params P;
  real *p0, *p, *phi;
  real *u, *v, *w, *u0, *v0, *w0;
  real *u_star, *v_star, *w_star;
  real *conv_u, *conv_v, *conv_w, *conv0_u, *conv0_v, *conv0_w;
  real *diff_u, *diff_v, *diff_w, *diff0_u, *diff0_v, *diff0_w;
  int *phase, *phase_shell, *flag_u, *flag_v, *flag_w;
  real *rhs_p;                /* un-ghosted Gcc.s3 */
  int nparts, coeff_stride;
  part_struct *parts;
  /* Lamb coefficients: [0..5] = pnm_re, pnm_im, phinm_re, phinm_im,
   * chinm_re, chinm_im; [6..11] the same "0" copies; [12..17] "00" */
  real *coef[18];
  /* statistics */
  int pp_iters, pp_converged, pp_solves, pp_iters_total;
  real pp_resid;
  int cg_iters[3], cg_converged[3];
  real cg_resid[3];
  int lamb_iters;
  real lamb_err;
} orc_state;

/* lifecycle */
orc_state *orc_create(const dom_struct *dom, int nparts, int coeff_stride);
void orc_destroy(orc_state *st);
/* pointer to a named array and its element count (see orc_fluid.c) */
void *orc_field(orc_state *st, const char *name, long *count);
orc_params *orc_params_ptr(orc_state *st);
void orc_get_stats(orc_state *st, int *iv, real *rv);
int orc_set_threads(int n);

/* boundary conditions: which = 0 (u,v,w,p), 1 (u*,v*,w*), 2 (phi), 3 (p) */
void orc_dom_BC(orc_state *st, int which);
void orc_compute_forcing(orc_state *st);
void orc_compute_vel_BC(orc_state *st);

/* fluid */
void orc_U_star_2(orc_state *st);
void orc_star_rhs(orc_state *st, int comp);
void orc_star_helmholtz(orc_state *st, int comp);
void orc_solvability(orc_state *st);
void orc_PP_rhs(orc_state *st);
void orc_PP_bicgstab(orc_state *st);
void orc_project(orc_state *st);
void orc_update_p(orc_state *st);
void orc_store_u(orc_state *st);
real orc_find_dt(orc_state *st);
real orc_compute_energy(orc_state *st);
void orc_divergence(orc_state *st, const real *uu, const real *vv,
  const real *ww, real *max_abs, real *l2);

/* operators for tests: apply the Poisson DIA matrix to an un-ghosted x */
void orc_poisson_apply(orc_state *st, const real *x, real *y);
/* solve the Poisson DIA system A x = b (un-ghosted) with the reference's
 * scaled Jacobi-BiCGSTAB; x holds the initial guess on entry */
int orc_poisson_solve(orc_state *st, const real *b, real *x, real tol,
  int maxit, real *resid);

/* particles */
void orc_build_cages(orc_state *st);
void orc_part_BC(orc_state *st, int star);
void orc_part_BC_p(orc_state *st);
void orc_part_p_fill(orc_state *st);
void orc_parts_internal(orc_state *st);
void orc_Lamb(orc_state *st);
real orc_lamb_err(orc_state *st);
void orc_store_coeffs(orc_state *st);
void orc_move_parts_sub(orc_state *st);
void orc_move_parts(orc_state *st);
void orc_quad_nodes(real *node_t, real *node_p, real *A1, real *A2,
  real *A3);

/* one whole step of src/bluebottle.c:603-708 */
int orc_step(orc_state *st);

#endif
