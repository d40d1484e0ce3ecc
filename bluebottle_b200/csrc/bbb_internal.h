/* bbb_internal.h -- shared declarations of libbbb200's CUDA layer.
 *
 * Device data layout (HBM):
 *  - Flow fields keep the reference's ghost-padded layouts (Gcc, Gfx, Gfy,
 *    Gfz with one ghost layer, x fastest), so push/pull are plain copies and
 *    the boundary-condition semantics stay identical.
 *  - Krylov vectors are un-ghosted and dense (n = nx*ny*nz for the
 *    pressure, (nx+1)*ny*nz etc. for the Helmholtz components), row length a
 *    multiple of 32 elements at the benchmark sizes, so every warp access is
 *    a full 128-byte line.  Periodic neighbours are found by index wrap.
 *  - The matrix is never stored: one byte per unknown (bbb_mask bits) holds
 *    the six face weights |flag| and the identity-row bit; diagonal and
 *    Jacobi scale are recomputed from it in registers.
 */
#ifndef BBB_INTERNAL_H
#define BBB_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/bluebottle_b200.h"

/* mask bits */
#define BBB_MW 0x01
#define BBB_ME 0x02
#define BBB_MS 0x04
#define BBB_MN 0x08
#define BBB_MB 0x10
#define BBB_MT 0x20
#define BBB_MID 0x40   /* identity row (particle cell / particle face) */

/* one linear system on a dense box nx*ny*nz */
struct bbb_box {
  int nx, ny, nz;
  int perx, pery, perz;     /* periodic wrap along each axis            */
  int dupx, dupy, dupz;     /* the axis carries the duplicated periodic
                               face (Gfx along x etc.): wrap skips it     */
  long long n;
};

/* constant part of a 7-point operator: off-diagonal weight along each axis
 * and the diagonal convention */
struct bbb_op {
  double wx, wy, wz;        /* weight of one face (|flag| = 1)            */
  int helmholtz;            /* 0: Poisson  A = sum w (x_nb - x_c)
                               1: Helmholtz A = x_c + sum w (x_c - x_nb) */
};

/* device-resident scalars of one Krylov solve; kernels read and write them
 * so that no host round trip is needed inside an iteration */
struct bbb_kry {
  double rho, alpha, omega, beta;  /* BiCGSTAB / CG recurrences           */
  double tol;                      /* absolute tolerance rtol*||b||       */
  double bnorm, rnorm;             /* ||b||, latest residual norm         */
  double sumx;                     /* sum of the solution (mean removal)  */
  double t_s, t_t, s_s;            /* (t,s), (t,t), (s,s) of the last K2  */
  double rhv;                      /* (rh, v) of the last BiCGSTAB pass A */
  double rstart;                   /* ||r|| at a residual replacement; a
                                      resumed solve whose ||r|| grows 1e3-
                                      fold past it stops (status -1)      */
  int iter, maxit, done, converged, s_conv, status, first, pad;
  int keep;                        /* 1: no early exit on ||s|| (the inner
                                      solve resumes after its last pass A) */
  int keep_pad;
  unsigned int ticket;             /* last-block election counter         */
};

/* device state of the library (one GPU) */
struct bbb_dev {
  int ready;
  int dev;
  cudaStream_t stream;
  /* ghosted flow fields */
  real *p0, *p, *phi;
  real *u, *v, *w, *u0, *v0, *w0, *us, *vs, *ws;
  real *conv_u, *conv_v, *conv_w, *conv0_u, *conv0_v, *conv0_w;
  real *diff_u, *diff_v, *diff_w, *diff0_u, *diff0_v, *diff0_w;
  int *phase, *phase_shell, *flag_u, *flag_v, *flag_w;
  /* matrix-free operator masks (dense, un-ghosted) */
  uint8_t *mask_p, *mask_u, *mask_v, *mask_w;
  int masks_valid;
  /* Krylov workspace, FP64 (dense; sized for the largest system) */
  long long nmax;
  double *kb, *kx, *kr, *krh, *kp[2], *kv[2], *ks, *kt;
  /* FP32 workspace of the mixed-precision form */
  float *fb, *fx, *fr, *frh, *fp[2], *fv[2], *fs, *ft;
  double *partials;                /* per-block reduction partials       */
  int max_blocks;
  bbb_kry *kry;                    /* device scalars                     */
  bbb_kry *kry_inner;              /* scalars of the FP32 inner solve    */
  bbb_kry *kry_host;               /* pinned mirror                      */
  /* particles */
  int np, stride;
  part_struct *parts;
  real *coef[18];
  real *node_pp, *node_ur, *node_ut, *node_up;   /* nparts*26 each */
  real *perr;                      /* per-particle Lamb error            */
  /* faces whose velocity the particle boundary condition sets: packed
   * (component << 30 | ghosted face index), owning particle, and the
   * face geometry in the particle frame (LF_NGEO arrays of lf_cap) */
  long long lf_cap, lf_n;
  int *lf_idx, *lf_part;
  double *lf_geo;
  unsigned int *lf_count;
  int *lf_pcnt, *lf_pstart, *lf_pfill;   /* faces per particle, list
                                            offsets, fill cursors      */
  int lf_np;                             /* particles they are sized for */
  int lf_valid, lf_geo_valid;
  real *red_host;                  /* pinned scratch for host reductions */
  double *red_dev;                 /* device scratch for small reductions */
  unsigned int *red_ticket;
  long long launches;
};

extern bbb_dev g_dev;

/* grid geometry passed to kernels by value */
struct bbb_geom {
  int nx, ny, nz;
  int cc_s1, cc_s2, fx_s1, fx_s2, fy_s1, fy_s2, fz_s1, fz_s2;
  long long cc_n, fx_n, fy_n, fz_n;          /* ghosted element counts */
  double dx, dy, dz, xs, ys, zs, xe, ye, ze, xl, yl, zl;
};

bbb_geom bbb_make_geom(void);

/* status / error plumbing (bbb_host.c) */
#ifdef __cplusplus
extern "C" {
#endif
void bbb_set_status(int status, const char *where);
void bbb_set_status_at(int status, const char *what, const char *file, int line);
int bbb_fail_exit(void);
extern bbb_options g_opt;
/* >0 while bbb_step runs a Lamb sub-iteration whose pressure solve takes
 * the loosened tolerance g_opt.lamb_pp_tol (bbb_pp_tol) */
extern real g_pp_tol_now;
extern bbb_stats g_stats;
void bbb_record_solver(const char *name, int niter, real resid);
#ifdef __cplusplus
}
#endif

/* relative tolerance of the pressure solve about to run */
static inline real bbb_pp_tol(void) { return g_pp_tol_now > 0 ? g_pp_tol_now : pp_residual; }

#define BBB_CK(call) do { cudaError_t e_ = (call); if(e_ != cudaSuccess) { \
  bbb_set_status_at(BBB_ERR_CUDA, cudaGetErrorString(e_), __FILE__, __LINE__); } } while(0)
#define BBB_LAUNCHED() do { g_dev.launches++; \
  cudaError_t e_ = cudaPeekAtLastError(); if(e_ != cudaSuccess) \
    bbb_set_status_at(BBB_ERR_CUDA, cudaGetErrorString(e_), __FILE__, __LINE__); } while(0)

/* per-launch CUDA-event timing of the solver and RHS kernels while
 * bbb_profile_enable(1) is on (bbb_krylov.cu): the slots, as
 * bbb_profile_get_pass numbers them */
#define BBB_PROF_PASS_A 0         /* BiCGSTAB pass A                       */
#define BBB_PROF_PASS_B 1         /* BiCGSTAB pass B                       */
#define BBB_PROF_OUTER 2          /* FP64 outer residual (defect correction) */
#define BBB_PROF_CG1 3            /* Helmholtz CG stencil pass             */
#define BBB_PROF_CG2 4            /* Helmholtz CG pointwise pass           */
#define BBB_PROF_RHS 5            /* momentum right-hand side              */
void bbb_prof_begin(int slot, double bytes);
void bbb_prof_end(void);

/* entry points between the .cu files */
void bbb_dev_require(void);
void bbb_build_masks(void);
int bbb_poisson_solve(int record);
int bbb_poisson_solve_mixed(int record);
int bbb_helmholtz_solve(int comp);
void bbb_part_BC_fields(real *uu, real *vv, real *ww);
void bbb_star_rhs(int comp_mask, int explicit_ab2);
void bbb_pp_rhs_to_b(void);
double bbb_dev_sum_interior_cc(const real *f);
double bbb_poisson_resid_norm(const double *x);
/* learned initial guess (bbb_learn.cu) */
int bbb_learn_pre_solve(void);
void bbb_learn_post_solve(void);
void bbb_learn_solve_done(double r_final);
void bbb_learn_step_boundary(void);
void bbb_learn_release(void);
void bbb_snapshot_release(void);
void bbb_bins_free(void);

#endif
