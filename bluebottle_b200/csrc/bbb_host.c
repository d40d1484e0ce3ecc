/* bbb_host.c -- host side of libbbb200: the reference's global state,
 * options and status, readers for the reference's input files, domain and
 * particle initialisation, a seeded particle packer, and the time-step
 * driver.  Plain C99; the GPU work is behind the cuda_* entry points.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../include/bluebottle_b200.h"

#define WEAK __attribute__((weak))

/* ------------------------------------------------ reference globals
 * Declared in src/bluebottle.h and src/particle.h, defined in
 * src/bluebottle.c:29-187 and src/particle.c:25-77.  Weak here so that the
 * reference's own definitions win when it links this library. */
WEAK int dev_start, dev_end, nsubdom;
WEAK dom_struct *dom;
WEAK dom_struct Dom;
WEAK real *p0, *p, *phi;
WEAK real *u, *u0, *v, *v0, *w, *w0;
WEAK real *f_x, *f_y, *f_z;
WEAK real *diff0_u, *diff0_v, *diff0_w;
WEAK real *conv0_u, *conv0_v, *conv0_w;
WEAK real *diff_u, *diff_v, *diff_w;
WEAK real *conv_u, *conv_v, *conv_w;
WEAK real *u_star, *v_star, *w_star;
WEAK real duration, ttime, vel_tDelay, p_tDelay, g_tDelay;
WEAK real dt, dt0, CFL;
WEAK int pp_max_iter;
WEAK real pp_residual;
real g_pp_tol_now = 0.;
WEAK int lamb_max_iter;
WEAK real lamb_residual, lamb_relax, lamb_cut;
WEAK int out_plane, stepnum, init_cond;
WEAK g_struct g;
WEAK real rho_f, mu, nu;
WEAK BC bc;
WEAK gradP_struct gradP;
WEAK long int cpumem, gpumem;
WEAK real pid_int, pid_back, Kp, Ki, Kd;
WEAK int *phase, *phase_shell, *flag_u, *flag_v, *flag_w;
WEAK int nparts;
WEAK real interactionLengthRatio;
WEAK dom_struct binDom;
WEAK part_struct *parts;
WEAK int coeff_stride;
WEAK real *pnm_re, *pnm_im, *phinm_re, *phinm_im, *chinm_re, *chinm_im;
WEAK real *pnm_re0, *pnm_im0, *phinm_re0, *phinm_im0, *chinm_re0, *chinm_im0;
WEAK real *pnm_re00, *pnm_im00, *phinm_re00, *phinm_im00, *chinm_re00,
  *chinm_im00;

/* ------------------------------------------------ options and status */
bbb_options g_opt;
bbb_stats g_stats;
static int g_status = BBB_OK;
static int g_exit_on_failure = 1;
static int g_opt_init = 0;
static char g_record_dir[1024] = "record";

void bbb_default_options(bbb_options *opt)
{
  memset(opt, 0, sizeof(*opt));
  opt->implicit = 1;
  opt->fixed_dt = 0.;
  opt->precision = BBB_PREC_FP64;
  opt->inner_tol = 1e-4;
  opt->max_outer = 20;
  opt->learned_guess = 0;
  opt->record = 0;
  opt->gravity_balance = 0;
  opt->lamb_max_iter_override = 0;
  opt->verbose = 0;
  opt->reliable = 0;
  opt->contact_overrun = 0;
  opt->lamb_pp_tol = 0.;
}

static void opt_init(void)
{
  if(!g_opt_init) { bbb_default_options(&g_opt); g_opt_init = 1; }
}

void bbb_set_options(const bbb_options *opt) { g_opt = *opt; g_opt_init = 1; }
void bbb_get_options(bbb_options *opt) { opt_init(); *opt = g_opt; }
void bbb_get_stats(bbb_stats *st) { *st = g_stats; }
int bbb_last_status(void) { return g_status; }
void bbb_clear_status(void) { g_status = BBB_OK; }
void bbb_set_exit_on_failure(int on) { g_exit_on_failure = on; }

const char *bbb_status_string(int s)
{
  switch(s) {
    case BBB_OK: return "ok";
    case BBB_ERR_CUDA: return "CUDA call failed";
    case BBB_ERR_NOT_CONVERGED: return "Krylov solve did not converge";
    case BBB_ERR_CONFIG: return "bad or missing input";
    case BBB_ERR_UNSUPPORTED: return "unsupported feature";
    case BBB_ERR_STATE: return "called in the wrong order";
    case BBB_ERR_DIVERGED: return "time step left [1e-10, 1e10]";
    case BBB_ERR_TOO_LARGE: return "size exceeds the stated limit";
    case BBB_ERR_NONFINITE: return "non-finite solver residual";
  }
  return "unknown status";
}

void bbb_set_status(int status, const char *where)
{
  if(status == BBB_OK) return;
  if(g_status == BBB_OK) g_status = status;
  if(g_opt.verbose || status == BBB_ERR_CUDA)
    fprintf(stderr, "bluebottle_b200: %s (%s)\n", bbb_status_string(status),
      where ? where : "");
}

/* as bbb_set_status, naming the source line of the failed call */
void bbb_set_status_at(int status, const char *what, const char *file, int line)
{
  char buf[256];
  const char *base = strrchr(file, '/');
  snprintf(buf, sizeof(buf), "%s at %s:%d", what ? what : "", base ? base + 1 : file, line);
  bbb_set_status(status, buf);
}

int bbb_fail_exit(void) { return g_exit_on_failure; }

/* record/solver_*.rec, the format of src/recorder.c:1891-1953 */
void bbb_record_solver(const char *name, int niter, real resid)
{
  opt_init();
  if(!g_opt.record) return;
  char path[1200];
  snprintf(path, sizeof(path), "%s/%s", g_record_dir, name);
  FILE *rec = fopen(path, "r+");
  if(rec == NULL) {
    rec = fopen(path, "w");
    if(rec == NULL) return;
    fprintf(rec, "%-12s", "stepnum");
    fprintf(rec, "%-15s", "ttime");
    fprintf(rec, "%-15s", "dt");
    fprintf(rec, "%-8s", "niter");
    fprintf(rec, "%-15s", "resid");
  }
  fseek(rec, 0, SEEK_END);
  fprintf(rec, "\n");
  fprintf(rec, "%-12d", stepnum);
  fprintf(rec, "%-15e", ttime);
  fprintf(rec, "%-15e", dt);
  fprintf(rec, "%-8d", niter);
  fprintf(rec, "%-15e", resid);
  fclose(rec);
}

void bbb_set_record_dir(const char *dir)
{
  snprintf(g_record_dir, sizeof(g_record_dir), "%s", dir);
}

/* ------------------------------------------------ input readers
 * The grammar is the reference's strict-order format: flow.config as read
 * by domain_read_input (src/domain.c:30-730) and part.config as read by
 * parts_read_input (src/particle.c:79-159). */

static int rd(FILE *f, const char *fmt, void *a, void *b, void *c, int want)
{
  int n = fscanf(f, fmt, a, b, c);
  return n == want;
}

static int read_pressure_bc(FILE *f, const char *key, int *type, real *ds)
{
  char fmt[64], buf[64];
  snprintf(fmt, sizeof(fmt), "%s %%63s", key);
  if(fscanf(f, fmt, buf) != 1) return 0;
  if(strcmp(buf, "PERIODIC") == 0) { *type = BBB_PERIODIC; *ds = 0; }
  else if(strcmp(buf, "NEUMANN") == 0) {
    *type = BBB_NEUMANN;
    if(fscanf(f, "%lf", ds) != 1) return 0;
  } else return 0;
  if(fscanf(f, "\n") < 0) return 0;
  return 1;
}

static int read_vel_bc(FILE *f, const char *key, int *type, real *Dm,
  real *D, real *Da)
{
  char fmt[64], buf[64];
  snprintf(fmt, sizeof(fmt), "%s %%63s", key);
  if(fscanf(f, fmt, buf) != 1) return 0;
  if(strcmp(buf, "PERIODIC") == 0) *type = BBB_PERIODIC;
  else if(strcmp(buf, "DIRICHLET") == 0 || strcmp(buf, "PRECURSOR") == 0) {
    *type = strcmp(buf, "DIRICHLET") == 0 ? BBB_DIRICHLET : BBB_PRECURSOR;
    if(fscanf(f, "%lf %lf", Dm, Da) != 2) return 0;
    *D = 0;
  } else if(strcmp(buf, "NEUMANN") == 0) {
    *type = BBB_NEUMANN; *Dm = 0; *Da = 0; *D = 0;
  } else return 0;
  if(fscanf(f, "\n") < 0) return 0;
  return 1;
}

static FILE *open_in(const char *dir, const char *name)
{
  char path[2048];
  snprintf(path, sizeof(path), "%s/%s", dir, name);
  return fopen(path, "r");
}

static int read_flow(const char *dir)
{
  FILE *f = open_in(dir, "flow.config");
  if(!f) return 0;
  char buf[64];
  int ok = 1;
  ok &= fscanf(f, "DOMAIN\n") >= 0;
  ok &= rd(f, "(Xs, Xe, Xn) %lf %lf %d\n", &Dom.xs, &Dom.xe, &Dom.xn, 3);
  ok &= rd(f, "(Ys, Ye, Yn) %lf %lf %d\n", &Dom.ys, &Dom.ye, &Dom.yn, 3);
  ok &= rd(f, "(Zs, Ze, Zn) %lf %lf %d\n", &Dom.zs, &Dom.ze, &Dom.zn, 3);
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "GPU DOMAIN DECOMPOSITION\n") >= 0;
  ok &= rd(f, "DEV RANGE %d %d\n", &dev_start, &dev_end, NULL, 2);
  ok &= rd(f, "n %d\n", &nsubdom, NULL, NULL, 1);
  if(!ok || nsubdom < 1) { fclose(f); return 0; }
  free(dom);
  dom = (dom_struct *)calloc((size_t)nsubdom, sizeof(dom_struct));
  for(int i = 0; i < nsubdom; i++) {
    ok &= rd(f, "(Xs, Xe, Xn) %lf %lf %d\n", &dom[i].xs, &dom[i].xe, &dom[i].xn, 3);
    ok &= rd(f, "(Ys, Ye, Yn) %lf %lf %d\n", &dom[i].ys, &dom[i].ye, &dom[i].yn, 3);
    ok &= rd(f, "(Zs, Ze, Zn) %lf %lf %d\n", &dom[i].zs, &dom[i].ze, &dom[i].zn, 3);
    int e, w_, n_, s, t, b;
    ok &= fscanf(f, "E %d W %d N %d S %d T %d B %d\n", &e, &w_, &n_, &s, &t, &b) == 6;
    dom[i].E = e; dom[i].W = w_; dom[i].N = n_; dom[i].S = s; dom[i].T = t; dom[i].B = b;
  }
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "PHYSICAL PARAMETERS\n") >= 0;
  ok &= rd(f, "rho_f %lf\n", &rho_f, NULL, NULL, 1);
  ok &= rd(f, "nu %lf\n", &nu, NULL, NULL, 1);
  mu = nu * rho_f;
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "SIMULATION PARAMETERS\n") >= 0;
  ok &= rd(f, "duration %lf\n", &duration, NULL, NULL, 1);
  ok &= rd(f, "CFL %lf\n", &CFL, NULL, NULL, 1);
  ok &= rd(f, "pp_max_iter %d\n", &pp_max_iter, NULL, NULL, 1);
  ok &= rd(f, "pp_residual %lf\n", &pp_residual, NULL, NULL, 1);
  ok &= rd(f, "lamb_max_iter %d\n", &lamb_max_iter, NULL, NULL, 1);
  ok &= rd(f, "lamb_residual %lf\n", &lamb_residual, NULL, NULL, 1);
  ok &= rd(f, "lamb_relax %lf\n", &lamb_relax, NULL, NULL, 1);
  ok &= rd(f, "lamb_cut %lf\n", &lamb_cut, NULL, NULL, 1);
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "BOUNDARY CONDITIONS\n") >= 0;
  ok &= rd(f, "vel_tDelay %lf\n", &vel_tDelay, NULL, NULL, 1);
  ok &= fscanf(f, "PRESSURE\n") >= 0;
  ok &= read_pressure_bc(f, "bc.pW", &bc.pW, &bc.dsW);
  ok &= read_pressure_bc(f, "bc.pE", &bc.pE, &bc.dsE);
  ok &= read_pressure_bc(f, "bc.pS", &bc.pS, &bc.dsS);
  ok &= read_pressure_bc(f, "bc.pN", &bc.pN, &bc.dsN);
  ok &= read_pressure_bc(f, "bc.pB", &bc.pB, &bc.dsB);
  ok &= read_pressure_bc(f, "bc.pT", &bc.pT, &bc.dsT);
  ok &= fscanf(f, "X-VELOCITY\n") >= 0;
  ok &= read_vel_bc(f, "bc.uW", &bc.uW, &bc.uWDm, &bc.uWD, &bc.uWDa);
  ok &= read_vel_bc(f, "bc.uE", &bc.uE, &bc.uEDm, &bc.uED, &bc.uEDa);
  ok &= read_vel_bc(f, "bc.uS", &bc.uS, &bc.uSDm, &bc.uSD, &bc.uSDa);
  ok &= read_vel_bc(f, "bc.uN", &bc.uN, &bc.uNDm, &bc.uND, &bc.uNDa);
  ok &= read_vel_bc(f, "bc.uB", &bc.uB, &bc.uBDm, &bc.uBD, &bc.uBDa);
  ok &= read_vel_bc(f, "bc.uT", &bc.uT, &bc.uTDm, &bc.uTD, &bc.uTDa);
  ok &= fscanf(f, "Y-VELOCITY\n") >= 0;
  ok &= read_vel_bc(f, "bc.vW", &bc.vW, &bc.vWDm, &bc.vWD, &bc.vWDa);
  ok &= read_vel_bc(f, "bc.vE", &bc.vE, &bc.vEDm, &bc.vED, &bc.vEDa);
  ok &= read_vel_bc(f, "bc.vS", &bc.vS, &bc.vSDm, &bc.vSD, &bc.vSDa);
  ok &= read_vel_bc(f, "bc.vN", &bc.vN, &bc.vNDm, &bc.vND, &bc.vNDa);
  ok &= read_vel_bc(f, "bc.vB", &bc.vB, &bc.vBDm, &bc.vBD, &bc.vBDa);
  ok &= read_vel_bc(f, "bc.vT", &bc.vT, &bc.vTDm, &bc.vTD, &bc.vTDa);
  ok &= fscanf(f, "Z-VELOCITY\n") >= 0;
  ok &= read_vel_bc(f, "bc.wW", &bc.wW, &bc.wWDm, &bc.wWD, &bc.wWDa);
  ok &= read_vel_bc(f, "bc.wE", &bc.wE, &bc.wEDm, &bc.wED, &bc.wEDa);
  ok &= read_vel_bc(f, "bc.wS", &bc.wS, &bc.wSDm, &bc.wSD, &bc.wSDa);
  ok &= read_vel_bc(f, "bc.wN", &bc.wN, &bc.wNDm, &bc.wND, &bc.wNDa);
  ok &= read_vel_bc(f, "bc.wB", &bc.wB, &bc.wBDm, &bc.wBD, &bc.wBDa);
  ok &= read_vel_bc(f, "bc.wT", &bc.wT, &bc.wTDm, &bc.wTD, &bc.wTDa);
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "INITIAL CONDITION\n") >= 0;
  ok &= fscanf(f, "init_cond %63s", buf) == 1;
  if(strcmp(buf, "QUIESCENT") == 0) init_cond = BBB_QUIESCENT;
  else if(strcmp(buf, "SHEAR") == 0) init_cond = BBB_SHEAR;
  else if(strcmp(buf, "CHANNEL") == 0) init_cond = BBB_CHANNEL;
  else ok = 0;
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "SOLVABILITY ENFORCEMENT PLANE\n") >= 0;
  ok &= fscanf(f, "out_plane %63s", buf) == 1;
  if(strcmp(buf, "WEST") == 0) out_plane = BBB_WEST;
  else if(strcmp(buf, "EAST") == 0) out_plane = BBB_EAST;
  else if(strcmp(buf, "SOUTH") == 0) out_plane = BBB_SOUTH;
  else if(strcmp(buf, "NORTH") == 0) out_plane = BBB_NORTH;
  else if(strcmp(buf, "BOTTOM") == 0) out_plane = BBB_BOTTOM;
  else if(strcmp(buf, "TOP") == 0) out_plane = BBB_TOP;
  else if(strcmp(buf, "HOMOGENEOUS") == 0) out_plane = BBB_HOMOGENEOUS;
  else ok = 0;
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "SIMULATION DRIVING CONDITIONS\n") >= 0;
  ok &= rd(f, "p_tDelay %lf\n", &p_tDelay, NULL, NULL, 1);
  ok &= rd(f, "gradP.x %lf %lf\n", &gradP.xm, &gradP.xa, NULL, 2);
  gradP.x = 0;
  ok &= rd(f, "gradP.y %lf %lf\n", &gradP.ym, &gradP.ya, NULL, 2);
  gradP.y = 0;
  ok &= rd(f, "gradP.z %lf %lf\n", &gradP.zm, &gradP.za, NULL, 2);
  gradP.z = 0;
  ok &= rd(f, "g_tDelay %lf\n", &g_tDelay, NULL, NULL, 1);
  ok &= rd(f, "g.x %lf %lf\n", &g.xm, &g.xa, NULL, 2);
  g.x = 0;
  ok &= rd(f, "g.y %lf %lf\n", &g.ym, &g.ya, NULL, 2);
  g.y = 0;
  ok &= rd(f, "g.z %lf %lf\n", &g.zm, &g.za, NULL, 2);
  g.z = 0;
  ok &= fscanf(f, "\n") >= 0;
  ok &= fscanf(f, "PID CONTROLLER GAINS\n") >= 0;
  ok &= rd(f, "Kp %lf\n", &Kp, NULL, NULL, 1);
  ok &= rd(f, "Ki %lf\n", &Ki, NULL, NULL, 1);
  ok &= rd(f, "Kd %lf\n", &Kd, NULL, NULL, 1);
  fclose(f);
  return ok;
}

static int read_parts(const char *dir)
{
  FILE *f = open_in(dir, "part.config");
  if(!f) { nparts = 0; return 1; }   /* no particle file: no particles */
  int ok = 1;
  ok &= rd(f, "n %d\n", &nparts, NULL, NULL, 1);
  if(!ok || nparts < 0) { fclose(f); return 0; }
  free(parts);
  parts = (part_struct *)calloc((size_t)(nparts > 0 ? nparts : 1),
    sizeof(part_struct));
  ok &= rd(f, "(l/a) %lf\n", &interactionLengthRatio, NULL, NULL, 1);
  for(int i = 0; i < nparts && ok; i++) {
    part_struct *q = &parts[i];
    ok &= fscanf(f, "\n") >= 0;
    ok &= rd(f, "r %lf\n", &q->r, NULL, NULL, 1);
    ok &= rd(f, "(x, y, z) %lf %lf %lf\n", &q->x, &q->y, &q->z, 3);
    ok &= rd(f, "(aFx, aFy, aFz) %lf %lf %lf\n", &q->aFx, &q->aFy, &q->aFz, 3);
    ok &= rd(f, "(aLx, aLy, aLz) %lf %lf %lf\n", &q->aLx, &q->aLy, &q->aLz, 3);
    ok &= rd(f, "rho %lf\n", &q->rho, NULL, NULL, 1);
    ok &= rd(f, "E %lf\n", &q->E, NULL, NULL, 1);
    ok &= rd(f, "sigma %lf\n", &q->sigma, NULL, NULL, 1);
    ok &= rd(f, "e_dry %lf\n", &q->e_dry, NULL, NULL, 1);
    ok &= rd(f, "coeff_fric %lf\n", &q->coeff_fric, NULL, NULL, 1);
    ok &= rd(f, "order %d\n", &q->order, NULL, NULL, 1);
    ok &= rd(f, "rs/r %lf\n", &q->rs, NULL, NULL, 1);
    ok &= rd(f, "spring_k %lf\n", &q->spring_k, NULL, NULL, 1);
    ok &= rd(f, "spring (x, y, z) %lf %lf %lf\n", &q->spring_x, &q->spring_y,
      &q->spring_z, 3);
    ok &= rd(f, "spring_l %lf\n", &q->spring_l, NULL, NULL, 1);
    ok &= rd(f, "translating %d\n", &q->translating, NULL, NULL, 1);
    ok &= rd(f, "rotating %d\n", &q->rotating, NULL, NULL, 1);
  }
  fclose(f);
  return ok;
}

int bbb_read_input(const char *dir)
{
  opt_init();
  if(!read_flow(dir)) {
    bbb_set_status(BBB_ERR_CONFIG, "flow.config");
    return BBB_ERR_CONFIG;
  }
  if(!read_parts(dir)) {
    bbb_set_status(BBB_ERR_CONFIG, "part.config");
    return BBB_ERR_CONFIG;
  }
  if(nsubdom != 1) {
    bbb_set_status(BBB_ERR_UNSUPPORTED, "one GPU subdomain only");
    return BBB_ERR_UNSUPPORTED;
  }
  return BBB_OK;
}

/* ------------------------------------------------ domain initialisation
 * src/domain.c:1591-2347: grid_info index spaces (one ghost layer), the
 * host field arrays, QUIESCENT / SHEAR / CHANNEL starts and the initial
 * dt. */
static void set_grid(grid_info *G, int nx, int ny, int nz, int local)
{
  G->is = BBB_DOM_BUF; G->isb = G->is - BBB_DOM_BUF; G->in = nx;
  G->inb = G->in + 2 * BBB_DOM_BUF; G->ie = G->is + G->in; G->ieb = G->ie + BBB_DOM_BUF;
  G->js = BBB_DOM_BUF; G->jsb = G->js - BBB_DOM_BUF; G->jn = ny;
  G->jnb = G->jn + 2 * BBB_DOM_BUF; G->je = G->js + G->jn; G->jeb = G->je + BBB_DOM_BUF;
  G->ks = BBB_DOM_BUF; G->ksb = G->ks - BBB_DOM_BUF; G->kn = nz;
  G->knb = G->kn + 2 * BBB_DOM_BUF; G->ke = G->ks + G->kn; G->keb = G->ke + BBB_DOM_BUF;
  G->s1 = G->in; G->s2 = G->s1 * G->jn; G->s3 = G->s2 * G->kn;
  G->s1b = G->inb; G->s2b = G->s1b * G->jnb; G->s3b = G->s2b * G->knb;
  /* the subdomain's own (underscored) indices are filled for dom[] only,
   * as src/domain.c:1777 does; with one subdomain they equal the global */
  if(!local) return;
  G->_is = G->is; G->_ie = G->ie; G->_in = G->in; G->_isb = G->isb;
  G->_ieb = G->ieb; G->_inb = G->inb;
  G->_js = G->js; G->_je = G->je; G->_jn = G->jn; G->_jsb = G->jsb;
  G->_jeb = G->jeb; G->_jnb = G->jnb;
  G->_ks = G->ks; G->_ke = G->ke; G->_kn = G->kn; G->_ksb = G->ksb;
  G->_keb = G->keb; G->_knb = G->knb;
  G->_s1 = G->s1; G->_s1b = G->s1b; G->_s2 = G->s2; G->_s2b = G->s2b;
  G->_s3 = G->s3; G->_s3b = G->s3b;
}

static void setup_dom(dom_struct *d, int local)
{
  d->xl = d->xe - d->xs; d->yl = d->ye - d->ys; d->zl = d->ze - d->zs;
  d->dx = d->xl / d->xn; d->dy = d->yl / d->yn; d->dz = d->zl / d->zn;
  set_grid(&d->Gcc, d->xn, d->yn, d->zn, local);
  set_grid(&d->Gfx, d->xn + 1, d->yn, d->zn, local);
  set_grid(&d->Gfy, d->xn, d->yn + 1, d->zn, local);
  set_grid(&d->Gfz, d->xn, d->yn, d->zn + 1, local);
}

static real *zalloc(long n)
{
  return (real *)calloc((size_t)(n > 0 ? n : 1), sizeof(real));
}

static void free_fields(void)
{
  real **fs[] = {&p0, &p, &phi, &u, &v, &w, &u0, &v0, &w0, &diff0_u,
    &diff0_v, &diff0_w, &conv0_u, &conv0_v, &conv0_w, &diff_u, &diff_v,
    &diff_w, &conv_u, &conv_v, &conv_w, &u_star, &v_star, &w_star, &f_x,
    &f_y, &f_z};
  for(size_t a = 0; a < sizeof(fs) / sizeof(fs[0]); a++) {
    free(*fs[a]); *fs[a] = NULL;
  }
}

int bbb_domain_init(void)
{
  opt_init();
  if(!dom || nsubdom != 1) {
    bbb_set_status(BBB_ERR_STATE, "bbb_domain_init before bbb_read_input");
    return BBB_ERR_STATE;
  }
  setup_dom(&Dom, 0);
  setup_dom(&dom[0], 1);
  free_fields();
  long ncc = Dom.Gcc.s3b, nfx = Dom.Gfx.s3b, nfy = Dom.Gfy.s3b,
       nfz = Dom.Gfz.s3b;
  p0 = zalloc(ncc); p = zalloc(ncc); phi = zalloc(ncc);
  u = zalloc(nfx); v = zalloc(nfy); w = zalloc(nfz);
  u0 = zalloc(nfx); v0 = zalloc(nfy); w0 = zalloc(nfz);
  diff0_u = zalloc(nfx); diff0_v = zalloc(nfy); diff0_w = zalloc(nfz);
  conv0_u = zalloc(nfx); conv0_v = zalloc(nfy); conv0_w = zalloc(nfz);
  diff_u = zalloc(nfx); diff_v = zalloc(nfy); diff_w = zalloc(nfz);
  conv_u = zalloc(nfx); conv_v = zalloc(nfy); conv_w = zalloc(nfz);
  u_star = zalloc(nfx); v_star = zalloc(nfy); w_star = zalloc(nfz);
  f_x = zalloc(nfx); f_y = zalloc(nfy); f_z = zalloc(nfz);
  cpumem += (long)sizeof(real) * (3 * ncc + 9 * (nfx + nfy + nfz));

  if(init_cond == BBB_SHEAR) {
    const grid_info *G = &Dom.Gfx;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real y = ((j - 0.5) * Dom.dy) + Dom.ys, z = ((k - 0.5) * Dom.dz) + Dom.zs;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      u[C] = (bc.uNDm - bc.uSDm) * (y - Dom.ys) / Dom.yl + bc.uSDm;
      u[C] += (bc.uTDm - bc.uBDm) * (z - Dom.zs) / Dom.zl + bc.uBDm;
      u0[C] = u[C];
    }
    G = &Dom.Gfy;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real x = ((i - 0.5) * Dom.dx) + Dom.xs, z = ((k - 0.5) * Dom.dz) + Dom.zs;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      v[C] = (bc.vEDm - bc.vWDm) * (x - Dom.xs) / Dom.xl + bc.vWDm;
      /* the reference divides by ze here (src/domain.c:2225) */
      v[C] += (bc.vTDm - bc.vBDm) * (z - Dom.zs) / Dom.ze + bc.vBDm;
      v0[C] = v[C];
    }
    G = &Dom.Gfz;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real x = ((i - 0.5) * Dom.dx) + Dom.xs, y = ((j - 0.5) * Dom.dy) + Dom.ys;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      w[C] = (bc.wEDm - bc.wWDm) * (x - Dom.xs) / Dom.xl + bc.wWDm;
      w[C] += (bc.wNDm - bc.wSDm) * (y - Dom.ys) / Dom.yl + bc.wSDm;
      w0[C] = w[C];
    }
  } else if(init_cond == BBB_CHANNEL) {
    const grid_info *G = &Dom.Gfx;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real y = ((j - 0.5) * Dom.dy) + Dom.ys, z = ((k - 0.5) * Dom.dz) + Dom.zs;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      u[C] = 0.5 / mu * gradP.xm * (y * y - (Dom.ys + Dom.ye) * y + Dom.ys * Dom.ye)
        * (bc.uS == BBB_DIRICHLET)
        + 0.5 / mu * gradP.xm * (z * z - (Dom.zs + Dom.ze) * z + Dom.zs * Dom.ze)
        * (bc.uB == BBB_DIRICHLET);
      u0[C] = u[C];
    }
    G = &Dom.Gfy;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real x = ((i - 0.5) * Dom.dx) + Dom.xs, z = ((k - 0.5) * Dom.dz) + Dom.zs;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      v[C] = 0.5 / mu * gradP.ym * (x * x - (Dom.xs + Dom.xe) * x + Dom.xs * Dom.xe)
        * (bc.vW == BBB_DIRICHLET)
        + 0.5 / mu * gradP.ym * (z * z - (Dom.zs + Dom.ze) * z + Dom.zs * Dom.ze)
        * (bc.vB == BBB_DIRICHLET);
      v0[C] = v[C];
    }
    G = &Dom.Gfz;
    for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
    for(int i = G->isb; i < G->ieb; i++) {
      real x = ((i - 0.5) * Dom.dx) + Dom.xs, y = ((j - 0.5) * Dom.dy) + Dom.ys;
      long C = i + (long)j * G->s1b + (long)k * G->s2b;
      w[C] = 0.5 / mu * gradP.zm * (x * x - (Dom.xs + Dom.xe) * x + Dom.xs * Dom.xe)
        * (bc.wW == BBB_DIRICHLET)
        + 0.5 / mu * gradP.zm * (y * y - (Dom.ys + Dom.ye) * y + Dom.ys * Dom.ye)
        * (bc.wS == BBB_DIRICHLET);
      w0[C] = w[C];
    }
  }
  real dx_min = Dom.dx;
  if(Dom.dy < dx_min) dx_min = Dom.dy;
  if(Dom.dz < dx_min) dx_min = Dom.dz;
  dt = 2. * nu / (dx_min * dx_min);
  dt += 2. * nu / (Dom.dy * Dom.dy);
  dt += 2. * nu / (Dom.dz * Dom.dz);
  dt = CFL / dt;
  dt0 = -1.;
  stepnum = 0;
  ttime = 0.;
  if(g_opt.fixed_dt > 0) dt = g_opt.fixed_dt;
  return BBB_OK;
}

void bbb_init_taylor_green(real U)
{
  /* positions as in the staggered layout: u on x-faces at x = (i-1) dx,
   * y = (j-0.5) dy, z = (k-0.5) dz (ghosted indices), and alike for v */
  const grid_info *G = &Dom.Gfx;
  for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
  for(int i = G->isb; i < G->ieb; i++) {
    real x = (i - 1) * Dom.dx + Dom.xs, y = (j - 0.5) * Dom.dy + Dom.ys,
         z = (k - 0.5) * Dom.dz + Dom.zs;
    long C = i + (long)j * G->s1b + (long)k * G->s2b;
    u[C] = U * sin(x) * cos(y) * cos(z);
    u0[C] = u[C];
  }
  G = &Dom.Gfy;
  for(int k = G->ksb; k < G->keb; k++) for(int j = G->jsb; j < G->jeb; j++)
  for(int i = G->isb; i < G->ieb; i++) {
    real x = (i - 0.5) * Dom.dx + Dom.xs, y = (j - 1) * Dom.dy + Dom.ys,
         z = (k - 0.5) * Dom.dz + Dom.zs;
    long C = i + (long)j * G->s1b + (long)k * G->s2b;
    v[C] = -U * cos(x) * sin(y) * cos(z);
    v0[C] = v[C];
  }
  G = &Dom.Gfz;
  for(long c = 0; c < G->s3b; c++) { w[c] = 0.; w0[c] = 0.; }
  init_cond = BBB_TAYLOR_GREEN;
}

/* ------------------------------------------------ particle initialisation
 * src/particle.c:295-535 */
static void free_parts_arrays(void)
{
  real **cs[] = {&pnm_re, &pnm_im, &phinm_re, &phinm_im, &chinm_re,
    &chinm_im, &pnm_re0, &pnm_im0, &phinm_re0, &phinm_im0, &chinm_re0,
    &chinm_im0, &pnm_re00, &pnm_im00, &phinm_re00, &phinm_im00, &chinm_re00,
    &chinm_im00};
  for(size_t a = 0; a < sizeof(cs) / sizeof(cs[0]); a++) { free(*cs[a]); *cs[a] = NULL; }
  free(phase); free(phase_shell); free(flag_u); free(flag_v); free(flag_w);
  phase = phase_shell = flag_u = flag_v = flag_w = NULL;
}

/* the collision bin grid (binDom_init, src/particle.c:598): bins of at
 * least 2 a_max + ratio a_max per side, cell-centred indices only */
static void bin_dom_init(void)
{
  real rmax = 0;
  for(int i = 0; i < nparts; i++)
    rmax = rmax + (parts[i].r > rmax) * (parts[i].r - rmax);
  memset(&binDom, 0, sizeof(binDom));
  real span = 2. * rmax + interactionLengthRatio * rmax;
  binDom.xs = Dom.xs; binDom.xe = Dom.xe; binDom.xl = Dom.xl;
  binDom.xn = (int)floor(Dom.xl / span);
  if(binDom.xn == 0) { binDom.xn = 1; binDom.dx = Dom.xl; }
  else binDom.dx = Dom.xl / binDom.xn;
  binDom.ys = Dom.ys; binDom.ye = Dom.ye; binDom.yl = Dom.yl;
  binDom.yn = (int)floor(Dom.yl / span);
  if(binDom.yn == 0) { binDom.yn = 1; binDom.dy = Dom.yl; }
  else binDom.dy = Dom.yl / binDom.yn;
  binDom.zs = Dom.zs; binDom.ze = Dom.ze; binDom.zl = Dom.zl;
  binDom.zn = (int)floor(Dom.zl / span);
  if(binDom.zn == 0) { binDom.zn = 1; binDom.dz = Dom.zl; }
  else binDom.dz = Dom.zl / binDom.zn;
  grid_info *G = &binDom.Gcc;
  G->is = BBB_DOM_BUF; G->in = binDom.xn; G->ie = G->is + G->in;
  G->js = BBB_DOM_BUF; G->jn = binDom.yn; G->je = G->js + G->jn;
  G->ks = BBB_DOM_BUF; G->kn = binDom.zn; G->ke = BBB_DOM_BUF + G->kn;
  G->s1 = G->in; G->s2 = G->s1 * G->jn; G->s3 = G->s2 * G->kn;
}

int bbb_parts_init(void)
{
  free_parts_arrays();
  long ncc = Dom.Gcc.s3b;
  phase = (int *)malloc(sizeof(int) * (size_t)ncc);
  phase_shell = (int *)malloc(sizeof(int) * (size_t)ncc);
  flag_u = (int *)malloc(sizeof(int) * (size_t)Dom.Gfx.s3b);
  flag_v = (int *)malloc(sizeof(int) * (size_t)Dom.Gfy.s3b);
  flag_w = (int *)malloc(sizeof(int) * (size_t)Dom.Gfz.s3b);
  for(long c = 0; c < ncc; c++) { phase[c] = -1; phase_shell[c] = 1; }
  for(long c = 0; c < Dom.Gfx.s3b; c++) flag_u[c] = 1;
  for(long c = 0; c < Dom.Gfy.s3b; c++) flag_v[c] = 1;
  for(long c = 0; c < Dom.Gfz.s3b; c++) flag_w[c] = 1;
  coeff_stride = 0;
  for(int i = 0; i < nparts; i++) {
    part_struct *q = &parts[i];
    memset(&q->cage, 0, sizeof(q->cage));
    q->rs = q->rs * q->r;
    q->ncoeff = 0;
    for(int j = 0; j <= q->order; j++) q->ncoeff += j + 1;
    q->x0 = q->x; q->y0 = q->y; q->z0 = q->z;
    q->u = q->v = q->w = 0.; q->u0 = q->v0 = q->w0 = 0.;
    q->udot = q->vdot = q->wdot = 0.; q->udot0 = q->vdot0 = q->wdot0 = 0.;
    q->axx = 1.; q->axy = 0.; q->axz = 0.;
    q->ayx = 0.; q->ayy = 1.; q->ayz = 0.;
    q->azx = 0.; q->azy = 0.; q->azz = 1.;
    q->ox = q->oy = q->oz = 0.; q->ox0 = q->oy0 = q->oz0 = 0.;
    q->oxdot = q->oydot = q->ozdot = 0.; q->oxdot0 = q->oydot0 = q->ozdot0 = 0.;
    if(init_cond == BBB_SHEAR) {
      if(q->translating) {
        q->u = (bc.uNDm - bc.uSDm) * (q->y - Dom.ys) / Dom.yl + bc.uSDm;
        q->u += (bc.uTDm - bc.uBDm) * (q->z - Dom.zs) / Dom.zl + bc.uBDm;
        q->u0 = q->u;
        q->v = (bc.vEDm - bc.vWDm) * (q->x - Dom.xs) / Dom.xl + bc.vWDm;
        q->v += (bc.vTDm - bc.vBDm) * (q->z - Dom.zs) / Dom.zl + bc.vBDm;
        q->v0 = q->v;
        q->w = (bc.wEDm - bc.wWDm) * (q->x - Dom.xs) / Dom.xl + bc.wWDm;
        q->w += (bc.wNDm - bc.wSDm) * (q->y - Dom.ys) / Dom.yl + bc.wSDm;
        q->w0 = q->w;
        q->x0 = q->x - dt * q->u; q->y0 = q->y - dt * q->v; q->z0 = q->z - dt * q->w;
      }
      if(q->rotating) {
        q->ox = -0.5 * (bc.vTDm - bc.vBDm) / Dom.zl;
        q->ox += 0.5 * (bc.wNDm - bc.wSDm) / Dom.yl;
        q->oy = 0.5 * (bc.uTDm - bc.uBDm) / Dom.zl;
        q->oy += -0.5 * (bc.wEDm - bc.wWDm) / Dom.xl;
        q->oz = -0.5 * (bc.uNDm - bc.uSDm) / Dom.yl;
        q->oz += 0.5 * (bc.vEDm - bc.vWDm) / Dom.xl;
        q->ox0 = q->ox; q->oy0 = q->oy; q->oz0 = q->oz;
      }
    } else if(init_cond == BBB_CHANNEL) {
      if(q->translating) {
        real x = q->x, y = q->y, z = q->z;
        q->u = 0.5 / mu * gradP.xm * (y * y - (Dom.ys + Dom.ye) * y + Dom.ys * Dom.ye)
          * (bc.uS == BBB_DIRICHLET)
          + 0.5 / mu * gradP.xm * (z * z - (Dom.zs + Dom.ze) * z + Dom.zs * Dom.ze)
          * (bc.uB == BBB_DIRICHLET);
        q->u0 = q->u;
        q->v = 0.5 / mu * gradP.ym * (x * x - (Dom.xs + Dom.xe) * x + Dom.xs * Dom.xe)
          * (bc.vW == BBB_DIRICHLET)
          + 0.5 / mu * gradP.ym * (z * z - (Dom.zs + Dom.ze) * z + Dom.zs * Dom.ze)
          * (bc.vB == BBB_DIRICHLET);
        q->v0 = q->v;
        q->w = 0.5 / mu * gradP.zm * (x * x - (Dom.xs + Dom.xe) * x + Dom.xs * Dom.xe)
          * (bc.wW == BBB_DIRICHLET)
          + 0.5 / mu * gradP.zm * (y * y - (Dom.ys + Dom.ye) * y + Dom.ys * Dom.ye)
          * (bc.wS == BBB_DIRICHLET);
        q->w0 = q->w;
        q->x0 = q->x - dt * q->u; q->y0 = q->y - dt * q->v; q->z0 = q->z - dt * q->w;
      }
    }
    q->Fx = q->Fy = q->Fz = 0.; q->Lx = q->Ly = q->Lz = 0.;
    q->kFx = q->kFy = q->kFz = 0.;
    q->iFx = q->iFy = q->iFz = 0.; q->iLx = q->iLy = q->iLz = 0.;
    if(q->ncoeff > coeff_stride) coeff_stride = q->ncoeff;
    for(int j = 0; j < BBB_NNODES; j++) q->nodes[j] = -1;
    for(int j = 0; j < BBB_MAX_NEIGHBORS; j++) { q->St[j] = 0.; q->iSt[j] = -1; }
  }
  long nc = (long)coeff_stride * nparts;
  real **cs[] = {&pnm_re, &pnm_im, &phinm_re, &phinm_im, &chinm_re,
    &chinm_im, &pnm_re0, &pnm_im0, &phinm_re0, &phinm_im0, &chinm_re0,
    &chinm_im0, &pnm_re00, &pnm_im00, &phinm_re00, &phinm_im00, &chinm_re00,
    &chinm_im00};
  for(size_t a = 0; a < sizeof(cs) / sizeof(cs[0]); a++) *cs[a] = zalloc(nc);
  if(g_opt.gravity_balance) {
    /* zero net weight of the periodic box: gradP.z = sum (rho_p - rho_f)
     * V_p g_z / V_box, so that the fluid's -gradP balances the particles'
     * buoyancy-reduced weight */
    real ex = 0.;
    for(int i = 0; i < nparts; i++)
      ex += (parts[i].rho - rho_f) * 4. / 3. * BBB_PI * parts[i].r * parts[i].r * parts[i].r;
    gradP.zm = ex * g.zm / (Dom.xl * Dom.yl * Dom.zl);
    gradP.za = 0.;
  }
  bin_dom_init();
  return BBB_OK;
}

/* ------------------------------------------------ seeded particle pack
 * Replaces src/seeder.c's unseeded generator (srand(time(NULL)),
 * src/seeder.c:234) with a reproducible one: splitmix64 stream, uniform
 * centres, rejection against every earlier sphere through a cell list.
 * The placement rules are the reference seeder's: centres inside the
 * domain less its screens bc.dsW .. bc.dsT (src/seeder.c:246-257), at
 * least a from a non-periodic wall of that region (:259-285; here a plus
 * half the surface gap), and a sphere's periodic images counted only along
 * the periodic axes (:390-700, whose velocity conditions bc.uW, bc.vS,
 * bc.wB decide).  Images are one domain length apart (the reference
 * shifts by the screened length, which differs only where a periodic axis
 * has a screen). */
static uint64_t sm64(uint64_t *s)
{
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static real urand(uint64_t *s) { return (sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

/* one axis of the pack: the sampled interval, the periodic length (0 when
 * not periodic) and the cell list's cells */
typedef struct {
  real lo, len;          /* centres in [lo, lo + len)                  */
  real origin, L;        /* domain start and length                    */
  int per, nc;
} pk_axis;

static int pk_axis_init(pk_axis *ax, real xs, real xl, real ds_lo, real ds_hi,
  int per, real wall, real dmin)
{
  ax->origin = xs;
  ax->L = xl;
  ax->per = per;
  ax->lo = xs + ds_lo + (per ? 0. : wall);
  ax->len = xl - ds_lo - ds_hi - (per ? 0. : 2. * wall);
  ax->nc = (int)floor(xl / dmin);
  if(ax->nc < 1) ax->nc = 1;
  return ax->len > 0.;
}

static int pk_cell(const pk_axis *ax, real x)
{
  int c = (int)((x - ax->origin) / ax->L * ax->nc);
  if(c < 0) c = 0;
  if(c >= ax->nc) c = ax->nc - 1;
  return c;
}

int bbb_seed_particles(int n, real a, real min_gap, real rho, int order,
  real rsr, unsigned long long seed)
{
  if(n < 0) return BBB_ERR_CONFIG;
  free(parts);
  parts = (part_struct *)calloc((size_t)(n > 0 ? n : 1), sizeof(part_struct));
  nparts = 0;
  uint64_t s = (uint64_t)seed;
  real dmin = 2. * a + min_gap * a;
  real wall = a + 0.5 * min_gap * a;
  pk_axis X[3];
  int fits = pk_axis_init(&X[0], Dom.xs, Dom.xl, bc.dsW, bc.dsE, bc.uW == BBB_PERIODIC, wall, dmin);
  fits &= pk_axis_init(&X[1], Dom.ys, Dom.yl, bc.dsS, bc.dsN, bc.vS == BBB_PERIODIC, wall, dmin);
  fits &= pk_axis_init(&X[2], Dom.zs, Dom.zl, bc.dsB, bc.dsT, bc.wB == BBB_PERIODIC, wall, dmin);
  if(!fits && n > 0) {
    bbb_set_status(BBB_ERR_CONFIG, "particle pack: no room between the walls");
    return BBB_ERR_CONFIG;
  }
  long ncell = (long)X[0].nc * X[1].nc * X[2].nc;
  int *head = (int *)malloc(sizeof(int) * (size_t)ncell);
  int *next = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for(long c = 0; c < ncell; c++) head[c] = -1;
  long tries = 0, max_tries = 2000L * (n > 0 ? n : 1) + 100000L;
  while(nparts < n && tries < max_tries) {
    tries++;
    real p[3];
    int ic[3];
    for(int d = 0; d < 3; d++) {
      p[d] = X[d].lo + urand(&s) * X[d].len;
      ic[d] = pk_cell(&X[d], p[d]);
    }
    int ok = 1;
    for(int dz = -1; dz <= 1 && ok; dz++) for(int dy = -1; dy <= 1 && ok; dy++)
    for(int dx = -1; dx <= 1 && ok; dx++) {
      int off[3] = {dx, dy, dz}, jc[3], inside = 1;
      for(int d = 0; d < 3; d++) {
        jc[d] = ic[d] + off[d];
        if(X[d].per) jc[d] = (jc[d] % X[d].nc + X[d].nc) % X[d].nc;
        else if(jc[d] < 0 || jc[d] >= X[d].nc) inside = 0;
      }
      /* with fewer than 3 cells along an axis the wrapped neighbours
       * repeat: visit each cell once */
      for(int d = 0; d < 3 && inside; d++)
        if(X[d].per && X[d].nc < 3 && off[d] != 0 && (X[d].nc == 1 || off[d] == 1))
          inside = 0;
      if(!inside) continue;
      for(int q = head[jc[0] + (long)X[0].nc * (jc[1] + (long)X[1].nc * jc[2])];
          q >= 0; q = next[q]) {
        real r[3] = {p[0] - parts[q].x, p[1] - parts[q].y, p[2] - parts[q].z};
        real r2 = 0.;
        for(int d = 0; d < 3; d++) {
          if(X[d].per) r[d] -= X[d].L * round(r[d] / X[d].L);
          r2 += r[d] * r[d];
        }
        if(r2 < dmin * dmin) { ok = 0; break; }
      }
    }
    if(!ok) continue;
    part_struct *q = &parts[nparts];
    memset(q, 0, sizeof(*q));
    q->r = a; q->x = p[0]; q->y = p[1]; q->z = p[2];
    q->rho = rho; q->E = 1.e6; q->sigma = 0.5; q->e_dry = 1.; q->coeff_fric = 0.5;
    q->order = order; q->rs = rsr;
    q->translating = 1; q->rotating = 1;
    long cell = ic[0] + (long)X[0].nc * (ic[1] + (long)X[1].nc * ic[2]);
    next[nparts] = head[cell];
    head[cell] = nparts;
    nparts++;
  }
  free(head);
  free(next);
  if(nparts < n) {
    bbb_set_status(BBB_ERR_CONFIG, "particle pack too dense for the box");
    return BBB_ERR_CONFIG;
  }
  return BBB_OK;
}

/* The particle list as the reference's part.config (the layout
 * src/seeder.c:786-815 writes and src/particle.c:79-159 reads), numbers
 * with 17 significant digits so the file reads back to the same doubles
 * (the reference's seeder prints %f).  path NULL or empty: the seeder's
 * own ./input/part_seeder.config. */
int bbb_write_part_config(const char *path)
{
  const char *fn = (path && path[0]) ? path : "./input/part_seeder.config";
  FILE *f = fopen(fn, "w");
  if(!f) {
    bbb_set_status(BBB_ERR_CONFIG, "write_part_config: cannot create the file");
    return BBB_ERR_CONFIG;
  }
  fprintf(f, "n %d\n", nparts);
  fprintf(f, "(l/a) %.17g\n", interactionLengthRatio);
  for(int i = 0; i < nparts; i++) {
    const part_struct *q = &parts[i];
    fprintf(f, "\n");
    fprintf(f, "r %.17g\n", q->r);
    fprintf(f, "(x, y, z) %.17g %.17g %.17g\n", q->x, q->y, q->z);
    fprintf(f, "(aFx, aFy, aFz) %.17g %.17g %.17g\n", q->aFx, q->aFy, q->aFz);
    fprintf(f, "(aLx, aLy, aLz) %.17g %.17g %.17g\n", q->aLx, q->aLy, q->aLz);
    fprintf(f, "rho %.17g\n", q->rho);
    fprintf(f, "E %.17g\n", q->E);
    fprintf(f, "sigma %.17g\n", q->sigma);
    fprintf(f, "e_dry %.17g\n", q->e_dry);
    fprintf(f, "coeff_fric %.17g\n", q->coeff_fric);
    fprintf(f, "order %d\n", q->order);
    fprintf(f, "rs/r %.17g\n", q->rs);
    fprintf(f, "spring_k %.17g\n", q->spring_k);
    fprintf(f, "spring (x, y, z) %.17g %.17g %.17g\n", q->spring_x, q->spring_y,
      q->spring_z);
    fprintf(f, "spring_l %.17g\n", q->spring_l);
    fprintf(f, "translating %d\n", q->translating);
    fprintf(f, "rotating %d\n", q->rotating);
  }
  if(fclose(f) != 0) {
    bbb_set_status(BBB_ERR_CONFIG, "write_part_config: write failed");
    return BBB_ERR_CONFIG;
  }
  return BBB_OK;
}

void bbb_host_free(void)
{
  free_fields();
  free_parts_arrays();
  free(parts); parts = NULL; nparts = 0;
  free(dom); dom = NULL;
}

/* ------------------------------------------------ time-step driver */

/* device set-up and the pre-loop sequence of src/bluebottle.c:415-543:
 * allocate, push, build cages, initial dt, boundary conditions and the
 * rigid-body fill inside particles */
int bbb_prepare(void)
{
  opt_init();
  cuda_dom_malloc();
  cuda_part_malloc();
  cuda_dom_push();
  cuda_part_push();
  cuda_build_cages();
  cuda_part_pull();
  real d = cuda_find_dt();
  dt = g_opt.fixed_dt > 0 ? g_opt.fixed_dt : d;
  if(nparts > 0) cuda_part_BC();
  cuda_dom_BC();
  cuda_parts_internal();
  cuda_dom_BC();
  if(g_opt.learned_guess) bbb_learn_enable(g_opt.learned_guess);
  return bbb_last_status();
}

void bbb_release(void)
{
  cuda_part_free();
  cuda_dom_free();
}

void bbb_advance_clock(void)
{
  ttime += dt;
  stepnum++;
}

int bbb_step(void)
{
  opt_init();
  int st0 = bbb_last_status();
  if(st0 != BBB_OK) return st0;
  memset(&g_stats, 0, sizeof(g_stats));
  g_stats.step_dt = dt;
  bbb_advance_clock();
  cuda_compute_forcing(&pid_int, &pid_back, Kp, Ki, Kd);
  /* compute_vel_BC (src/domain.c:3144) */
  real delta = ttime - vel_tDelay;
  if(delta >= 0) {
#define RAMP(D, Dm, Da) do { if((Da) == 0) (D) = (Dm); \
    else if(fabs(delta * (Da)) > fabs(Dm)) (D) = (Dm); else (D) = delta * (Da); } while(0)
    RAMP(bc.uWD, bc.uWDm, bc.uWDa); RAMP(bc.uED, bc.uEDm, bc.uEDa);
    RAMP(bc.uSD, bc.uSDm, bc.uSDa); RAMP(bc.uND, bc.uNDm, bc.uNDa);
    RAMP(bc.uBD, bc.uBDm, bc.uBDa); RAMP(bc.uTD, bc.uTDm, bc.uTDa);
    RAMP(bc.vWD, bc.vWDm, bc.vWDa); RAMP(bc.vED, bc.vEDm, bc.vEDa);
    RAMP(bc.vSD, bc.vSDm, bc.vSDa); RAMP(bc.vND, bc.vNDm, bc.vNDa);
    RAMP(bc.vBD, bc.vBDm, bc.vBDa); RAMP(bc.vTD, bc.vTDm, bc.vTDa);
    RAMP(bc.wWD, bc.wWDm, bc.wWDa); RAMP(bc.wED, bc.wEDm, bc.wEDa);
    RAMP(bc.wSD, bc.wSDm, bc.wSDa); RAMP(bc.wND, bc.wNDm, bc.wNDa);
    RAMP(bc.wBD, bc.wBDm, bc.wBDa); RAMP(bc.wTD, bc.wTDm, bc.wTDa);
#undef RAMP
  }
  cuda_build_cages();
  int lmax = g_opt.lamb_max_iter_override > 0 ? g_opt.lamb_max_iter_override
                                               : lamb_max_iter;
  int iter = 0;
  real iter_err = FLT_MAX;
  /* with options.lamb_pp_tol the pressure solves of all but the last
   * sub-iteration stop at that looser tolerance; the step still ends on a
   * solve to pp_residual (force_full: one more sub-iteration after a
   * loosened one that met the coefficient criterion) */
  const real loose = g_opt.lamb_pp_tol;
  int force_full = 0;
  while(iter_err > lamb_residual || force_full) {
    if(g_opt.implicit) {
      cuda_ustar_helmholtz(0);
      cuda_vstar_helmholtz(0);
      cuda_wstar_helmholtz(0);
    } else {
      cuda_U_star_2();
    }
    if(nparts > 0) cuda_part_BC_star();
    cuda_dom_BC_star();
    cuda_solvability();
    if(nparts > 0) cuda_part_BC_star();
    cuda_dom_BC_star();
    const int loose_now = loose > 0 && !force_full && iter + 1 < lmax;
    g_pp_tol_now = loose_now ? loose : 0.;
    cuda_PP_bicgstab(0);
    g_pp_tol_now = 0.;
    cuda_dom_BC_phi();
    cuda_project();
    if(nparts > 0) cuda_part_BC();
    cuda_dom_BC();
    cuda_update_p();
    if(nparts > 0) {
      cuda_part_BC();
      cuda_part_p_fill();
    }
    cuda_dom_BC_p();
    cuda_move_parts_sub();
    cuda_Lamb();
    iter_err = cuda_lamb_err();
    iter++;
    if(bbb_last_status() != BBB_OK) return bbb_last_status();
    if(force_full || iter == lmax) break;
    if(loose_now && iter_err <= lamb_residual) force_full = 1;
  }
  g_stats.lamb_iters = iter;
  g_stats.lamb_err = iter_err;
  cuda_move_parts();
  cuda_parts_internal();
  cuda_dom_BC();
  cuda_store_u();
  if(nparts > 0) cuda_store_coeffs();
  dt0 = dt;
  dt = cuda_find_dt();
  if(g_opt.fixed_dt > 0) dt = g_opt.fixed_dt;
  if(dt < 1.e-10 || dt > 1.e10) {
    bbb_set_status(BBB_ERR_DIVERGED, "bbb_step");
    return BBB_ERR_DIVERGED;
  }
  return bbb_last_status();
}
