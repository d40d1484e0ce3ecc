/* orc_fluid.c -- CPU FP64 oracle: domain boundary conditions, momentum
 * right-hand sides, Helmholtz and pressure-Poisson Krylov solves, projection
 * and pressure update.  TEST INFRASTRUCTURE ONLY (see orc.h). */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "orc.h"

#define CCI(G, i, j, k) ((i) + (j) * (G).s1b + (k) * (G).s2b)

/* ---------------------------------------------------------------- state */

static real *alloc_r(long n)
{
  real *a = (real *)calloc((size_t)(n > 0 ? n : 1), sizeof(real));
  return a;
}
static int *alloc_i(long n)
{
  int *a = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
  return a;
}

orc_state *orc_create(const dom_struct *dom, int nparts, int coeff_stride)
{
  orc_state *st = (orc_state *)calloc(1, sizeof(orc_state));
  st->dom = *dom;
  long ncc = dom->Gcc.s3b, nfx = dom->Gfx.s3b, nfy = dom->Gfy.s3b,
       nfz = dom->Gfz.s3b;
  st->p0 = alloc_r(ncc); st->p = alloc_r(ncc); st->phi = alloc_r(ncc);
  st->u = alloc_r(nfx); st->u0 = alloc_r(nfx); st->u_star = alloc_r(nfx);
  st->v = alloc_r(nfy); st->v0 = alloc_r(nfy); st->v_star = alloc_r(nfy);
  st->w = alloc_r(nfz); st->w0 = alloc_r(nfz); st->w_star = alloc_r(nfz);
  st->conv_u = alloc_r(nfx); st->conv0_u = alloc_r(nfx);
  st->diff_u = alloc_r(nfx); st->diff0_u = alloc_r(nfx);
  st->conv_v = alloc_r(nfy); st->conv0_v = alloc_r(nfy);
  st->diff_v = alloc_r(nfy); st->diff0_v = alloc_r(nfy);
  st->conv_w = alloc_r(nfz); st->conv0_w = alloc_r(nfz);
  st->diff_w = alloc_r(nfz); st->diff0_w = alloc_r(nfz);
  st->phase = alloc_i(ncc); st->phase_shell = alloc_i(ncc);
  st->flag_u = alloc_i(nfx); st->flag_v = alloc_i(nfy);
  st->flag_w = alloc_i(nfz);
  for(long c = 0; c < ncc; c++) { st->phase[c] = -1; st->phase_shell[c] = 1; }
  for(long c = 0; c < nfx; c++) st->flag_u[c] = 1;
  for(long c = 0; c < nfy; c++) st->flag_v[c] = 1;
  for(long c = 0; c < nfz; c++) st->flag_w[c] = 1;
  st->rhs_p = alloc_r(dom->Gcc.s3);
  st->nparts = nparts;
  st->coeff_stride = coeff_stride;
  st->parts = (part_struct *)calloc((size_t)(nparts > 0 ? nparts : 1),
    sizeof(part_struct));
  for(int a = 0; a < 18; a++)
    st->coef[a] = alloc_r((long)nparts * coeff_stride);
  st->P.dt0 = -1.;
  return st;
}

void orc_destroy(orc_state *st)
{
  if(!st) return;
  real **rs[] = {&st->p0, &st->p, &st->phi, &st->u, &st->u0, &st->u_star,
    &st->v, &st->v0, &st->v_star, &st->w, &st->w0, &st->w_star,
    &st->conv_u, &st->conv0_u, &st->diff_u, &st->diff0_u,
    &st->conv_v, &st->conv0_v, &st->diff_v, &st->diff0_v,
    &st->conv_w, &st->conv0_w, &st->diff_w, &st->diff0_w, &st->rhs_p};
  for(size_t a = 0; a < sizeof(rs) / sizeof(rs[0]); a++) free(*rs[a]);
  free(st->phase); free(st->phase_shell);
  free(st->flag_u); free(st->flag_v); free(st->flag_w);
  free(st->parts);
  for(int a = 0; a < 18; a++) free(st->coef[a]);
  free(st);
}

orc_params *orc_params_ptr(orc_state *st) { return &st->P; }

/* iv: pp_iters, pp_converged, pp_solves, pp_iters_total, cg_iters[3],
 * lamb_iters; rv: pp_resid, lamb_err, cg_resid[3] */
void orc_get_stats(orc_state *st, int *iv, real *rv)
{
  iv[0] = st->pp_iters; iv[1] = st->pp_converged; iv[2] = st->pp_solves;
  iv[3] = st->pp_iters_total; iv[4] = st->cg_iters[0];
  iv[5] = st->cg_iters[1]; iv[6] = st->cg_iters[2]; iv[7] = st->lamb_iters;
  rv[0] = st->pp_resid; rv[1] = st->lamb_err; rv[2] = st->cg_resid[0];
  rv[3] = st->cg_resid[1]; rv[4] = st->cg_resid[2];
}

int orc_set_threads(int n)
{
  if(n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

static const char *coef_names[18] = {
  "pnm_re", "pnm_im", "phinm_re", "phinm_im", "chinm_re", "chinm_im",
  "pnm_re0", "pnm_im0", "phinm_re0", "phinm_im0", "chinm_re0", "chinm_im0",
  "pnm_re00", "pnm_im00", "phinm_re00", "phinm_im00", "chinm_re00",
  "chinm_im00"};

void *orc_field(orc_state *st, const char *name, long *count)
{
  const dom_struct *d = &st->dom;
  long ncc = d->Gcc.s3b, nfx = d->Gfx.s3b, nfy = d->Gfy.s3b,
       nfz = d->Gfz.s3b;
#define F(nm, ptr, n) if(strcmp(name, nm) == 0) { *count = (n); return (void *)(ptr); }
  F("p0", st->p0, ncc) F("p", st->p, ncc) F("phi", st->phi, ncc)
  F("u", st->u, nfx) F("u0", st->u0, nfx) F("u_star", st->u_star, nfx)
  F("v", st->v, nfy) F("v0", st->v0, nfy) F("v_star", st->v_star, nfy)
  F("w", st->w, nfz) F("w0", st->w0, nfz) F("w_star", st->w_star, nfz)
  F("conv_u", st->conv_u, nfx) F("conv0_u", st->conv0_u, nfx)
  F("diff_u", st->diff_u, nfx) F("diff0_u", st->diff0_u, nfx)
  F("conv_v", st->conv_v, nfy) F("conv0_v", st->conv0_v, nfy)
  F("diff_v", st->diff_v, nfy) F("diff0_v", st->diff0_v, nfy)
  F("conv_w", st->conv_w, nfz) F("conv0_w", st->conv0_w, nfz)
  F("diff_w", st->diff_w, nfz) F("diff0_w", st->diff0_w, nfz)
  F("phase", st->phase, ncc) F("phase_shell", st->phase_shell, ncc)
  F("flag_u", st->flag_u, nfx) F("flag_v", st->flag_v, nfy)
  F("flag_w", st->flag_w, nfz)
  F("rhs_p", st->rhs_p, (long)d->Gcc.s3)
  F("parts", st->parts, (long)st->nparts)
#undef F
  for(int a = 0; a < 18; a++)
    if(strcmp(name, coef_names[a]) == 0) {
      *count = (long)st->nparts * st->coeff_stride;
      return st->coef[a];
    }
  *count = 0;
  return NULL;
}

/* ---------------------------------------------- boundary conditions
 * Restates the face kernels of src/bluebottle_kernel.cu:26-1248 and the
 * dispatch order of cuda_dom_BC (src/cuda_bluebottle.cu:1549-2300): faces
 * W, E, S, N, B, T in turn, and within each face p, u, v, w.  Every face
 * loop spans the full ghosted extent of the other two directions. */

/* normal-component faces (u on W/E, v on S/N, w on B/T).  `ax` selects the
 * normal axis; lo = 1 for the low face. */
static void bc_normal(real *f, const grid_info *G, int ax, int lo, int type,
  real bcv)
{
  int n1 = ax == 0 ? G->jnb : G->inb;
  int n2 = ax == 2 ? G->jnb : G->knb;
  int st0 = ax == 0 ? 1 : (ax == 1 ? G->s1b : G->s2b);
  int sA = ax == 0 ? G->s1b : 1;
  int sB = ax == 2 ? G->s1b : G->s2b;
  int s = ax == 0 ? G->is : (ax == 1 ? G->js : G->ks);
  int e = ax == 0 ? G->ie : (ax == 1 ? G->je : G->ke);
  int sb = ax == 0 ? G->isb : (ax == 1 ? G->jsb : G->ksb);
  int eb = ax == 0 ? G->ieb : (ax == 1 ? G->jeb : G->keb);
  for(int b = 0; b < n2; b++) for(int a = 0; a < n1; a++) {
    long base = (long)a * sA + (long)b * sB;
#define AT(q) f[base + (long)(q) * st0]
    if(lo) {
      if(type == BBB_PERIODIC) { AT(sb) = AT(e - 2); AT(s) = AT(e - 1); }
      else if(type == BBB_DIRICHLET) { AT(sb) = 2. * bcv - AT(s + 1); AT(s) = bcv; }
      else if(type == BBB_NEUMANN) { AT(sb) = AT(s); }
    } else {
      if(type == BBB_PERIODIC) { AT(eb - 1) = AT(s + 1); AT(e - 1) = AT(s); }
      else if(type == BBB_DIRICHLET) { AT(eb - 1) = 2. * bcv - AT(e - 2); AT(e - 1) = bcv; }
      else if(type == BBB_NEUMANN) { AT(eb - 1) = AT(e - 1); }
    }
#undef AT
  }
}

/* tangential faces and cell-centred fields (p, phi): only the ghost layer
 * changes.  `cell` = 1 for p/phi (no Dirichlet kernel in the reference). */
static void bc_tangent(real *f, const grid_info *G, int ax, int lo, int type,
  real bcv)
{
  int n1 = ax == 0 ? G->jnb : G->inb;
  int n2 = ax == 2 ? G->jnb : G->knb;
  int st0 = ax == 0 ? 1 : (ax == 1 ? G->s1b : G->s2b);
  int sA = ax == 0 ? G->s1b : 1;
  int sB = ax == 2 ? G->s1b : G->s2b;
  int s = ax == 0 ? G->is : (ax == 1 ? G->js : G->ks);
  int e = ax == 0 ? G->ie : (ax == 1 ? G->je : G->ke);
  int sb = ax == 0 ? G->isb : (ax == 1 ? G->jsb : G->ksb);
  int eb = ax == 0 ? G->ieb : (ax == 1 ? G->jeb : G->keb);
  for(int b = 0; b < n2; b++) for(int a = 0; a < n1; a++) {
    long base = (long)a * sA + (long)b * sB;
#define AT(q) f[base + (long)(q) * st0]
    if(lo) {
      if(type == BBB_PERIODIC) AT(sb) = AT(e - 1);
      else if(type == BBB_DIRICHLET)
        AT(sb) = 8. / 3. * bcv - 2. * AT(s) + 1. / 3. * AT(s + 1);
      else if(type == BBB_NEUMANN) AT(sb) = AT(s);
    } else {
      if(type == BBB_PERIODIC) AT(eb - 1) = AT(s);
      else if(type == BBB_DIRICHLET)
        AT(eb - 1) = 8. / 3. * bcv - 2. * AT(e - 1) + 1. / 3. * AT(e - 2);
      else if(type == BBB_NEUMANN) AT(eb - 1) = AT(e - 1);
    }
#undef AT
  }
}

static void bc_apply(orc_state *st, real *pp, real *uu, real *vv, real *ww)
{
  const dom_struct *d = &st->dom;
  const BC *b = &st->P.bc;
  /* per face: {axis, lo, p type, u type, u value, v type, v value, w...} */
  int   pt[6] = {b->pW, b->pE, b->pS, b->pN, b->pB, b->pT};
  int   ut[6] = {b->uW, b->uE, b->uS, b->uN, b->uB, b->uT};
  real  uv[6] = {b->uWD, b->uED, b->uSD, b->uND, b->uBD, b->uTD};
  int   vt[6] = {b->vW, b->vE, b->vS, b->vN, b->vB, b->vT};
  real  vv_[6] = {b->vWD, b->vED, b->vSD, b->vND, b->vBD, b->vTD};
  int   wt[6] = {b->wW, b->wE, b->wS, b->wN, b->wB, b->wT};
  real  wv[6] = {b->wWD, b->wED, b->wSD, b->wND, b->wBD, b->wTD};
  for(int face = 0; face < 6; face++) {
    int ax = face / 2, lo = (face % 2) == 0;
    if(pp && (pt[face] == BBB_PERIODIC || pt[face] == BBB_NEUMANN))
      bc_tangent(pp, &d->Gcc, ax, lo, pt[face], 0.);
    if(uu) {
      if(ax == 0) bc_normal(uu, &d->Gfx, ax, lo, ut[face], uv[face]);
      else bc_tangent(uu, &d->Gfx, ax, lo, ut[face], uv[face]);
    }
    if(vv) {
      if(ax == 1) bc_normal(vv, &d->Gfy, ax, lo, vt[face], vv_[face]);
      else bc_tangent(vv, &d->Gfy, ax, lo, vt[face], vv_[face]);
    }
    if(ww) {
      if(ax == 2) bc_normal(ww, &d->Gfz, ax, lo, wt[face], wv[face]);
      else bc_tangent(ww, &d->Gfz, ax, lo, wt[face], wv[face]);
    }
  }
}

void orc_dom_BC(orc_state *st, int which)
{
  switch(which) {
    case 0: bc_apply(st, st->p, st->u, st->v, st->w); break;
    case 1: bc_apply(st, NULL, st->u_star, st->v_star, st->w_star); break;
    case 2: bc_apply(st, st->phi, NULL, NULL, NULL); break;
    case 3: bc_apply(st, st->p, NULL, NULL, NULL); break;
  }
}

/* ramp helper of src/cuda_bluebottle.cu:3716-3760 and src/domain.c:3144 */
static real ramp(real delta, real a, real m)
{
  if(a == 0) return m;
  if(fabs(delta * a) > fabs(m)) return m;
  return delta * a;
}

/* src/cuda_bluebottle.cu:3674-3814; the forcing field the reference fills
 * is uniform (-gradP/rho_f), so the oracle keeps it as a scalar. */
void orc_compute_forcing(orc_state *st)
{
  orc_params *P = &st->P;
  real delta = P->ttime - P->p_tDelay;
  int pid = (P->Kp > 0 || P->Ki > 0 || P->Kd > 0);
  if(delta >= 0) {
    P->gradP.x = ramp(delta, P->gradP.xa, P->gradP.xm);
    P->gradP.y = ramp(delta, P->gradP.ya, P->gradP.ym);
    if(!pid) P->gradP.z = ramp(delta, P->gradP.za, P->gradP.zm);
  }
  delta = P->ttime - P->g_tDelay;
  if(delta >= 0) {
    P->g.x = ramp(delta, P->g.xa, P->g.xm);
    P->g.y = ramp(delta, P->g.ya, P->g.ym);
    P->g.z = ramp(delta, P->g.za, P->g.zm);
  }
  delta = P->ttime - P->p_tDelay;
  if(delta >= 0 && pid) {
    real acc_z = 0, volp = 0, massp = 0;
    for(int i = 0; i < st->nparts; i++) {
      part_struct *q = &st->parts[i];
      volp += q->r * q->r * q->r;
      massp += q->rho * q->r * q->r * q->r;
      acc_z += q->wdot;
    }
    volp *= 4. / 3. * BBB_PI;
    massp *= 4. / 3. * BBB_PI;
    real volfrac = volp / (st->dom.xl * st->dom.yl * st->dom.zl);
    real rho_avg = massp / volp * volfrac + P->rho_f * (1. - volfrac);
    acc_z /= st->nparts;
    P->pid_int = P->pid_int + acc_z * P->dt;
    P->gradP.z = P->gradP.z + (P->Kp * acc_z + P->Ki * P->pid_int / P->ttime
      + P->Kd * (acc_z - P->pid_back)) * rho_avg;
    P->pid_back = acc_z;
  }
}

/* src/domain.c:3144-3222 */
void orc_compute_vel_BC(orc_state *st)
{
  orc_params *P = &st->P;
  BC *b = &P->bc;
  real delta = P->ttime - P->vel_tDelay;
  if(delta < 0) return;
  b->uWD = ramp(delta, b->uWDa, b->uWDm); b->uED = ramp(delta, b->uEDa, b->uEDm);
  b->uSD = ramp(delta, b->uSDa, b->uSDm); b->uND = ramp(delta, b->uNDa, b->uNDm);
  b->uBD = ramp(delta, b->uBDa, b->uBDm); b->uTD = ramp(delta, b->uTDa, b->uTDm);
  b->vWD = ramp(delta, b->vWDa, b->vWDm); b->vED = ramp(delta, b->vEDa, b->vEDm);
  b->vSD = ramp(delta, b->vSDa, b->vSDm); b->vND = ramp(delta, b->vNDa, b->vNDm);
  b->vBD = ramp(delta, b->vBDa, b->vBDm); b->vTD = ramp(delta, b->vTDa, b->vTDm);
  b->wWD = ramp(delta, b->wWDa, b->wWDm); b->wED = ramp(delta, b->wEDa, b->wEDm);
  b->wSD = ramp(delta, b->wSDa, b->wSDm); b->wND = ramp(delta, b->wNDa, b->wNDm);
  b->wBD = ramp(delta, b->wBDa, b->wBDm); b->wTD = ramp(delta, b->wTDa, b->wTDm);
}

/* ------------------------------------------------ momentum RHS
 * One routine serves all three components by permuting axes.  For the
 * component along axis `c` (0 = u on Gfx, 1 = v on Gfy, 2 = w on Gfz) the
 * arithmetic, including the order of every sum, follows u_star_2 /
 * v_star_2 / w_star_2 (src/bluebottle_kernel.cu:1504-2004, explicit AB2)
 * and ustar_rhs / vstar_rhs / wstar_rhs (src/bicgstab_kernel.cu:27-481,
 * Crank-Nicolson).  Faces computed: all interior faces of the component's
 * grid, interior rows of the other two directions. */
static void star_rhs_core(orc_state *st, int c, int explicit_ab2)
{
  const dom_struct *d = &st->dom;
  const orc_params *P = &st->P;
  const grid_info *G[3] = {&d->Gfx, &d->Gfy, &d->Gfz};
  const grid_info *Gc = G[c];
  real *vel0[3] = {st->u0, st->v0, st->w0};
  real *conv0[3] = {st->conv0_u, st->conv0_v, st->conv0_w};
  real *conv[3] = {st->conv_u, st->conv_v, st->conv_w};
  real *diff0[3] = {st->diff0_u, st->diff0_v, st->diff0_w};
  real *diff[3] = {st->diff_u, st->diff_v, st->diff_w};
  real *star[3] = {st->u_star, st->v_star, st->w_star};
  real dd[3] = {1. / d->dx, 1. / d->dy, 1. / d->dz};
  real fc[3] = {-P->gradP.x / P->rho_f, -P->gradP.y / P->rho_f,
    -P->gradP.z / P->rho_f};
  real ab0 = 0.5 * P->dt / P->dt0;
  real ab = 1. + ab0;
  real rho_f = P->rho_f, nu = P->nu, dt = P->dt, dt0 = P->dt0;
  /* unit offsets along each axis, per grid */
  long off[4][3];
  for(int g = 0; g < 3; g++) {
    off[g][0] = 1; off[g][1] = G[g]->s1b; off[g][2] = G[g]->s2b;
  }
  off[3][0] = 1; off[3][1] = d->Gcc.s1b; off[3][2] = d->Gcc.s2b;
  int a1 = (c + 1) % 3, a2 = (c + 2) % 3;   /* the two transverse axes */
  int lo[3] = {Gc->is, Gc->js, Gc->ks}, hi[3] = {Gc->ie, Gc->je, Gc->ke};
  real *vc = vel0[c];

  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = lo[2]; k < hi[2]; k++)
  for(int j = lo[1]; j < hi[1]; j++)
  for(int i = lo[0]; i < hi[0]; i++) {
    int idx[3] = {i, j, k};
    long C = idx[0] * off[c][0] + idx[1] * off[c][1] + idx[2] * off[c][2];
    long Cp = idx[0] * off[3][0] + idx[1] * off[3][1] + idx[2] * off[3][2];
    /* this component along the three axes */
    real m[3], pl[3], x0 = vc[C];
    for(int a = 0; a < 3; a++) { m[a] = vc[C - off[c][a]]; pl[a] = vc[C + off[c][a]]; }
    /* transverse components: for axis t, the velocity along t at the
     * faces bracketing this face: (t at idx - e_c), (t at idx),
     * (t at idx - e_c + e_t), (t at idx + e_t) */
    real tr[3][4];
    for(int tt = 0; tt < 2; tt++) {
      int t = tt == 0 ? a1 : a2;
      real *vt = vel0[t];
      long Ct = idx[0] * off[t][0] + idx[1] * off[t][1] + idx[2] * off[t][2];
      tr[t][0] = vt[Ct - off[t][c]];
      tr[t][1] = vt[Ct];
      tr[t][2] = vt[Ct - off[t][c] + off[t][t]];
      tr[t][3] = vt[Ct + off[t][t]];
    }
    /* previous-step pressure p0, as launched at src/cuda_bicgstab.cu:1115
     * and src/cuda_bluebottle.cu:2946-2965 */
    real s = (st->p0[Cp - off[3][c]] - st->p0[Cp]) * dd[c] / rho_f;
    /* convection: d(u_c u_a)/dx_a in axis order x, y, z */
    real term[3];
    for(int a = 0; a < 3; a++) {
      real t;
      if(a == c) {
        t = (pl[a] + x0) * (pl[a] + x0) - (x0 + m[a]) * (x0 + m[a]);
      } else {
        t = (pl[a] + x0) * (tr[a][3] + tr[a][2])
          - (x0 + m[a]) * (tr[a][1] + tr[a][0]);
      }
      term[a] = t * (0.25 * dd[a]);
    }
    real cv = term[0] + term[1] + term[2];
    if(explicit_ab2) {
      if(dt0 > 0) s += (-ab * cv + ab0 * conv0[c][C]);
      else s += -cv;
    } else {
      if(dt0 > 0) s += (-ab * cv + ab0 * conv0[c][C]);
      else s += -cv;
    }
    real lap[3];
    for(int a = 0; a < 3; a++) {
      real d1 = (pl[a] - x0) * dd[a];
      real d0 = (x0 - m[a]) * dd[a];
      lap[a] = (d1 - d0) * dd[a];
    }
    real df = nu * (lap[0] + lap[1] + lap[2]);
    if(explicit_ab2) {
      if(dt0 > 0) s += (ab * df - ab0 * diff0[c][C]);
      else s += df;
    } else {
      s += 0.5 * df;
    }
    s += fc[c];
    s *= dt;
    s += x0;
    if(explicit_ab2) {
      s *= (st->phase[Cp - off[3][c]] < 0 && st->phase[Cp] < 0);
      diff[c][C] = df;
    }
    star[c][C] = s;
    conv[c][C] = cv;
  }
}

/* src/cuda_bluebottle.cu:2930-3026 (explicit build's cuda_U_star_2) */
void orc_U_star_2(orc_state *st)
{
  star_rhs_core(st, 0, 1);
  star_rhs_core(st, 1, 1);
  star_rhs_core(st, 2, 1);
}

/* src/cuda_bicgstab.cu:1091-1175 */
void orc_star_rhs(orc_state *st, int comp)
{
  star_rhs_core(st, comp, 0);
}

/* ------------------------------------------------ DIA matrices and BLAS */

typedef struct dia13 {
  long n;
  long off[13];
  real *val;   /* val[d*n + row] */
} dia13;

static void dia_alloc(dia13 *A, long n, long s1, long s2, long s3, int sw)
{
  A->n = n;
  /* sw = 1 for Poisson (x-wrap +-1), 2 for Gfx Helmholtz (duplicated face) */
  A->off[0] = -s3 + s2; A->off[1] = -s2; A->off[2] = -s2 + s1;
  A->off[3] = -s1; A->off[4] = -s1 + sw; A->off[5] = -1; A->off[6] = 0;
  A->off[7] = 1; A->off[8] = s1 - sw; A->off[9] = s1; A->off[10] = s2 - s1;
  A->off[11] = s2; A->off[12] = s3 - s2;
  A->val = (real *)calloc((size_t)(13 * n), sizeof(real));
}

/* DIA SpMV: y[r] = sum_d val[d][r] * x[r + off[d]] over in-range columns,
 * diagonals in index order */
static void dia_spmv(const dia13 *A, const real *x, real *y)
{
  long n = A->n;
  #pragma omp parallel for schedule(static)
  for(long r = 0; r < n; r++) {
    real s = 0.;
    for(int d = 0; d < 13; d++) {
      long col = r + A->off[d];
      if(col >= 0 && col < n) s += A->val[d * n + r] * x[col];
    }
    y[r] = s;
  }
}

/* Dot product with a summation order fixed by n alone (chunks of VCHUNK
 * summed in index order), so the oracle's iterates do not depend on the
 * host's thread count. */
#define VCHUNK 4096
static real vdot(long n, const real *a, const real *b)
{
  long nc = (n + VCHUNK - 1) / VCHUNK;
  real part_stack[64];
  real *part = nc <= 64 ? part_stack : (real *)malloc(sizeof(real) * (size_t)nc);
  #pragma omp parallel for schedule(static)
  for(long c = 0; c < nc; c++) {
    long i1 = (c + 1) * VCHUNK < n ? (c + 1) * VCHUNK : n;
    real s = 0.;
    for(long i = c * VCHUNK; i < i1; i++) s += a[i] * b[i];
    part[c] = s;
  }
  real s = 0.;
  for(long c = 0; c < nc; c++) s += part[c];
  if(part != part_stack) free(part);
  return s;
}
static real vnrm2(long n, const real *a) { return sqrt(vdot(n, a, a)); }

/* Right-preconditioned BiCGSTAB with CUSP's monitor semantics:
 * converged when ||r|| <= tol*||b||, iteration count advanced once per full
 * iteration, early exit on ||s|| (x += alpha*M*p) without advancing it. */
static int bicgstab(const dia13 *A, const real *dinv, const real *b, real *x,
  int maxit, real rtol, int *iters, real *resid)
{
  long n = A->n;
  real *y = alloc_r(n), *p = alloc_r(n), *r = alloc_r(n), *rs = alloc_r(n),
       *s = alloc_r(n), *Mp = alloc_r(n), *AMp = alloc_r(n), *Ms = alloc_r(n),
       *AMs = alloc_r(n);
  real tol = rtol * vnrm2(n, b);
  dia_spmv(A, x, y);
  for(long i = 0; i < n; i++) { r[i] = 1. * b[i] + -1. * y[i]; }
  memcpy(p, r, n * sizeof(real));
  memcpy(rs, r, n * sizeof(real));
  real rr_old = vdot(n, rs, r);
  int it = 0, conv = 0;
  real rn = vnrm2(n, r);
  for(;;) {
    if(rn <= tol) { conv = 1; break; }
    if(it >= maxit) break;
    if(!isfinite(rn)) break;
    for(long i = 0; i < n; i++) Mp[i] = dinv[i] * p[i];
    dia_spmv(A, Mp, AMp);
    real alpha = rr_old / vdot(n, rs, AMp);
    for(long i = 0; i < n; i++) s[i] = 1. * r[i] + -alpha * AMp[i];
    real sn = vnrm2(n, s);
    if(sn <= tol) {
      for(long i = 0; i < n; i++) x[i] = 1. * x[i] + alpha * Mp[i];
      rn = sn;
      conv = 1;
      break;
    }
    for(long i = 0; i < n; i++) Ms[i] = dinv[i] * s[i];
    dia_spmv(A, Ms, AMs);
    real omega = vdot(n, AMs, s) / vdot(n, AMs, AMs);
    #pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++) {
      x[i] = 1. * x[i] + alpha * Mp[i] + omega * Ms[i];
      r[i] = 1. * s[i] + -omega * AMs[i];
    }
    real rr_new = vdot(n, rs, r);
    real beta = (rr_new / rr_old) * (alpha / omega);
    rr_old = rr_new;
    #pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++)
      p[i] = 1. * r[i] + beta * p[i] + -beta * omega * AMp[i];
    it++;
    rn = vnrm2(n, r);
  }
  *iters = it;
  *resid = rn;
  free(y); free(p); free(r); free(rs); free(s); free(Mp); free(AMp);
  free(Ms); free(AMs);
  return conv;
}

/* Jacobi-preconditioned CG with the same monitor semantics */
static int pcg(const dia13 *A, const real *dinv, const real *b, real *x,
  int maxit, real rtol, int *iters, real *resid)
{
  long n = A->n;
  real *y = alloc_r(n), *r = alloc_r(n), *z = alloc_r(n), *p = alloc_r(n);
  real tol = rtol * vnrm2(n, b);
  dia_spmv(A, x, y);
  for(long i = 0; i < n; i++) r[i] = 1. * b[i] + -1. * y[i];
  for(long i = 0; i < n; i++) z[i] = dinv[i] * r[i];
  memcpy(p, z, n * sizeof(real));
  real rz_old = vdot(n, r, z);
  int it = 0, conv = 0;
  real rn = vnrm2(n, r);
  for(;;) {
    if(rn <= tol) { conv = 1; break; }
    if(it >= maxit) break;
    if(!isfinite(rn)) break;
    dia_spmv(A, p, y);
    real alpha = rz_old / vdot(n, y, p);
    #pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++) {
      x[i] = alpha * p[i] + x[i];
      r[i] = -alpha * y[i] + r[i];
      z[i] = dinv[i] * r[i];
    }
    real rz_new = vdot(n, r, z);
    real beta = rz_new / rz_old;
    #pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++) p[i] = 1. * z[i] + beta * p[i];
    rz_old = rz_new;
    it++;
    rn = vnrm2(n, r);
  }
  *iters = it;
  *resid = rn;
  free(y); free(r); free(z); free(p);
  return conv;
}

/* ------------------------------------------------ Helmholtz (CN) solve
 * src/cuda_bicgstab.cu:44-712 with the coefficient kernels of
 * src/bicgstab_kernel.cu:643-1652.  Component c on grid G: unknowns are the
 * interior faces (G.s3 of them, un-ghosted ordering), matrix
 * I - 0.5 nu dt Lap_flags, rows with flag < 0 replaced by identity,
 * periodic wraps on the 13-diagonal pattern. */
void orc_star_helmholtz(orc_state *st, int comp)
{
  const dom_struct *d = &st->dom;
  orc_params *P = &st->P;
  const grid_info *G = comp == 0 ? &d->Gfx : (comp == 1 ? &d->Gfy : &d->Gfz);
  real *star = comp == 0 ? st->u_star : (comp == 1 ? st->v_star : st->w_star);
  int *fself = comp == 0 ? st->flag_u : (comp == 1 ? st->flag_v : st->flag_w);

  orc_star_rhs(st, comp);
  orc_dom_BC(st, 1);
  if(st->nparts > 0) orc_part_BC(st, 1);

  long n = G->s3;
  dia13 A;
  /* the duplicated periodic face makes the wrap offset s1-2 along the
   * component's own axis (src/cuda_bicgstab.cu:72-76) */
  dia_alloc(&A, n, G->s1, G->s2, G->s3, comp == 0 ? 2 : 1);
  if(comp == 1) { A.off[10] = G->s2 - 2 * G->s1; A.off[2] = -G->s2 + 2 * G->s1; }
  if(comp == 2) { A.off[12] = G->s3 - 2 * G->s2; A.off[0] = -G->s3 + 2 * G->s2; }
  real ddx = 1. / (d->dx * d->dx), ddy = 1. / (d->dy * d->dy),
       ddz = 1. / (d->dz * d->dz);
  real nu = P->nu, dt = P->dt;
  real *b = alloc_r(n), *x = alloc_r(n);

  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    long W = CCI(d->Gfx, i, j, k), E = CCI(d->Gfx, i + 1, j, k);
    long S = CCI(d->Gfy, i, j, k), N = CCI(d->Gfy, i, j + 1, k);
    long B = CCI(d->Gfz, i, j, k), T = CCI(d->Gfz, i, j, k + 1);
    long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
    real fW = abs(st->flag_u[W]), fE = abs(st->flag_u[E]);
    real fS = abs(st->flag_v[S]), fN = abs(st->flag_v[N]);
    real fB = abs(st->flag_w[B]), fT = abs(st->flag_w[T]);
    real *v = A.val;
    v[1 * n + C] -= fB * 0.5 * nu * dt * ddz;
    v[3 * n + C] -= fS * 0.5 * nu * dt * ddy;
    v[5 * n + C] -= fW * 0.5 * nu * dt * ddx;
    v[6 * n + C] += 1.;
    v[6 * n + C] += fW * 0.5 * nu * dt * ddx;
    v[6 * n + C] += fE * 0.5 * nu * dt * ddx;
    v[6 * n + C] += fS * 0.5 * nu * dt * ddy;
    v[6 * n + C] += fN * 0.5 * nu * dt * ddy;
    v[6 * n + C] += fB * 0.5 * nu * dt * ddz;
    v[6 * n + C] += fT * 0.5 * nu * dt * ddz;
    v[7 * n + C] -= fE * 0.5 * nu * dt * ddx;
    v[9 * n + C] -= fN * 0.5 * nu * dt * ddy;
    v[11 * n + C] -= fT * 0.5 * nu * dt * ddz;
    b[C] = star[CCI(*G, i, j, k)];
  }
  /* periodic wraps (src/bicgstab_kernel.cu:1348-1652) */
  const BC *bc = &P->bc;
  int perW = comp == 0 ? bc->uW : (comp == 1 ? bc->vW : bc->wW);
  int perE = comp == 0 ? bc->uE : (comp == 1 ? bc->vE : bc->wE);
  int perS = comp == 0 ? bc->uS : (comp == 1 ? bc->vS : bc->wS);
  int perN = comp == 0 ? bc->uN : (comp == 1 ? bc->vN : bc->wN);
  int perB = comp == 0 ? bc->uB : (comp == 1 ? bc->vB : bc->wB);
  int perT = comp == 0 ? bc->uT : (comp == 1 ? bc->vT : bc->wT);
  real cx = 0.5 * nu * dt * ddx, cy = 0.5 * nu * dt * ddy,
       cz = 0.5 * nu * dt * ddz;
  for(int k = 0; k < G->kn; k++) for(int j = 0; j < G->jn; j++) {
    if(perW == BBB_PERIODIC) {
      long C = 0 + (long)j * G->s1 + (long)k * G->s2;
      A.val[5 * n + C] += cx; A.val[8 * n + C] -= cx;
    }
    if(perE == BBB_PERIODIC) {
      long C = (G->in - 1) + (long)j * G->s1 + (long)k * G->s2;
      A.val[4 * n + C] -= cx; A.val[7 * n + C] += cx;
    }
  }
  for(int k = 0; k < G->kn; k++) for(int i = 0; i < G->in; i++) {
    if(perS == BBB_PERIODIC) {
      long C = i + 0 + (long)k * G->s2;
      A.val[3 * n + C] += cy; A.val[10 * n + C] -= cy;
    }
    if(perN == BBB_PERIODIC) {
      long C = i + (long)(G->jn - 1) * G->s1 + (long)k * G->s2;
      A.val[2 * n + C] -= cy; A.val[9 * n + C] += cy;
    }
  }
  for(int j = 0; j < G->jn; j++) for(int i = 0; i < G->in; i++) {
    if(perB == BBB_PERIODIC) {
      long C = i + (long)j * G->s1;
      A.val[1 * n + C] += cz; A.val[12 * n + C] -= cz;
    }
    if(perT == BBB_PERIODIC) {
      long C = i + (long)j * G->s1 + (long)(G->kn - 1) * G->s2;
      A.val[0 * n + C] -= cz; A.val[11 * n + C] += cz;
    }
  }
  /* Dirichlet walls (src/bicgstab_kernel.cu:946-1348, launched by
   * src/cuda_bicgstab.cu:213-260 and the v, w counterparts): the wall
   * normal to the component turns its face rows into identity rows; a
   * tangential wall drops the coupling across it */
  int dir[6] = {perW == BBB_DIRICHLET, perE == BBB_DIRICHLET, perS == BBB_DIRICHLET,
                perN == BBB_DIRICHLET, perB == BBB_DIRICHLET, perT == BBB_DIRICHLET};
  for(int k = 0; k < G->kn; k++) for(int j = 0; j < G->jn; j++)
  for(int i = 0; i < G->in; i++) {
    long C = i + (long)j * G->s1 + (long)k * G->s2;
    int at[6] = {i == 0, i == G->in - 1, j == 0, j == G->jn - 1, k == 0, k == G->kn - 1};
    static const int cross[6] = {5, 7, 3, 9, 1, 11};
    for(int f = 0; f < 6; f++) {
      if(!dir[f] || !at[f]) continue;
      if(f / 2 == comp) {
        for(int dd = 0; dd < 13; dd++) A.val[dd * n + C] = 0.;
        A.val[6 * n + C] = 1.;
      } else {
        A.val[cross[f] * n + C] = 0.;
      }
    }
  }
  /* particle identity rows (src/bicgstab_kernel.cu:730-827) */
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    if(fself[CCI(*G, i, j, k)] < 0) {
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      for(int dd = 0; dd < 13; dd++) A.val[dd * n + C] = 0.;
      A.val[6 * n + C] = 1.;
    }
  }
  real *dinv = alloc_r(n);
  for(long r = 0; r < n; r++) dinv[r] = 1. / A.val[6 * n + r];
  real norm = vnrm2(n, b);
  if(norm == 0) norm = 1.;
  real inv = 1. / norm;
  for(long r = 0; r < n; r++) b[r] *= inv;
  int it; real res;
  int conv = pcg(&A, dinv, b, x, P->pp_max_iter, P->pp_residual, &it, &res);
  st->cg_iters[comp] = it;
  st->cg_resid[comp] = res;
  st->cg_converged[comp] = conv;
  for(long r = 0; r < n; r++) x[r] *= norm;
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++)
    star[CCI(*G, i, j, k)] =
      x[(i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2];
  free(A.val); free(b); free(x); free(dinv);
}

/* ------------------------------------------------ solvability
 * src/cuda_bluebottle.cu:4122-4314, kernels src/bluebottle_kernel.cu:
 * 2133-2245 */
void orc_solvability(orc_state *st)
{
  const dom_struct *d = &st->dom;
  real ex = 0, ey = 0, ez = 0;
  const grid_info *X = &d->Gfx, *Y = &d->Gfy, *Z = &d->Gfz;
  for(int k = 0; k < X->kn; k++) for(int j = 0; j < X->jn; j++)
    ex += -st->u_star[CCI(*X, X->is, j + 1, k + 1)];
  for(int k = 0; k < X->kn; k++) for(int j = 0; j < X->jn; j++)
    ex += st->u_star[CCI(*X, X->ie - 1, j + 1, k + 1)];
  ex = ex * d->dy * d->dz;
  for(int k = 0; k < Y->kn; k++) for(int i = 0; i < Y->in; i++)
    ey += -st->v_star[CCI(*Y, i + 1, Y->js, k + 1)];
  for(int k = 0; k < Y->kn; k++) for(int i = 0; i < Y->in; i++)
    ey += st->v_star[CCI(*Y, i + 1, Y->je - 1, k + 1)];
  ey = ey * d->dx * d->dz;
  for(int j = 0; j < Z->jn; j++) for(int i = 0; i < Z->in; i++)
    ez += -st->w_star[CCI(*Z, i + 1, j + 1, Z->ks)];
  for(int j = 0; j < Z->jn; j++) for(int i = 0; i < Z->in; i++)
    ez += st->w_star[CCI(*Z, i + 1, j + 1, Z->ke - 1)];
  ez = ez * d->dx * d->dy;
  int op = st->P.out_plane;
  real area;
  real eps;
#define PLANE_X(ii, sign) for(int k = 0; k < X->kn; k++) for(int j = 0; j < X->jn; j++) \
    st->u_star[CCI(*X, ii, j + 1, k + 1)] += (sign) * eps;
#define PLANE_Y(jj, sign) for(int k = 0; k < Y->kn; k++) for(int i = 0; i < Y->in; i++) \
    st->v_star[CCI(*Y, i + 1, jj, k + 1)] += (sign) * eps;
#define PLANE_Z(kk, sign) for(int j = 0; j < Z->jn; j++) for(int i = 0; i < Z->in; i++) \
    st->w_star[CCI(*Z, i + 1, j + 1, kk)] += (sign) * eps;
  switch(op) {
    case BBB_WEST: case BBB_EAST:
      ex = ex / d->yl / d->zl; ey = ey / d->yl / d->zl; ez = ez / d->yl / d->zl;
      eps = ex + ey + ez;
      if(op == BBB_WEST) { PLANE_X(X->is, 1.) } else { PLANE_X(X->ie - 1, -1.) }
      break;
    case BBB_SOUTH: case BBB_NORTH:
      ex = ex / d->zl / d->xl; ey = ey / d->zl / d->xl; ez = ez / d->zl / d->xl;
      eps = ex + ey + ez;
      if(op == BBB_SOUTH) { PLANE_Y(Y->js, 1.) } else { PLANE_Y(Y->je - 1, -1.) }
      break;
    case BBB_BOTTOM: case BBB_TOP:
      ex = ex / d->xl / d->yl; ey = ey / d->xl / d->yl; ez = ez / d->xl / d->yl;
      eps = ex + ey + ez;
      if(op == BBB_BOTTOM) { PLANE_Z(Z->ks, 1.) } else { PLANE_Z(Z->ke - 1, -1.) }
      break;
    case BBB_HOMOGENEOUS:
      ex = 0.5 * ex / d->yl / d->zl;
      ey = 0.5 * ey / d->zl / d->xl;
      ez = 0.5 * ez / d->xl / d->yl;
      eps = ex; PLANE_X(X->is, 1.) PLANE_X(X->ie - 1, -1.)
      eps = ey; PLANE_Y(Y->js, 1.) PLANE_Y(Y->je - 1, -1.)
      eps = ez; PLANE_Z(Z->ks, 1.) PLANE_Z(Z->ke - 1, -1.)
      break;
  }
  (void)area;
#undef PLANE_X
#undef PLANE_Y
#undef PLANE_Z
}

/* ------------------------------------------------ pressure Poisson */

/* src/bicgstab_kernel.cu:483-562: b = rho_f/dt * div(u*) on interior
 * cells, un-ghosted */
void orc_PP_rhs(orc_state *st)
{
  const dom_struct *d = &st->dom;
  real ddx = 1. / d->dx, ddy = 1. / d->dy, ddz = 1. / d->dz;
  real rho_f = st->P.rho_f, dt = st->P.dt;
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = d->Gcc.ks; k < d->Gcc.ke; k++)
  for(int j = d->Gcc.js; j < d->Gcc.je; j++)
  for(int i = d->Gcc.is; i < d->Gcc.ie; i++) {
    real s = (st->u_star[CCI(d->Gfx, i + 1, j, k)]
      - st->u_star[CCI(d->Gfx, i, j, k)]) * ddx;
    s += (st->v_star[CCI(d->Gfy, i, j + 1, k)]
      - st->v_star[CCI(d->Gfy, i, j, k)]) * ddy;
    s += (st->w_star[CCI(d->Gfz, i, j, k + 1)]
      - st->w_star[CCI(d->Gfz, i, j, k)]) * ddz;
    s *= rho_f / dt;
    st->rhs_p[(i - 1) + (long)(j - 1) * d->Gcc.s1 + (long)(k - 1) * d->Gcc.s2] = s;
  }
}

/* src/bicgstab_kernel.cu:1654-1856 */
static void poisson_dia(orc_state *st, dia13 *A)
{
  const dom_struct *d = &st->dom;
  const grid_info *G = &d->Gcc;
  long n = G->s3;
  dia_alloc(A, n, G->s1, G->s2, G->s3, 1);
  real ddx = 1. / (d->dx * d->dx), ddy = 1. / (d->dy * d->dy),
       ddz = 1. / (d->dz * d->dz);
  real *v = A->val;
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    long W = CCI(d->Gfx, i, j, k), E = CCI(d->Gfx, i + 1, j, k);
    long S = CCI(d->Gfy, i, j, k), N = CCI(d->Gfy, i, j + 1, k);
    long B = CCI(d->Gfz, i, j, k), T = CCI(d->Gfz, i, j, k + 1);
    long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
    v[1 * n + C] += (real)abs(st->flag_w[B]) * ddz;
    v[3 * n + C] += (real)abs(st->flag_v[S]) * ddy;
    v[5 * n + C] += (real)abs(st->flag_u[W]) * ddx;
    v[6 * n + C] -= (real)(abs(st->flag_u[W]) + abs(st->flag_u[E])) * ddx;
    v[6 * n + C] -= (real)(abs(st->flag_v[S]) + abs(st->flag_v[N])) * ddy;
    v[6 * n + C] -= (real)(abs(st->flag_w[B]) + abs(st->flag_w[T])) * ddz;
    v[7 * n + C] += (real)abs(st->flag_u[E]) * ddx;
    v[9 * n + C] += (real)abs(st->flag_v[N]) * ddy;
    v[11 * n + C] += (real)abs(st->flag_w[T]) * ddz;
  }
  const BC *bc = &st->P.bc;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++) {
    if(bc->pW == BBB_PERIODIC) {
      int i = G->is;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_u[CCI(d->Gfx, i, j, k)]) * ddx;
      v[5 * n + C] -= f; v[8 * n + C] += f;
    }
    if(bc->pE == BBB_PERIODIC) {
      int i = G->ie - 1;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_u[CCI(d->Gfx, i + 1, j, k)]) * ddx;
      v[4 * n + C] += f; v[7 * n + C] -= f;
    }
  }
  for(int k = G->ks; k < G->ke; k++) for(int i = G->is; i < G->ie; i++) {
    if(bc->pS == BBB_PERIODIC) {
      int j = G->js;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_v[CCI(d->Gfy, i, j, k)]) * ddy;
      v[3 * n + C] -= f; v[10 * n + C] += f;
    }
    if(bc->pN == BBB_PERIODIC) {
      int j = G->je - 1;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_v[CCI(d->Gfy, i, j + 1, k)]) * ddy;
      v[2 * n + C] += f; v[9 * n + C] -= f;
    }
  }
  for(int j = G->js; j < G->je; j++) for(int i = G->is; i < G->ie; i++) {
    if(bc->pB == BBB_PERIODIC) {
      int k = G->ks;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_w[CCI(d->Gfz, i, j, k)]) * ddz;
      v[1 * n + C] -= f; v[12 * n + C] += f;
    }
    if(bc->pT == BBB_PERIODIC) {
      int k = G->ke - 1;
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      real f = (real)abs(st->flag_w[CCI(d->Gfz, i, j, k + 1)]) * ddz;
      v[0 * n + C] += f; v[11 * n + C] -= f;
    }
  }
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    if(st->phase[CCI(*G, i, j, k)] > -1) {
      long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
      for(int dd = 0; dd < 13; dd++) v[dd * n + C] = 0.;
      v[6 * n + C] = 1.;
    }
  }
}

void orc_poisson_apply(orc_state *st, const real *x, real *y)
{
  dia13 A;
  poisson_dia(st, &A);
  dia_spmv(&A, x, y);
  free(A.val);
}

int orc_poisson_solve(orc_state *st, const real *b_in, real *x, real tol,
  int maxit, real *resid)
{
  dia13 A;
  poisson_dia(st, &A);
  long n = A.n;
  real *dinv = alloc_r(n), *b = alloc_r(n);
  for(long r = 0; r < n; r++) dinv[r] = 1. / A.val[6 * n + r];
  real norm = vnrm2(n, b_in);
  if(norm == 0) norm = 1.;
  real inv = 1. / norm;
  for(long r = 0; r < n; r++) { b[r] = b_in[r] * inv; x[r] *= inv; }
  int it;
  int conv = bicgstab(&A, dinv, b, x, maxit, tol, &it, resid);
  for(long r = 0; r < n; r++) x[r] *= norm;
  free(A.val); free(dinv); free(b);
  st->pp_iters = it;
  st->pp_converged = conv;
  return it;
}

/* src/cuda_bicgstab.cu:715-1073 */
void orc_PP_bicgstab(orc_state *st)
{
  const dom_struct *d = &st->dom;
  const grid_info *G = &d->Gcc;
  orc_PP_rhs(st);
  if(st->nparts > 0) orc_part_BC_p(st);
  long n = G->s3;
  real *x = alloc_r(n);
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++)
    x[(i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2] =
      st->phi[CCI(*G, i, j, k)];
  real res;
  orc_poisson_solve(st, st->rhs_p, x, st->P.pp_residual, st->P.pp_max_iter,
    &res);
  st->pp_resid = res;
  st->pp_solves++;
  st->pp_iters_total += st->pp_iters;
  real sum = 0.;
  for(long r = 0; r < n; r++) sum += x[r];
  real avg = sum / n;
  for(long r = 0; r < n; r++) x[r] = x[r] + -avg * 1.;
  for(int k = G->ks; k < G->ke; k++)
  for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++)
    st->phi[CCI(*G, i, j, k)] =
      x[(i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2];
  free(x);
}

/* src/bluebottle_kernel.cu:1250-1302 */
void orc_project(orc_state *st)
{
  const dom_struct *d = &st->dom;
  real rho_f = st->P.rho_f, dt = st->P.dt;
  real ddx = 1. / d->dx, ddy = 1. / d->dy, ddz = 1. / d->dz;
  const grid_info *X = &d->Gfx, *Y = &d->Gfy, *Z = &d->Gfz;
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = X->ks; k < X->ke; k++) for(int j = X->js; j < X->je; j++)
  for(int i = X->is; i < X->ie; i++) {
    long C = CCI(*X, i, j, k);
    real g = abs(st->flag_u[C]) * ddx * (st->phi[CCI(d->Gcc, i, j, k)]
      - st->phi[CCI(d->Gcc, i - 1, j, k)]);
    st->u[C] = st->u_star[C] - dt / rho_f * g;
  }
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = Y->ks; k < Y->ke; k++) for(int j = Y->js; j < Y->je; j++)
  for(int i = Y->is; i < Y->ie; i++) {
    long C = CCI(*Y, i, j, k);
    real g = abs(st->flag_v[C]) * ddy * (st->phi[CCI(d->Gcc, i, j, k)]
      - st->phi[CCI(d->Gcc, i, j - 1, k)]);
    st->v[C] = st->v_star[C] - dt / rho_f * g;
  }
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = Z->ks; k < Z->ke; k++) for(int j = Z->js; j < Z->je; j++)
  for(int i = Z->is; i < Z->ie; i++) {
    long C = CCI(*Z, i, j, k);
    real g = abs(st->flag_w[C]) * ddz * (st->phi[CCI(d->Gcc, i, j, k)]
      - st->phi[CCI(d->Gcc, i, j, k - 1)]);
    st->w[C] = st->w_star[C] - dt / rho_f * g;
  }
}

/* rows (or planes) 1 .. the returned index that forcing_add_c_const
 * (src/bluebottle_kernel.cu:2042) reaches under the launch shape of
 * src/cuda_bluebottle.cu:3629-3644: min(n, 16) threads, ceil(n / threads)
 * blocks, offset by the one ghost layer and bounded by the ghosted count
 * -- the interior, plus the far ghost row when n > 16 is not a multiple
 * of 16 */
static int add_const_cover(int n)
{
  int r = n < 16 ? n : (n + 15) / 16 * 16;
  return r < n + 1 ? r : n + 1;
}

/* src/cuda_bluebottle.cu:3616-3671, src/bluebottle_kernel.cu:1326-1338 and
 * forcing_add_c_const :2042 (all columns, the rows and planes
 * add_const_cover names) */
void orc_update_p(orc_state *st)
{
  const grid_info *G = &st->dom.Gcc;
  #pragma omp parallel for collapse(2) schedule(static)
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    long C = CCI(*G, i, j, k);
    st->p[C] = (st->phase[C] < 0) * (st->p0[C] + st->phi[C]);
  }
  real sum = 0.;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) sum += st->p[CCI(*G, i, j, k)];
  real mean = sum / G->s3;
  int jmax = add_const_cover(G->jn), kmax = add_const_cover(G->kn);
  for(int k = 1; k <= kmax; k++) for(int j = 1; j <= jmax; j++)
  for(int i = G->isb; i < G->ieb; i++) st->p[CCI(*G, i, j, k)] += -mean;
}

/* src/cuda_bluebottle.cu:3580-3613 */
void orc_store_u(orc_state *st)
{
  const dom_struct *d = &st->dom;
  size_t fx = d->Gfx.s3b * sizeof(real), fy = d->Gfy.s3b * sizeof(real),
         fz = d->Gfz.s3b * sizeof(real);
  memcpy(st->conv0_u, st->conv_u, fx);
  memcpy(st->conv0_v, st->conv_v, fy);
  memcpy(st->conv0_w, st->conv_w, fz);
  if(!st->P.implicit) {
    memcpy(st->diff0_u, st->diff_u, fx);
    memcpy(st->diff0_v, st->diff_v, fy);
    memcpy(st->diff0_w, st->diff_w, fz);
  }
  memcpy(st->p0, st->p, d->Gcc.s3b * sizeof(real));
  memcpy(st->u0, st->u, fx);
  memcpy(st->v0, st->v, fy);
  memcpy(st->w0, st->w, fz);
}

/* src/cuda_bluebottle.cu:3500-3577 (maximum, not maximum magnitude, over
 * the full ghosted arrays, starting from 0) */
real orc_find_dt(orc_state *st)
{
  const dom_struct *d = &st->dom;
  orc_params *P = &st->P;
  if(P->fixed_dt > 0) return P->fixed_dt;
  real umax = 0., vmax = 0., wmax = 0.;
  for(long c = 0; c < d->Gfx.s3b; c++) if(st->u[c] > umax) umax = st->u[c];
  for(long c = 0; c < d->Gfy.s3b; c++) if(st->v[c] > vmax) vmax = st->v[c];
  for(long c = 0; c < d->Gfz.s3b; c++) if(st->w[c] > wmax) wmax = st->w[c];
  real tmp;
  if(!P->implicit) {
    tmp = umax / d->dx + 2. * P->nu / d->dx / d->dx;
    tmp += vmax / d->dy + 2. * P->nu / d->dy / d->dy;
    tmp += wmax / d->dz + 2. * P->nu / d->dz / d->dz;
  } else {
    tmp = umax / d->dx;
    tmp += vmax / d->dy;
    tmp += wmax / d->dz;
  }
  real dtn = P->CFL / tmp;
  if(dtn > FLT_MAX) dtn = FLT_MAX;
  if(P->implicit && dtn > 1.1 * P->dt) dtn = 1.1 * P->dt;
  return dtn;
}

/* src/cuda_bluebottle.cu:3944-4015 with src/bluebottle_kernel.cu:
 * 3849-3905: half the mean over the cells of |u|^2, each component taken
 * to the cell centre as the average of its two faces (colocate_Gf?), the
 * squares summed u, v, w (energy_multiply) */
real orc_compute_energy(orc_state *st)
{
  const dom_struct *d = &st->dom;
  const grid_info *G = &d->Gcc;
  real e = 0.;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    real uc = 0.5 * (st->u[CCI(d->Gfx, i, j, k)] + st->u[CCI(d->Gfx, i + 1, j, k)]);
    real vc = 0.5 * (st->v[CCI(d->Gfy, i, j, k)] + st->v[CCI(d->Gfy, i, j + 1, k)]);
    real wc = 0.5 * (st->w[CCI(d->Gfz, i, j, k)] + st->w[CCI(d->Gfz, i, j, k + 1)]);
    e += uc * uc + vc * vc + wc * wc;
  }
  return e / G->s3 * 0.5;
}

void orc_divergence(orc_state *st, const real *uu, const real *vv,
  const real *ww, real *max_abs, real *l2)
{
  const dom_struct *d = &st->dom;
  real ddx = 1. / d->dx, ddy = 1. / d->dy, ddz = 1. / d->dz;
  real mx = 0., s2 = 0.;
  for(int k = d->Gcc.ks; k < d->Gcc.ke; k++)
  for(int j = d->Gcc.js; j < d->Gcc.je; j++)
  for(int i = d->Gcc.is; i < d->Gcc.ie; i++) {
    if(st->phase[CCI(d->Gcc, i, j, k)] > -1) continue;
    real s = (uu[CCI(d->Gfx, i + 1, j, k)] - uu[CCI(d->Gfx, i, j, k)]) * ddx
      + (vv[CCI(d->Gfy, i, j + 1, k)] - vv[CCI(d->Gfy, i, j, k)]) * ddy
      + (ww[CCI(d->Gfz, i, j, k + 1)] - ww[CCI(d->Gfz, i, j, k)]) * ddz;
    if(fabs(s) > mx) mx = fabs(s);
    s2 += s * s;
  }
  *max_abs = mx;
  *l2 = sqrt(s2);
}

/* one step of src/bluebottle.c:603-708 */
int orc_step(orc_state *st)
{
  orc_params *P = &st->P;
  P->ttime += P->dt;
  P->stepnum++;
  st->pp_solves = 0;
  st->pp_iters_total = 0;
  orc_compute_forcing(st);
  orc_compute_vel_BC(st);
  orc_build_cages(st);
  int iter = 0;
  real err = FLT_MAX;
  while(err > P->lamb_residual) {
    if(P->implicit) {
      orc_star_helmholtz(st, 0);
      orc_star_helmholtz(st, 1);
      orc_star_helmholtz(st, 2);
    } else {
      orc_U_star_2(st);
    }
    if(st->nparts > 0) orc_part_BC(st, 1);
    orc_dom_BC(st, 1);
    orc_solvability(st);
    if(st->nparts > 0) orc_part_BC(st, 1);
    orc_dom_BC(st, 1);
    orc_PP_bicgstab(st);
    orc_dom_BC(st, 2);
    orc_project(st);
    if(st->nparts > 0) orc_part_BC(st, 0);
    orc_dom_BC(st, 0);
    orc_update_p(st);
    if(st->nparts > 0) {
      orc_part_BC(st, 0);
      orc_part_p_fill(st);
    }
    orc_dom_BC(st, 3);
    orc_move_parts_sub(st);
    orc_Lamb(st);
    err = orc_lamb_err(st);
    iter++;
    if(iter == P->lamb_max_iter) break;
  }
  st->lamb_iters = iter;
  st->lamb_err = err;
  orc_move_parts(st);
  orc_parts_internal(st);
  orc_dom_BC(st, 0);
  orc_store_u(st);
  if(st->nparts > 0) orc_store_coeffs(st);
  P->dt0 = P->dt;
  P->dt = orc_find_dt(st);
  if(P->dt < 1.e-10 || P->dt > 1.e10) return 1;
  return 0;
}
