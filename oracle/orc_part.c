/* orc_part.c -- CPU FP64 oracle: Physalis particle coupling.
 * Cage/phase/flag construction (integer work), Lamb's-series boundary
 * conditions, 26-node surface quadrature, Lamb coefficients, hydrodynamic
 * force/torque, coefficient error and the Newton-Euler update.
 * TEST INFRASTRUCTURE ONLY (see orc.h). */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc.h"

#define CCI(G, i, j, k) ((i) + (j) * (G).s1b + (k) * (G).s2b)
#define PI BBB_PI
#define DIV_ST BBB_DIV_ST

/* ------------------------------------------------ cage construction
 * src/cuda_particle.cu:357-896 with kernels src/particle_kernel.cu:25-533.
 * Particles are processed in index order, so where cages overlap the
 * highest index wins. */

static void build_phase_box(orc_state *st, int p, real X, real Y, real Z,
  int is, int ie, int js, int je, int ks, int ke)
{
  const dom_struct *d = &st->dom;
  real r = st->parts[p].r;
  for(int tk = ks; tk < ke; tk++)
  for(int tj = js; tj < je; tj++)
  for(int ti = is; ti < ie; ti++) {
    if(ti < 0 || ti >= d->Gcc.inb || tj < 0 || tj >= d->Gcc.jnb || tk < 0
      || tk >= d->Gcc.knb) continue;
    real xx = (ti - 0.5) * d->dx - (X - d->xs);
    real yy = (tj - 0.5) * d->dy - (Y - d->ys);
    real zz = (tk - 0.5) * d->dz - (Z - d->zs);
    real dd = sqrt(xx * xx + yy * yy + zz * zz);
    long C = CCI(d->Gcc, ti, tj, tk);
    int cutoff = (floor(dd / r)) < 1;
    st->phase[C] = cutoff * p + (1 - cutoff) * st->phase[C];
  }
}

/* ghost copy of a cell-centred int field (cage_phases_periodic_*) */
static void periodic_cc(orc_state *st, int *f, int ax)
{
  const grid_info *G = &st->dom.Gcc;
  if(ax == 0) {
    for(int k = 0; k < G->knb; k++) for(int j = 0; j < G->jnb; j++) {
      f[CCI(*G, G->isb, j, k)] = f[CCI(*G, G->ie - 1, j, k)];
      f[CCI(*G, G->ieb - 1, j, k)] = f[CCI(*G, G->is, j, k)];
    }
  } else if(ax == 1) {
    for(int k = 0; k < G->knb; k++) for(int i = 0; i < G->inb; i++) {
      f[CCI(*G, i, G->jsb, k)] = f[CCI(*G, i, G->je - 1, k)];
      f[CCI(*G, i, G->jeb - 1, k)] = f[CCI(*G, i, G->js, k)];
    }
  } else {
    for(int j = 0; j < G->jnb; j++) for(int i = 0; i < G->inb; i++) {
      f[CCI(*G, i, j, G->ksb)] = f[CCI(*G, i, j, G->ke - 1)];
      f[CCI(*G, i, j, G->keb - 1)] = f[CCI(*G, i, j, G->ks)];
    }
  }
}

/* ghost copy of a face flag field along axis `ax`; `normal` = 1 when ax is
 * the field's own component (the duplicated face shifts the source by one,
 * cage_flag_u_periodic_x etc.) */
static void periodic_face(int *f, const grid_info *G, int ax, int normal)
{
  int sh = normal ? 1 : 0;
  if(ax == 0) {
    for(int k = 0; k < G->knb; k++) for(int j = 0; j < G->jnb; j++) {
      f[CCI(*G, G->isb, j, k)] = f[CCI(*G, G->ie - 1 - sh, j, k)];
      f[CCI(*G, G->ieb - 1, j, k)] = f[CCI(*G, G->is + sh, j, k)];
    }
  } else if(ax == 1) {
    for(int k = 0; k < G->knb; k++) for(int i = 0; i < G->inb; i++) {
      f[CCI(*G, i, G->jsb, k)] = f[CCI(*G, i, G->je - 1 - sh, k)];
      f[CCI(*G, i, G->jeb - 1, k)] = f[CCI(*G, i, G->js + sh, k)];
    }
  } else {
    for(int j = 0; j < G->jnb; j++) for(int i = 0; i < G->inb; i++) {
      f[CCI(*G, i, j, G->ksb)] = f[CCI(*G, i, j, G->ke - 1 - sh)];
      f[CCI(*G, i, j, G->keb - 1)] = f[CCI(*G, i, j, G->ks + sh)];
    }
  }
}

static void cage_extent(int n_in, real pos, real s, real dlt, int gs, int ge,
  int *cs, int *cbs, int *ce, int *cbe)
{
  int is = (int)(round((pos - s) / dlt) - 0.5 * n_in + BBB_DOM_BUF);
  int ie = is + n_in;
  int ibs, ibe;
  if(is < gs) { is = is + ge; ibs = ge; ibe = gs; }
  else if(ie > ge) { ie = ie - ge; ibs = ge; ibe = gs; }
  else { ibs = ie; ibe = ie; }
  *cs = is; *cbs = ibs; *ce = ie; *cbe = ibe;
}

void orc_build_cages(orc_state *st)
{
  const dom_struct *d = &st->dom;
  const BC *bc = &st->P.bc;
  long ncc = d->Gcc.s3b;
  for(long c = 0; c < ncc; c++) { st->phase[c] = -1; st->phase_shell[c] = 1; }
  for(long c = 0; c < d->Gfx.s3b; c++) st->flag_u[c] = 1;
  for(long c = 0; c < d->Gfy.s3b; c++) st->flag_v[c] = 1;
  for(long c = 0; c < d->Gfz.s3b; c++) st->flag_w[c] = 1;

  for(int i = 0; i < st->nparts; i++) {
    part_struct *q = &st->parts[i];
    cage_struct *cg = &q->cage;
    cg->in = (int)(2.0 * ceil(q->r / d->dx)) + 2;
    cg->jn = (int)(2.0 * ceil(q->r / d->dy)) + 2;
    cg->kn = (int)(2.0 * ceil(q->r / d->dz)) + 2;
    if(d->xn % 2) cg->in = cg->in - 1;
    if(d->yn % 2) cg->jn = cg->jn - 1;
    if(d->zn % 2) cg->kn = cg->kn - 1;
    cg->cx = (int)((q->x - d->xs + 0.5 * d->dx) / d->dx);
    cg->cy = (int)((q->y - d->ys + 0.5 * d->dy) / d->dy);
    cg->cz = (int)((q->z - d->zs + 0.5 * d->dz) / d->dz);
    cage_extent(cg->in, q->x, d->xs, d->dx, d->Gcc.is, d->Gcc.ie,
      &cg->is, &cg->ibs, &cg->ie, &cg->ibe);
    cage_extent(cg->jn, q->y, d->ys, d->dy, d->Gcc.js, d->Gcc.je,
      &cg->js, &cg->jbs, &cg->je, &cg->jbe);
    cage_extent(cg->kn, q->z, d->zs, d->dz, d->Gcc.ks, d->Gcc.ke,
      &cg->ks, &cg->kbs, &cg->ke, &cg->kbe);
  }

  int xPer = (bc->uE == BBB_PERIODIC);
  int yPer = (bc->vN == BBB_PERIODIC);
  int zPer = (bc->wT == BBB_PERIODIC);
  for(int i = 0; i < st->nparts; i++) {
    part_struct *q = &st->parts[i];
    cage_struct *c = &q->cage;
    if(c->in <= 0 || c->jn <= 0 || c->kn <= 0) continue;
    real x = q->x, y = q->y, z = q->z, r = q->r;
    real Xp = x + (x < d->xs + r) * d->xl * xPer;
    real Xm = x - d->xl * (x > (d->xe - r)) * xPer;
    real Yp = y + (y < d->ys + r) * d->yl * yPer;
    real Ym = y - d->yl * (y > (d->ye - r)) * yPer;
    real Zp = z + (z < d->zs + r) * d->zl * zPer;
    real Zm = z - d->zl * (z > (d->ze - r)) * zPer;
    int sx = c->ibe < c->ie, sy = c->jbe < c->je, sz = c->kbe < c->ke;
    build_phase_box(st, i, Xp, Yp, Zp, c->is, c->ibs, c->js, c->jbs, c->ks, c->kbs);
    if(sx) build_phase_box(st, i, Xm, Yp, Zp, c->ibe, c->ie, c->js, c->jbs, c->ks, c->kbs);
    if(sy) build_phase_box(st, i, Xp, Ym, Zp, c->is, c->ibs, c->jbe, c->je, c->ks, c->kbs);
    if(sz) build_phase_box(st, i, Xp, Yp, Zm, c->is, c->ibs, c->js, c->jbs, c->kbe, c->ke);
    if(sx && sy) build_phase_box(st, i, Xm, Ym, Zp, c->ibe, c->ie, c->jbe, c->je, c->ks, c->kbs);
    if(sx && sz) build_phase_box(st, i, Xm, Yp, Zm, c->ibe, c->ie, c->js, c->jbs, c->kbe, c->ke);
    if(sy && sz) build_phase_box(st, i, Xp, Ym, Zm, c->is, c->ibs, c->jbe, c->je, c->kbe, c->ke);
    if(sx && sy && sz) build_phase_box(st, i, Xm, Ym, Zm, c->ibe, c->ie, c->jbe, c->je, c->kbe, c->ke);
  }

  int perx = bc->uW == BBB_PERIODIC && bc->uE == BBB_PERIODIC;
  int pery = bc->uS == BBB_PERIODIC && bc->uN == BBB_PERIODIC;
  int perz = bc->uB == BBB_PERIODIC && bc->uT == BBB_PERIODIC;
  if(perx) periodic_cc(st, st->phase, 0);
  if(pery) periodic_cc(st, st->phase, 1);
  if(perz) periodic_cc(st, st->phase, 2);

  const grid_info *G = &d->Gcc;
  int *ph = st->phase, *sh = st->phase_shell;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i <= G->ie; i++) {
    long W = CCI(*G, i - 1, j, k), E = CCI(*G, i, j, k);
    sh[E] = sh[E] * (1 - (ph[W] < 0 && ph[E] > -1));
    sh[W] = sh[W] * (1 - (ph[W] > -1 && ph[E] < 0));
  }
  for(int k = G->ks; k < G->ke; k++) for(int i = G->is; i < G->ie; i++)
  for(int j = G->js; j <= G->je; j++) {
    long S = CCI(*G, i, j - 1, k), N = CCI(*G, i, j, k);
    sh[N] = sh[N] * (1 - (ph[S] < 0 && ph[N] > -1));
    sh[S] = sh[S] * (1 - (ph[S] > -1 && ph[N] < 0));
  }
  for(int j = G->js; j < G->je; j++) for(int i = G->is; i < G->ie; i++)
  for(int k = G->ks; k <= G->ke; k++) {
    long B = CCI(*G, i, j, k - 1), T = CCI(*G, i, j, k);
    sh[T] = sh[T] * (1 - (ph[B] < 0 && ph[T] > -1));
    sh[B] = sh[B] * (1 - (ph[B] > -1 && ph[T] < 0));
  }
  if(perx) periodic_cc(st, sh, 0);
  if(pery) periodic_cc(st, sh, 1);
  if(perz) periodic_cc(st, sh, 2);

#define FLAG(a, b) (1 - 2 * ((ph[a] < 0 && ph[b] > -1) || (ph[a] > -1 && ph[b] < 0) \
    || (sh[a] < 1 && sh[b] < 1)))
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i <= G->ie; i++)
    st->flag_u[CCI(d->Gfx, i, j, k)] =
      FLAG(CCI(*G, i - 1, j, k), CCI(*G, i, j, k));
  for(int k = G->ks; k < G->ke; k++) for(int i = G->is; i < G->ie; i++)
  for(int j = G->js; j <= G->je; j++)
    st->flag_v[CCI(d->Gfy, i, j, k)] =
      FLAG(CCI(*G, i, j - 1, k), CCI(*G, i, j, k));
  for(int j = G->js; j < G->je; j++) for(int i = G->is; i < G->ie; i++)
  for(int k = G->ks; k <= G->ke; k++)
    st->flag_w[CCI(d->Gfz, i, j, k)] =
      FLAG(CCI(*G, i, j, k - 1), CCI(*G, i, j, k));
#undef FLAG

  /* external (wall) faces, src/particle_kernel.cu:499-533 */
  if(bc->uW != BBB_PERIODIC && bc->uE != BBB_PERIODIC) {
    const grid_info *F = &d->Gfx;
    for(int k = 0; k < F->knb; k++) for(int j = 0; j < F->jnb; j++) {
      st->flag_u[CCI(*F, F->is, j, k)] = 0;
      st->flag_u[CCI(*F, F->ie - 1, j, k)] = 0;
    }
  }
  if(bc->vS != BBB_PERIODIC && bc->vN != BBB_PERIODIC) {
    const grid_info *F = &d->Gfy;
    for(int k = 0; k < F->knb; k++) for(int i = 0; i < F->inb; i++) {
      st->flag_v[CCI(*F, i, F->js, k)] = 0;
      st->flag_v[CCI(*F, i, F->je - 1, k)] = 0;
    }
  }
  if(bc->wB != BBB_PERIODIC && bc->wT != BBB_PERIODIC) {
    const grid_info *F = &d->Gfz;
    for(int j = 0; j < F->jnb; j++) for(int i = 0; i < F->inb; i++) {
      st->flag_w[CCI(*F, i, j, F->ks)] = 0;
      st->flag_w[CCI(*F, i, j, F->ke - 1)] = 0;
    }
  }
  /* periodic ghosts of the flags; the v test on bc.vW twice is the
   * reference's (src/cuda_particle.cu:845) */
  if(bc->uW == BBB_PERIODIC && bc->uE == BBB_PERIODIC) periodic_face(st->flag_u, &d->Gfx, 0, 1);
  if(bc->uS == BBB_PERIODIC && bc->uN == BBB_PERIODIC) periodic_face(st->flag_u, &d->Gfx, 1, 0);
  if(bc->uB == BBB_PERIODIC && bc->uT == BBB_PERIODIC) periodic_face(st->flag_u, &d->Gfx, 2, 0);
  if(bc->vW == BBB_PERIODIC && bc->vW == BBB_PERIODIC) periodic_face(st->flag_v, &d->Gfy, 0, 0);
  if(bc->vS == BBB_PERIODIC && bc->vN == BBB_PERIODIC) periodic_face(st->flag_v, &d->Gfy, 1, 1);
  if(bc->vB == BBB_PERIODIC && bc->vT == BBB_PERIODIC) periodic_face(st->flag_v, &d->Gfy, 2, 0);
  if(bc->wW == BBB_PERIODIC && bc->wE == BBB_PERIODIC) periodic_face(st->flag_w, &d->Gfz, 0, 0);
  if(bc->wS == BBB_PERIODIC && bc->wN == BBB_PERIODIC) periodic_face(st->flag_w, &d->Gfz, 1, 0);
  if(bc->wB == BBB_PERIODIC && bc->wT == BBB_PERIODIC) periodic_face(st->flag_w, &d->Gfz, 2, 1);
}

/* ------------------------------------------------ Lamb's series
 * src/particle_kernel.cu:1020-1369: normalisation N_nm, associated Legendre
 * functions P_nm (n <= 5, Condon-Shortley sign), Cartesian -> spherical, the
 * X/Y/Z angular sums of each coefficient family, and the velocity field. */

static real Nnm(int n, int m)
{
  real top = 1, bot = 1;
  for(int i = 1; i <= (n - m); i++) top *= (real)i;
  for(int i = 1; i <= (n + m); i++) bot *= (real)i;
  return sqrt((2. * n + 1.) / 4. / PI * top / bot);
}

static real Pnm(int n, int m, real theta)
{
  real x = cos(theta), y = sin(theta);
  switch(n * 10 + m) {
    case 0: return 1;
    case 10: return x;
    case 11: return -y;
    case 20: return 0.5 * (3. * x * x - 1.);
    case 21: return -3. * x * y;
    case 22: return 3. * y * y;
    case 30: return 0.5 * x * (5. * x * x - 3.);
    case 31: return -1.5 * (5. * x * x - 1.) * y;
    case 32: return 15. * x * y * y;
    case 33: return -15. * y * y * y;
    case 40: return 0.125 * (35. * x * x * x * x - 30. * x * x + 3.);
    case 41: return -2.5 * (7. * x * x - 3.) * x * y;
    case 42: return 7.5 * (7. * x * x - 1.) * y * y;
    case 43: return -105. * x * y * y * y;
    case 44: return 105. * y * y * y * y;
    case 50: return 0.125 * x * (63. * x * x * x * x - 70. * x * x + 15.);
    case 51: return -1.875 * y * (21. * x * x * x * x - 14. * x * x + 1.);
    case 52: return 52.5 * x * y * y * (3. * x * x - 1.);
    case 53: return -52.5 * y * y * y * (9. * x * x - 1.);
    case 54: return 945. * x * y * y * y * y;
    case 55: return -945. * y * y * y * y * y;
  }
  return 0;
}

static void xyz2rtp(real x, real y, real z, real *r, real *theta, real *phi)
{
  real XY = x * x + y * y;
  real XYZ = XY + z * z;
  if(XYZ >= 0 && XYZ < DIV_ST) XYZ = DIV_ST;
  *r = sqrt(XYZ);
  *theta = acos(z / *r);
  if(XY >= 0 && XY < DIV_ST) XY = DIV_ST;
  *phi = acos(x / sqrt(XY));
  if(y < 0.) *phi = 2. * PI - *phi;
}

static int coeff_base(int n) { int c = 0; for(int j = 0; j < n; j++) c += j + 1; return c; }

/* X: sum N P (re cos - im sin) with m=0 term single */
static real Xsum(int n, real theta, real phi, const real *re, const real *im,
  int pp, int stride)
{
  int c = coeff_base(n) + pp * stride;
  real sum = Nnm(n, 0) * Pnm(n, 0, theta) * re[c];
  for(int m = 1; m <= n; m++) {
    c++;
    sum += 2. * Nnm(n, m) * Pnm(n, m, theta)
      * (re[c] * cos(m * phi) - im[c] * sin(m * phi));
  }
  return sum;
}

static real clamp_st(real st)
{
  if(st >= 0 && st < DIV_ST) st = DIV_ST;
  else if(st < 0 && st > -DIV_ST) st = -DIV_ST;
  return st;
}

/* Y: theta-derivative family */
static real Ysum(int n, real theta, real phi, const real *re, const real *im,
  int pp, int stride)
{
  real ct = cos(theta);
  real st = clamp_st(sin(theta));
  int c = coeff_base(n) + pp * stride;
  int m = 0;
  real sum = Nnm(n, m)
    * (-(n + 1) * ct / st * Pnm(n, m, theta) + (n - m + 1) / st * Pnm(n + 1, m, theta))
    * re[c];
  for(m = 1; m <= n; m++) {
    c++;
    sum += 2. * Nnm(n, m)
      * (-(n + 1) * ct / st * Pnm(n, m, theta) + (n - m + 1) / st * Pnm(n + 1, m, theta))
      * (re[c] * cos(m * phi) - im[c] * sin(m * phi));
  }
  return sum;
}

/* Z: phi-derivative family */
static real Zsum(int n, real theta, real phi, const real *re, const real *im,
  int pp, int stride)
{
  real st = clamp_st(sin(theta));
  int c = coeff_base(n) + pp * stride;
  real sum = 0.;
  for(int m = 1; m <= n; m++) {
    c++;
    sum += -2. * m / st * Nnm(n, m) * Pnm(n, m, theta)
      * (re[c] * sin(m * phi) + im[c] * cos(m * phi));
  }
  return sum;
}

static void lamb_vel(int order, real a, real r, real theta, real phi, real nu,
  real *const *cf, int p, int stride, real *Ux, real *Uy, real *Uz)
{
  const real *pre = cf[0], *pim = cf[1], *fre = cf[2], *fim = cf[3],
             *cre = cf[4], *cim = cf[5];
  real ar = a / r, ra = r / a;
  real ur = 0.;
  real ut = 0.5 * ra * Ysum(0, theta, phi, pre, pim, p, stride);
  real up = 0.5 * ra * Zsum(0, theta, phi, pre, pim, p, stride);
  for(int n = 1; n <= order; n++) {
    real powranp1 = pow(ra, n + 1.);
    real powranm1 = pow(ra, n - 1.);
    real powarnp2 = pow(ar, n + 2.);
    real powarnp1 = pow(ar, n + 1.);
    real powarn = pow(ar, n);
    real od2np3 = 1. / (2. * n + 3.);
    real odnp1 = 1. / (n + 1.);
    ur += (0.5 * n * od2np3 * powranp1
      + 0.25 * n * ((2. * n + 1.) * od2np3 * ar * ar - 1.) * powarn)
      * Xsum(n, theta, phi, pre, pim, p, stride);
    ur += (n * powranm1
      + 0.5 * n * (2. * n - 1. - (2. * n + 1.) * ra * ra) * pow(ar, n + 2.))
      * Xsum(n, theta, phi, fre, fim, p, stride);
    ut += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
      + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn)
      * Ysum(n, theta, phi, pre, pim, p, stride);
    ut += (powranm1
      + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2)
      * Ysum(n, theta, phi, fre, fim, p, stride);
    ut += (powranm1 - powarnp1) * Zsum(n, theta, phi, cre, cim, p, stride);
    up += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
      + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn)
      * Zsum(n, theta, phi, pre, pim, p, stride);
    up += (powranm1
      + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2)
      * Zsum(n, theta, phi, fre, fim, p, stride);
    up += (-powranm1 + powarnp1) * Ysum(n, theta, phi, cre, cim, p, stride);
  }
  ur *= nu / a;
  ut *= nu / a;
  up *= nu / a;
  *Ux = ur * sin(theta) * cos(phi) + ut * cos(theta) * cos(phi) - up * sin(phi);
  *Uy = ur * sin(theta) * sin(phi) + ut * cos(theta) * sin(phi) + up * cos(phi);
  *Uz = ur * cos(theta) - ut * sin(theta);
}

static real wrap_rel(real x, real a, real L)
{
  if(x <= 2. * a - L) x += L;
  if(x >= L - 2. * a) x -= L;
  return x;
}

/* src/cuda_particle.cu:899-992, kernels src/particle_kernel.cu:535-838.
 * Every interior face of each component, ghost rows included, whose flag
 * is < 1 and which borders a particle cell takes the Lamb velocity plus the
 * rigid-body motion. */
void orc_part_BC(orc_state *st, int star)
{
  const dom_struct *d = &st->dom;
  real nu = st->P.nu;
  int stride = st->coeff_stride;
  real *uu = star ? st->u_star : st->u;
  real *vv = star ? st->v_star : st->v;
  real *ww = star ? st->w_star : st->w;
  const grid_info *Gc = &d->Gcc;
  for(int comp = 0; comp < 3; comp++) {
    const grid_info *G = comp == 0 ? &d->Gfx : (comp == 1 ? &d->Gfy : &d->Gfz);
    real *f = comp == 0 ? uu : (comp == 1 ? vv : ww);
    int *flag = comp == 0 ? st->flag_u : (comp == 1 ? st->flag_v : st->flag_w);
    int ilo = comp == 0 ? G->is : G->isb, ihi = comp == 0 ? G->ie : G->ieb;
    int jlo = comp == 1 ? G->js : G->jsb, jhi = comp == 1 ? G->je : G->jeb;
    int klo = comp == 2 ? G->ks : G->ksb, khi = comp == 2 ? G->ke : G->keb;
    #pragma omp parallel for collapse(2) schedule(static)
    for(int k = klo; k < khi; k++) for(int j = jlo; j < jhi; j++)
    for(int i = ilo; i < ihi; i++) {
      long C = CCI(*G, i, j, k);
      int im = i - (comp == 0), jm = j - (comp == 1), km = k - (comp == 2);
      int P0 = st->phase[CCI(*Gc, im, jm, km)];
      int P1 = st->phase[CCI(*Gc, i, j, k)];
      int P = P0 > -1 ? P0 : (P1 > -1 ? P1 : -1);
      if(P < 0 || flag[C] >= 1) continue;
      const part_struct *q = &st->parts[P];
      real a = q->r;
      real x = (comp == 0 ? (i - BBB_DOM_BUF) * d->dx : (i - 0.5) * d->dx) + d->xs - q->x;
      real y = (comp == 1 ? (j - BBB_DOM_BUF) * d->dy : (j - 0.5) * d->dy) + d->ys - q->y;
      real z = (comp == 2 ? (k - BBB_DOM_BUF) * d->dz : (k - 0.5) * d->dz) + d->zs - q->z;
      x = wrap_rel(x, a, d->xl);
      y = wrap_rel(y, a, d->yl);
      z = wrap_rel(z, a, d->zl);
      real r, theta, phi;
      xyz2rtp(x, y, z, &r, &theta, &phi);
      real Ux, Uy, Uz;
      lamb_vel(q->order, a, r, theta, phi, nu, st->coef, P, stride, &Ux, &Uy, &Uz);
      real val;
      real rr = 0.1 / nu * (r * r * r * r * r - a * a * a * a * a) / (r * r * r);
      if(comp == 0) {
        real ocr = q->oy * z - q->oz * y;
        real odcr = q->oydot * z - q->ozdot * y;
        val = Ux + q->u + ocr;
        val += rr * odcr;
      } else if(comp == 1) {
        real ocr = -(q->ox * z - q->oz * x);
        real odcr = -(q->oxdot * z - q->ozdot * x);
        val = Uy + q->v + ocr;
        val += rr * odcr;
      } else {
        real ocr = q->ox * y - q->oy * x;
        real odcr = q->oxdot * y - q->oydot * x;
        val = Uz + q->w + ocr;
        val += rr * odcr;
      }
      f[C] = val;
    }
  }
}

/* src/cuda_particle.cu:996-1017, src/particle_kernel.cu:840-940.  The
 * reference computes a Lamb pressure for shell cells and then multiplies
 * the result by (phase < 0 && phase_shell); for finite values the net
 * effect is rhs = 0 in every particle cell and unchanged elsewhere. */
void orc_part_BC_p(orc_state *st)
{
  const grid_info *G = &st->dom.Gcc;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    long CC = CCI(*G, i, j, k);
    long C = (i - 1) + (long)(j - 1) * G->s1 + (long)(k - 1) * G->s2;
    if(!(st->phase[CC] < 0 && st->phase_shell[CC])) st->rhs_p[C] = 0.;
  }
}

/* src/cuda_particle.cu:1019-1043, src/particle_kernel.cu:942-1018 */
void orc_part_p_fill(orc_state *st)
{
  const dom_struct *d = &st->dom;
  const grid_info *G = &d->Gcc;
  const orc_params *P = &st->P;
  for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
  for(int i = G->is; i < G->ie; i++) {
    long CC = CCI(*G, i, j, k);
    int p = st->phase[CC];
    if(p < 0) continue;
    const part_struct *q = &st->parts[p];
    real a = q->r;
    real x = wrap_rel((i - 0.5) * d->dx + d->xs - q->x, a, d->xl);
    real y = wrap_rel((j - 0.5) * d->dy + d->ys - q->y, a, d->yl);
    real z = wrap_rel((k - 0.5) * d->dz + d->zs - q->z, a, d->zl);
    real r, theta, phi;
    xyz2rtp(x, y, z, &r, &theta, &phi);
    real pp = Xsum(0, theta, phi, st->coef[0], st->coef[1], p, st->coeff_stride);
    pp *= P->mu * P->nu / (a * a);
    real ocr2 = (q->oy * z - q->oz * y) * (q->oy * z - q->oz * y);
    ocr2 += (q->ox * z - q->oz * x) * (q->ox * z - q->oz * x);
    ocr2 += (q->ox * y - q->oy * x) * (q->ox * y - q->oy * x);
    real rhoV = P->rho_f;
    real acc = (-P->gradP.x / rhoV - q->udot) * x + (-P->gradP.y / rhoV - q->vdot) * y
      + (-P->gradP.z / rhoV - q->wdot) * z;
    pp += 0.5 * P->rho_f * ocr2 + P->rho_f * acc;
    st->p[CC] = pp;
  }
}

/* src/cuda_bluebottle.cu:4822-4900, src/bluebottle_kernel.cu:3916-4022 */
void orc_parts_internal(orc_state *st)
{
  if(st->nparts <= 0) return;
  const dom_struct *d = &st->dom;
  const grid_info *Gc = &d->Gcc;
  for(int comp = 0; comp < 3; comp++) {
    const grid_info *G = comp == 0 ? &d->Gfx : (comp == 1 ? &d->Gfy : &d->Gfz);
    real *f = comp == 0 ? st->u : (comp == 1 ? st->v : st->w);
    int *flag = comp == 0 ? st->flag_u : (comp == 1 ? st->flag_v : st->flag_w);
    for(int k = G->ks; k < G->ke; k++) for(int j = G->js; j < G->je; j++)
    for(int i = G->is; i < G->ie; i++) {
      long C = CCI(*G, i, j, k);
      int pw = st->phase[CCI(*Gc, i - (comp == 0), j - (comp == 1), k - (comp == 2))];
      int pe = st->phase[CCI(*Gc, i, j, k)];
      int fl = flag[C];
      if(!(pw > -1 && pe > -1 && fl != -1)) continue;
      const part_struct *q = &st->parts[pe];
      real rx = (comp == 0 ? (i - BBB_DOM_BUF) * d->dx : (i - 0.5) * d->dx) + d->xs - q->x;
      real ry = (comp == 1 ? (j - BBB_DOM_BUF) * d->dy : (j - 0.5) * d->dy) + d->ys - q->y;
      real rz = (comp == 2 ? (k - BBB_DOM_BUF) * d->dz : (k - 0.5) * d->dz) + d->zs - q->z;
      rx = wrap_rel(rx, q->r, d->xl);
      ry = wrap_rel(ry, q->r, d->yl);
      rz = wrap_rel(rz, q->r, d->zl);
      if(comp == 0) f[C] = (q->oy * rz - q->oz * ry) + q->u;
      else if(comp == 1) f[C] = (q->oz * rx - q->ox * rz) + q->v;
      else f[C] = (q->ox * ry - q->oy * rx) + q->w;
    }
  }
}

/* ------------------------------------------------ quadrature
 * 26-node degree-7 Lebedev rule of src/cuda_quadrature.cu:86-150: the 6
 * axis nodes (polar ones nudged off the pole by DIV_ST), 12 edge midpoints,
 * 8 cube vertices; weights 4 pi {1/21, 4/105, 27/840}. */
void orc_quad_nodes(real *node_t, real *node_p, real *A1, real *A2, real *A3)
{
  real PI14 = 0.25 * PI, PI12 = 0.5 * PI, PI34 = 0.75 * PI,
       PI54 = 1.25 * PI, PI32 = 1.5 * PI, PI74 = 1.75 * PI;
  real alph1 = 0.955316618124509, alph2 = 2.186276035465284;
  real t1[6] = {PI12, PI12, PI12, PI12, 0. + DIV_ST, PI - DIV_ST};
  real p1[6] = {0., PI12, PI, PI32, 0., 0.};
  real t2[12] = {PI12, PI12, PI12, PI12, PI14, PI14, PI14, PI14,
    PI34, PI34, PI34, PI34};
  real p2[12] = {PI14, PI34, PI54, PI74, 0., PI12, PI, PI32, 0., PI12, PI,
    PI32};
  real t3[8] = {alph1, alph1, alph1, alph1, alph2, alph2, alph2, alph2};
  real p3[8] = {PI14, PI34, PI54, PI74, PI14, PI34, PI54, PI74};
  for(int i = 0; i < 6; i++) { node_t[i] = t1[i]; node_p[i] = p1[i]; }
  for(int i = 0; i < 12; i++) { node_t[6 + i] = t2[i]; node_p[6 + i] = p2[i]; }
  for(int i = 0; i < 8; i++) { node_t[18 + i] = t3[i]; node_p[18 + i] = p3[i]; }
  *A1 = 0.598398600683775;
  *A2 = 0.478718880547015;
  *A3 = 0.403919055461543;
}

/* src/cuda_quadrature.cu:64-313 with kernels check_nodes (:45),
 * interpolate_nodes (:95), cuda_get_coeffs (:377), cuda_calc_forces (:545) */
void orc_Lamb(orc_state *st)
{
  if(st->nparts <= 0) return;
  const dom_struct *d = &st->dom;
  const orc_params *P = &st->P;
  const BC *bc = &P->bc;
  int nnodes = BBB_NNODES;
  real node_t[BBB_NNODES], node_p[BBB_NNODES], A1, A2, A3;
  orc_quad_nodes(node_t, node_p, &A1, &A2, &A3);
  static const int nn[15] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 4};
  static const int mm[15] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3, 0, 1, 2, 3, 4};
  int np = st->nparts, stride = st->coeff_stride;
  real *pp = (real *)calloc((size_t)np * nnodes, sizeof(real));
  real *ur = (real *)calloc((size_t)np * nnodes, sizeof(real));
  real *ut = (real *)calloc((size_t)np * nnodes, sizeof(real));
  real *up = (real *)calloc((size_t)np * nnodes, sizeof(real));
  real ddx = 1. / d->dx, ddy = 1. / d->dy, ddz = 1. / d->dz;
  real mu = P->mu, nu = P->nu, rho_f = P->rho_f;

  #pragma omp parallel for schedule(static)
  for(int part = 0; part < np; part++) {
    part_struct *q = &st->parts[part];
    for(int node = 0; node < nnodes; node++) {
      real xp = q->rs * sin(node_t[node]) * cos(node_p[node]);
      real yp = q->rs * sin(node_t[node]) * sin(node_p[node]);
      real zp = q->rs * cos(node_t[node]);
      real x = xp + q->x, y = yp + q->y, z = zp + q->z;
      /* check_nodes: wall interference codes */
      q->nodes[node] = -1;
      if(x - d->xs < 0) {
        if(bc->uW == BBB_DIRICHLET || bc->vW == BBB_DIRICHLET || bc->wW == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -10;
      } if(x - d->xe > 0) {
        if(bc->uE == BBB_DIRICHLET || bc->vE == BBB_DIRICHLET || bc->wE == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -11;
      } if(y - d->ys < 0) {
        if(bc->uS == BBB_DIRICHLET || bc->vS == BBB_DIRICHLET || bc->wS == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -12;
      } if(y - d->ye > 0) {
        if(bc->uN == BBB_DIRICHLET || bc->vN == BBB_DIRICHLET || bc->wN == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -13;
      } if(z - d->zs < 0) {
        if(bc->uB == BBB_DIRICHLET || bc->vB == BBB_DIRICHLET || bc->wB == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -14;
      } if(z - d->ze > 0) {
        if(bc->uT == BBB_DIRICHLET || bc->vT == BBB_DIRICHLET || bc->wT == BBB_DIRICHLET)
          if(q->nodes[node] == -1) q->nodes[node] = -15;
      }
    }
  }

  #pragma omp parallel for schedule(static)
  for(int part = 0; part < np; part++) {
    const part_struct *q = &st->parts[part];
    real ox = q->ox, oy = q->oy, oz = q->oz;
    real oxdot = q->oxdot, oydot = q->oydot, ozdot = q->ozdot;
    real udot = q->udot, vdot = q->vdot, wdot = q->wdot;
    for(int node = 0; node < nnodes; node++) {
      int nd = q->nodes[node];
      real xp = q->rs * sin(node_t[node]) * cos(node_p[node]);
      real yp = q->rs * sin(node_t[node]) * sin(node_p[node]);
      real zp = q->rs * cos(node_t[node]);
      real x = xp + q->x, y = yp + q->y, z = zp + q->z;
      if(x < d->xs && bc->uW == BBB_PERIODIC) x = x + d->xl;
      else if(x > d->xe && bc->uE == BBB_PERIODIC) x = x - d->xl;
      if(y < d->ys && bc->vS == BBB_PERIODIC) y = y + d->yl;
      else if(y > d->ye && bc->vN == BBB_PERIODIC) y = y - d->yl;
      if(z < d->zs && bc->wB == BBB_PERIODIC) z = z + d->zl;
      else if(z > d->ze && bc->wT == BBB_PERIODIC) z = z - d->zl;
      /* pressure: cell containing the node, central-difference gradient */
      int i = (int)floor((x - d->xs) * ddx) + BBB_DOM_BUF;
      int j = (int)floor((y - d->ys) * ddy) + BBB_DOM_BUF;
      int k = (int)floor((z - d->zs) * ddz) + BBB_DOM_BUF;
      if(i < d->Gcc.is) i = d->Gcc.is;
      if(j < d->Gcc.js) j = d->Gcc.js;
      if(k < d->Gcc.ks) k = d->Gcc.ks;
      if(i > d->Gcc.ie - 1) i = d->Gcc.ie - 1;
      if(j > d->Gcc.je - 1) j = d->Gcc.je - 1;
      if(k > d->Gcc.ke - 1) k = d->Gcc.ke - 1;
      long C = CCI(d->Gcc, i, j, k);
      real xx = (i - 0.5) * d->dx + d->xs;
      real yy = (j - 0.5) * d->dy + d->ys;
      real zz = (k - 0.5) * d->dz + d->zs;
      const real *p = st->p;
      real dpdx = 0.5 * (p[C + 1] - p[C - 1]) * ddx;
      real dpdy = 0.5 * (p[C + d->Gcc.s1b] - p[C - d->Gcc.s1b]) * ddy;
      real dpdz = 0.5 * (p[C + d->Gcc.s2b] - p[C - d->Gcc.s2b]) * ddz;
      real pv = p[C] + dpdx * (x - xx) + dpdy * (y - yy) + dpdz * (z - zz);
      real ocr2 = (oy * zp - oz * yp) * (oy * zp - oz * yp);
      ocr2 += (ox * zp - oz * xp) * (ox * zp - oz * xp);
      ocr2 += (ox * yp - oy * xp) * (ox * yp - oy * xp);
      real rhoV = rho_f;
      real acc = (-P->gradP.x / rhoV - udot) * xp + (-P->gradP.y / rhoV - vdot) * yp
        + (-P->gradP.z / rhoV - wdot) * zp;
      pv -= 0.5 * rho_f * ocr2 + rho_f * acc;
      pp[node + nnodes * part] = (nd == -1) * pv;

      real rs3 = q->rs * q->rs * q->rs;
      real rs5 = rs3 * q->rs * q->rs;
      real a5 = q->r * q->r * q->r * q->r * q->r;
      real vel[3];
      const real *fld[3] = {st->u, st->v, st->w};
      const grid_info *Gs[3] = {&d->Gfx, &d->Gfy, &d->Gfz};
      real wall[3][6] = {{bc->uWD, bc->uED, bc->uSD, bc->uND, bc->uBD, bc->uTD},
        {bc->vWD, bc->vED, bc->vSD, bc->vND, bc->vBD, bc->vTD},
        {bc->wWD, bc->wED, bc->wSD, bc->wND, bc->wBD, bc->wTD}};
      real ocr[3] = {oy * zp - oz * yp, -(ox * zp - oz * xp), ox * yp - oy * xp};
      real odcr[3] = {oydot * zp - ozdot * yp, -(oxdot * zp - ozdot * xp),
        oxdot * yp - oydot * xp};
      real pu[3] = {q->u, q->v, q->w};
      for(int c = 0; c < 3; c++) {
        const grid_info *G = Gs[c];
        int ii = c == 0 ? (int)round((x - d->xs) * ddx) + BBB_DOM_BUF
                        : (int)floor((x - d->xs) * ddx) + BBB_DOM_BUF;
        int jj = c == 1 ? (int)round((y - d->ys) * ddy) + BBB_DOM_BUF
                        : (int)floor((y - d->ys) * ddy) + BBB_DOM_BUF;
        int kk = c == 2 ? (int)round((z - d->zs) * ddz) + BBB_DOM_BUF
                        : (int)floor((z - d->zs) * ddz) + BBB_DOM_BUF;
        if(ii < G->is) ii = G->is;
        if(jj < G->js) jj = G->js;
        if(kk < G->ks) kk = G->ks;
        if(ii > G->ie - 1) ii = G->ie - 1;
        if(jj > G->je - 1) jj = G->je - 1;
        if(kk > G->ke - 1) kk = G->ke - 1;
        real fx = c == 0 ? (ii - BBB_DOM_BUF) * d->dx + d->xs : (ii - 0.5) * d->dx + d->xs;
        real fy = c == 1 ? (jj - BBB_DOM_BUF) * d->dy + d->ys : (jj - 0.5) * d->dy + d->ys;
        real fz = c == 2 ? (kk - BBB_DOM_BUF) * d->dz + d->zs : (kk - 0.5) * d->dz + d->zs;
        long CF = CCI(*G, ii, jj, kk);
        const real *f = fld[c];
        real dfdx = 0.5 * (f[CF + 1] - f[CF - 1]) * ddx;
        real dfdy = 0.5 * (f[CF + G->s1b] - f[CF - G->s1b]) * ddy;
        real dfdz = 0.5 * (f[CF + G->s2b] - f[CF - G->s2b]) * ddz;
        real val = f[CF] + dfdx * (x - fx) + dfdy * (y - fy) + dfdz * (z - fz);
        real vwall = (nd == -10) * wall[c][0] + (nd == -11) * wall[c][1]
          + (nd == -12) * wall[c][2] + (nd == -13) * wall[c][3]
          + (nd == -14) * wall[c][4] + (nd == -15) * wall[c][5];
        val -= pu[c] + ocr[c];
        val -= 0.1 / nu * (rs5 - a5) / rs3 * odcr[c];
        vwall -= pu[c] + ocr[c];
        vwall -= 0.1 / nu * (rs5 - a5) / rs3 * odcr[c];
        vel[c] = (nd == -1) * val + (nd < -1) * vwall;
      }
      real stt = sin(node_t[node]), ctt = cos(node_t[node]);
      real sp = sin(node_p[node]), cp = cos(node_p[node]);
      ur[node + part * nnodes] = stt * (vel[0] * cp + vel[1] * sp) + vel[2] * ctt;
      ut[node + part * nnodes] = ctt * (vel[0] * cp + vel[1] * sp) - vel[2] * stt;
      up[node + part * nnodes] = -vel[0] * sp + vel[1] * cp;
    }
  }

  /* inner products and coefficient solve (node-0 serial sums of the
   * reference, weights A1 for nodes 0-5, A2 for 6-17, A3 for 18-25) */
  real relax = P->lamb_relax;
  #pragma omp parallel for schedule(static)
  for(int part = 0; part < np; part++) {
    part_struct *q = &st->parts[part];
    real ars = q->r / q->rs, rsa = q->rs / q->r;
    for(int coeff = 0; coeff < q->ncoeff && coeff < 15; coeff++) {
      int n = nn[coeff], m = mm[coeff];
      real I[6][BBB_NNODES];
      for(int node = 0; node < nnodes; node++) {
        real theta = node_t[node], phi = node_p[node];
        real N_nm = Nnm(n, m);
        real P_nm = Pnm(n, m, theta);
        real P_n1m = Pnm(n + 1, m, theta);
        real dPdt = (n - m + 1.) * P_n1m - (n + 1.) * cos(theta) * P_nm;
        real dPdp = m * P_nm;
        real pv = pp[node + part * nnodes], tv = ut[node + part * nnodes],
             fv = up[node + part * nnodes];
        I[0][node] = N_nm * P_nm * pv * cos(m * phi);
        I[1][node] = -N_nm * P_nm * pv * sin(m * phi);
        I[2][node] = N_nm / sin(theta) * (dPdt * tv * cos(m * phi) - dPdp * fv * sin(m * phi));
        I[3][node] = N_nm / sin(theta) * (-dPdt * tv * sin(m * phi) - dPdp * fv * cos(m * phi));
        I[4][node] = N_nm / sin(theta) * (dPdp * tv * sin(m * phi) + dPdt * fv * cos(m * phi));
        I[5][node] = N_nm / sin(theta) * (dPdp * tv * cos(m * phi) - dPdt * fv * sin(m * phi));
      }
      real S[6];
      for(int a = 0; a < 6; a++) {
        real s = I[a][0] * A1;
        for(int i = 1; i < 6; i++) s += A1 * I[a][i];
        for(int i = 6; i < 18; i++) s += A2 * I[a][i];
        for(int i = 18; i < 26; i++) s += A3 * I[a][i];
        S[a] = s;
      }
      long ci = (long)stride * part + coeff;
      real **cf = st->coef;
      real r = q->r;
      if(n == 0) {
        cf[0][ci] = cf[6][ci] + relax * (r * r / mu / nu * S[0] * pow(ars, n) - cf[6][ci]);
        cf[1][ci] = cf[7][ci] + relax * (r * r / mu / nu * S[1] * pow(ars, n) - cf[7][ci]);
        cf[2][ci] = 0.; cf[3][ci] = 0.; cf[4][ci] = 0.; cf[5][ci] = 0.;
      } else {
        real A = (1. - 0.5 * n * (2. * n - 1.) / (n + 1.) * pow(ars, 2. * n + 1.)) * pow(rsa, n);
        real B = n * (2. * n - 1.) * (2. * n + 1.) / (n + 1.) * pow(ars, n + 1.);
        real Cc = 0.25 * n * (2. * (n + 3.) / (2. * n + 3.)
          + (n - 2. - n * (2. * n + 1.) / (2. * n + 3.) * ars * ars) * pow(ars, 2. * n + 1.))
          * pow(rsa, n + 1.);
        real D = n * (n + 1. + 0.5 * ((n - 2.) * (2. * n + 1.) * rsa * rsa
          - n * (2. * n - 1.)) * pow(ars, 2. * n + 1.)) * pow(rsa, n - 1.);
        real den = A * D + B * Cc;
        real pre = (r * r / mu / nu * S[0] * D + r / nu * S[2] * B) / den;
        real pim = (r * r / mu / nu * S[1] * D + r / nu * S[3] * B) / den;
        real fre = (r / nu * S[2] * A - r * r / mu / nu * S[0] * Cc) / den;
        real fim = (r / nu * S[3] * A - r * r / mu / nu * S[1] * Cc) / den;
        real E = n * (n + 1.) * (pow(ars, 2. * n + 1.) - 1.) * pow(rsa, n);
        real cre = r / nu * S[4] / E;
        real cim = r / nu * S[5] / E;
        cf[0][ci] = cf[6][ci] * (1. - relax) + relax * pre;
        cf[1][ci] = cf[7][ci] * (1. - relax) + relax * pim;
        cf[2][ci] = cf[8][ci] * (1. - relax) + relax * fre;
        cf[3][ci] = cf[9][ci] * (1. - relax) + relax * fim;
        cf[4][ci] = cf[10][ci] * (1. - relax) + relax * cre;
        cf[5][ci] = cf[11][ci] * (1. - relax) + relax * cim;
      }
    }
    /* forces and torques, src/quadrature_kernel.cu:545-576 */
    real vol = 4. / 3. * PI * q->r * q->r * q->r;
    real N10 = sqrt(3. / 4. / PI), N11 = sqrt(3. / 8. / PI);
    real **cf = st->coef;
    long b = (long)stride * part;
    q->Fx = rho_f * vol * (q->udot + P->gradP.x)
      - PI * mu * nu * 2. * N11 * (cf[0][b + 2] + 6. * cf[2][b + 2]);
    q->Fy = rho_f * vol * (q->vdot + P->gradP.y)
      + PI * mu * nu * 2. * N11 * (cf[1][b + 2] + 6. * cf[3][b + 2]);
    q->Fz = rho_f * vol * (q->wdot + P->gradP.z)
      + PI * mu * nu * N10 * (cf[0][b + 1] + 6. * cf[2][b + 1]);
    q->Lx = rho_f * vol * q->r * q->r * q->oxdot
      - 8. * PI * mu * nu * 2. * N11 * q->r * cf[4][b + 2];
    q->Ly = rho_f * vol * q->r * q->r * q->oydot
      + 8. * PI * mu * nu * 2. * N11 * q->r * cf[5][b + 2];
    q->Lz = rho_f * vol * q->r * q->r * q->ozdot
      + 8. * PI * mu * nu * N10 * q->r * cf[4][b + 1];
  }
  free(pp); free(ur); free(ut); free(up);
}

/* src/cuda_quadrature.cu:316-398 with compute_error
 * (src/quadrature_kernel.cu:578-654).  Per particle: among its 6*stride
 * coefficients, those whose square exceeds FLT_MIN are ranked by
 * magnitude; each one larger than lamb_cut times the largest contributes
 * |c - c0| / max(|c|, 1e-16); the particle error is the largest of these
 * (at least FLT_MIN).  The reference writes its per-particle sort scratch
 * with a stride of `stride` although each particle needs 6*stride entries,
 * so neighbouring particles race; this restatement gives each particle its
 * own list, which is the computation the kernel intends. */
real orc_lamb_err(orc_state *st)
{
  if(st->nparts <= 0) return 0.;
  int stride = st->coeff_stride, np = st->nparts;
  real lamb_cut = st->P.lamb_cut;
  real maxe = FLT_MIN;
  for(int part = 0; part < np; part++) {
    real c[6 * 32], c0[6 * 32];
    for(int a = 0; a < 6; a++) for(int i = 0; i < stride; i++) {
      c[a * stride + i] = st->coef[a][(long)part * stride + i];
      c0[a * stride + i] = st->coef[6 + a][(long)part * stride + i];
    }
    int nt = 6 * stride;
    real big = -1.;
    for(int j = 0; j < nt; j++) {
      if(c[j] * c[j] > FLT_MIN && fabs(c[j]) > big) big = fabs(c[j]);
    }
    real e = FLT_MIN;
    if(big >= 0.) {
      for(int j = 0; j < nt; j++) {
        if(!(c[j] * c[j] > FLT_MIN)) continue;
        if(fabs(c[j]) > lamb_cut * big) {
          real div = fabs(c[j]);
          if(div < 1e-16) div = 1e-16;
          real er = fabs((c[j] - c0[j]) / div);
          if(er > e) e = er;
        }
      }
    }
    if(e > maxe) maxe = e;
  }
  for(int a = 0; a < 6; a++)
    memcpy(st->coef[6 + a], st->coef[a], sizeof(real) * (size_t)np * stride);
  return maxe;
}

/* src/cuda_particle.cu:1046-1081 */
void orc_store_coeffs(orc_state *st)
{
  size_t n = sizeof(real) * (size_t)st->nparts * st->coeff_stride;
  for(int a = 0; a < 6; a++) memcpy(st->coef[12 + a], st->coef[a], n);
}

/* ------------------------------------------------ interaction forces
 * src/cuda_bluebottle.cu:4317-4554 (sequence), src/bluebottle_kernel.cu:
 * collision_init :2400, bin_fill :2422, bin_start :2454, collision_parts
 * :2500, collision_walls :2875, spring_parts :3592; the bin grid of
 * binDom_init src/particle.c:598.
 *
 * Kept as the reference computes them:
 * - the kernels take interactionLengthRatio as an int (truncated), so the
 *   lubrication range hN = (int)ratio * a;
 * - the contact-list searches test iSt[q] before q < MAX_NEIGHBORS, so they
 *   read (and, in the lubrication branch, write) slot 12: the 4 bytes after
 *   iSt (the low word of e_dry) and, for St[12], the 8 bytes after St
 *   (iSt[0], iSt[1]); both are emulated byte for byte below;
 * - every wall's contact branch takes the tangential wall velocity from the
 *   south wall's Dirichlet values (bc.uSD, bc.vSD, bc.wSD);
 * - the east-wall contact torque uses the function-scope Ftx, which only an
 *   earlier lubrication branch of the same call assigns (0 there); it is 0
 *   here (the reference reads an unassigned local otherwise);
 * - the x walls' contact slip takes omega_x in place of omega_y.
 * Where the reference's new-contact search would run past slot 12 (all 12
 * slots taken) it stops at 12. */
#define ORC_MAXN BBB_MAX_NEIGHBORS

static int ist_get(const part_struct *q, int k)
{
  int v;
  memcpy(&v, (const char *)q->iSt + sizeof(int) * (size_t)k, sizeof(int));
  return v;
}
static void ist_set(part_struct *q, int k, int v)
{
  memcpy((char *)q->iSt + sizeof(int) * (size_t)k, &v, sizeof(int));
}
static real st_get(const part_struct *q, int k)
{
  real v;
  memcpy(&v, (const char *)q->St + sizeof(real) * (size_t)k, sizeof(real));
  return v;
}
static void st_set(part_struct *q, int k, real v)
{
  memcpy((char *)q->St + sizeof(real) * (size_t)k, &v, sizeof(real));
}

/* 1 while the current interaction pass emulates the reference's slot-12
 * accesses (orc_params.contact_overrun); 0 keeps the searches inside the
 * 12 slots, as the library does by default */
static int g_overrun;

/* lubrication range entered: drop `key` from the contact list */
static void contact_forget(part_struct *q, int key)
{
  int k = 0;
  if(g_overrun) {
    while(ist_get(q, k) != key && k < ORC_MAXN) k++;
    if(ist_get(q, k) == key) { ist_set(q, k, -1); st_set(q, k, 0.); }
    return;
  }
  while(k < ORC_MAXN && ist_get(q, k) != key) k++;
  if(k < ORC_MAXN) { ist_set(q, k, -1); st_set(q, k, 0.); }
}

/* contact: slot of `key`, adding it with Stokes number `St` when new;
 * without the emulation -1 when the list is full (nothing stored) */
static int contact_slot(part_struct *q, int key, real St)
{
  int k = 0;
  if(g_overrun) {
    while(ist_get(q, k) != key && k < ORC_MAXN) k++;
    if(k == ORC_MAXN) {
      k = 0;
      while(ist_get(q, k) != -1 && k < ORC_MAXN) k++;
      ist_set(q, k, key);
      st_set(q, k, St);
    }
    return k;
  }
  while(k < ORC_MAXN && ist_get(q, k) != key) k++;
  if(k < ORC_MAXN) return k;
  k = 0;
  while(k < ORC_MAXN && ist_get(q, k) != -1) k++;
  if(k == ORC_MAXN) return -1;
  ist_set(q, k, key);
  st_set(q, k, St);
  return k;
}

/* stored Stokes number of a contact slot, or St when it has none */
static real contact_st(const part_struct *q, int slot, real St)
{
  return slot >= 0 ? st_get(q, slot) : St;
}

typedef struct orc_bins {
  int xn, yn, zn, s1, s2, s3;
  real xs, ys, zs, dx, dy, dz;
  int *start, *end, *ind, *bin;
} orc_bins;

static void bins_geometry(const orc_state *st, orc_bins *B)
{
  const dom_struct *D = &st->dom;
  real rmax = 0;
  for(int i = 0; i < st->nparts; i++)
    rmax = rmax + (st->parts[i].r > rmax) * (st->parts[i].r - rmax);
  real ilr = st->P.interactionLengthRatio;
  B->xs = D->xs; B->ys = D->ys; B->zs = D->zs;
  B->xn = (int)floor(D->xl / (2. * rmax + ilr * rmax));
  if(B->xn == 0) { B->xn = 1; B->dx = D->xl; } else B->dx = D->xl / B->xn;
  B->yn = (int)floor(D->yl / (2. * rmax + ilr * rmax));
  if(B->yn == 0) { B->yn = 1; B->dy = D->yl; } else B->dy = D->yl / B->yn;
  B->zn = (int)floor(D->zl / (2. * rmax + ilr * rmax));
  if(B->zn == 0) { B->zn = 1; B->dz = D->zl; } else B->dz = D->zl / B->zn;
  B->s1 = B->xn; B->s2 = B->s1 * B->yn; B->s3 = B->s2 * B->zn;
}

/* bin of every particle, particles ordered by (bin, index) */
static void bins_fill(orc_state *st, orc_bins *B)
{
  int n = st->nparts;
  B->start = (int *)malloc(sizeof(int) * (size_t)B->s3);
  B->end = (int *)malloc(sizeof(int) * (size_t)B->s3);
  B->ind = (int *)malloc(sizeof(int) * (size_t)n);
  B->bin = (int *)malloc(sizeof(int) * (size_t)n);
  for(int c = 0; c < B->s3; c++) { B->start[c] = -1; B->end[c] = -1; }
  for(int pp = 0; pp < n; pp++) {
    part_struct *q = &st->parts[pp];
    int ib = (int)floor((q->x - B->xs) / B->dx);
    int jb = (int)floor((q->y - B->ys) / B->dy);
    int kb = (int)floor((q->z - B->zs) / B->dz);
    int c = ib + jb * B->s1 + kb * B->s2;
    q->bin = c;
    B->ind[pp] = pp;
    B->bin[pp] = c;
  }
  /* stable sort by bin (insertion: particle counts are small) */
  for(int a = 1; a < n; a++) {
    int kb = B->bin[a], ki = B->ind[a], b = a - 1;
    while(b >= 0 && B->bin[b] > kb) {
      B->bin[b + 1] = B->bin[b]; B->ind[b + 1] = B->ind[b]; b--;
    }
    B->bin[b + 1] = kb; B->ind[b + 1] = ki;
  }
  for(int a = 0; a < n; a++) {
    if(a == 0 || B->bin[a] != B->bin[a - 1]) {
      B->start[B->bin[a]] = a;
      if(a > 0) B->end[B->bin[a - 1]] = a;
    }
    if(a == n - 1) B->end[B->bin[a]] = a + 1;
  }
}

static void bins_free(orc_bins *B)
{
  free(B->start); free(B->end); free(B->ind); free(B->bin);
}

static void interaction_init(orc_state *st)
{
  for(int i = 0; i < st->nparts; i++) {
    part_struct *q = &st->parts[i];
    q->iFx = 0.; q->iFy = 0.; q->iFz = 0.;
    q->iLx = 0.; q->iLy = 0.; q->iLz = 0.;
  }
}

static void springs(orc_state *st)
{
  for(int i = 0; i < st->nparts; i++) {
    part_struct *q = &st->parts[i];
    if(!(q->spring_k > 0.)) continue;
    real nx = q->x - q->spring_x, ny = q->y - q->spring_y, nz = q->z - q->spring_z;
    real n = sqrt(nx * nx + ny * ny + nz * nz);
    real lx = q->spring_l * (nx / n), ly = q->spring_l * (ny / n),
         lz = q->spring_l * (nz / n);
    q->kFx = -q->spring_k * (q->x - q->spring_x - lx);
    q->kFy = -q->spring_k * (q->y - q->spring_y - ly);
    q->kFz = -q->spring_k * (q->z - q->spring_z - lz);
  }
}

/* nearest periodic image of the separation along one axis */
static real min_image(real a, real b, real L, int periodic)
{
  real r = a - b, r1 = a - (b + L), r2 = a - (b - L);
  if(r1 * r1 < r * r) r = r1;
  if(r2 * r2 < r * r) r = r2;
  return periodic * r + (!periodic) * (a - b);
}

/* force and torque on particle i from particle j (collision_parts body) */
static void pair_force(orc_state *st, int i, int j)
{
  const orc_params *P = &st->P;
  const dom_struct *D = &st->dom;
  part_struct *pi = &st->parts[i];
  const part_struct *pj = &st->parts[j];
  real eps = 0.01, mu = P->mu, rhof = P->rho_f, nu = P->nu, dt = P->dt;
  int ilr = (int)P->interactionLengthRatio;
  real ai = pi->r, aj = pj->r, B = aj / ai, hN = ilr * pi->r;
  real rx = min_image(pi->x, pj->x, D->xl, P->bc.uW == BBB_PERIODIC);
  real ry = min_image(pi->y, pj->y, D->yl, P->bc.vS == BBB_PERIODIC);
  real rz = min_image(pi->z, pj->z, D->zl, P->bc.wB == BBB_PERIODIC);
  real ux = 0.5 * ((pi->u - pj->u) + (pi->u0 - pj->u0));
  real uy = 0.5 * ((pi->v - pj->v) + (pi->v0 - pj->v0));
  real uz = 0.5 * ((pi->w - pj->w) + (pi->w0 - pj->w0));
  real r = sqrt(rx * rx + ry * ry + rz * rz);
  real omx = 0.5 * ((pi->ox + pj->ox) + (pi->ox0 + pj->ox0));
  real omy = 0.5 * ((pi->oy + pj->oy) + (pi->oy0 + pj->oy0));
  real omz = 0.5 * ((pi->oz + pj->oz) + (pi->oz0 + pj->oz0));
  real om = sqrt(omx * omx + omy * omy + omz * omz);
  real h = r - ai - aj;
  real nx = rx / r, ny = ry / r, nz = rz / r;
  real udotn = ux * nx + uy * ny + uz * nz;
  real unx = udotn * nx, uny = udotn * ny, unz = udotn * nz;
  real utx = ux - unx, uty = uy - uny, utz = uz - unz;
  real ut = sqrt(utx * utx + uty * uty + utz * utz);
  real tx, ty, tz, bx, by, bz;
  if(ut > 0) {
    tx = utx / ut; ty = uty / ut; tz = utz / ut;
    bx = ny * tz - nz * ty; by = -nx * tz + nz * tx; bz = nx * ty - ny * tx;
    real b = sqrt(bx * bx + by * by + bz * bz);
    bx = bx / b; by = by / b; bz = bz / b;
  } else if(om > 0) {
    bx = omx / om; by = omy / om; bz = omz / om;
    tx = by * nz - bz * ny; ty = -bx * nz + bz * nx; tz = bx * ny - by * nx;
    real t = sqrt(tx * tx + ty * ty + tz * tz);
    tx = tx / t; ty = ty / t; tz = tz / t;
  } else {
    tx = 1.; ty = 0.; tz = 0.;
    bx = ny * tz - nz * ty; by = -nx * tz + nz * tx; bz = nx * ty - ny * tx;
    real b = sqrt(bx * bx + by * by + bz * bz);
    bx = bx / b; by = by / b; bz = bz / b;
  }
  (void)bx; (void)by; (void)bz;
  real opB = 1 + B;
  real ocnx = omy * nz - omz * ny, ocny = -omx * nz + omz * nx, ocnz = omx * ny - omy * nx;
  real ucnx = uty * nz - utz * ny, ucny = -utx * nz + utz * nx, ucnz = utx * ny - uty * nx;
  real Fnx, Fny, Fnz, Ftx, Fty, Ftz, Lox, Loy, Loz;
  if(h < hN && h > 0) {
    contact_forget(pi, j);
    if(h < eps * pi->r) h = eps * pi->r;
    real ah = ai / h - ai / hN, lnah = log(hN / h);
    Fnx = -1. * B * B / (opB * opB) * ah - B * (1. + 7. * B + B * B) / (5. * opB * opB * opB) * lnah;
    Fny = Fnx; Fnz = Fnx;
    Fnx *= 6. * PI * mu * ai * unx;
    Fny *= 6. * PI * mu * ai * uny;
    Fnz *= 6. * PI * mu * ai * unz;
    Ftx = -6. * PI * mu * ai * utx * 4. * B * (2. + B + 2. * B * B) / (15. * opB * opB * opB) * lnah;
    Fty = -6. * PI * mu * ai * uty * 4. * B * (2. + B + 2. * B * B) / (15. * opB * opB * opB) * lnah;
    Ftz = -6. * PI * mu * ai * utz * 4. * B * (2. + B + 2. * B * B) / (15. * opB * opB * opB) * lnah;
    Ftx += 8. * PI * mu * ai * ai * ocnx * B * (4. + B) / (10. * opB * opB) * lnah;
    Fty += 8. * PI * mu * ai * ai * ocny * B * (4. + B) / (10. * opB * opB) * lnah;
    Ftz += 8. * PI * mu * ai * ai * ocnz * B * (4. + B) / (10. * opB * opB) * lnah;
    Lox = -8. * PI * mu * ai * ai * ucnx * B * (4. + B) / (10. * opB * opB) * lnah;
    Loy = -8. * PI * mu * ai * ai * ucny * B * (4. + B) / (10. * opB * opB) * lnah;
    Loz = -8. * PI * mu * ai * ai * ucnz * B * (4. + B) / (10. * opB * opB) * lnah;
    Lox += -8. * PI * mu * ai * ai * ai * omx * 2. * B / (5. * opB) * lnah;
    Loy += -8. * PI * mu * ai * ai * ai * omy * 2. * B / (5. * opB) * lnah;
    Loz += -8. * PI * mu * ai * ai * ai * omz * 2. * B / (5. * opB) * lnah;
  } else {
    Fnx = 0; Fny = 0; Fnz = 0; Ftx = 0; Fty = 0; Ftz = 0; Lox = 0; Loy = 0; Loz = 0;
  }
  if(h < 0) {
    real St_now = 1. / 9. * pi->rho / rhof * 2. * pi->r * fabs(udotn) / nu;
    int q = contact_slot(pi, j, St_now);
    real Vx = -utx + 0.5 * (ai + aj + h) * ocnx;
    real Vy = -uty + 0.5 * (ai + aj + h) * ocny;
    real Vz = -utz + 0.5 * (ai + aj + h) * ocnz;
    real Hi = 0.5 * pi->E / (1. + pi->sigma);
    real kt = 8. / ((1. - pi->sigma * pi->sigma) / Hi + (1. - pi->sigma * pi->sigma) / Hi)
      / sqrt(1. / ai) * sqrt(-h);
    real Vdotn = Vx * nx + Vy * ny + Vz * nz;
    real sx = (Vx - Vdotn * nx) * dt, sy = (Vy - Vdotn * ny) * dt, sz = (Vz - Vdotn * nz) * dt;
    real k = 4. / 3. / ((1. - pi->sigma * pi->sigma) / pi->E
      + (1. - pj->sigma * pj->sigma) / pj->E) / sqrt(1. / ai + 1. / aj);
    real xcx0 = 1.e-4;
    real e = pi->e_dry + (1. + pi->e_dry) / contact_st(pi, q, St_now) * log(xcx0);
    if(e < 0) e = 0;
    real alpha = -2.263 * pow(e, 0.3948) + 2.22;
    real eta = alpha * sqrt(4. / 3. * PI * ai * ai * ai * pi->rho * k * sqrt(-h));
    Fnx = (sqrt(-h * h * h) * k - eta * udotn) * nx;
    Fny = (sqrt(-h * h * h) * k - eta * udotn) * ny;
    Fnz = (sqrt(-h * h * h) * k - eta * udotn) * nz;
    real cf = 0.5 * (pi->coeff_fric + pj->coeff_fric);
    Ftx = -kt * sx; Fty = -kt * sy; Ftz = -kt * sz;
    real Ftdotn = Ftx * nx + Fty * ny + Ftz * nz;
    Ftx = Ftx - Ftdotn * nx; Fty = Fty - Ftdotn * ny; Ftz = Ftz - Ftdotn * nz;
    real Ft = sqrt(Ftx * Ftx + Fty * Fty + Ftz * Ftz);
    real Fn = sqrt(Fnx * Fnx + Fny * Fny + Fnz * Fnz);
    if(Ft > cf * Fn) {
      Ftx = cf * Fn * Ftx / Ft; Fty = cf * Fn * Fty / Ft; Ftz = cf * Fn * Ftz / Ft;
    }
    Lox = -(ai + 0.5 * h) * ((Fny + Fty) * nz - (Fnz + Ftz) * ny);
    Loy = (ai + 0.5 * h) * ((Fnx + Ftx) * nz - (Fnz + Ftz) * nx);
    Loz = -(ai + 0.5 * h) * ((Fnx + Ftx) * ny - (Fny + Fty) * nx);
  }
  pi->iFx += Fnx + Ftx;
  pi->iFy += Fny + Fty;
  pi->iFz += Fnz + Ftz;
  pi->iLx += Lox;
  pi->iLy += Loy;
  pi->iLz += Loz;
}

/* neighbour bins in the reference's order (z, y, x; -1..1), wrapping only
 * across periodic faces with more than two bins */
static void collide_parts(orc_state *st, const orc_bins *B)
{
  const BC *bc = &st->P.bc;
  int fW = 0, fE = B->xn - 1, fS = 0, fN = B->yn - 1, fB = 0, fT = B->zn - 1;
  int xnb = B->xn > 2, ynb = B->yn > 2, znb = B->zn > 2;
  for(int index = 0; index < st->nparts; index++) {
    int i = B->ind[index], bin = B->bin[index];
    int kbin = bin / B->s2, jbin = (bin - kbin * B->s2) / B->s1;
    int ibin = bin - kbin * B->s2 - jbin * B->s1;
    for(int n = -1; n <= 1; n++) {
      int ks;
      if((n == -1 && kbin == fB && bc->uB != BBB_PERIODIC) ||
         (n == 1 && kbin == fT && bc->uT != BBB_PERIODIC) ||
         (n == -1 && kbin == fB && bc->uB == BBB_PERIODIC && znb == 0) ||
         (n == 1 && kbin == fT && bc->uT == BBB_PERIODIC && znb == 0)) continue;
      else if(n == -1 && kbin == fB) ks = fT * B->s2;
      else if(n == 1 && kbin == fT) ks = fB * B->s2;
      else ks = (kbin + n) * B->s2;
      for(int m = -1; m <= 1; m++) {
        int js;
        if((m == -1 && jbin == fS && bc->uS != BBB_PERIODIC) ||
           (m == 1 && jbin == fN && bc->uN != BBB_PERIODIC) ||
           (m == -1 && jbin == fS && bc->uS == BBB_PERIODIC && ynb == 0) ||
           (m == 1 && jbin == fN && bc->uN == BBB_PERIODIC && ynb == 0)) continue;
        else if(m == -1 && jbin == fS) js = fN * B->s1;
        else if(m == 1 && jbin == fN) js = fS * B->s1;
        else js = (jbin + m) * B->s1;
        for(int l = -1; l <= 1; l++) {
          int is;
          if((l == -1 && ibin == fW && bc->uW != BBB_PERIODIC) ||
             (l == 1 && ibin == fE && bc->uE != BBB_PERIODIC) ||
             (l == -1 && ibin == fW && bc->uW == BBB_PERIODIC && xnb == 0) ||
             (l == 1 && ibin == fE && bc->uE == BBB_PERIODIC && xnb == 0)) continue;
          else if(l == -1 && ibin == fW) is = fE;
          else if(l == 1 && ibin == fE) is = fW;
          else is = ibin + l;
          int adj = is + js + ks;
          if(B->start[adj] == -1) continue;
          for(int t = B->start[adj]; t < B->end[adj]; t++) {
            int j = B->ind[t];
            if(j != i) pair_force(st, i, j);
          }
        }
      }
    }
  }
}

/* one wall (collision_walls).  ax: normal axis 0/1/2; hi: 0 for the W/S/B
 * wall, 1 for E/N/T; key -10..-15. */
static void wall_force(orc_state *st, part_struct *p, int ax, int hi, real *Ftx_scope)
{
  const orc_params *P = &st->P;
  const dom_struct *D = &st->dom;
  const BC *bc = &P->bc;
  real eps = 0.01, mu = P->mu, rhof = P->rho_f, nu = P->nu, dt = P->dt;
  int ilr = (int)P->interactionLengthRatio;
  real ai = p->r, hN = ilr * p->r;
  real pos[3] = {p->x, p->y, p->z}, vel[3] = {p->u, p->v, p->w};
  real vel0[3] = {p->u0, p->v0, p->w0};
  real om[3] = {p->ox, p->oy, p->oz}, om0[3] = {p->ox0, p->oy0, p->oz0};
  real wallpos, ds;
  int press;
  /* Dirichlet wall velocities of this wall, per component */
  real wv[3];
  int key = -10 - (2 * ax + hi);
  if(ax == 0) {
    ds = hi ? bc->dsE : bc->dsW;
    wallpos = hi ? D->xe - ds : D->xs + ds;
    press = hi ? bc->pE : bc->pW;
    wv[0] = hi ? bc->uED : bc->uWD; wv[1] = hi ? bc->vED : bc->vWD; wv[2] = hi ? bc->wED : bc->wWD;
  } else if(ax == 1) {
    ds = hi ? bc->dsN : bc->dsS;
    wallpos = hi ? D->ye - ds : D->ys + ds;
    press = hi ? bc->pN : bc->pS;
    wv[0] = hi ? bc->uND : bc->uSD; wv[1] = hi ? bc->vND : bc->vSD; wv[2] = hi ? bc->wND : bc->wSD;
  } else {
    ds = hi ? bc->dsT : bc->dsB;
    wallpos = hi ? D->ze - ds : D->zs + ds;
    press = hi ? bc->pT : bc->pB;
    wv[0] = hi ? bc->uTD : bc->uBD; wv[1] = hi ? bc->vTD : bc->vBD; wv[2] = hi ? bc->wTD : bc->wBD;
  }
  real sd[3] = {bc->uSD, bc->vSD, bc->wSD};
  real h = fabs(pos[ax] - wallpos) - ai;
  real isTrue = (press == BBB_NEUMANN);
  /* tangential axes in the reference's order and the sign pattern of the
   * rotation terms: lo walls (W, S, B) and hi walls mirror each other */
  int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
  real sg = hi ? -1. : 1.;
  if(h < hN && h > 0) {
    contact_forget(p, key);
    if(h < eps * p->r) h = eps * p->r;
    real ah = ai / h - ai / hN, lnah = log(hN / h);
    real Un = vel[ax] - wv[ax];
    real Ut[3] = {vel[0] - wv[0], vel[1] - wv[1], vel[2] - wv[2]};
    Ut[ax] = 0.;
    real F[3] = {0., 0., 0.}, Ft[3] = {0., 0., 0.}, L[3] = {0., 0., 0.};
    F[ax] = -6. * PI * mu * ai * Un * ah;
    Ft[t1] = -6. * PI * mu * ai * Ut[t1] * 8. / 15. * lnah;
    Ft[t2] = -6. * PI * mu * ai * Ut[t2] * 8. / 15. * lnah;
    /* rotation coupling: (t1, t2) = (y, z) for x walls, (x, z) for y walls,
     * (x, y) for z walls; the y walls carry the opposite orientation */
    real so = (ax == 1) ? -sg : sg;
    Ft[t1] += so * 8. * PI * mu * ai * ai * om[t2] * 1. / 10. * lnah;
    Ft[t2] += -so * 8. * PI * mu * ai * ai * om[t1] * 1. / 10. * lnah;
    L[t1] = -so * 8. * PI * mu * ai * ai * Ut[t2] * 1. / 10. * lnah;
    L[t2] = so * 8. * PI * mu * ai * ai * Ut[t1] * 1. / 10. * lnah;
    L[t1] += -8. * PI * mu * ai * ai * ai * om[t1] * 2. / 5. * lnah;
    L[t2] += -8. * PI * mu * ai * ai * ai * om[t2] * 2. / 5. * lnah;
    *Ftx_scope = Ft[0];
    p->iFx += isTrue * (F[0] + Ft[0]);
    p->iFy += isTrue * (F[1] + Ft[1]);
    p->iFz += isTrue * (F[2] + Ft[2]);
    p->iLx += isTrue * L[0];
    p->iLy += isTrue * L[1];
    p->iLz += isTrue * L[2];
  }
  if(h < 0) {
    real Un = sg * (vel[ax] - wv[ax]);
    real Ut1 = 0.5 * (vel[t1] + vel0[t1]) - sd[t1];
    real Ut2 = 0.5 * (vel[t2] + vel0[t2]) - sd[t2];
    real St_now = 1. / 9. * p->rho / rhof * 2. * p->r * fabs(Un) / nu;
    int q = contact_slot(p, key, St_now);
    real o[3] = {0.5 * (om[0] + om0[0]), 0.5 * (om[1] + om0[1]), 0.5 * (om[2] + om0[2])};
    /* slip velocity at the contact point; the x walls take omega_x where
     * omega_y belongs (src/bluebottle_kernel.cu:2977, :3091) */
    real so = (ax == 1) ? -1. : 1.;
    real o2 = ax == 0 ? o[0] : o[t1];
    real V1 = sg * (Ut1 - so * (ai + 0.5 * h) * o[t2]);
    real V2 = sg * (Ut2 + so * (ai + 0.5 * h) * o2);
    real Hi = 0.5 * p->E / (1. + p->sigma);
    real kt = 8. / ((1. - p->sigma * p->sigma) / Hi + (1. - p->sigma * p->sigma) / Hi)
      / sqrt(1. / ai) * sqrt(-h);
    real s1 = V1 * dt, s2 = V2 * dt;
    real k = 4. / 3. / ((1. - p->sigma * p->sigma) / p->E + (1. - p->sigma * p->sigma) / p->E)
      / sqrt(1. / ai);
    real xcx0 = 1.e-4;
    real e = p->e_dry + (1. + p->e_dry) / contact_st(p, q, St_now) * log(xcx0);
    if(e < 0) e = 0;
    real alpha = -2.263 * pow(e, 0.3948) + 2.22;
    real eta = alpha * sqrt(4. / 3. * PI * ai * ai * ai * p->rho * k * sqrt(-h));
    real cf = p->coeff_fric;
    real F1 = -kt * s1, F2 = -kt * s2;
    real Ft = sqrt(F1 * F1 + F2 * F2);
    real Fn = sqrt(-h * h * h) * k - eta * Un;
    if(Ft > fabs(cf * Fn)) {
      F1 = cf * Fn * F1 / Ft;
      F2 = cf * Fn * F2 / Ft;
    }
    real arm = ai + 0.5 * h;
    if(ax == 0) {
      p->iFx += sg * isTrue * Fn;
      p->iFy += isTrue * F1;
      p->iFz += isTrue * F2;
      if(!hi) { p->iLy += isTrue * arm * F2; p->iLz -= isTrue * arm * F1; }
      else { p->iLy -= isTrue * arm * F2; p->iLz += isTrue * arm * (*Ftx_scope); }
    } else if(ax == 1) {
      p->iFx += isTrue * F1;
      p->iFy += sg * isTrue * Fn;
      p->iFz += isTrue * F2;
      if(!hi) { p->iLx -= isTrue * arm * F2; p->iLz += isTrue * arm * F1; }
      else { p->iLx += isTrue * arm * F2; p->iLz -= isTrue * arm * F1; }
    } else {
      p->iFx += isTrue * F1;
      p->iFy += isTrue * F2;
      p->iFz += sg * isTrue * Fn;
      if(!hi) { p->iLx += isTrue * arm * F2; p->iLy -= isTrue * arm * F1; }
      else { p->iLx -= isTrue * arm * F2; p->iLy += isTrue * arm * F1; }
    }
  }
}

static void collide_walls(orc_state *st)
{
  for(int i = 0; i < st->nparts; i++) {
    real Ftx_scope = 0.;
    for(int w = 0; w < 6; w++) wall_force(st, &st->parts[i], w / 2, w % 2, &Ftx_scope);
  }
}

static void rotate(real qr, real qi, real qj, real qk, real *pi, real *pj,
  real *pk)
{
  real Pr = *pi * qi + *pj * qj + *pk * qk;
  real Pi = *pi * qr - *pj * qk + *pk * qj;
  real Pj = *pi * qk + *pj * qr - *pk * qi;
  real Pk = -*pi * qj + *pj * qi + *pk * qr;
  *pi = qr * Pi + qi * Pr + qj * Pk - qk * Pj;
  *pj = qr * Pj - qi * Pk + qj * Pr + qk * Pi;
  *pk = qr * Pk + qi * Pj - qj * Pi + qk * Pr;
}

static void move_parts(orc_state *st, int final)
{
  const dom_struct *d = &st->dom;
  const orc_params *P = &st->P;
  real dt = P->dt;
  for(int pp = 0; pp < st->nparts; pp++) {
    part_struct *q = &st->parts[pp];
    real vol = 4. / 3. * PI * q->r * q->r * q->r;
    real m = vol * q->rho;
    if(q->translating) {
      q->udot = (q->Fx + q->kFx + q->iFx + q->aFx - vol * P->gradP.x) / m
        + (q->rho - P->rho_f) / q->rho * P->g.x;
      q->vdot = (q->Fy + q->kFy + q->iFy + q->aFy - vol * P->gradP.y) / m
        + (q->rho - P->rho_f) / q->rho * P->g.y;
      q->wdot = (q->Fz + q->kFz + q->iFz + q->aFz - vol * P->gradP.z) / m
        + (q->rho - P->rho_f) / q->rho * P->g.z;
      q->u = q->u0 + 0.5 * dt * (q->udot + q->udot0);
      q->v = q->v0 + 0.5 * dt * (q->vdot + q->vdot0);
      q->w = q->w0 + 0.5 * dt * (q->wdot + q->wdot0);
      if(final) {
        q->x = q->x0 + 0.5 * dt * (q->u + q->u0);
        if(q->x < d->xs) q->x = q->x + d->xl;
        else if(q->x > d->xe) q->x = q->x - d->xl;
        q->y = q->y0 + 0.5 * dt * (q->v + q->v0);
        if(q->y < d->ys) q->y = q->y + d->yl;
        else if(q->y > d->ye) q->y = q->y - d->yl;
        q->z = q->z0 + 0.5 * dt * (q->w + q->w0);
        if(q->z < d->zs) q->z = q->z + d->zl;
        else if(q->z > d->ze) q->z = q->z - d->zl;
        q->x0 = q->x; q->y0 = q->y; q->z0 = q->z;
        q->u0 = q->u; q->v0 = q->v; q->w0 = q->w;
        q->udot0 = q->udot; q->vdot0 = q->vdot; q->wdot0 = q->wdot;
      }
    }
    if(q->rotating) {
      real I = 0.4 * m * q->r * q->r;
      q->oxdot = (q->Lx + q->iLx + q->aLx) / I;
      q->oydot = (q->Ly + q->iLy + q->aLy) / I;
      q->ozdot = (q->Lz + q->iLz + q->aLz) / I;
      q->ox = q->ox0 + 0.5 * dt * (q->oxdot + q->oxdot0);
      q->oy = q->oy0 + 0.5 * dt * (q->oydot + q->oydot0);
      q->oz = q->oz0 + 0.5 * dt * (q->ozdot + q->ozdot0);
      if(final) {
        real mag = 0.5 * sqrt(q->ox * q->ox + q->oy * q->oy + q->oz * q->oz);
        mag += 0.5 * sqrt(q->ox0 * q->ox0 + q->oy0 * q->oy0 + q->oz0 * q->oz0);
        real X = 0, Y = 0, Z = 0;
        if(mag > 0) {
          X = 0.5 * (q->ox + q->ox0) / mag;
          Y = 0.5 * (q->oy + q->oy0) / mag;
          Z = 0.5 * (q->oz + q->oz0) / mag;
        }
        real theta = mag * dt;
        real qr = cos(0.5 * theta);
        real qi = X * sin(0.5 * theta);
        real qj = Y * sin(0.5 * theta);
        real qk = Z * sin(0.5 * theta);
        rotate(qr, qi, qj, qk, &q->axx, &q->axy, &q->axz);
        rotate(qr, qi, qj, qk, &q->ayx, &q->ayy, &q->ayz);
        rotate(qr, qi, qj, qk, &q->azx, &q->azy, &q->azz);
        q->ox0 = q->ox; q->oy0 = q->oy; q->oz0 = q->oz;
        q->oxdot0 = q->oxdot; q->oydot0 = q->oydot; q->ozdot0 = q->ozdot;
      }
    }
  }
}

/* src/cuda_bluebottle.cu:4317-4433: interaction forces, the first
 * Newton-Euler half step, interaction forces again; the final call adds
 * the position update (move_parts_b) */
static void interactions(orc_state *st, int final)
{
  int n = st->nparts;
  if(n <= 0) return;
  g_overrun = st->P.contact_overrun;
  orc_bins B;
  memset(&B, 0, sizeof(B));
  if(n > 1) {
    bins_geometry(st, &B);
    bins_fill(st, &B);
  }
  for(int pass = 0; pass < 2; pass++) {
    interaction_init(st);
    if(n > 1) collide_parts(st, &B);
    springs(st);
    collide_walls(st);
    if(pass == 0) move_parts(st, 0);
  }
  if(n > 1) bins_free(&B);
  if(final) move_parts(st, 1);
}

void orc_move_parts_sub(orc_state *st)
{
  interactions(st, 0);
}

/* src/cuda_bluebottle.cu:4435-4554 */
void orc_move_parts(orc_state *st)
{
  interactions(st, 1);
}
