/* bluebottle_b200_types.h -- data types shared across the C ABI.
 *
 * These structs are the ones bluebottle's host code (bluebottle.c, domain.c,
 * particle.c) hands to its GPU layer through global variables.  Their member
 * order and types are kept identical to the reference so that the reference's
 * own time loop can link against this library unchanged:
 *   grid_info, dom_struct ........ src/domain.h:39-236
 *   g_struct, BC, gradP_struct ... src/bluebottle.h:2061-2334
 *   cage_struct, part_struct ..... src/particle.h:193-326
 * The build is FP64 only (the reference's PREC=DOUBLE, Makefile:36), so
 * `real` is double.
 */
#ifndef BLUEBOTTLE_B200_TYPES_H
#define BLUEBOTTLE_B200_TYPES_H

typedef double real;

#define BBB_PI 3.14159265358979323846
#define BBB_DIV_ST 1e-10          /* src/bluebottle.h:69 */
#define BBB_DOM_BUF 1             /* src/bluebottle.h:142 */
#define BBB_NNODES 26             /* src/particle.h:41 */
#define BBB_MAX_NEIGHBORS 12      /* src/particle.h */

/* boundary-condition codes, src/bluebottle.h:155-205 */
#define BBB_PERIODIC 0
#define BBB_DIRICHLET 1
#define BBB_NEUMANN 2
#define BBB_PRECURSOR 3
#define BBB_HOMOGENEOUS 10
#define BBB_WEST 0
#define BBB_EAST 1
#define BBB_SOUTH 2
#define BBB_NORTH 3
#define BBB_BOTTOM 4
#define BBB_TOP 5

/* initial-condition codes, src/bluebottle.h:328-352; TAYLOR_GREEN is an
 * addition of this library (3-D Taylor-Green vortex) */
#define BBB_QUIESCENT 0
#define BBB_SHEAR 1
#define BBB_CHANNEL 2
#define BBB_TAYLOR_GREEN 100

typedef struct grid_info {
  int is, ie, in, isb, ieb, inb;
  int js, je, jn, jsb, jeb, jnb;
  int ks, ke, kn, ksb, keb, knb;
  int s1, s1b, s2, s2b, s3, s3b;
  int _is, _ie, _in, _isb, _ieb, _inb;
  int _js, _je, _jn, _jsb, _jeb, _jnb;
  int _ks, _ke, _kn, _ksb, _keb, _knb;
  int _s1, _s1b, _s2, _s2b, _s3, _s3b;
} grid_info;

typedef struct dom_struct {
  grid_info Gcc;
  grid_info Gfx;
  grid_info Gfy;
  grid_info Gfz;
  real xs, xe, xl; int xn; real dx;
  real ys, ye, yl; int yn; real dy;
  real zs, ze, zl; int zn; real dz;
  int E, W, N, S, T, B;
} dom_struct;

typedef struct g_struct {
  real x, xm, xa;
  real y, ym, ya;
  real z, zm, za;
} g_struct;

typedef struct gradP_struct {
  real x, xm, xa;
  real y, ym, ya;
  real z, zm, za;
} gradP_struct;

typedef struct BC {
  int pW; real pWD; int pE; real pED; int pS; real pSD;
  int pN; real pND; int pB; real pBD; int pT; real pTD;
  int uW; real uWDm, uWD, uWDa; int uE; real uEDm, uED, uEDa;
  int uS; real uSDm, uSD, uSDa; int uN; real uNDm, uND, uNDa;
  int uB; real uBDm, uBD, uBDa; int uT; real uTDm, uTD, uTDa;
  int vW; real vWDm, vWD, vWDa; int vE; real vEDm, vED, vEDa;
  int vS; real vSDm, vSD, vSDa; int vN; real vNDm, vND, vNDa;
  int vB; real vBDm, vBD, vBDa; int vT; real vTDm, vTD, vTDa;
  int wW; real wWDm, wWD, wWDa; int wE; real wEDm, wED, wEDa;
  int wS; real wSDm, wSD, wSDa; int wN; real wNDm, wND, wNDa;
  int wB; real wBDm, wBD, wBDa; int wT; real wTDm, wTD, wTDa;
  real dsW, dsE, dsS, dsN, dsB, dsT;
} BC;

typedef struct cage_struct {
  int cx, cy, cz;
  int is, ibs, ie, ibe, in;
  int js, jbs, je, jbe, jn;
  int ks, kbs, ke, kbe, kn;
} cage_struct;

typedef struct part_struct {
  real r;
  real x, y, z;
  real x0, y0, z0;
  real u, v, w;
  real u0, v0, w0;
  real udot, vdot, wdot;
  real udot0, vdot0, wdot0;
  real axx, axy, axz, ayx, ayy, ayz, azx, azy, azz;
  real ox, oy, oz;
  real ox0, oy0, oz0;
  real oxdot, oydot, ozdot;
  real oxdot0, oydot0, ozdot0;
  real Fx, Fy, Fz;
  real Lx, Ly, Lz;
  real aFx, aFy, aFz;
  real aLx, aLy, aLz;
  real kFx, kFy, kFz;
  real iFx, iFy, iFz;
  real iLx, iLy, iLz;
  int nodes[BBB_NNODES];
  real rho;
  real E;
  real sigma;
  cage_struct cage;
  int order;
  real rs;
  int ncoeff;
  real spring_k;
  real spring_x, spring_y, spring_z;
  real spring_l;
  int translating;
  int rotating;
  int bin;
  real St[BBB_MAX_NEIGHBORS];
  int iSt[BBB_MAX_NEIGHBORS];
  real e_dry;
  real coeff_fric;
} part_struct;

#endif
