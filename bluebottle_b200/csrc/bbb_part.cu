/* bbb_part.cu -- Physalis particle coupling on the device.
 *
 *  - cage build (src/cuda_particle.cu:357-896): the reference computes the
 *    cage extents on the host and launches up to seven build_phase kernels
 *    per particle from a host loop; here one kernel computes every extent
 *    and one CTA per particle marks its cells.  Overlapping cages resolve
 *    to the highest particle index (atomicMax), which is what the
 *    reference's index-ordered launches produce.  Distances use explicitly
 *    rounded operations (no fused multiply-add) so the integer results
 *    (phase, phase_shell, flag_u/v/w) match an FP64 CPU evaluation bit for
 *    bit.
 *  - Lamb boundary velocities, internal rigid-body fill and the in-particle
 *    pressure (src/particle_kernel.cu:535-1018, src/bluebottle_kernel.cu:
 *    3916-4022).
 *  - quadrature, coefficients and forces (src/quadrature_kernel.cu:45-576)
 *    with one 32-thread block per particle, node per lane.
 *  - coefficient error (src/quadrature_kernel.cu:578-654) and the
 *    Newton-Euler update (src/bluebottle_kernel.cu:2247-2398).
 */
#include <float.h>
#include <math.h>
#include <string.h>
#include "bbb_internal.h"
#include "bbb_reduce.cuh"

#define PI BBB_PI
#define DIV_ST BBB_DIV_ST

/* ------------------------------------------------ cage build */

__global__ void k_reset_cages(int *phs, int *shl, long long ncc, int *fu,
  long long nfx, int *fv, long long nfy, int *fw, long long nfz)
{
  long long st = (long long)gridDim.x * blockDim.x;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncc; t += st) {
    phs[t] = -1; shl[t] = 1;
  }
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nfx; t += st) fu[t] = 1;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nfy; t += st) fv[t] = 1;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nfz; t += st) fw[t] = 1;
}

__device__ __forceinline__ void cage_extent(int n_in, double pos, double s,
  double dlt, int gs, int ge, int *cs, int *cbs, int *ce, int *cbe)
{
  double q = round(__ddiv_rn(__dsub_rn(pos, s), dlt));
  int is = (int)__dadd_rn(__dsub_rn(q, __dmul_rn(0.5, (double)n_in)), (double)BBB_DOM_BUF);
  int ie = is + n_in;
  int ibs, ibe;
  if(is < gs) { is = is + ge; ibs = ge; ibe = gs; }
  else if(ie > ge) { ie = ie - ge; ibs = ge; ibe = gs; }
  else { ibs = ie; ibe = ie; }
  *cs = is; *cbs = ibs; *ce = ie; *cbe = ibe;
}

/* cage extents, src/cuda_particle.cu:462-531 */
__global__ void k_cage_extents(part_struct *parts, int np, bbb_geom G,
  int gis, int gie, int gjs, int gje, int gks, int gke)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= np) return;
  part_struct *q = &parts[i];
  cage_struct c;
  c.in = (int)(2.0 * ceil(__ddiv_rn(q->r, G.dx))) + 2;
  c.jn = (int)(2.0 * ceil(__ddiv_rn(q->r, G.dy))) + 2;
  c.kn = (int)(2.0 * ceil(__ddiv_rn(q->r, G.dz))) + 2;
  if(G.nx % 2) c.in = c.in - 1;
  if(G.ny % 2) c.jn = c.jn - 1;
  if(G.nz % 2) c.kn = c.kn - 1;
  c.cx = (int)__ddiv_rn(__dadd_rn(__dsub_rn(q->x, G.xs), __dmul_rn(0.5, G.dx)), G.dx);
  c.cy = (int)__ddiv_rn(__dadd_rn(__dsub_rn(q->y, G.ys), __dmul_rn(0.5, G.dy)), G.dy);
  c.cz = (int)__ddiv_rn(__dadd_rn(__dsub_rn(q->z, G.zs), __dmul_rn(0.5, G.dz)), G.dz);
  cage_extent(c.in, q->x, G.xs, G.dx, gis, gie, &c.is, &c.ibs, &c.ie, &c.ibe);
  cage_extent(c.jn, q->y, G.ys, G.dy, gjs, gje, &c.js, &c.jbs, &c.je, &c.jbe);
  cage_extent(c.kn, q->z, G.zs, G.dz, gks, gke, &c.ks, &c.kbs, &c.ke, &c.kbe);
  q->cage = c;
}

/* one CTA per particle: the (up to eight) periodic pieces of its cage,
 * src/cuda_particle.cu:544-667 with build_phase src/particle_kernel.cu:93 */
__global__ void k_build_phase(const part_struct *parts, int *phs, bbb_geom G,
  int xPer, int yPer, int zPer)
{
  int p = blockIdx.x;
  const part_struct *q = &parts[p];
  cage_struct c = q->cage;
  if(c.in <= 0 || c.jn <= 0 || c.kn <= 0) return;
  double x = q->x, y = q->y, z = q->z, r = q->r;
  double Xp = __dadd_rn(x, (double)(x < __dadd_rn(G.xs, r)) * G.xl * xPer);
  double Xm = __dsub_rn(x, G.xl * (double)(x > __dsub_rn(G.xe, r)) * xPer);
  double Yp = __dadd_rn(y, (double)(y < __dadd_rn(G.ys, r)) * G.yl * yPer);
  double Ym = __dsub_rn(y, G.yl * (double)(y > __dsub_rn(G.ye, r)) * yPer);
  double Zp = __dadd_rn(z, (double)(z < __dadd_rn(G.zs, r)) * G.zl * zPer);
  double Zm = __dsub_rn(z, G.zl * (double)(z > __dsub_rn(G.ze, r)) * zPer);
  int sx = c.ibe < c.ie, sy = c.jbe < c.je, sz = c.kbe < c.ke;
  for(int piece = 0; piece < 8; piece++) {
    int px = piece & 1, py = (piece >> 1) & 1, pz = (piece >> 2) & 1;
    if((px && !sx) || (py && !sy) || (pz && !sz)) continue;
    int is = px ? c.ibe : c.is, ie = px ? c.ie : c.ibs;
    int js = py ? c.jbe : c.js, je = py ? c.je : c.jbs;
    int ks = pz ? c.kbe : c.ks, ke = pz ? c.ke : c.kbs;
    double X = px ? Xm : Xp, Y = py ? Ym : Yp, Z = pz ? Zm : Zp;
    int ni = ie - is, nj = je - js, nk = ke - ks;
    if(ni <= 0 || nj <= 0 || nk <= 0) continue;
    double cxo = __dsub_rn(X, G.xs), cyo = __dsub_rn(Y, G.ys), czo = __dsub_rn(Z, G.zs);
    long long tot = (long long)ni * nj * nk;
    for(long long t = threadIdx.x; t < tot; t += blockDim.x) {
      int ti = is + (int)(t % ni);
      long long rr = t / ni;
      int tj = js + (int)(rr % nj), tk = ks + (int)(rr / nj);
      /* a cage wider than the domain can reach past the ghost layer */
      if(ti < 0 || ti > G.nx + 1 || tj < 0 || tj > G.ny + 1 || tk < 0
        || tk > G.nz + 1) continue;
      double xx = __dsub_rn(__dmul_rn(__dsub_rn((double)ti, 0.5), G.dx), cxo);
      double yy = __dsub_rn(__dmul_rn(__dsub_rn((double)tj, 0.5), G.dy), cyo);
      double zz = __dsub_rn(__dmul_rn(__dsub_rn((double)tk, 0.5), G.dz), czo);
      double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(xx, xx), __dmul_rn(yy, yy)),
        __dmul_rn(zz, zz)));
      if(floor(__ddiv_rn(d, r)) < 1)
        atomicMax(&phs[ti + (long long)tj * G.cc_s1 + (long long)tk * G.cc_s2], p);
    }
  }
}

/* ghost copies of a cell-centred int field along one axis
 * (cage_phases_periodic_*, src/particle_kernel.cu:174-221) */
__global__ void k_periodic_cc(int *f, bbb_geom G, int ax)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y * blockDim.y + threadIdx.y;
  int ni = G.nx + 2, nj = G.ny + 2, nk = G.nz + 2;
  long long s1 = G.cc_s1, s2 = G.cc_s2;
  if(ax == 0) {
    if(a >= nj || b >= nk) return;
    long long base = a * s1 + b * s2;
    f[base + 0] = f[base + (ni - 2)];
    f[base + (ni - 1)] = f[base + 1];
  } else if(ax == 1) {
    if(a >= ni || b >= nk) return;
    long long base = a + b * s2;
    f[base + 0] = f[base + (nj - 2) * s1];
    f[base + (nj - 1) * s1] = f[base + 1 * s1];
  } else {
    if(a >= ni || b >= nj) return;
    long long base = a + b * s1;
    f[base + 0] = f[base + (nk - 2) * s2];
    f[base + (nk - 1) * s2] = f[base + 1 * s2];
  }
}

/* phase_shell sweeps, one thread per line as src/particle_kernel.cu:223-291 */
__global__ void k_phase_shell(const int *phs, int *shl, bbb_geom G, int ax)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int b = blockIdx.y * blockDim.y + threadIdx.y + 1;
  long long s1 = G.cc_s1, s2 = G.cc_s2;
  long long base, st;
  int n;
  if(ax == 0) { if(a > G.ny || b > G.nz) return; base = a * s1 + b * s2; st = 1; n = G.nx; }
  else if(ax == 1) { if(a > G.nx || b > G.nz) return; base = a + b * s2; st = s1; n = G.ny; }
  else { if(a > G.nx || b > G.ny) return; base = a + b * s1; st = s2; n = G.nz; }
  for(int i = 1; i <= n + 1; i++) {
    long long W = base + (i - 1) * st, E = base + i * st;
    shl[E] = shl[E] * (1 - (phs[W] < 0 && phs[E] > -1));
    shl[W] = shl[W] * (1 - (phs[W] > -1 && phs[E] < 0));
  }
}

/* cage_flag_u/v/w, src/particle_kernel.cu:410-497 */
__global__ void k_cage_flags(const int *phs, const int *shl, int *fu, int *fv,
  int *fw, bbb_geom G)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int k = blockIdx.z + 1;
  if(i > G.nx + 1 || j > G.ny + 1) return;
  long long C = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
#define FLAG(a, b) (1 - 2 * ((phs[a] < 0 && phs[b] > -1) || (phs[a] > -1 && phs[b] < 0) \
    || (shl[a] < 1 && shl[b] < 1)))
  if(j <= G.ny && k <= G.nz)
    fu[i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2] = FLAG(C - 1, C);
  if(i <= G.nx && k <= G.nz)
    fv[i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2] = FLAG(C - G.cc_s1, C);
  if(i <= G.nx && j <= G.ny)
    fw[i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2] = FLAG(C - G.cc_s2, C);
#undef FLAG
}

/* flag_external_*, src/particle_kernel.cu:499-533 */
__global__ void k_flag_external(int *f, int s1, int s2, int ni, int nj, int nk,
  int ax)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y * blockDim.y + threadIdx.y;
  if(ax == 0) {
    if(a >= nj || b >= nk) return;
    long long base = (long long)a * s1 + (long long)b * s2;
    f[base + 1] = 0; f[base + (ni - 2)] = 0;
  } else if(ax == 1) {
    if(a >= ni || b >= nk) return;
    long long base = a + (long long)b * s2;
    f[base + 1LL * s1] = 0; f[base + (long long)(nj - 2) * s1] = 0;
  } else {
    if(a >= ni || b >= nj) return;
    long long base = a + (long long)b * s1;
    f[base + 1LL * s2] = 0; f[base + (long long)(nk - 2) * s2] = 0;
  }
}

/* periodic ghost copies of a face flag field (cage_flag_*_periodic_*,
 * src/particle_kernel.cu:293-408); `normal` shifts the source by the
 * duplicated face */
__global__ void k_periodic_face(int *f, int s1, int s2, int ni, int nj, int nk,
  int ax, int normal)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y * blockDim.y + threadIdx.y;
  int sh = normal ? 1 : 0;
  if(ax == 0) {
    if(a >= nj || b >= nk) return;
    long long base = (long long)a * s1 + (long long)b * s2;
    f[base + 0] = f[base + (ni - 2 - sh)];
    f[base + (ni - 1)] = f[base + 1 + sh];
  } else if(ax == 1) {
    if(a >= ni || b >= nk) return;
    long long base = a + (long long)b * s2;
    f[base + 0] = f[base + (long long)(nj - 2 - sh) * s1];
    f[base + (long long)(nj - 1) * s1] = f[base + (long long)(1 + sh) * s1];
  } else {
    if(a >= ni || b >= nj) return;
    long long base = a + (long long)b * s1;
    f[base + 0] = f[base + (long long)(nk - 2 - sh) * s2];
    f[base + (long long)(nk - 1) * s2] = f[base + (long long)(1 + sh) * s2];
  }
}

static dim3 face_grid(int n1, int n2) { return dim3((n1 + 31) / 32, (n2 + 7) / 8); }

extern "C" void cuda_build_cages(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  const dom_struct *d = &Dom;
  bbb_geom G = bbb_make_geom();
  cudaStream_t s = g_dev.stream;
  dim3 blk(32, 8);
  k_reset_cages<<<1184, 256, 0, s>>>(g_dev.phase, g_dev.phase_shell, d->Gcc.s3b,
    g_dev.flag_u, d->Gfx.s3b, g_dev.flag_v, d->Gfy.s3b, g_dev.flag_w, d->Gfz.s3b);
  BBB_LAUNCHED();
  if(nparts > 0 && g_dev.np == nparts) {
    k_cage_extents<<<(nparts + 127) / 128, 128, 0, s>>>(g_dev.parts, nparts, G,
      d->Gcc.is, d->Gcc.ie, d->Gcc.js, d->Gcc.je, d->Gcc.ks, d->Gcc.ke);
    BBB_LAUNCHED();
    k_build_phase<<<nparts, 256, 0, s>>>(g_dev.parts, g_dev.phase, G,
      bc.uE == BBB_PERIODIC, bc.vN == BBB_PERIODIC, bc.wT == BBB_PERIODIC);
    BBB_LAUNCHED();
  }
  int perx = bc.uW == BBB_PERIODIC && bc.uE == BBB_PERIODIC;
  int pery = bc.uS == BBB_PERIODIC && bc.uN == BBB_PERIODIC;
  int perz = bc.uB == BBB_PERIODIC && bc.uT == BBB_PERIODIC;
  int ni = G.nx + 2, nj = G.ny + 2, nk = G.nz + 2;
  int *pers[2] = {g_dev.phase, g_dev.phase_shell};
  for(int f = 0; f < 2; f++) {
    if(f == 1) {
      k_phase_shell<<<face_grid(G.ny, G.nz), blk, 0, s>>>(g_dev.phase, g_dev.phase_shell, G, 0);
      BBB_LAUNCHED();
      k_phase_shell<<<face_grid(G.nx, G.nz), blk, 0, s>>>(g_dev.phase, g_dev.phase_shell, G, 1);
      BBB_LAUNCHED();
      k_phase_shell<<<face_grid(G.nx, G.ny), blk, 0, s>>>(g_dev.phase, g_dev.phase_shell, G, 2);
      BBB_LAUNCHED();
    }
    if(perx) { k_periodic_cc<<<face_grid(nj, nk), blk, 0, s>>>(pers[f], G, 0); BBB_LAUNCHED(); }
    if(pery) { k_periodic_cc<<<face_grid(ni, nk), blk, 0, s>>>(pers[f], G, 1); BBB_LAUNCHED(); }
    if(perz) { k_periodic_cc<<<face_grid(ni, nj), blk, 0, s>>>(pers[f], G, 2); BBB_LAUNCHED(); }
  }
  dim3 grd((G.nx + 1 + 31) / 32, (G.ny + 1 + 7) / 8, G.nz + 1);
  k_cage_flags<<<grd, blk, 0, s>>>(g_dev.phase, g_dev.phase_shell, g_dev.flag_u,
    g_dev.flag_v, g_dev.flag_w, G);
  BBB_LAUNCHED();
  const grid_info *X = &d->Gfx, *Y = &d->Gfy, *Z = &d->Gfz;
  if(bc.uW != BBB_PERIODIC && bc.uE != BBB_PERIODIC) {
    k_flag_external<<<face_grid(X->jnb, X->knb), blk, 0, s>>>(g_dev.flag_u, X->s1b, X->s2b,
      X->inb, X->jnb, X->knb, 0);
    BBB_LAUNCHED();
  }
  if(bc.vS != BBB_PERIODIC && bc.vN != BBB_PERIODIC) {
    k_flag_external<<<face_grid(Y->inb, Y->knb), blk, 0, s>>>(g_dev.flag_v, Y->s1b, Y->s2b,
      Y->inb, Y->jnb, Y->knb, 1);
    BBB_LAUNCHED();
  }
  if(bc.wB != BBB_PERIODIC && bc.wT != BBB_PERIODIC) {
    k_flag_external<<<face_grid(Z->inb, Z->jnb), blk, 0, s>>>(g_dev.flag_w, Z->s1b, Z->s2b,
      Z->inb, Z->jnb, Z->knb, 2);
    BBB_LAUNCHED();
  }
  /* periodic flag ghosts; v's x test reads bc.vW twice as the reference
   * does (src/cuda_particle.cu:845) */
  struct { int *f; const grid_info *g; int per[3]; int comp; } F[3] = {
    {g_dev.flag_u, X, {bc.uW == BBB_PERIODIC && bc.uE == BBB_PERIODIC,
      bc.uS == BBB_PERIODIC && bc.uN == BBB_PERIODIC,
      bc.uB == BBB_PERIODIC && bc.uT == BBB_PERIODIC}, 0},
    {g_dev.flag_v, Y, {bc.vW == BBB_PERIODIC && bc.vW == BBB_PERIODIC,
      bc.vS == BBB_PERIODIC && bc.vN == BBB_PERIODIC,
      bc.vB == BBB_PERIODIC && bc.vT == BBB_PERIODIC}, 1},
    {g_dev.flag_w, Z, {bc.wW == BBB_PERIODIC && bc.wE == BBB_PERIODIC,
      bc.wS == BBB_PERIODIC && bc.wN == BBB_PERIODIC,
      bc.wB == BBB_PERIODIC && bc.wT == BBB_PERIODIC}, 2}};
  for(int f = 0; f < 3; f++) {
    const grid_info *g = F[f].g;
    int n[3] = {g->inb, g->jnb, g->knb};
    for(int ax = 0; ax < 3; ax++) {
      if(!F[f].per[ax]) continue;
      int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
      k_periodic_face<<<face_grid(n[t1], n[t2]), blk, 0, s>>>(F[f].f, g->s1b, g->s2b,
        g->inb, g->jnb, g->knb, ax, F[f].comp == ax);
      BBB_LAUNCHED();
    }
  }
  g_dev.masks_valid = 0;
  g_dev.lf_valid = 0;
}

/* ------------------------------------------------ Lamb's series */

__device__ __forceinline__ double d_Nnm(int n, int m)
{
  double top = 1, bot = 1;
  for(int i = 1; i <= (n - m); i++) top *= (double)i;
  for(int i = 1; i <= (n + m); i++) bot *= (double)i;
  return sqrt((2. * n + 1.) / 4. / PI * top / bot);
}

__device__ __forceinline__ double d_Pnm(int n, int m, double theta)
{
  double x = cos(theta), y = sin(theta);
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

__device__ __forceinline__ void d_xyz2rtp(double x, double y, double z,
  double *r, double *theta, double *phi)
{
  double XY = x * x + y * y;
  double XYZ = XY + z * z;
  if(XYZ >= 0 && XYZ < DIV_ST) XYZ = DIV_ST;
  *r = sqrt(XYZ);
  *theta = acos(z / *r);
  if(XY >= 0 && XY < DIV_ST) XY = DIV_ST;
  *phi = acos(x / sqrt(XY));
  if(y < 0.) *phi = 2. * PI - *phi;
}

__device__ __forceinline__ int d_cbase(int n)
{ int c = 0; for(int j = 0; j < n; j++) c += j + 1; return c; }

__device__ __forceinline__ double d_clamp_st(double st)
{
  if(st >= 0 && st < DIV_ST) st = DIV_ST;
  else if(st < 0 && st > -DIV_ST) st = -DIV_ST;
  return st;
}

__device__ double d_X(int n, double theta, double phi, const double *re,
  const double *im, int pp, int stride)
{
  int c = d_cbase(n) + pp * stride;
  double sum = d_Nnm(n, 0) * d_Pnm(n, 0, theta) * re[c];
  for(int m = 1; m <= n; m++) {
    c++;
    sum += 2. * d_Nnm(n, m) * d_Pnm(n, m, theta)
      * (re[c] * cos(m * phi) - im[c] * sin(m * phi));
  }
  return sum;
}

__device__ double d_Y(int n, double theta, double phi, const double *re,
  const double *im, int pp, int stride)
{
  double ct = cos(theta);
  double st = d_clamp_st(sin(theta));
  int c = d_cbase(n) + pp * stride;
  int m = 0;
  double sum = d_Nnm(n, m)
    * (-(n + 1) * ct / st * d_Pnm(n, m, theta) + (n - m + 1) / st * d_Pnm(n + 1, m, theta))
    * re[c];
  for(m = 1; m <= n; m++) {
    c++;
    sum += 2. * d_Nnm(n, m)
      * (-(n + 1) * ct / st * d_Pnm(n, m, theta) + (n - m + 1) / st * d_Pnm(n + 1, m, theta))
      * (re[c] * cos(m * phi) - im[c] * sin(m * phi));
  }
  return sum;
}

__device__ double d_Z(int n, double theta, double phi, const double *re,
  const double *im, int pp, int stride)
{
  double st = d_clamp_st(sin(theta));
  int c = d_cbase(n) + pp * stride;
  double sum = 0.;
  for(int m = 1; m <= n; m++) {
    c++;
    sum += -2. * m / st * d_Nnm(n, m) * d_Pnm(n, m, theta)
      * (re[c] * sin(m * phi) + im[c] * cos(m * phi));
  }
  return sum;
}

struct coef_ptrs { const double *c[6]; };

__device__ void d_lamb_vel(int order, double a, double r, double theta,
  double phi, double nu, const coef_ptrs &cf, int p, int stride, double *Ux,
  double *Uy, double *Uz)
{
  const double *pre = cf.c[0], *pim = cf.c[1], *fre = cf.c[2], *fim = cf.c[3],
               *cre = cf.c[4], *cim = cf.c[5];
  double ar = a / r, ra = r / a;
  double ur = 0.;
  double ut = 0.5 * ra * d_Y(0, theta, phi, pre, pim, p, stride);
  double up = 0.5 * ra * d_Z(0, theta, phi, pre, pim, p, stride);
  for(int n = 1; n <= order; n++) {
    double powranp1 = pow(ra, n + 1.);
    double powranm1 = pow(ra, n - 1.);
    double powarnp2 = pow(ar, n + 2.);
    double powarnp1 = pow(ar, n + 1.);
    double powarn = pow(ar, (double)n);
    double od2np3 = 1. / (2. * n + 3.);
    double odnp1 = 1. / (n + 1.);
    ur += (0.5 * n * od2np3 * powranp1
      + 0.25 * n * ((2. * n + 1.) * od2np3 * ar * ar - 1.) * powarn)
      * d_X(n, theta, phi, pre, pim, p, stride);
    ur += (n * powranm1
      + 0.5 * n * (2. * n - 1. - (2. * n + 1.) * ra * ra) * pow(ar, n + 2.))
      * d_X(n, theta, phi, fre, fim, p, stride);
    ut += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
      + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn)
      * d_Y(n, theta, phi, pre, pim, p, stride);
    ut += (powranm1
      + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2)
      * d_Y(n, theta, phi, fre, fim, p, stride);
    ut += (powranm1 - powarnp1) * d_Z(n, theta, phi, cre, cim, p, stride);
    up += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
      + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn)
      * d_Z(n, theta, phi, pre, pim, p, stride);
    up += (powranm1
      + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2)
      * d_Z(n, theta, phi, fre, fim, p, stride);
    up += (-powranm1 + powarnp1) * d_Y(n, theta, phi, cre, cim, p, stride);
  }
  ur *= nu / a;
  ut *= nu / a;
  up *= nu / a;
  *Ux = ur * sin(theta) * cos(phi) + ut * cos(theta) * cos(phi) - up * sin(phi);
  *Uy = ur * sin(theta) * sin(phi) + ut * cos(theta) * sin(phi) + up * cos(phi);
  *Uz = ur * cos(theta) - ut * sin(theta);
}

__device__ __forceinline__ double d_wrap_rel(double x, double a, double L)
{
  if(x <= 2. * a - L) x += L;
  if(x >= L - 2. * a) x -= L;
  return x;
}

/* ------------------------------------------------ particle BC faces
 * part_BC_u/v/w (src/particle_kernel.cu:535-838) visit every interior
 * face of each component, ghost rows included, and overwrite those with
 * flag < 1 that border a particle cell with the Lamb velocity plus the
 * rigid-body motion.  Those faces depend only on phase and flags, which
 * change only in the cage build, and their positions relative to the
 * particle change only when particles move; the Lamb loop applies the
 * condition about seven times per sub-iteration.  So the faces are listed
 * once per cage build, their particle-frame geometry (r, cos/sin theta,
 * cos/sin m phi) once per particle move, and each application evaluates
 * the series from that list with no transcendental calls. */

#define LF_NGEO 14   /* x y z r ct st cp1 sp1 cp2 sp2 cp3 sp3 cp4 sp4 */
__constant__ double c_Nnm[6][6];
__constant__ double c_od2np3[6], c_odnp1[6];   /* 1/(2n+3), 1/(n+1) */
static int g_nnm_ready = 0;

static void upload_nnm(void)
{
  if(g_nnm_ready) return;
  double t[6][6];
  for(int n = 0; n < 6; n++) for(int m = 0; m < 6; m++) {
    double top = 1, bot = 1;
    for(int i = 1; i <= (n - m); i++) top *= (double)i;
    for(int i = 1; i <= (n + m); i++) bot *= (double)i;
    t[n][m] = m <= n ? sqrt((2. * n + 1.) / 4. / PI * top / bot) : 0.;
  }
  BBB_CK(cudaMemcpyToSymbol(c_Nnm, t, sizeof(t)));
  double a[6], b[6];
  for(int n = 0; n < 6; n++) { a[n] = 1. / (2. * n + 3.); b[n] = 1. / (n + 1.); }
  BBB_CK(cudaMemcpyToSymbol(c_od2np3, a, sizeof(a)));
  BBB_CK(cudaMemcpyToSymbol(c_odnp1, b, sizeof(b)));
  g_nnm_ready = 1;
}

/* the faces part_BC would change: flag < 1 and a particle cell on either
 * side (the first side wins, as in the reference) */
__device__ __forceinline__ int lf_owner(int comp, int i, int j, int k,
  const int *phs, const int *fu, const int *fv, const int *fw,
  const bbb_geom &G, long long *Cout)
{
  int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
  int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
  long long C = i + (long long)j * s1 + (long long)k * s2;
  const int *flag = comp == 0 ? fu : (comp == 1 ? fv : fw);
  if(flag[C] >= 1) return -1;
  long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
  long long cstep = comp == 0 ? 1 : (comp == 1 ? G.cc_s1 : G.cc_s2);
  int P0 = phs[cc - cstep], P1 = phs[cc];
  *Cout = C;
  return P0 > -1 ? P0 : (P1 > -1 ? P1 : -1);
}

/* pass 0 counts the faces per particle, pass 1 fills each particle's
 * faces into its own run of the list, so that the threads of a warp
 * evaluating the list mostly share one particle and its coefficients (the
 * order inside a run is irrelevant: every face is written by exactly one
 * entry).  The threads of a warp that hold faces of one particle update
 * its counter with one atomic. */
__global__ void k_lf_collect(const int *phs, const int *fu, const int *fv,
  const int *fw, bbb_geom G, int pass, int *pcnt, const int *pstart,
  int *pfill, int *idx, int *part, long long cap)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  int lane = (threadIdx.x + blockDim.x * threadIdx.y) & 31;
  bool in = !(i > G.nx + 1 || j > G.ny + 1 || k > G.nz + 1);
  unsigned alive = __ballot_sync(0xffffffffu, in);
  if(!in) return;
  for(int comp = 0; comp < 3; comp++) {
    bool skip = (comp == 0 && i < 1) || (comp == 1 && j < 1) || (comp == 2 && k < 1);
    long long C = 0;
    int P = skip ? -1 : lf_owner(comp, i, j, k, phs, fu, fv, fw, G, &C);
    unsigned faces = __ballot_sync(alive, P >= 0);
    if(P < 0) continue;
    unsigned peers = __match_any_sync(faces, P);
    int lead = __ffs(peers) - 1, n = __popc(peers);
    if(pass == 0) {
      if(lane == lead) atomicAdd(&pcnt[P], n);
    } else {
      int base = 0;
      if(lane == lead) base = atomicAdd(&pfill[P], n);
      base = __shfl_sync(peers, base, lead);
      long long slot = (long long)pstart[P] + base
        + __popc(peers & ((1u << lane) - 1u));
      if(slot < cap) {
        idx[slot] = (int)(((unsigned int)comp << 30) | (unsigned int)C);
        part[slot] = P;
      }
    }
  }
}

/* total of the per-particle face counts (after their scan) */
__global__ void k_lf_total(const int *pcnt, const int *pstart, int np,
  unsigned int *count)
{
  if(threadIdx.x == 0 && blockIdx.x == 0)
    *count = np > 0 ? (unsigned int)(pstart[np - 1] + pcnt[np - 1]) : 0u;
}

/* particle-frame geometry of every listed face, from the current
 * particle positions */
__global__ void k_lf_geom(long long n, const int *idx, const int *part,
  const part_struct *parts, bbb_geom G, double *geo, long long cap)
{
  for(long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
      e += (long long)gridDim.x * blockDim.x) {
    unsigned int pk = (unsigned int)idx[e];
    int comp = (int)(pk >> 30);
    long long C = (long long)(pk & 0x3fffffffu);
    int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
    int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
    int k = (int)(C / s2), rem = (int)(C % s2);
    int j = rem / s1, i = rem % s1;
    const part_struct *q = &parts[part[e]];
    double a = q->r;
    double x = (comp == 0 ? (i - BBB_DOM_BUF) * G.dx : (i - 0.5) * G.dx) + G.xs - q->x;
    double y = (comp == 1 ? (j - BBB_DOM_BUF) * G.dy : (j - 0.5) * G.dy) + G.ys - q->y;
    double z = (comp == 2 ? (k - BBB_DOM_BUF) * G.dz : (k - 0.5) * G.dz) + G.zs - q->z;
    x = d_wrap_rel(x, a, G.xl);
    y = d_wrap_rel(y, a, G.yl);
    z = d_wrap_rel(z, a, G.zl);
    double r, theta, phi;
    d_xyz2rtp(x, y, z, &r, &theta, &phi);
    double g[LF_NGEO];
    g[0] = x; g[1] = y; g[2] = z; g[3] = r;
    g[4] = cos(theta); g[5] = sin(theta);
    for(int m = 1; m <= 4; m++) { g[4 + 2 * m] = cos(m * phi); g[5 + 2 * m] = sin(m * phi); }
#pragma unroll
    for(int a2 = 0; a2 < LF_NGEO; a2++) geo[a2 * cap + e] = g[a2];
  }
}

/* associated Legendre P_n^m from x = cos theta, y = sin theta (n <= 5) */
__device__ __forceinline__ double lf_P(int n, int m, double x, double y)
{
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

/* Lamb velocity (src/particle_kernel.cu:1311-1369) from the stored face
 * geometry; the X/Y/Z angular sums of :1107-1309 with cos(m phi),
 * sin(m phi), cos theta, sin theta precomputed and powers of r/a formed
 * by multiplication */
__global__ void __launch_bounds__(256) k_lf_eval(long long n, const int *idx,
  const int *part, const double *__restrict__ geo, long long cap,
  const part_struct *parts, coef_ptrs cf, int stride, double nu, real *uu,
  real *vv, real *ww)
{
  for(long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
      e += (long long)gridDim.x * blockDim.x) {
    unsigned int pk = (unsigned int)idx[e];
    int comp = (int)(pk >> 30);
    long long C = (long long)(pk & 0x3fffffffu);
    int P = part[e];
    const part_struct *q = &parts[P];
    double x = geo[0 * cap + e], y = geo[1 * cap + e], z = geo[2 * cap + e];
    double r = geo[3 * cap + e], ct = geo[4 * cap + e], st = geo[5 * cap + e];
    double cm[5], sm[5];
    cm[0] = 1.; sm[0] = 0.;
#pragma unroll
    for(int m = 1; m <= 4; m++) { cm[m] = geo[(4 + 2 * m) * cap + e]; sm[m] = geo[(5 + 2 * m) * cap + e]; }
    double stc = st;
    if(stc >= 0 && stc < DIV_ST) stc = DIV_ST;
    else if(stc < 0 && stc > -DIV_ST) stc = -DIV_ST;
    double a = q->r;
    double ar = a / r, ra = r / a;
    int order = q->order;
    const double *pre = cf.c[0], *pim = cf.c[1], *fre = cf.c[2], *fim = cf.c[3],
                 *cre = cf.c[4], *cim = cf.c[5];
    int base = P * stride;
    /* n = 0 terms */
    /* one division per face: the reference divides by sin(theta) in
     * every (n, m) term; multiplying by its reciprocal differs by at most
     * an ulp per term and takes the ~50 FP64 divisions per face (most of
     * this kernel's time) out of the loop */
    const double inv_stc = 1. / stc;
    double Y0 = c_Nnm[0][0] * (-1. * ct * inv_stc * 1. + inv_stc * lf_P(1, 0, ct, st)) * pre[base];
    double ur = 0.;
    double ut = 0.5 * ra * Y0;
    double up = 0.;
    double ran = 1., arn = 1.;   /* ra^(n-1), ar^n at the loop head */
    int c0 = 1;
    /* both loops unrolled over the orders the tables hold (n <= 5): every
     * P_n^m becomes a fixed polynomial and cos(m phi), sin(m phi) stay in
     * registers; the guard keeps the particle's own order */
#pragma unroll
    for(int nn_ = 1; nn_ <= 5; nn_++) {
      if(nn_ > order) break;
      double n = nn_;
      arn *= ar;
      double powranm1 = ran;
      double powranp1 = ran * ra * ra;
      double powarn = arn;
      double powarnp1 = arn * ar;
      double powarnp2 = powarnp1 * ar;
      double od2np3 = c_od2np3[nn_];    /* 1 / (2n + 3), 1 / (n + 1) */
      double odnp1 = c_odnp1[nn_];
      double Xp = 0., Xf = 0., Yp = 0., Yf = 0., Yc = 0., Zp = 0., Zf = 0., Zc = 0.;
#pragma unroll
      for(int m = 0; m <= nn_; m++) {
        int c = base + c0 + m;
        double N = c_Nnm[nn_][m];
        double Pn = lf_P(nn_, m, ct, st);
        double dY = -(n + 1) * ct * inv_stc * Pn + (nn_ - m + 1) * inv_stc * lf_P(nn_ + 1, m, ct, st);
        double w = m == 0 ? 1. : 2.;
        double Rp = pre[c] * cm[m] - pim[c] * sm[m];
        double Rf = fre[c] * cm[m] - fim[c] * sm[m];
        double Rc = cre[c] * cm[m] - cim[c] * sm[m];
        Xp += w * N * Pn * Rp;
        Xf += w * N * Pn * Rf;
        Yp += w * N * dY * Rp;
        Yf += w * N * dY * Rf;
        Yc += w * N * dY * Rc;
        if(m > 0) {
          double zf = -2. * m * inv_stc * N * Pn;
          Zp += zf * (pre[c] * sm[m] + pim[c] * cm[m]);
          Zf += zf * (fre[c] * sm[m] + fim[c] * cm[m]);
          Zc += zf * (cre[c] * sm[m] + cim[c] * cm[m]);
        }
      }
      ur += (0.5 * n * od2np3 * powranp1
        + 0.25 * n * ((2. * n + 1.) * od2np3 * ar * ar - 1.) * powarn) * Xp;
      ur += (n * powranm1
        + 0.5 * n * (2. * n - 1. - (2. * n + 1.) * ra * ra) * powarnp2) * Xf;
      ut += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
        + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn) * Yp;
      ut += (powranm1
        + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2) * Yf;
      ut += (powranm1 - powarnp1) * Zc;
      up += (0.5 * (n + 3.) * odnp1 * od2np3 * powranp1
        + 0.25 * odnp1 * (n - 2. - n * (2. * n + 1.) * od2np3 * ar * ar) * powarn) * Zp;
      up += (powranm1
        + 0.5 * odnp1 * ((n - 2.) * (2. * n + 1.) * ra * ra - n * (2. * n - 1.)) * powarnp2) * Zf;
      up += (-powranm1 + powarnp1) * Yc;
      ran *= ra;
      c0 += nn_ + 1;
    }
    ur *= nu / a;
    ut *= nu / a;
    up *= nu / a;
    double rr = 0.1 / nu * (r * r * r * r * r - a * a * a * a * a) / (r * r * r);
    if(comp == 0) {
      double Ux = ur * st * cm[1] + ut * ct * cm[1] - up * sm[1];
      double val = Ux + q->u + (q->oy * z - q->oz * y);
      val += rr * (q->oydot * z - q->ozdot * y);
      uu[C] = val;
    } else if(comp == 1) {
      double Uy = ur * st * sm[1] + ut * ct * sm[1] + up * cm[1];
      double val = Uy + q->v + (-(q->ox * z - q->oz * x));
      val += rr * (-(q->oxdot * z - q->ozdot * x));
      vv[C] = val;
    } else {
      double Uz = ur * ct - ut * st;
      double val = Uz + q->w + (q->ox * y - q->oy * x);
      val += rr * (q->oxdot * y - q->oydot * x);
      ww[C] = val;
    }
  }
}

__global__ void k_bin_scan(const int *cnt, int *start, int n);

static void lf_build(void)
{
  bbb_geom G = bbb_make_geom();
  dim3 blk(32, 8), grd((G.nx + 2 + 31) / 32, (G.ny + 2 + 7) / 8, G.nz + 2);
  if(!g_dev.lf_count) {
    if(cudaMalloc((void **)&g_dev.lf_count, sizeof(unsigned int)) != cudaSuccess) {
      bbb_set_status(BBB_ERR_CUDA, "cudaMalloc face list");
      return;
    }
  }
  if(g_dev.lf_np != nparts) {
    if(g_dev.lf_pcnt) cudaFree(g_dev.lf_pcnt);
    if(g_dev.lf_pstart) cudaFree(g_dev.lf_pstart);
    if(g_dev.lf_pfill) cudaFree(g_dev.lf_pfill);
    g_dev.lf_pcnt = g_dev.lf_pstart = g_dev.lf_pfill = NULL;
    g_dev.lf_np = 0;
    size_t b = sizeof(int) * (size_t)(nparts > 0 ? nparts : 1);
    if(cudaMalloc((void **)&g_dev.lf_pcnt, b) != cudaSuccess
      || cudaMalloc((void **)&g_dev.lf_pstart, b) != cudaSuccess
      || cudaMalloc((void **)&g_dev.lf_pfill, b) != cudaSuccess) {
      bbb_set_status(BBB_ERR_CUDA, "cudaMalloc face list");
      return;
    }
    g_dev.lf_np = nparts;
  }
  size_t pb = sizeof(int) * (size_t)nparts;
  for(int pass = 0; pass < 2; pass++) {
    if(pass == 0) BBB_CK(cudaMemsetAsync(g_dev.lf_pcnt, 0, pb, g_dev.stream));
    else BBB_CK(cudaMemsetAsync(g_dev.lf_pfill, 0, pb, g_dev.stream));
    k_lf_collect<<<grd, blk, 0, g_dev.stream>>>(g_dev.phase, g_dev.flag_u,
      g_dev.flag_v, g_dev.flag_w, G, pass, g_dev.lf_pcnt, g_dev.lf_pstart,
      g_dev.lf_pfill, g_dev.lf_idx, g_dev.lf_part, g_dev.lf_cap);
    BBB_LAUNCHED();
    if(pass == 0) {
      k_bin_scan<<<1, 1024, 0, g_dev.stream>>>(g_dev.lf_pcnt, g_dev.lf_pstart, nparts);
      BBB_LAUNCHED();
      k_lf_total<<<1, 32, 0, g_dev.stream>>>(g_dev.lf_pcnt, g_dev.lf_pstart, nparts,
        g_dev.lf_count);
      BBB_LAUNCHED();
      unsigned int cnt = 0;
      BBB_CK(cudaMemcpyAsync(&cnt, g_dev.lf_count, sizeof(cnt),
        cudaMemcpyDeviceToHost, g_dev.stream));
      BBB_CK(cudaStreamSynchronize(g_dev.stream));
      g_dev.lf_n = cnt;
      if((long long)cnt > g_dev.lf_cap) {
        long long cap = (long long)cnt + cnt / 4 + 1024;
        if(g_dev.lf_idx) cudaFree(g_dev.lf_idx);
        if(g_dev.lf_part) cudaFree(g_dev.lf_part);
        if(g_dev.lf_geo) cudaFree(g_dev.lf_geo);
        g_dev.lf_idx = NULL; g_dev.lf_part = NULL; g_dev.lf_geo = NULL;
        if(cudaMalloc((void **)&g_dev.lf_idx, sizeof(int) * cap) != cudaSuccess
          || cudaMalloc((void **)&g_dev.lf_part, sizeof(int) * cap) != cudaSuccess
          || cudaMalloc((void **)&g_dev.lf_geo, sizeof(double) * LF_NGEO * cap) != cudaSuccess) {
          bbb_set_status(BBB_ERR_CUDA, "cudaMalloc face list");
          g_dev.lf_cap = 0;
          return;
        }
        g_dev.lf_cap = cap;
      }
    }
  }
  g_dev.lf_valid = 1;
  g_dev.lf_geo_valid = 0;
}

static coef_ptrs cur_coefs(void)
{
  coef_ptrs c;
  for(int a = 0; a < 6; a++) c.c[a] = g_dev.coef[a];
  return c;
}

void bbb_part_BC_fields(real *uu, real *vv, real *ww)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  upload_nnm();
  if(!g_dev.lf_valid) lf_build();
  if(bbb_last_status() == BBB_ERR_CUDA) return;
  long long n = g_dev.lf_n;
  if(n <= 0) return;
  int blocks = (int)((n + 255) / 256);
  if(blocks > 148 * 16) blocks = 148 * 16;
  if(!g_dev.lf_geo_valid) {
    k_lf_geom<<<blocks, 256, 0, g_dev.stream>>>(n, g_dev.lf_idx, g_dev.lf_part,
      g_dev.parts, bbb_make_geom(), g_dev.lf_geo, g_dev.lf_cap);
    BBB_LAUNCHED();
    g_dev.lf_geo_valid = 1;
  }
  k_lf_eval<<<blocks, 256, 0, g_dev.stream>>>(n, g_dev.lf_idx, g_dev.lf_part,
    g_dev.lf_geo, g_dev.lf_cap, g_dev.parts, cur_coefs(), coeff_stride, nu,
    uu, vv, ww);
  BBB_LAUNCHED();
}

/* src/cuda_particle.cu:899-944 */
extern "C" void cuda_part_BC(void) { bbb_part_BC_fields(g_dev.u, g_dev.v, g_dev.w); }
/* src/cuda_particle.cu:947-992 */
extern "C" void cuda_part_BC_star(void) { bbb_part_BC_fields(g_dev.us, g_dev.vs, g_dev.ws); }

/* src/cuda_particle.cu:996-1017: zero the Poisson right-hand side inside
 * particles (the net effect of part_BC_p for finite values) */
__global__ void k_zero_rhs_solid(double *b, const int *phs, bbb_geom G)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    if(phs[i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2] > -1) b[t] = 0.;
  }
}

extern "C" void cuda_part_BC_p(int dev)
{
  (void)dev;
  bbb_dev_require();
  if(!g_dev.ready) return;
  bbb_geom G = bbb_make_geom();
  k_zero_rhs_solid<<<1184, 256, 0, g_dev.stream>>>(g_dev.kb, g_dev.phase, G);
  BBB_LAUNCHED();
}

/* part_BC_p_fill, src/particle_kernel.cu:942-1018 */
__global__ void k_p_fill(real *pp, const int *phs, const part_struct *parts,
  coef_ptrs cf, int stride, double mu, double nu, double rho_f, double gpx,
  double gpy, double gpz, bbb_geom G)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    long long CC = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    int p = phs[CC];
    if(p < 0) continue;
    const part_struct *q = &parts[p];
    double a = q->r;
    double x = d_wrap_rel((i - 0.5) * G.dx + G.xs - q->x, a, G.xl);
    double y = d_wrap_rel((j - 0.5) * G.dy + G.ys - q->y, a, G.yl);
    double z = d_wrap_rel((k - 0.5) * G.dz + G.zs - q->z, a, G.zl);
    double r, theta, phi;
    d_xyz2rtp(x, y, z, &r, &theta, &phi);
    double v = d_X(0, theta, phi, cf.c[0], cf.c[1], p, stride);
    v *= mu * nu / (a * a);
    double o2 = (q->oy * z - q->oz * y) * (q->oy * z - q->oz * y);
    o2 += (q->ox * z - q->oz * x) * (q->ox * z - q->oz * x);
    o2 += (q->ox * y - q->oy * x) * (q->ox * y - q->oy * x);
    double acc = (-gpx / rho_f - q->udot) * x + (-gpy / rho_f - q->vdot) * y
      + (-gpz / rho_f - q->wdot) * z;
    v += 0.5 * rho_f * o2 + rho_f * acc;
    pp[CC] = v;
  }
}

extern "C" void cuda_part_p_fill(void)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  bbb_geom G = bbb_make_geom();
  k_p_fill<<<1184, 256, 0, g_dev.stream>>>(g_dev.p, g_dev.phase, g_dev.parts,
    cur_coefs(), coeff_stride, mu, nu, rho_f, gradP.x, gradP.y, gradP.z, G);
  BBB_LAUNCHED();
}

/* internal_u/v/w, src/bluebottle_kernel.cu:3916-4022 */
__global__ void k_internal(real *uu, real *vv, real *ww, const int *phs,
  const int *fu, const int *fv, const int *fw, const part_struct *parts,
  bbb_geom G)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int k = blockIdx.z + 1;
  if(i > G.nx + 1 || j > G.ny + 1) return;
  long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
  for(int comp = 0; comp < 3; comp++) {
    if(comp == 0 && (j > G.ny || k > G.nz)) continue;
    if(comp == 1 && (i > G.nx || k > G.nz)) continue;
    if(comp == 2 && (i > G.nx || j > G.ny)) continue;
    int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
    int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
    long long C = i + (long long)j * s1 + (long long)k * s2;
    long long cstep = comp == 0 ? 1 : (comp == 1 ? G.cc_s1 : G.cc_s2);
    int pw = phs[cc - cstep], pe = phs[cc];
    const int *flag = comp == 0 ? fu : (comp == 1 ? fv : fw);
    if(!(pw > -1 && pe > -1 && flag[C] != -1)) continue;
    const part_struct *q = &parts[pe];
    double rx = (comp == 0 ? (i - BBB_DOM_BUF) * G.dx : (i - 0.5) * G.dx) + G.xs - q->x;
    double ry = (comp == 1 ? (j - BBB_DOM_BUF) * G.dy : (j - 0.5) * G.dy) + G.ys - q->y;
    double rz = (comp == 2 ? (k - BBB_DOM_BUF) * G.dz : (k - 0.5) * G.dz) + G.zs - q->z;
    rx = d_wrap_rel(rx, q->r, G.xl);
    ry = d_wrap_rel(ry, q->r, G.yl);
    rz = d_wrap_rel(rz, q->r, G.zl);
    if(comp == 0) uu[C] = (q->oy * rz - q->oz * ry) + q->u;
    else if(comp == 1) vv[C] = (q->oz * rx - q->ox * rz) + q->v;
    else ww[C] = (q->ox * ry - q->oy * rx) + q->w;
  }
}

extern "C" void cuda_parts_internal(void)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  bbb_geom G = bbb_make_geom();
  dim3 blk(32, 8), grd((G.nx + 1 + 31) / 32, (G.ny + 1 + 7) / 8, G.nz + 1);
  k_internal<<<grd, blk, 0, g_dev.stream>>>(g_dev.u, g_dev.v, g_dev.w,
    g_dev.phase, g_dev.flag_u, g_dev.flag_v, g_dev.flag_w, g_dev.parts, G);
  BBB_LAUNCHED();
}

/* ------------------------------------------------ quadrature
 * 26-node degree-7 Lebedev rule (src/cuda_quadrature.cu:86-150): 6 axis
 * nodes (poles nudged by DIV_ST), 12 edge midpoints, 8 cube vertices;
 * weights 4 pi {1/21, 4/105, 27/840}. */
__constant__ double c_node_t[26];
__constant__ double c_node_p[26];
static int g_nodes_ready = 0;

static void upload_nodes(void)
{
  if(g_nodes_ready) return;
  double PI14 = 0.25 * PI, PI12 = 0.5 * PI, PI34 = 0.75 * PI,
         PI54 = 1.25 * PI, PI32 = 1.5 * PI, PI74 = 1.75 * PI;
  double alph1 = 0.955316618124509, alph2 = 2.186276035465284;
  double t[26] = {PI12, PI12, PI12, PI12, 0. + DIV_ST, PI - DIV_ST,
    PI12, PI12, PI12, PI12, PI14, PI14, PI14, PI14, PI34, PI34, PI34, PI34,
    alph1, alph1, alph1, alph1, alph2, alph2, alph2, alph2};
  double p[26] = {0., PI12, PI, PI32, 0., 0.,
    PI14, PI34, PI54, PI74, 0., PI12, PI, PI32, 0., PI12, PI, PI32,
    PI14, PI34, PI54, PI74, PI14, PI34, PI54, PI74};
  BBB_CK(cudaMemcpyToSymbol(c_node_t, t, sizeof(t)));
  BBB_CK(cudaMemcpyToSymbol(c_node_p, p, sizeof(p)));
  g_nodes_ready = 1;
}

struct lamb_args {
  part_struct *parts;
  const real *p, *u, *v, *w;
  coef_ptrs cur;
  double *cf[6];          /* writable current coefficients */
  const double *cf0[6];   /* previous iterate             */
  int stride, np;
  double mu, nu, rho_f, relax, gpx, gpy, gpz;
  BC bc;
  bbb_geom G;
  int s_cc1, s_cc2;
};

__global__ void __launch_bounds__(32) k_lamb(lamb_args L)
{
  const double A1 = 0.598398600683775, A2 = 0.478718880547015,
               A3 = 0.403919055461543;
  int part = blockIdx.x;
  int node = threadIdx.x;
  __shared__ double s_pp[32], s_ut[32], s_up[32];
  __shared__ double s_I[6][32];
  part_struct *q = &L.parts[part];
  const bbb_geom &G = L.G;
  const BC &bc = L.bc;
  if(node < 26) {
    double th = c_node_t[node], ph_ = c_node_p[node];
    double xp = q->rs * sin(th) * cos(ph_);
    double yp = q->rs * sin(th) * sin(ph_);
    double zp = q->rs * cos(th);
    double x = xp + q->x, y = yp + q->y, z = zp + q->z;
    int nd = -1;
    if(x - G.xs < 0) {
      if(bc.uW == BBB_DIRICHLET || bc.vW == BBB_DIRICHLET || bc.wW == BBB_DIRICHLET)
        if(nd == -1) nd = -10;
    } if(x - G.xe > 0) {
      if(bc.uE == BBB_DIRICHLET || bc.vE == BBB_DIRICHLET || bc.wE == BBB_DIRICHLET)
        if(nd == -1) nd = -11;
    } if(y - G.ys < 0) {
      if(bc.uS == BBB_DIRICHLET || bc.vS == BBB_DIRICHLET || bc.wS == BBB_DIRICHLET)
        if(nd == -1) nd = -12;
    } if(y - G.ye > 0) {
      if(bc.uN == BBB_DIRICHLET || bc.vN == BBB_DIRICHLET || bc.wN == BBB_DIRICHLET)
        if(nd == -1) nd = -13;
    } if(z - G.zs < 0) {
      if(bc.uB == BBB_DIRICHLET || bc.vB == BBB_DIRICHLET || bc.wB == BBB_DIRICHLET)
        if(nd == -1) nd = -14;
    } if(z - G.ze > 0) {
      if(bc.uT == BBB_DIRICHLET || bc.vT == BBB_DIRICHLET || bc.wT == BBB_DIRICHLET)
        if(nd == -1) nd = -15;
    }
    q->nodes[node] = nd;
    if(x < G.xs && bc.uW == BBB_PERIODIC) x = x + G.xl;
    else if(x > G.xe && bc.uE == BBB_PERIODIC) x = x - G.xl;
    if(y < G.ys && bc.vS == BBB_PERIODIC) y = y + G.yl;
    else if(y > G.ye && bc.vN == BBB_PERIODIC) y = y - G.yl;
    if(z < G.zs && bc.wB == BBB_PERIODIC) z = z + G.zl;
    else if(z > G.ze && bc.wT == BBB_PERIODIC) z = z - G.zl;
    double ddx = 1. / G.dx, ddy = 1. / G.dy, ddz = 1. / G.dz;
    int i = (int)floor(__dmul_rn(__dsub_rn(x, G.xs), ddx)) + BBB_DOM_BUF;
    int j = (int)floor(__dmul_rn(__dsub_rn(y, G.ys), ddy)) + BBB_DOM_BUF;
    int k = (int)floor(__dmul_rn(__dsub_rn(z, G.zs), ddz)) + BBB_DOM_BUF;
    i = max(1, min(i, G.nx)); j = max(1, min(j, G.ny)); k = max(1, min(k, G.nz));
    long long C = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    double xx = (i - 0.5) * G.dx + G.xs, yy = (j - 0.5) * G.dy + G.ys,
           zz = (k - 0.5) * G.dz + G.zs;
    const real *p = L.p;
    double dpdx = 0.5 * (p[C + 1] - p[C - 1]) * ddx;
    double dpdy = 0.5 * (p[C + G.cc_s1] - p[C - G.cc_s1]) * ddy;
    double dpdz = 0.5 * (p[C + G.cc_s2] - p[C - G.cc_s2]) * ddz;
    double pv = p[C] + dpdx * (x - xx) + dpdy * (y - yy) + dpdz * (z - zz);
    double ox = q->ox, oy = q->oy, oz = q->oz;
    double o2 = (oy * zp - oz * yp) * (oy * zp - oz * yp);
    o2 += (ox * zp - oz * xp) * (ox * zp - oz * xp);
    o2 += (ox * yp - oy * xp) * (ox * yp - oy * xp);
    double acc = (-L.gpx / L.rho_f - q->udot) * xp + (-L.gpy / L.rho_f - q->vdot) * yp
      + (-L.gpz / L.rho_f - q->wdot) * zp;
    pv -= 0.5 * L.rho_f * o2 + L.rho_f * acc;
    pv = (nd == -1) * pv;

    double rs3 = q->rs * q->rs * q->rs, rs5 = rs3 * q->rs * q->rs;
    double a5 = q->r * q->r * q->r * q->r * q->r;
    double ocr[3] = {oy * zp - oz * yp, -(ox * zp - oz * xp), ox * yp - oy * xp};
    double odcr[3] = {q->oydot * zp - q->ozdot * yp, -(q->oxdot * zp - q->ozdot * xp),
      q->oxdot * yp - q->oydot * xp};
    double pu[3] = {q->u, q->v, q->w};
    double wall[3][6] = {{bc.uWD, bc.uED, bc.uSD, bc.uND, bc.uBD, bc.uTD},
      {bc.vWD, bc.vED, bc.vSD, bc.vND, bc.vBD, bc.vTD},
      {bc.wWD, bc.wED, bc.wSD, bc.wND, bc.wBD, bc.wTD}};
    double vel[3];
    for(int c = 0; c < 3; c++) {
      const real *f = c == 0 ? L.u : (c == 1 ? L.v : L.w);
      int s1 = c == 0 ? G.fx_s1 : (c == 1 ? G.fy_s1 : G.fz_s1);
      int s2 = c == 0 ? G.fx_s2 : (c == 1 ? G.fy_s2 : G.fz_s2);
      double fxr = __dmul_rn(__dsub_rn(x, G.xs), ddx);
      double fyr = __dmul_rn(__dsub_rn(y, G.ys), ddy);
      double fzr = __dmul_rn(__dsub_rn(z, G.zs), ddz);
      int ii = (int)(c == 0 ? round(fxr) : floor(fxr)) + BBB_DOM_BUF;
      int jj = (int)(c == 1 ? round(fyr) : floor(fyr)) + BBB_DOM_BUF;
      int kk = (int)(c == 2 ? round(fzr) : floor(fzr)) + BBB_DOM_BUF;
      int ihi = G.nx + (c == 0), jhi = G.ny + (c == 1), khi = G.nz + (c == 2);
      ii = max(1, min(ii, ihi)); jj = max(1, min(jj, jhi)); kk = max(1, min(kk, khi));
      double fx = c == 0 ? (ii - BBB_DOM_BUF) * G.dx + G.xs : (ii - 0.5) * G.dx + G.xs;
      double fy = c == 1 ? (jj - BBB_DOM_BUF) * G.dy + G.ys : (jj - 0.5) * G.dy + G.ys;
      double fz = c == 2 ? (kk - BBB_DOM_BUF) * G.dz + G.zs : (kk - 0.5) * G.dz + G.zs;
      long long CF = ii + (long long)jj * s1 + (long long)kk * s2;
      double dfdx = 0.5 * (f[CF + 1] - f[CF - 1]) * ddx;
      double dfdy = 0.5 * (f[CF + s1] - f[CF - s1]) * ddy;
      double dfdz = 0.5 * (f[CF + s2] - f[CF - s2]) * ddz;
      double val = f[CF] + dfdx * (x - fx) + dfdy * (y - fy) + dfdz * (z - fz);
      double vw = (nd == -10) * wall[c][0] + (nd == -11) * wall[c][1]
        + (nd == -12) * wall[c][2] + (nd == -13) * wall[c][3]
        + (nd == -14) * wall[c][4] + (nd == -15) * wall[c][5];
      val -= pu[c] + ocr[c];
      val -= 0.1 / L.nu * (rs5 - a5) / rs3 * odcr[c];
      vw -= pu[c] + ocr[c];
      vw -= 0.1 / L.nu * (rs5 - a5) / rs3 * odcr[c];
      vel[c] = (nd == -1) * val + (nd < -1) * vw;
    }
    double stt = sin(th), ctt = cos(th), sp = sin(ph_), cp = cos(ph_);
    s_pp[node] = pv;
    s_ut[node] = ctt * (vel[0] * cp + vel[1] * sp) - vel[2] * stt;
    s_up[node] = -vel[0] * sp + vel[1] * cp;
  }
  __syncwarp();
  /* inner products and the coefficient solve, one coefficient at a time */
  double ars = q->r / q->rs, rsa = q->rs / q->r;
  int ncoef = q->ncoeff < 15 ? q->ncoeff : 15;
  const int nn_[15] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 4};
  const int mm_[15] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3, 0, 1, 2, 3, 4};
  double mu = L.mu, nu = L.nu, relax = L.relax, r = q->r;
  for(int coeff = 0; coeff < ncoef; coeff++) {
    int n = nn_[coeff], m = mm_[coeff];
    if(node < 26) {
      double theta = c_node_t[node], phi = c_node_p[node];
      double N_nm = d_Nnm(n, m);
      double P_nm = d_Pnm(n, m, theta);
      double P_n1m = d_Pnm(n + 1, m, theta);
      double dPdt = (n - m + 1.) * P_n1m - (n + 1.) * cos(theta) * P_nm;
      double dPdp = m * P_nm;
      double pv = s_pp[node], tv = s_ut[node], fv = s_up[node];
      s_I[0][node] = N_nm * P_nm * pv * cos(m * phi);
      s_I[1][node] = -N_nm * P_nm * pv * sin(m * phi);
      s_I[2][node] = N_nm / sin(theta) * (dPdt * tv * cos(m * phi) - dPdp * fv * sin(m * phi));
      s_I[3][node] = N_nm / sin(theta) * (-dPdt * tv * sin(m * phi) - dPdp * fv * cos(m * phi));
      s_I[4][node] = N_nm / sin(theta) * (dPdp * tv * sin(m * phi) + dPdt * fv * cos(m * phi));
      s_I[5][node] = N_nm / sin(theta) * (dPdp * tv * cos(m * phi) - dPdt * fv * sin(m * phi));
    }
    __syncwarp();
    if(node < 6) {
      /* lane a sums integrand a in the reference's serial node order */
      int a = node;
      double s = s_I[a][0] * A1;
      for(int i = 1; i < 6; i++) s += A1 * s_I[a][i];
      for(int i = 6; i < 18; i++) s += A2 * s_I[a][i];
      for(int i = 18; i < 26; i++) s += A3 * s_I[a][i];
      s_I[a][31] = s;
    }
    __syncwarp();
    if(node == 0) {
      double S[6];
      for(int a = 0; a < 6; a++) S[a] = s_I[a][31];
      long long ci = (long long)L.stride * part + coeff;
      if(n == 0) {
        L.cf[0][ci] = L.cf0[0][ci] + relax * (r * r / mu / nu * S[0] * pow(ars, (double)n) - L.cf0[0][ci]);
        L.cf[1][ci] = L.cf0[1][ci] + relax * (r * r / mu / nu * S[1] * pow(ars, (double)n) - L.cf0[1][ci]);
        L.cf[2][ci] = 0.; L.cf[3][ci] = 0.; L.cf[4][ci] = 0.; L.cf[5][ci] = 0.;
      } else {
        double A = (1. - 0.5 * n * (2. * n - 1.) / (n + 1.) * pow(ars, 2. * n + 1.)) * pow(rsa, (double)n);
        double B = n * (2. * n - 1.) * (2. * n + 1.) / (n + 1.) * pow(ars, n + 1.);
        double Cc = 0.25 * n * (2. * (n + 3.) / (2. * n + 3.)
          + (n - 2. - n * (2. * n + 1.) / (2. * n + 3.) * ars * ars) * pow(ars, 2. * n + 1.))
          * pow(rsa, n + 1.);
        double D = n * (n + 1. + 0.5 * ((n - 2.) * (2. * n + 1.) * rsa * rsa
          - n * (2. * n - 1.)) * pow(ars, 2. * n + 1.)) * pow(rsa, n - 1.);
        double den = A * D + B * Cc;
        double pre = (r * r / mu / nu * S[0] * D + r / nu * S[2] * B) / den;
        double pim = (r * r / mu / nu * S[1] * D + r / nu * S[3] * B) / den;
        double fre = (r / nu * S[2] * A - r * r / mu / nu * S[0] * Cc) / den;
        double fim = (r / nu * S[3] * A - r * r / mu / nu * S[1] * Cc) / den;
        double E = n * (n + 1.) * (pow(ars, 2. * n + 1.) - 1.) * pow(rsa, (double)n);
        double cre = r / nu * S[4] / E;
        double cim = r / nu * S[5] / E;
        L.cf[0][ci] = L.cf0[0][ci] * (1. - relax) + relax * pre;
        L.cf[1][ci] = L.cf0[1][ci] * (1. - relax) + relax * pim;
        L.cf[2][ci] = L.cf0[2][ci] * (1. - relax) + relax * fre;
        L.cf[3][ci] = L.cf0[3][ci] * (1. - relax) + relax * fim;
        L.cf[4][ci] = L.cf0[4][ci] * (1. - relax) + relax * cre;
        L.cf[5][ci] = L.cf0[5][ci] * (1. - relax) + relax * cim;
      }
    }
    __syncwarp();
  }
  if(node == 0) {
    /* forces and torques, src/quadrature_kernel.cu:545-576 */
    double vol = 4. / 3. * PI * q->r * q->r * q->r;
    double N10 = sqrt(3. / 4. / PI), N11 = sqrt(3. / 8. / PI);
    long long b = (long long)L.stride * part;
    double *const *cf = L.cf;
    q->Fx = L.rho_f * vol * (q->udot + L.gpx)
      - PI * mu * nu * 2. * N11 * (cf[0][b + 2] + 6. * cf[2][b + 2]);
    q->Fy = L.rho_f * vol * (q->vdot + L.gpy)
      + PI * mu * nu * 2. * N11 * (cf[1][b + 2] + 6. * cf[3][b + 2]);
    q->Fz = L.rho_f * vol * (q->wdot + L.gpz)
      + PI * mu * nu * N10 * (cf[0][b + 1] + 6. * cf[2][b + 1]);
    q->Lx = L.rho_f * vol * q->r * q->r * q->oxdot
      - 8. * PI * mu * nu * 2. * N11 * q->r * cf[4][b + 2];
    q->Ly = L.rho_f * vol * q->r * q->r * q->oydot
      + 8. * PI * mu * nu * 2. * N11 * q->r * cf[5][b + 2];
    q->Lz = L.rho_f * vol * q->r * q->r * q->ozdot
      + 8. * PI * mu * nu * N10 * q->r * cf[4][b + 1];
  }
}

/* src/cuda_quadrature.cu:64-313 */
extern "C" void cuda_Lamb(void)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  upload_nodes();
  lamb_args L;
  L.parts = g_dev.parts;
  L.p = g_dev.p; L.u = g_dev.u; L.v = g_dev.v; L.w = g_dev.w;
  L.cur = cur_coefs();
  for(int a = 0; a < 6; a++) { L.cf[a] = g_dev.coef[a]; L.cf0[a] = g_dev.coef[6 + a]; }
  L.stride = coeff_stride; L.np = nparts;
  L.mu = mu; L.nu = nu; L.rho_f = rho_f; L.relax = lamb_relax;
  L.gpx = gradP.x; L.gpy = gradP.y; L.gpz = gradP.z;
  L.bc = bc;
  L.G = bbb_make_geom();
  k_lamb<<<nparts, 32, 0, g_dev.stream>>>(L);
  BBB_LAUNCHED();
}

/* per-particle coefficient change, the computation compute_error
 * (src/quadrature_kernel.cu:578-654) intends, with a private sort list per
 * particle; then the device maximum */
__global__ void k_lamb_err(const double *const *unused, int np, int stride,
  double lamb_cut, const double *c0, const double *c1, const double *c2,
  const double *c3, const double *c4, const double *c5, const double *o0,
  const double *o1, const double *o2, const double *o3, const double *o4,
  const double *o5, double *partials, unsigned int *ticket, double *out)
{
  (void)unused;
  __shared__ double sh[32];
  double e = FLT_MIN;
  for(int part = blockIdx.x * blockDim.x + threadIdx.x; part < np;
      part += gridDim.x * blockDim.x) {
    const double *cs[6] = {c0, c1, c2, c3, c4, c5};
    const double *os[6] = {o0, o1, o2, o3, o4, o5};
    double big = -1.;
    for(int a = 0; a < 6; a++) for(int i = 0; i < stride; i++) {
      double c = cs[a][(long long)part * stride + i];
      if(c * c > FLT_MIN && fabs(c) > big) big = fabs(c);
    }
    double pe = FLT_MIN;
    if(big >= 0.) {
      for(int a = 0; a < 6; a++) for(int i = 0; i < stride; i++) {
        double c = cs[a][(long long)part * stride + i];
        if(!(c * c > FLT_MIN)) continue;
        if(fabs(c) > lamb_cut * big) {
          double div = fabs(c);
          if(div < 1e-16) div = 1e-16;
          double er = fabs((c - os[a][(long long)part * stride + i]) / div);
          if(er > pe) pe = er;
        }
      }
    }
    if(pe > e) e = pe;
  }
  double v[1] = {e};
  bbb_block_max<1>(v, sh);
  __shared__ unsigned int s_last;
  if(threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if(!s_last) return;
  __threadfence();
  double m[1] = {FLT_MIN};
  for(int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    m[0] = fmax(m[0], ((volatile double *)partials)[b]);
  bbb_block_max<1>(m, sh);
  if(threadIdx.x == 0) { *out = m[0]; *ticket = 0u; }
}

/* src/cuda_quadrature.cu:316-398 */
extern "C" real cuda_lamb_err(void)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return 0.;
  int blocks = (nparts + 255) / 256;
  if(blocks > 1184) blocks = 1184;
  double **c = g_dev.coef;
  k_lamb_err<<<blocks, 256, 0, g_dev.stream>>>(NULL, nparts, coeff_stride,
    lamb_cut, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9],
    c[10], c[11], g_dev.partials, g_dev.red_ticket + 8, g_dev.red_dev + 32);
  BBB_LAUNCHED();
  size_t n = sizeof(real) * (size_t)coeff_stride * nparts;
  for(int a = 0; a < 6; a++)
    BBB_CK(cudaMemcpyAsync(g_dev.coef[6 + a], g_dev.coef[a], n,
      cudaMemcpyDeviceToDevice, g_dev.stream));
  BBB_CK(cudaMemcpyAsync(g_dev.red_host, g_dev.red_dev + 32, sizeof(double),
    cudaMemcpyDeviceToHost, g_dev.stream));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  return g_dev.red_host[0];
}

/* src/cuda_particle.cu:1046-1081 */
extern "C" void cuda_store_coeffs(void)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  size_t n = sizeof(real) * (size_t)coeff_stride * nparts;
  for(int a = 0; a < 6; a++)
    BBB_CK(cudaMemcpyAsync(g_dev.coef[12 + a], g_dev.coef[a], n,
      cudaMemcpyDeviceToDevice, g_dev.stream));
}

/* ------------------------------------------------ Newton-Euler
 * move_parts_a/b and rotate (src/bluebottle_kernel.cu:2247-2398); the
 * interaction forces they integrate are computed below. */
__device__ void d_rotate(double qr, double qi, double qj, double qk,
  double *pi, double *pj, double *pk)
{
  double Pr = *pi * qi + *pj * qj + *pk * qk;
  double Pi = *pi * qr - *pj * qk + *pk * qj;
  double Pj = *pi * qk + *pj * qr - *pk * qi;
  double Pk = -*pi * qj + *pj * qi + *pk * qr;
  *pi = qr * Pi + qi * Pr + qj * Pk - qk * Pj;
  *pj = qr * Pj - qi * Pk + qj * Pr + qk * Pi;
  *pk = qr * Pk + qi * Pj - qj * Pi + qk * Pr;
}

__device__ void d_move(part_struct *q, int final, double dt, double rho_f,
  g_struct g, gradP_struct gp, bbb_geom G)
{
  double vol = 4. / 3. * PI * q->r * q->r * q->r;
  double m = vol * q->rho;
  if(q->translating) {
    q->udot = (q->Fx + q->kFx + q->iFx + q->aFx - vol * gp.x) / m
      + (q->rho - rho_f) / q->rho * g.x;
    q->vdot = (q->Fy + q->kFy + q->iFy + q->aFy - vol * gp.y) / m
      + (q->rho - rho_f) / q->rho * g.y;
    q->wdot = (q->Fz + q->kFz + q->iFz + q->aFz - vol * gp.z) / m
      + (q->rho - rho_f) / q->rho * g.z;
    q->u = q->u0 + 0.5 * dt * (q->udot + q->udot0);
    q->v = q->v0 + 0.5 * dt * (q->vdot + q->vdot0);
    q->w = q->w0 + 0.5 * dt * (q->wdot + q->wdot0);
    if(final) {
      q->x = q->x0 + 0.5 * dt * (q->u + q->u0);
      if(q->x < G.xs) q->x = q->x + G.xl;
      else if(q->x > G.xe) q->x = q->x - G.xl;
      q->y = q->y0 + 0.5 * dt * (q->v + q->v0);
      if(q->y < G.ys) q->y = q->y + G.yl;
      else if(q->y > G.ye) q->y = q->y - G.yl;
      q->z = q->z0 + 0.5 * dt * (q->w + q->w0);
      if(q->z < G.zs) q->z = q->z + G.zl;
      else if(q->z > G.ze) q->z = q->z - G.zl;
      q->x0 = q->x; q->y0 = q->y; q->z0 = q->z;
      q->u0 = q->u; q->v0 = q->v; q->w0 = q->w;
      q->udot0 = q->udot; q->vdot0 = q->vdot; q->wdot0 = q->wdot;
    }
  }
  if(q->rotating) {
    double I = 0.4 * m * q->r * q->r;
    q->oxdot = (q->Lx + q->iLx + q->aLx) / I;
    q->oydot = (q->Ly + q->iLy + q->aLy) / I;
    q->ozdot = (q->Lz + q->iLz + q->aLz) / I;
    q->ox = q->ox0 + 0.5 * dt * (q->oxdot + q->oxdot0);
    q->oy = q->oy0 + 0.5 * dt * (q->oydot + q->oydot0);
    q->oz = q->oz0 + 0.5 * dt * (q->ozdot + q->ozdot0);
    if(final) {
      double mag = 0.5 * sqrt(q->ox * q->ox + q->oy * q->oy + q->oz * q->oz);
      mag += 0.5 * sqrt(q->ox0 * q->ox0 + q->oy0 * q->oy0 + q->oz0 * q->oz0);
      double X = 0, Y = 0, Z = 0;
      if(mag > 0) {
        X = 0.5 * (q->ox + q->ox0) / mag;
        Y = 0.5 * (q->oy + q->oy0) / mag;
        Z = 0.5 * (q->oz + q->oz0) / mag;
      }
      double th = mag * dt;
      double qr = cos(0.5 * th), qi = X * sin(0.5 * th), qj = Y * sin(0.5 * th),
             qk = Z * sin(0.5 * th);
      d_rotate(qr, qi, qj, qk, &q->axx, &q->axy, &q->axz);
      d_rotate(qr, qi, qj, qk, &q->ayx, &q->ayy, &q->ayz);
      d_rotate(qr, qi, qj, qk, &q->azx, &q->azy, &q->azz);
      q->ox0 = q->ox; q->oy0 = q->oy; q->oz0 = q->oz;
      q->oxdot0 = q->oxdot; q->oydot0 = q->oydot; q->ozdot0 = q->ozdot;
    }
  }
}

/* ------------------------------------------------ interaction forces
 * Lubrication and Hertz contact between spheres and with Neumann walls,
 * springs (src/bluebottle_kernel.cu: collision_init :2400, bin_fill :2422,
 * bin_start :2454, collision_parts :2500, collision_walls :2875,
 * spring_parts :3592; sequence src/cuda_bluebottle.cu:4317-4554).  One
 * thread per particle does the reference's four per-particle kernels in
 * their order (each writes only its own particle and reads the others'
 * kinematics, which these kernels do not change).  Neighbours come from a
 * bin grid (binDom_init src/particle.c:598) built on the device by count,
 * scan, scatter and a per-bin sort by index, so a particle's partners are
 * visited in the reference's order: bins z, y, x from -1 to 1, particles
 * by index within a bin (its sort by bin is stable).  Kept as the
 * reference computes them: interactionLengthRatio enters as an int; the
 * contact-list searches read and write one slot past iSt / St (the bytes
 * that follow in part_struct); every wall's contact branch uses the south
 * wall's Dirichlet velocities; the east-wall contact torque takes the
 * function-scope Ftx (0 unless assigned earlier in the call); the x walls'
 * contact slip takes omega_x in place of omega_y. */
#define D_MAXN BBB_MAX_NEIGHBORS

struct bin_geom {
  int xn, yn, zn, s1, s2, s3;
  double xs, ys, zs, dx, dy, dz;
};

struct coll_args {
  double mu, rho_f, nu, dt;
  int ilr;                        /* (int) interactionLengthRatio */
  int overrun;                    /* option contact_overrun */
  double xs, xe, xl, ys, ye, yl, zs, ze, zl;
  BC bc;
};

static struct {
  int s3, np;
  bin_geom bg;
  int *cnt, *start, *fill, *list;
} g_bins;

__device__ __forceinline__ int d_ist_get(const part_struct *q, int k)
{
  int v;
  memcpy(&v, (const char *)q->iSt + sizeof(int) * k, sizeof(int));
  return v;
}
__device__ __forceinline__ void d_ist_set(part_struct *q, int k, int v)
{ memcpy((char *)q->iSt + sizeof(int) * k, &v, sizeof(int)); }
__device__ __forceinline__ double d_st_get(const part_struct *q, int k)
{
  double v;
  memcpy(&v, (const char *)q->St + sizeof(double) * k, sizeof(double));
  return v;
}
__device__ __forceinline__ void d_st_set(part_struct *q, int k, double v)
{ memcpy((char *)q->St + sizeof(double) * k, &v, sizeof(double)); }

/* The contact list of a sphere: partner keys iSt[0..11] with the impact
 * Stokes numbers St[0..11].  With `overrun` the searches test the slot
 * before the bound, as the reference's collision kernels do, and so reach
 * slot 12: the bytes that follow iSt and St in part_struct (the low word
 * of e_dry; iSt[0..1]) -- read, and written when all 12 slots are taken.
 * Without it they stop at the list's end: a partner not found is not
 * removed, and a new contact with no free slot is not stored (slot -1, its
 * current Stokes number is used). */
__device__ void d_contact_forget(part_struct *q, int key, int overrun)
{
  int k = 0;
  if(overrun) {
    while(d_ist_get(q, k) != key && k < D_MAXN) k++;
    if(d_ist_get(q, k) == key) { d_ist_set(q, k, -1); d_st_set(q, k, 0.); }
    return;
  }
  while(k < D_MAXN && d_ist_get(q, k) != key) k++;
  if(k < D_MAXN) { d_ist_set(q, k, -1); d_st_set(q, k, 0.); }
}

__device__ int d_contact_slot(part_struct *q, int key, double St, int overrun)
{
  int k = 0;
  if(overrun) {
    while(d_ist_get(q, k) != key && k < D_MAXN) k++;
    if(k == D_MAXN) {
      k = 0;
      while(d_ist_get(q, k) != -1 && k < D_MAXN) k++;
      d_ist_set(q, k, key);
      d_st_set(q, k, St);
    }
    return k;
  }
  while(k < D_MAXN && d_ist_get(q, k) != key) k++;
  if(k < D_MAXN) return k;
  k = 0;
  while(k < D_MAXN && d_ist_get(q, k) != -1) k++;
  if(k == D_MAXN) return -1;
  d_ist_set(q, k, key);
  d_st_set(q, k, St);
  return k;
}

/* the stored Stokes number of contact slot q, or St when it has none */
__device__ __forceinline__ double d_contact_st(const part_struct *q, int slot,
  double St)
{
  return slot >= 0 ? d_st_get(q, slot) : St;
}

__device__ __forceinline__ double d_min_image(double a, double b, double L,
  int periodic)
{
  double r = a - b, r1 = a - (b + L), r2 = a - (b - L);
  if(r1 * r1 < r * r) r = r1;
  if(r2 * r2 < r * r) r = r2;
  return periodic * r + (!periodic) * (a - b);
}

/* force and torque on particle pi from particle pj */
__device__ void d_pair_force(part_struct *pi, const part_struct *pj, int j,
  const coll_args &A)
{
  double eps = 0.01, mu = A.mu, rhof = A.rho_f, nu = A.nu, dt = A.dt;
  double ai = pi->r, aj = pj->r, B = aj / ai, hN = A.ilr * pi->r;
  double rx = d_min_image(pi->x, pj->x, A.xl, A.bc.uW == BBB_PERIODIC);
  double ry = d_min_image(pi->y, pj->y, A.yl, A.bc.vS == BBB_PERIODIC);
  double rz = d_min_image(pi->z, pj->z, A.zl, A.bc.wB == BBB_PERIODIC);
  double ux = 0.5 * ((pi->u - pj->u) + (pi->u0 - pj->u0));
  double uy = 0.5 * ((pi->v - pj->v) + (pi->v0 - pj->v0));
  double uz = 0.5 * ((pi->w - pj->w) + (pi->w0 - pj->w0));
  double r = sqrt(rx * rx + ry * ry + rz * rz);
  double omx = 0.5 * ((pi->ox + pj->ox) + (pi->ox0 + pj->ox0));
  double omy = 0.5 * ((pi->oy + pj->oy) + (pi->oy0 + pj->oy0));
  double omz = 0.5 * ((pi->oz + pj->oz) + (pi->oz0 + pj->oz0));
  double h = r - ai - aj;
  double nx = rx / r, ny = ry / r, nz = rz / r;
  double udotn = ux * nx + uy * ny + uz * nz;
  double unx = udotn * nx, uny = udotn * ny, unz = udotn * nz;
  double utx = ux - unx, uty = uy - uny, utz = uz - unz;
  double opB = 1 + B;
  double ocnx = omy * nz - omz * ny, ocny = -omx * nz + omz * nx, ocnz = omx * ny - omy * nx;
  double ucnx = uty * nz - utz * ny, ucny = -utx * nz + utz * nx, ucnz = utx * ny - uty * nx;
  double Fnx, Fny, Fnz, Ftx, Fty, Ftz, Lox, Loy, Loz;
  if(h < hN && h > 0) {
    d_contact_forget(pi, j, A.overrun);
    if(h < eps * pi->r) h = eps * pi->r;
    double ah = ai / h - ai / hN, lnah = log(hN / h);
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
    double St_now = 1. / 9. * pi->rho / rhof * 2. * pi->r * fabs(udotn) / nu;
    int q = d_contact_slot(pi, j, St_now, A.overrun);
    double Vx = -utx + 0.5 * (ai + aj + h) * ocnx;
    double Vy = -uty + 0.5 * (ai + aj + h) * ocny;
    double Vz = -utz + 0.5 * (ai + aj + h) * ocnz;
    double Hi = 0.5 * pi->E / (1. + pi->sigma);
    double kt = 8. / ((1. - pi->sigma * pi->sigma) / Hi + (1. - pi->sigma * pi->sigma) / Hi)
      / sqrt(1. / ai) * sqrt(-h);
    double Vdotn = Vx * nx + Vy * ny + Vz * nz;
    double sx = (Vx - Vdotn * nx) * dt, sy = (Vy - Vdotn * ny) * dt, sz = (Vz - Vdotn * nz) * dt;
    double k = 4. / 3. / ((1. - pi->sigma * pi->sigma) / pi->E
      + (1. - pj->sigma * pj->sigma) / pj->E) / sqrt(1. / ai + 1. / aj);
    double xcx0 = 1.e-4;
    double e = pi->e_dry + (1. + pi->e_dry) / d_contact_st(pi, q, St_now) * log(xcx0);
    if(e < 0) e = 0;
    double alpha = -2.263 * pow(e, 0.3948) + 2.22;
    double eta = alpha * sqrt(4. / 3. * PI * ai * ai * ai * pi->rho * k * sqrt(-h));
    Fnx = (sqrt(-h * h * h) * k - eta * udotn) * nx;
    Fny = (sqrt(-h * h * h) * k - eta * udotn) * ny;
    Fnz = (sqrt(-h * h * h) * k - eta * udotn) * nz;
    double cf = 0.5 * (pi->coeff_fric + pj->coeff_fric);
    Ftx = -kt * sx; Fty = -kt * sy; Ftz = -kt * sz;
    double Ftdotn = Ftx * nx + Fty * ny + Ftz * nz;
    Ftx = Ftx - Ftdotn * nx; Fty = Fty - Ftdotn * ny; Ftz = Ftz - Ftdotn * nz;
    double Ft = sqrt(Ftx * Ftx + Fty * Fty + Ftz * Ftz);
    double Fn = sqrt(Fnx * Fnx + Fny * Fny + Fnz * Fnz);
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

/* one wall: ax the normal axis, hi = 0 for W/S/B, 1 for E/N/T */
__device__ void d_wall_force(part_struct *p, int ax, int hi, const coll_args &A,
  double *Ftx_scope)
{
  const BC &bc = A.bc;
  double eps = 0.01, mu = A.mu, rhof = A.rho_f, nu = A.nu, dt = A.dt;
  double ai = p->r, hN = A.ilr * p->r;
  double pos[3] = {p->x, p->y, p->z}, vel[3] = {p->u, p->v, p->w};
  double vel0[3] = {p->u0, p->v0, p->w0};
  double om[3] = {p->ox, p->oy, p->oz}, om0[3] = {p->ox0, p->oy0, p->oz0};
  double wallpos, wv[3];
  int press, key = -10 - (2 * ax + hi);
  if(ax == 0) {
    wallpos = hi ? A.xe - bc.dsE : A.xs + bc.dsW;
    press = hi ? bc.pE : bc.pW;
    wv[0] = hi ? bc.uED : bc.uWD; wv[1] = hi ? bc.vED : bc.vWD; wv[2] = hi ? bc.wED : bc.wWD;
  } else if(ax == 1) {
    wallpos = hi ? A.ye - bc.dsN : A.ys + bc.dsS;
    press = hi ? bc.pN : bc.pS;
    wv[0] = hi ? bc.uND : bc.uSD; wv[1] = hi ? bc.vND : bc.vSD; wv[2] = hi ? bc.wND : bc.wSD;
  } else {
    wallpos = hi ? A.ze - bc.dsT : A.zs + bc.dsB;
    press = hi ? bc.pT : bc.pB;
    wv[0] = hi ? bc.uTD : bc.uBD; wv[1] = hi ? bc.vTD : bc.vBD; wv[2] = hi ? bc.wTD : bc.wBD;
  }
  double sd[3] = {bc.uSD, bc.vSD, bc.wSD};
  double h = fabs(pos[ax] - wallpos) - ai;
  double isTrue = (press == BBB_NEUMANN);
  int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
  double sg = hi ? -1. : 1.;
  if(h < hN && h > 0) {
    d_contact_forget(p, key, A.overrun);
    if(h < eps * p->r) h = eps * p->r;
    double ah = ai / h - ai / hN, lnah = log(hN / h);
    double Un = vel[ax] - wv[ax];
    double Ut[3] = {vel[0] - wv[0], vel[1] - wv[1], vel[2] - wv[2]};
    Ut[ax] = 0.;
    double F[3] = {0., 0., 0.}, Ft[3] = {0., 0., 0.}, L[3] = {0., 0., 0.};
    F[ax] = -6. * PI * mu * ai * Un * ah;
    Ft[t1] = -6. * PI * mu * ai * Ut[t1] * 8. / 15. * lnah;
    Ft[t2] = -6. * PI * mu * ai * Ut[t2] * 8. / 15. * lnah;
    double so = (ax == 1) ? -sg : sg;
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
    double Un = sg * (vel[ax] - wv[ax]);
    double Ut1 = 0.5 * (vel[t1] + vel0[t1]) - sd[t1];
    double Ut2 = 0.5 * (vel[t2] + vel0[t2]) - sd[t2];
    double St_now = 1. / 9. * p->rho / rhof * 2. * p->r * fabs(Un) / nu;
    int q = d_contact_slot(p, key, St_now, A.overrun);
    double o[3] = {0.5 * (om[0] + om0[0]), 0.5 * (om[1] + om0[1]), 0.5 * (om[2] + om0[2])};
    double so = (ax == 1) ? -1. : 1.;
    double o2 = ax == 0 ? o[0] : o[t1];
    double V1 = sg * (Ut1 - so * (ai + 0.5 * h) * o[t2]);
    double V2 = sg * (Ut2 + so * (ai + 0.5 * h) * o2);
    double Hi = 0.5 * p->E / (1. + p->sigma);
    double kt = 8. / ((1. - p->sigma * p->sigma) / Hi + (1. - p->sigma * p->sigma) / Hi)
      / sqrt(1. / ai) * sqrt(-h);
    double s1 = V1 * dt, s2 = V2 * dt;
    double k = 4. / 3. / ((1. - p->sigma * p->sigma) / p->E + (1. - p->sigma * p->sigma) / p->E)
      / sqrt(1. / ai);
    double xcx0 = 1.e-4;
    double e = p->e_dry + (1. + p->e_dry) / d_contact_st(p, q, St_now) * log(xcx0);
    if(e < 0) e = 0;
    double alpha = -2.263 * pow(e, 0.3948) + 2.22;
    double eta = alpha * sqrt(4. / 3. * PI * ai * ai * ai * p->rho * k * sqrt(-h));
    double cf = p->coeff_fric;
    double F1 = -kt * s1, F2 = -kt * s2;
    double Ft = sqrt(F1 * F1 + F2 * F2);
    double Fn = sqrt(-h * h * h) * k - eta * Un;
    if(Ft > fabs(cf * Fn)) {
      F1 = cf * Fn * F1 / Ft;
      F2 = cf * Fn * F2 / Ft;
    }
    double arm = ai + 0.5 * h;
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

__global__ void k_bin_count(part_struct *parts, int np, bin_geom bg, int *cnt)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= np) return;
  part_struct *q = &parts[i];
  int ib = (int)floor((q->x - bg.xs) / bg.dx);
  int jb = (int)floor((q->y - bg.ys) / bg.dy);
  int kb = (int)floor((q->z - bg.zs) / bg.dz);
  int c = ib + jb * bg.s1 + kb * bg.s2;
  q->bin = c;
  if(c >= 0 && c < bg.s3) atomicAdd(&cnt[c], 1);
}

/* exclusive scan of the bin counts (one block) */
__global__ void k_bin_scan(const int *cnt, int *start, int n)
{
  __shared__ int part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int per = (n + nt - 1) / nt, a = t * per, b = min(n, a + per);
  int s = 0;
  for(int c = a; c < b; c++) s += cnt[c];
  part[t] = s;
  __syncthreads();
  if(t == 0) {
    int run = 0;
    for(int q = 0; q < nt; q++) { int v = part[q]; part[q] = run; run += v; }
  }
  __syncthreads();
  s = part[t];
  for(int c = a; c < b; c++) { start[c] = s; s += cnt[c]; }
}

__global__ void k_bin_scatter(const part_struct *parts, int np, bin_geom bg,
  const int *start, int *fill, int *list)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= np) return;
  int c = parts[i].bin;
  if(c < 0 || c >= bg.s3) return;
  int slot = atomicAdd(&fill[c], 1);
  list[start[c] + slot] = i;
}

/* particles of each bin by index (the order of a stable sort by bin) */
__global__ void k_bin_sort(const int *start, const int *cnt, int *list, int n)
{
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= n) return;
  int a = start[c], m = cnt[c];
  for(int x = 1; x < m; x++) {
    int v = list[a + x], y = x - 1;
    while(y >= 0 && list[a + y] > v) { list[a + y + 1] = list[a + y]; y--; }
    list[a + y + 1] = v;
  }
}

__global__ void k_interact(part_struct *parts, int np, bin_geom bg,
  const int *start, const int *cnt, const int *list, coll_args A)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= np) return;
  part_struct *pi = &parts[i];
  pi->iFx = 0.; pi->iFy = 0.; pi->iFz = 0.;
  pi->iLx = 0.; pi->iLy = 0.; pi->iLz = 0.;
  if(np > 1) {
    int bin = pi->bin;
    int kbin = bin / bg.s2, jbin = (bin - kbin * bg.s2) / bg.s1;
    int ibin = bin - kbin * bg.s2 - jbin * bg.s1;
    int fW = 0, fE = bg.xn - 1, fS = 0, fN = bg.yn - 1, fB = 0, fT = bg.zn - 1;
    int xnb = bg.xn > 2, ynb = bg.yn > 2, znb = bg.zn > 2;
    const BC &bc = A.bc;
    for(int n = -1; n <= 1; n++) {
      int ks;
      if((n == -1 && kbin == fB && bc.uB != BBB_PERIODIC) ||
         (n == 1 && kbin == fT && bc.uT != BBB_PERIODIC) ||
         (n == -1 && kbin == fB && bc.uB == BBB_PERIODIC && znb == 0) ||
         (n == 1 && kbin == fT && bc.uT == BBB_PERIODIC && znb == 0)) continue;
      else if(n == -1 && kbin == fB) ks = fT * bg.s2;
      else if(n == 1 && kbin == fT) ks = fB * bg.s2;
      else ks = (kbin + n) * bg.s2;
      for(int m = -1; m <= 1; m++) {
        int js;
        if((m == -1 && jbin == fS && bc.uS != BBB_PERIODIC) ||
           (m == 1 && jbin == fN && bc.uN != BBB_PERIODIC) ||
           (m == -1 && jbin == fS && bc.uS == BBB_PERIODIC && ynb == 0) ||
           (m == 1 && jbin == fN && bc.uN == BBB_PERIODIC && ynb == 0)) continue;
        else if(m == -1 && jbin == fS) js = fN * bg.s1;
        else if(m == 1 && jbin == fN) js = fS * bg.s1;
        else js = (jbin + m) * bg.s1;
        for(int l = -1; l <= 1; l++) {
          int is;
          if((l == -1 && ibin == fW && bc.uW != BBB_PERIODIC) ||
             (l == 1 && ibin == fE && bc.uE != BBB_PERIODIC) ||
             (l == -1 && ibin == fW && bc.uW == BBB_PERIODIC && xnb == 0) ||
             (l == 1 && ibin == fE && bc.uE == BBB_PERIODIC && xnb == 0)) continue;
          else if(l == -1 && ibin == fW) is = fE;
          else if(l == 1 && ibin == fE) is = fW;
          else is = ibin + l;
          int adj = is + js + ks;
          if(adj < 0 || adj >= bg.s3) continue;
          int a = start[adj], m2 = cnt[adj];
          for(int t = a; t < a + m2; t++) {
            int j = list[t];
            if(j != i) d_pair_force(pi, &parts[j], j, A);
          }
        }
      }
    }
  }
  if(pi->spring_k > 0.) {
    double nx = pi->x - pi->spring_x, ny = pi->y - pi->spring_y, nz = pi->z - pi->spring_z;
    double n = sqrt(nx * nx + ny * ny + nz * nz);
    double lx = pi->spring_l * (nx / n), ly = pi->spring_l * (ny / n),
           lz = pi->spring_l * (nz / n);
    pi->kFx = -pi->spring_k * (pi->x - pi->spring_x - lx);
    pi->kFy = -pi->spring_k * (pi->y - pi->spring_y - ly);
    pi->kFz = -pi->spring_k * (pi->z - pi->spring_z - lz);
  }
  double Ftx_scope = 0.;
  for(int w = 0; w < 6; w++) d_wall_force(pi, w / 2, w % 2, A, &Ftx_scope);
}

__global__ void k_move(part_struct *parts, int np, int final, double dt,
  double rho_f, g_struct g, gradP_struct gp, bbb_geom G)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= np) return;
  d_move(&parts[i], final, dt, rho_f, g, gp, G);
}

/* the bin grid of binDom (binDom_init, src/particle.c:598, filled on the
 * host by bbb_parts_init or by the reference's own host code) */
static void bins_setup(void)
{
  if(g_bins.cnt && g_bins.np == nparts) return;
  bin_geom &b = g_bins.bg;
  b.xs = binDom.xs; b.ys = binDom.ys; b.zs = binDom.zs;
  b.dx = binDom.dx; b.dy = binDom.dy; b.dz = binDom.dz;
  b.xn = binDom.xn; b.yn = binDom.yn; b.zn = binDom.zn;
  b.s1 = binDom.Gcc.s1; b.s2 = binDom.Gcc.s2; b.s3 = binDom.Gcc.s3;
  if(b.s3 <= 0 || b.s1 <= 0 || b.s2 <= 0) {
    bbb_set_status(BBB_ERR_CONFIG, "collision bins (binDom) not set up");
    b.s3 = 0;
    return;
  }
  g_bins.s3 = b.s3;
  g_bins.np = nparts;
  int *ps[3];
  for(int a = 0; a < 3; a++)
    if(cudaMalloc((void **)&ps[a], sizeof(int) * (size_t)b.s3) != cudaSuccess)
      bbb_set_status(BBB_ERR_CUDA, "cudaMalloc bins");
  g_bins.cnt = ps[0]; g_bins.start = ps[1]; g_bins.fill = ps[2];
  if(cudaMalloc((void **)&g_bins.list, sizeof(int) * (size_t)(nparts > 0 ? nparts : 1)) != cudaSuccess)
    bbb_set_status(BBB_ERR_CUDA, "cudaMalloc bins");
}

void bbb_bins_free(void)
{
  if(g_bins.cnt) {
    cudaFree(g_bins.cnt); cudaFree(g_bins.start); cudaFree(g_bins.fill);
    cudaFree(g_bins.list);
  }
  memset(&g_bins, 0, sizeof(g_bins));
}

static coll_args make_coll_args(void)
{
  coll_args A;
  A.mu = mu; A.rho_f = rho_f; A.nu = nu; A.dt = dt;
  A.ilr = (int)interactionLengthRatio;
  A.overrun = g_opt.contact_overrun;
  A.xs = Dom.xs; A.xe = Dom.xe; A.xl = Dom.xl;
  A.ys = Dom.ys; A.ye = Dom.ye; A.yl = Dom.yl;
  A.zs = Dom.zs; A.ze = Dom.ze; A.zl = Dom.zl;
  A.bc = bc;
  return A;
}

/* interaction forces, Newton-Euler half step, interaction forces again;
 * the final call adds the position update */
static void move_parts_seq(int final)
{
  bbb_dev_require();
  if(!g_dev.ready || nparts <= 0 || g_dev.np != nparts) return;
  int nb = (nparts + 127) / 128;
  coll_args A = make_coll_args();
  bbb_geom G = bbb_make_geom();
  if(nparts > 1) {
    bins_setup();
    if(g_bins.bg.s3 <= 0) return;
    const bin_geom &bg = g_bins.bg;
    BBB_CK(cudaMemsetAsync(g_bins.cnt, 0, sizeof(int) * (size_t)bg.s3, g_dev.stream));
    BBB_CK(cudaMemsetAsync(g_bins.fill, 0, sizeof(int) * (size_t)bg.s3, g_dev.stream));
    k_bin_count<<<nb, 128, 0, g_dev.stream>>>(g_dev.parts, nparts, bg, g_bins.cnt);
    BBB_LAUNCHED();
    k_bin_scan<<<1, 1024, 0, g_dev.stream>>>(g_bins.cnt, g_bins.start, bg.s3);
    BBB_LAUNCHED();
    k_bin_scatter<<<nb, 128, 0, g_dev.stream>>>(g_dev.parts, nparts, bg,
      g_bins.start, g_bins.fill, g_bins.list);
    BBB_LAUNCHED();
    k_bin_sort<<<(bg.s3 + 255) / 256, 256, 0, g_dev.stream>>>(g_bins.start,
      g_bins.cnt, g_bins.list, bg.s3);
    BBB_LAUNCHED();
  }
  bin_geom bg = g_bins.bg;
  for(int pass = 0; pass < 2; pass++) {
    k_interact<<<nb, 128, 0, g_dev.stream>>>(g_dev.parts, nparts, bg,
      g_bins.start, g_bins.cnt, g_bins.list, A);
    BBB_LAUNCHED();
    if(pass == 0) {
      k_move<<<nb, 128, 0, g_dev.stream>>>(g_dev.parts, nparts, 0, dt, rho_f, g,
        gradP, G);
      BBB_LAUNCHED();
    }
  }
  if(final) {
    k_move<<<nb, 128, 0, g_dev.stream>>>(g_dev.parts, nparts, 1, dt, rho_f, g,
      gradP, G);
    BBB_LAUNCHED();
  }
}

/* src/cuda_bluebottle.cu:4317-4433 */
extern "C" void cuda_move_parts_sub(void)
{
  move_parts_seq(0);
}

/* src/cuda_bluebottle.cu:4435-4554 */
extern "C" void cuda_move_parts(void)
{
  move_parts_seq(1);
  g_dev.lf_geo_valid = 0;   /* positions moved */
}
