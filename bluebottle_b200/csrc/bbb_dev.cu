/* bbb_dev.cu -- device state, host<->device transfer, domain boundary
 * conditions, forcing, solvability, projection, pressure update, history
 * store and the CFL time step.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "bbb_internal.h"
#include "bbb_reduce.cuh"

bbb_dev g_dev;

bbb_geom bbb_make_geom(void)
{
  bbb_geom g;
  const dom_struct *d = &Dom;
  g.nx = d->xn; g.ny = d->yn; g.nz = d->zn;
  g.cc_s1 = d->Gcc.s1b; g.cc_s2 = d->Gcc.s2b;
  g.fx_s1 = d->Gfx.s1b; g.fx_s2 = d->Gfx.s2b;
  g.fy_s1 = d->Gfy.s1b; g.fy_s2 = d->Gfy.s2b;
  g.fz_s1 = d->Gfz.s1b; g.fz_s2 = d->Gfz.s2b;
  g.cc_n = d->Gcc.s3b; g.fx_n = d->Gfx.s3b; g.fy_n = d->Gfy.s3b;
  g.fz_n = d->Gfz.s3b;
  g.dx = d->dx; g.dy = d->dy; g.dz = d->dz;
  g.xs = d->xs; g.ys = d->ys; g.zs = d->zs;
  g.xe = d->xe; g.ye = d->ye; g.ze = d->ze;
  g.xl = d->xl; g.yl = d->yl; g.zl = d->zl;
  return g;
}

void bbb_dev_require(void)
{
  if(!g_dev.ready) bbb_set_status(BBB_ERR_STATE, "cuda_dom_malloc not called");
}

extern "C" long long bbb_kernel_launches(void) { return g_dev.launches; }
extern "C" void bbb_reset_kernel_launches(void) { g_dev.launches = 0; }

extern "C" int bbb_device_count(void)
{
  int n = 0;
  if(cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

/* ------------------------------------------------ allocation */

template <typename T>
static T *dalloc(long long n)
{
  T *p = NULL;
  if(n < 1) n = 1;
  cudaError_t e = cudaMalloc((void **)&p, sizeof(T) * (size_t)n);
  if(e != cudaSuccess) { bbb_set_status(BBB_ERR_CUDA, "cudaMalloc"); return NULL; }
  cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, g_dev.stream);
  gpumem += (long)(sizeof(T) * n);
  return p;
}

template <typename T>
static void dfree(T *&p) { if(p) cudaFree(p); p = NULL; }

/* src/cuda_bluebottle.cu:36-297 */
extern "C" void cuda_dom_malloc(void)
{
  /* a second set-up (a new domain in the same process) releases the
   * previous device state first: its arrays are sized for the old domain */
  if(g_dev.ready) {
    cuda_part_free();
    cuda_dom_free();
  }
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    bbb_set_status(BBB_ERR_CUDA, "no CUDA device");
    return;
  }
  g_dev.dev = dev_start < ndev ? dev_start : 0;
  BBB_CK(cudaSetDevice(g_dev.dev));
  BBB_CK(cudaStreamCreateWithFlags(&g_dev.stream, cudaStreamNonBlocking));
  const dom_struct *d = &Dom;
  long long ncc = d->Gcc.s3b, nfx = d->Gfx.s3b, nfy = d->Gfy.s3b,
            nfz = d->Gfz.s3b;
  g_dev.p0 = dalloc<real>(ncc); g_dev.p = dalloc<real>(ncc);
  g_dev.phi = dalloc<real>(ncc);
  g_dev.u = dalloc<real>(nfx); g_dev.u0 = dalloc<real>(nfx); g_dev.us = dalloc<real>(nfx);
  g_dev.v = dalloc<real>(nfy); g_dev.v0 = dalloc<real>(nfy); g_dev.vs = dalloc<real>(nfy);
  g_dev.w = dalloc<real>(nfz); g_dev.w0 = dalloc<real>(nfz); g_dev.ws = dalloc<real>(nfz);
  g_dev.conv_u = dalloc<real>(nfx); g_dev.conv0_u = dalloc<real>(nfx);
  g_dev.conv_v = dalloc<real>(nfy); g_dev.conv0_v = dalloc<real>(nfy);
  g_dev.conv_w = dalloc<real>(nfz); g_dev.conv0_w = dalloc<real>(nfz);
  g_dev.diff_u = dalloc<real>(nfx); g_dev.diff0_u = dalloc<real>(nfx);
  g_dev.diff_v = dalloc<real>(nfy); g_dev.diff0_v = dalloc<real>(nfy);
  g_dev.diff_w = dalloc<real>(nfz); g_dev.diff0_w = dalloc<real>(nfz);
  g_dev.phase = dalloc<int>(ncc); g_dev.phase_shell = dalloc<int>(ncc);
  g_dev.flag_u = dalloc<int>(nfx); g_dev.flag_v = dalloc<int>(nfy);
  g_dev.flag_w = dalloc<int>(nfz);
  long long nx = d->xn, ny = d->yn, nz = d->zn;
  long long np_ = nx * ny * nz, nu_ = (nx + 1) * ny * nz, nv_ = nx * (ny + 1) * nz,
            nw_ = nx * ny * (nz + 1);
  g_dev.mask_p = dalloc<uint8_t>(np_); g_dev.mask_u = dalloc<uint8_t>(nu_);
  g_dev.mask_v = dalloc<uint8_t>(nv_); g_dev.mask_w = dalloc<uint8_t>(nw_);
  g_dev.masks_valid = 0;
  long long nmax = np_;
  if(nu_ > nmax) nmax = nu_;
  if(nv_ > nmax) nmax = nv_;
  if(nw_ > nmax) nmax = nw_;
  g_dev.nmax = nmax;
  g_dev.kb = dalloc<double>(nmax); g_dev.kx = dalloc<double>(nmax);
  g_dev.kr = dalloc<double>(nmax); g_dev.krh = dalloc<double>(nmax);
  g_dev.kp[0] = dalloc<double>(nmax); g_dev.kp[1] = dalloc<double>(nmax);
  g_dev.kv[0] = dalloc<double>(nmax); g_dev.kv[1] = dalloc<double>(nmax);
  g_dev.ks = dalloc<double>(nmax); g_dev.kt = dalloc<double>(nmax);
  g_dev.max_blocks = 1 << 20;
  g_dev.partials = dalloc<double>((long long)g_dev.max_blocks * 8);
  g_dev.kry = dalloc<bbb_kry>(1);
  BBB_CK(cudaMallocHost((void **)&g_dev.kry_host, sizeof(bbb_kry)));
  BBB_CK(cudaMallocHost((void **)&g_dev.red_host, sizeof(real) * 64));
  g_dev.red_dev = dalloc<double>(64);
  g_dev.red_ticket = dalloc<unsigned int>(16);
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  g_dev.ready = (bbb_last_status() == BBB_OK);
}

/* src/cuda_particle.cu:28-167 */
extern "C" void cuda_part_malloc(void)
{
  g_dev.np = nparts;
  g_dev.stride = coeff_stride;
  long long nc = (long long)nparts * coeff_stride;
  g_dev.parts = dalloc<part_struct>(nparts);
  for(int a = 0; a < 18; a++) g_dev.coef[a] = dalloc<real>(nc);
  long long nn = (long long)nparts * BBB_NNODES;
  g_dev.node_pp = dalloc<real>(nn); g_dev.node_ur = dalloc<real>(nn);
  g_dev.node_ut = dalloc<real>(nn); g_dev.node_up = dalloc<real>(nn);
  g_dev.perr = dalloc<real>(nparts);
}

static real **host_coef(int a)
{
  static real **tab[18] = {&pnm_re, &pnm_im, &phinm_re, &phinm_im, &chinm_re,
    &chinm_im, &pnm_re0, &pnm_im0, &phinm_re0, &phinm_im0, &chinm_re0,
    &chinm_im0, &pnm_re00, &pnm_im00, &phinm_re00, &phinm_im00, &chinm_re00,
    &chinm_im00};
  return tab[a];
}

static void h2d(void *dst, const void *src, size_t n)
{
  if(dst && src && n) BBB_CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, g_dev.stream));
}
static void d2h(void *dst, const void *src, size_t n)
{
  if(dst && src && n) BBB_CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, g_dev.stream));
}

/* src/cuda_bluebottle.cu:299-528 */
extern "C" void cuda_dom_push(void)
{
  bbb_dev_require();
  const dom_struct *d = &Dom;
  size_t cc = sizeof(real) * d->Gcc.s3b, fx = sizeof(real) * d->Gfx.s3b,
         fy = sizeof(real) * d->Gfy.s3b, fz = sizeof(real) * d->Gfz.s3b;
  h2d(g_dev.p0, p0, cc); h2d(g_dev.p, p, cc); h2d(g_dev.phi, phi, cc);
  h2d(g_dev.u, u, fx); h2d(g_dev.v, v, fy); h2d(g_dev.w, w, fz);
  h2d(g_dev.u0, u0, fx); h2d(g_dev.v0, v0, fy); h2d(g_dev.w0, w0, fz);
  h2d(g_dev.us, u_star, fx); h2d(g_dev.vs, v_star, fy); h2d(g_dev.ws, w_star, fz);
  h2d(g_dev.diff0_u, diff0_u, fx); h2d(g_dev.diff0_v, diff0_v, fy);
  h2d(g_dev.diff0_w, diff0_w, fz);
  h2d(g_dev.conv0_u, conv0_u, fx); h2d(g_dev.conv0_v, conv0_v, fy);
  h2d(g_dev.conv0_w, conv0_w, fz);
  h2d(g_dev.diff_u, diff_u, fx); h2d(g_dev.diff_v, diff_v, fy);
  h2d(g_dev.diff_w, diff_w, fz);
  h2d(g_dev.conv_u, conv_u, fx); h2d(g_dev.conv_v, conv_v, fy);
  h2d(g_dev.conv_w, conv_w, fz);
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
}

/* src/cuda_bluebottle.cu:794-1195 */
extern "C" void cuda_dom_pull(void)
{
  bbb_dev_require();
  const dom_struct *d = &Dom;
  size_t cc = sizeof(real) * d->Gcc.s3b, fx = sizeof(real) * d->Gfx.s3b,
         fy = sizeof(real) * d->Gfy.s3b, fz = sizeof(real) * d->Gfz.s3b;
  d2h(p0, g_dev.p0, cc); d2h(p, g_dev.p, cc); d2h(phi, g_dev.phi, cc);
  d2h(u, g_dev.u, fx); d2h(v, g_dev.v, fy); d2h(w, g_dev.w, fz);
  d2h(u0, g_dev.u0, fx); d2h(v0, g_dev.v0, fy); d2h(w0, g_dev.w0, fz);
  d2h(u_star, g_dev.us, fx); d2h(v_star, g_dev.vs, fy); d2h(w_star, g_dev.ws, fz);
  d2h(diff0_u, g_dev.diff0_u, fx); d2h(diff0_v, g_dev.diff0_v, fy);
  d2h(diff0_w, g_dev.diff0_w, fz);
  d2h(conv0_u, g_dev.conv0_u, fx); d2h(conv0_v, g_dev.conv0_v, fy);
  d2h(conv0_w, g_dev.conv0_w, fz);
  d2h(diff_u, g_dev.diff_u, fx); d2h(diff_v, g_dev.diff_v, fy);
  d2h(diff_w, g_dev.diff_w, fz);
  d2h(conv_u, g_dev.conv_u, fx); d2h(conv_v, g_dev.conv_v, fy);
  d2h(conv_w, g_dev.conv_w, fz);
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
}

/* src/cuda_particle.cu:170-232 */
extern "C" void cuda_part_push(void)
{
  bbb_dev_require();
  const dom_struct *d = &Dom;
  if(nparts > 0 && g_dev.np == nparts) {
    h2d(g_dev.parts, parts, sizeof(part_struct) * nparts);
    size_t nc = sizeof(real) * (size_t)coeff_stride * nparts;
    for(int a = 0; a < 18; a++) h2d(g_dev.coef[a], *host_coef(a), nc);
  }
  h2d(g_dev.phase, phase, sizeof(int) * d->Gcc.s3b);
  h2d(g_dev.phase_shell, phase_shell, sizeof(int) * d->Gcc.s3b);
  h2d(g_dev.flag_u, flag_u, sizeof(int) * d->Gfx.s3b);
  h2d(g_dev.flag_v, flag_v, sizeof(int) * d->Gfy.s3b);
  h2d(g_dev.flag_w, flag_w, sizeof(int) * d->Gfz.s3b);
  g_dev.masks_valid = 0;
  g_dev.lf_valid = 0;
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
}

/* src/cuda_particle.cu:234-354 */
extern "C" void cuda_part_pull(void)
{
  bbb_dev_require();
  const dom_struct *d = &Dom;
  if(nparts > 0 && g_dev.np == nparts) {
    d2h(parts, g_dev.parts, sizeof(part_struct) * nparts);
    size_t nc = sizeof(real) * (size_t)coeff_stride * nparts;
    for(int a = 0; a < 18; a++) d2h(*host_coef(a), g_dev.coef[a], nc);
  }
  d2h(phase, g_dev.phase, sizeof(int) * d->Gcc.s3b);
  d2h(phase_shell, g_dev.phase_shell, sizeof(int) * d->Gcc.s3b);
  d2h(flag_u, g_dev.flag_u, sizeof(int) * d->Gfx.s3b);
  d2h(flag_v, g_dev.flag_v, sizeof(int) * d->Gfy.s3b);
  d2h(flag_w, g_dev.flag_w, sizeof(int) * d->Gfz.s3b);
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
}

/* the host particle array is page-locked on first use so that the
 * per-step exchange runs as a DMA from pinned memory */
static part_struct *g_pinned_parts = NULL;
static void pin_parts(void)
{
  if(nparts <= 0 || parts == g_pinned_parts) return;
  if(g_pinned_parts) cudaHostUnregister(g_pinned_parts);
  g_pinned_parts = NULL;
  if(cudaHostRegister(parts, sizeof(part_struct) * nparts, cudaHostRegisterDefault)
    == cudaSuccess) g_pinned_parts = parts;
  else cudaGetLastError();
}

extern "C" void bbb_part_state_push(void)
{
  bbb_dev_require();
  pin_parts();
  if(nparts > 0 && g_dev.np == nparts)
    h2d(g_dev.parts, parts, sizeof(part_struct) * nparts);
  g_dev.lf_geo_valid = 0;
}

/* device-side time marks on the library stream */
static cudaEvent_t g_marks[8];
extern "C" void bbb_mark(int i)
{
  if(i < 0 || i >= 8) return;
  if(!g_marks[i]) BBB_CK(cudaEventCreate(&g_marks[i]));
  BBB_CK(cudaEventRecord(g_marks[i], g_dev.stream));
}

extern "C" double bbb_mark_elapsed(int a, int b)
{
  if(a < 0 || a >= 8 || b < 0 || b >= 8 || !g_marks[a] || !g_marks[b]) return -1.;
  BBB_CK(cudaEventSynchronize(g_marks[b]));
  float ms = 0.f;
  if(cudaEventElapsedTime(&ms, g_marks[a], g_marks[b]) != cudaSuccess) return -1.;
  return ms;
}

extern "C" void bbb_part_state_pull(void)
{
  bbb_dev_require();
  if(nparts > 0 && g_dev.np == nparts)
    d2h(parts, g_dev.parts, sizeof(part_struct) * nparts);
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
}

extern "C" void cuda_dom_free(void)
{
  if(!g_dev.ready) return;
  cudaStreamSynchronize(g_dev.stream);
  bbb_learn_release();
  bbb_snapshot_release();
  real **rs[] = {&g_dev.p0, &g_dev.p, &g_dev.phi, &g_dev.u, &g_dev.v, &g_dev.w,
    &g_dev.u0, &g_dev.v0, &g_dev.w0, &g_dev.us, &g_dev.vs, &g_dev.ws,
    &g_dev.conv_u, &g_dev.conv_v, &g_dev.conv_w, &g_dev.conv0_u,
    &g_dev.conv0_v, &g_dev.conv0_w, &g_dev.diff_u, &g_dev.diff_v,
    &g_dev.diff_w, &g_dev.diff0_u, &g_dev.diff0_v, &g_dev.diff0_w};
  for(size_t a = 0; a < sizeof(rs) / sizeof(rs[0]); a++) dfree(*rs[a]);
  dfree(g_dev.phase); dfree(g_dev.phase_shell);
  dfree(g_dev.flag_u); dfree(g_dev.flag_v); dfree(g_dev.flag_w);
  dfree(g_dev.mask_p); dfree(g_dev.mask_u); dfree(g_dev.mask_v); dfree(g_dev.mask_w);
  double **ks[] = {&g_dev.kb, &g_dev.kx, &g_dev.kr, &g_dev.krh, &g_dev.kp[0],
    &g_dev.kp[1], &g_dev.kv[0], &g_dev.kv[1], &g_dev.ks, &g_dev.kt,
    &g_dev.partials, &g_dev.red_dev};
  for(size_t a = 0; a < sizeof(ks) / sizeof(ks[0]); a++) dfree(*ks[a]);
  float **fs[] = {&g_dev.fb, &g_dev.fx, &g_dev.fr, &g_dev.frh, &g_dev.fp[0],
    &g_dev.fp[1], &g_dev.fv[0], &g_dev.fv[1], &g_dev.fs, &g_dev.ft};
  for(size_t a = 0; a < sizeof(fs) / sizeof(fs[0]); a++) dfree(*fs[a]);
  dfree(g_dev.kry); dfree(g_dev.kry_inner); dfree(g_dev.red_ticket);
  if(g_pinned_parts) { cudaHostUnregister(g_pinned_parts); g_pinned_parts = NULL; }
  if(g_dev.kry_host) cudaFreeHost(g_dev.kry_host);
  if(g_dev.red_host) cudaFreeHost(g_dev.red_host);
  g_dev.kry_host = NULL; g_dev.red_host = NULL;
  cudaStreamDestroy(g_dev.stream);
  g_dev.ready = 0;
}

extern "C" void cuda_part_free(void)
{
  bbb_bins_free();
  dfree(g_dev.parts);
  for(int a = 0; a < 18; a++) dfree(g_dev.coef[a]);
  dfree(g_dev.node_pp); dfree(g_dev.node_ur); dfree(g_dev.node_ut);
  dfree(g_dev.node_up); dfree(g_dev.perr);
  dfree(g_dev.lf_idx); dfree(g_dev.lf_part); dfree(g_dev.lf_geo);
  dfree(g_dev.lf_count);
  dfree(g_dev.lf_pcnt); dfree(g_dev.lf_pstart); dfree(g_dev.lf_pfill);
  g_dev.lf_np = 0;
  g_dev.lf_cap = 0; g_dev.lf_n = 0; g_dev.lf_valid = 0; g_dev.lf_geo_valid = 0;
  g_dev.np = 0;
}

/* ------------------------------------------------ boundary conditions
 * Face kernels of src/bluebottle_kernel.cu:26-1248 in the dispatch order of
 * src/cuda_bluebottle.cu:1549-3420.  One launch per axis handles both faces
 * of that axis for every requested field, low face first, so the result
 * equals the reference's face-by-face sequence: the y launch reads the x
 * ghosts the x launch wrote, and the z launch reads both. */

struct bc_face_set {
  real *f[4];          /* p (cell), u, v, w; NULL = skip            */
  int type[4][2];      /* [field][lo/hi]                           */
  real val[4][2];      /* Dirichlet values                         */
  int s1[4], s2[4];    /* ghosted strides                          */
  int n[4][3];         /* ghosted extents nb per axis              */
};

__device__ __forceinline__ void bc_line(real *f, long long base, long long st,
  int nb, int type_lo, int type_hi, real vlo, real vhi, int normal)
{
  /* indices along the line: 0 = ghost, 1 = first interior, nb-2 = last
   * interior, nb-1 = ghost */
  int s = 1, e = nb - 1, sb = 0, eb = nb;
#define AT(q) f[base + (long long)(q) * st]
  if(normal) {
    if(type_lo == BBB_PERIODIC) { AT(sb) = AT(e - 2); AT(s) = AT(e - 1); }
    else if(type_lo == BBB_DIRICHLET) { AT(sb) = 2. * vlo - AT(s + 1); AT(s) = vlo; }
    else if(type_lo == BBB_NEUMANN) { AT(sb) = AT(s); }
    if(type_hi == BBB_PERIODIC) { AT(eb - 1) = AT(s + 1); AT(e - 1) = AT(s); }
    else if(type_hi == BBB_DIRICHLET) { AT(eb - 1) = 2. * vhi - AT(e - 2); AT(e - 1) = vhi; }
    else if(type_hi == BBB_NEUMANN) { AT(eb - 1) = AT(e - 1); }
  } else {
    if(type_lo == BBB_PERIODIC) AT(sb) = AT(e - 1);
    else if(type_lo == BBB_DIRICHLET) AT(sb) = 8. / 3. * vlo - 2. * AT(s) + 1. / 3. * AT(s + 1);
    else if(type_lo == BBB_NEUMANN) AT(sb) = AT(s);
    if(type_hi == BBB_PERIODIC) AT(eb - 1) = AT(s);
    else if(type_hi == BBB_DIRICHLET) AT(eb - 1) = 8. / 3. * vhi - 2. * AT(e - 1) + 1. / 3. * AT(e - 2);
    else if(type_hi == BBB_NEUMANN) AT(eb - 1) = AT(e - 1);
  }
#undef AT
}

__global__ void k_bc_axis(bc_face_set S, int ax)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y * blockDim.y + threadIdx.y;
  for(int fi = 0; fi < 4; fi++) {
    real *f = S.f[fi];
    if(!f) continue;
    /* the two transverse axes of this face */
    int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    if(a >= S.n[fi][t1] || b >= S.n[fi][t2]) continue;
    long long str[3] = {1, S.s1[fi], S.s2[fi]};
    long long base = a * str[t1] + b * str[t2];
    int normal = (fi == ax + 1);
    bc_line(f, base, str[ax], S.n[fi][ax], S.type[fi][0], S.type[fi][1],
      S.val[fi][0], S.val[fi][1], normal);
  }
}

static void bc_run(int which)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  const dom_struct *d = &Dom;
  bc_face_set S;
  memset(&S, 0, sizeof(S));
  const grid_info *G[4] = {&d->Gcc, &d->Gfx, &d->Gfy, &d->Gfz};
  for(int fi = 0; fi < 4; fi++) {
    S.s1[fi] = G[fi]->s1b; S.s2[fi] = G[fi]->s2b;
    S.n[fi][0] = G[fi]->inb; S.n[fi][1] = G[fi]->jnb; S.n[fi][2] = G[fi]->knb;
  }
  if(which == 0) { S.f[0] = g_dev.p; S.f[1] = g_dev.u; S.f[2] = g_dev.v; S.f[3] = g_dev.w; }
  else if(which == 1) { S.f[1] = g_dev.us; S.f[2] = g_dev.vs; S.f[3] = g_dev.ws; }
  else if(which == 2) { S.f[0] = g_dev.phi; }
  else { S.f[0] = g_dev.p; }
  int pt[6] = {bc.pW, bc.pE, bc.pS, bc.pN, bc.pB, bc.pT};
  int ut[6] = {bc.uW, bc.uE, bc.uS, bc.uN, bc.uB, bc.uT};
  int vt[6] = {bc.vW, bc.vE, bc.vS, bc.vN, bc.vB, bc.vT};
  int wt[6] = {bc.wW, bc.wE, bc.wS, bc.wN, bc.wB, bc.wT};
  real uv[6] = {bc.uWD, bc.uED, bc.uSD, bc.uND, bc.uBD, bc.uTD};
  real vv[6] = {bc.vWD, bc.vED, bc.vSD, bc.vND, bc.vBD, bc.vTD};
  real wv[6] = {bc.wWD, bc.wED, bc.wSD, bc.wND, bc.wBD, bc.wTD};
  int ext[6] = {dom[0].W, dom[0].E, dom[0].S, dom[0].N, dom[0].B, dom[0].T};
  for(int ax = 0; ax < 3; ax++) {
    for(int lh = 0; lh < 2; lh++) {
      int face = 2 * ax + lh;
      int on = ext[face] == -1;
      /* pressure has only periodic and Neumann kernels */
      S.type[0][lh] = on && (pt[face] == BBB_PERIODIC || pt[face] == BBB_NEUMANN) ? pt[face] : -1;
      S.type[1][lh] = on ? ut[face] : -1; S.val[1][lh] = uv[face];
      S.type[2][lh] = on ? vt[face] : -1; S.val[2][lh] = vv[face];
      S.type[3][lh] = on ? wt[face] : -1; S.val[3][lh] = wv[face];
      if(ut[face] == BBB_PRECURSOR || vt[face] == BBB_PRECURSOR || wt[face] == BBB_PRECURSOR)
        bbb_set_status(BBB_ERR_UNSUPPORTED, "PRECURSOR boundary condition");
    }
    int n1 = 0, n2 = 0;
    int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    for(int fi = 0; fi < 4; fi++) {
      if(S.n[fi][t1] > n1) n1 = S.n[fi][t1];
      if(S.n[fi][t2] > n2) n2 = S.n[fi][t2];
    }
    dim3 blk(32, 8), grd((n1 + 31) / 32, (n2 + 7) / 8);
    k_bc_axis<<<grd, blk, 0, g_dev.stream>>>(S, ax);
    BBB_LAUNCHED();
  }
}

extern "C" void cuda_dom_BC(void) { bc_run(0); }
extern "C" void cuda_dom_BC_star(void) { bc_run(1); }
extern "C" void cuda_dom_BC_phi(void) { bc_run(2); }
extern "C" void cuda_dom_BC_p(void) { bc_run(3); }

/* ------------------------------------------------ forcing
 * src/cuda_bluebottle.cu:3674-3814.  The forcing field the reference fills
 * is uniform (-gradP/rho_f along each axis); the momentum kernels take it
 * as a scalar, so only the ramps and the PID controller run here. */
static real ramp(real delta, real a, real m)
{
  if(a == 0) return m;
  if(fabs(delta * a) > fabs(m)) return m;
  return delta * a;
}

extern "C" void cuda_compute_forcing(real *pid_int_, real *pid_back_,
  real Kp_, real Ki_, real Kd_)
{
  real delta = ttime - p_tDelay;
  int pid = (Kp_ > 0 || Ki_ > 0 || Kd_ > 0);
  if(delta >= 0) {
    gradP.x = ramp(delta, gradP.xa, gradP.xm);
    gradP.y = ramp(delta, gradP.ya, gradP.ym);
    if(!pid) gradP.z = ramp(delta, gradP.za, gradP.zm);
  }
  delta = ttime - g_tDelay;
  if(delta >= 0) {
    g.x = ramp(delta, g.xa, g.xm);
    g.y = ramp(delta, g.ya, g.ym);
    g.z = ramp(delta, g.za, g.zm);
  }
  delta = ttime - p_tDelay;
  if(delta >= 0 && pid && nparts > 0) {
    cuda_part_pull();
    real acc_z = 0, volp = 0, massp = 0;
    for(int i = 0; i < nparts; i++) {
      volp += parts[i].r * parts[i].r * parts[i].r;
      massp += parts[i].rho * parts[i].r * parts[i].r * parts[i].r;
      acc_z += parts[i].wdot;
    }
    volp *= 4. / 3. * BBB_PI;
    massp *= 4. / 3. * BBB_PI;
    real volfrac = volp / (Dom.xl * Dom.yl * Dom.zl);
    real rho_avg = massp / volp * volfrac + rho_f * (1. - volfrac);
    acc_z /= nparts;
    *pid_int_ = *pid_int_ + acc_z * dt;
    gradP.z = gradP.z + (Kp_ * acc_z + Ki_ * (*pid_int_) / ttime
      + Kd_ * (acc_z - *pid_back_)) * rho_avg;
    *pid_back_ = acc_z;
  }
}

/* ------------------------------------------------ solvability
 * src/cuda_bluebottle.cu:4122-4314: net boundary flux of u* folded into
 * the outflow plane.  Two launches: a flux reduction and a plane update
 * that reads the flux from device memory. */

__global__ void k_surf_flux(const real *us, const real *vs, const real *ws,
  bbb_geom G, double *partials, unsigned int *ticket, double *out)
{
  __shared__ double sh[32 * 3];
  double v[3] = {0., 0., 0.};
  long long nyz = (long long)G.ny * G.nz, nxz = (long long)G.nx * G.nz,
            nxy = (long long)G.nx * G.ny;
  long long tot = nyz + nxz + nxy;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
      t += (long long)gridDim.x * blockDim.x) {
    if(t < nyz) {
      int j = (int)(t % G.ny) + 1, k = (int)(t / G.ny) + 1;
      long long r = (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
      v[0] += -us[r + 1] + us[r + (G.nx + 1)];
    } else if(t < nyz + nxz) {
      long long q = t - nyz;
      int i = (int)(q % G.nx) + 1, k = (int)(q / G.nx) + 1;
      long long r = i + (long long)k * G.fy_s2;
      v[1] += -vs[r + 1LL * G.fy_s1] + vs[r + (long long)(G.ny + 1) * G.fy_s1];
    } else {
      long long q = t - nyz - nxz;
      int i = (int)(q % G.nx) + 1, j = (int)(q / G.nx) + 1;
      long long r = i + (long long)j * G.fz_s1;
      v[2] += -ws[r + 1LL * G.fz_s2] + ws[r + (long long)(G.nz + 1) * G.fz_s2];
    }
  }
  if(bbb_grid_partial<3>(v, partials, ticket, sh)) {
    bbb_grid_finish_sum<3>(v, partials, ticket, sh);
    if(threadIdx.x == 0) {
      out[0] = v[0] * G.dy * G.dz;
      out[1] = v[1] * G.dx * G.dz;
      out[2] = v[2] * G.dx * G.dy;
    }
  }
}

__global__ void k_plane_eps(real *us, real *vs, real *ws, bbb_geom G,
  const double *eps3, int out_plane_)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y * blockDim.y + threadIdx.y;
  double ex = eps3[0], ey = eps3[1], ez = eps3[2];
  switch(out_plane_) {
    case BBB_WEST: case BBB_EAST: {
      if(a >= G.ny || b >= G.nz) return;
      double e = ex / G.yl / G.zl + ey / G.yl / G.zl + ez / G.yl / G.zl;
      long long r = (long long)(a + 1) * G.fx_s1 + (long long)(b + 1) * G.fx_s2;
      if(out_plane_ == BBB_WEST) us[r + 1] = us[r + 1] + e;
      else us[r + G.nx + 1] = us[r + G.nx + 1] - e;
      break;
    }
    case BBB_SOUTH: case BBB_NORTH: {
      if(a >= G.nx || b >= G.nz) return;
      double e = ex / G.zl / G.xl + ey / G.zl / G.xl + ez / G.zl / G.xl;
      long long r = (a + 1) + (long long)(b + 1) * G.fy_s2;
      if(out_plane_ == BBB_SOUTH) vs[r + G.fy_s1] = vs[r + G.fy_s1] + e;
      else vs[r + (long long)(G.ny + 1) * G.fy_s1] = vs[r + (long long)(G.ny + 1) * G.fy_s1] - e;
      break;
    }
    case BBB_BOTTOM: case BBB_TOP: {
      if(a >= G.nx || b >= G.ny) return;
      double e = ex / G.xl / G.yl + ey / G.xl / G.yl + ez / G.xl / G.yl;
      long long r = (a + 1) + (long long)(b + 1) * G.fz_s1;
      if(out_plane_ == BBB_BOTTOM) ws[r + G.fz_s2] = ws[r + G.fz_s2] + e;
      else ws[r + (long long)(G.nz + 1) * G.fz_s2] = ws[r + (long long)(G.nz + 1) * G.fz_s2] - e;
      break;
    }
    case BBB_HOMOGENEOUS: {
      double eX = 0.5 * ex / G.yl / G.zl, eY = 0.5 * ey / G.zl / G.xl,
             eZ = 0.5 * ez / G.xl / G.yl;
      if(a < G.ny && b < G.nz) {
        long long r = (long long)(a + 1) * G.fx_s1 + (long long)(b + 1) * G.fx_s2;
        us[r + 1] = us[r + 1] + eX;
        us[r + G.nx + 1] = us[r + G.nx + 1] - eX;
      }
      if(a < G.nx && b < G.nz) {
        long long r = (a + 1) + (long long)(b + 1) * G.fy_s2;
        vs[r + G.fy_s1] = vs[r + G.fy_s1] + eY;
        vs[r + (long long)(G.ny + 1) * G.fy_s1] = vs[r + (long long)(G.ny + 1) * G.fy_s1] - eY;
      }
      if(a < G.nx && b < G.ny) {
        long long r = (a + 1) + (long long)(b + 1) * G.fz_s1;
        ws[r + G.fz_s2] = ws[r + G.fz_s2] + eZ;
        ws[r + (long long)(G.nz + 1) * G.fz_s2] = ws[r + (long long)(G.nz + 1) * G.fz_s2] - eZ;
      }
      break;
    }
  }
}

extern "C" void cuda_solvability(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  bbb_geom G = bbb_make_geom();
  k_surf_flux<<<296, 256, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws, G,
    g_dev.partials, g_dev.red_ticket, g_dev.red_dev);
  BBB_LAUNCHED();
  int m = G.nx > G.ny ? G.nx : G.ny;
  if(G.nz > m) m = G.nz;
  dim3 blk(32, 8), grd((m + 31) / 32, (m + 7) / 8);
  k_plane_eps<<<grd, blk, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws, G,
    g_dev.red_dev, out_plane);
  BBB_LAUNCHED();
}

/* ------------------------------------------------ projection
 * src/bluebottle_kernel.cu:1250-1302: u = u* - dt/rho |flag| d(phi), all
 * three components in one pass over the union of the face index spaces. */
__global__ void k_project(const real *us, const real *vs, const real *ws,
  const real *ph, const int *fu, const int *fv, const int *fw,
  real *uu, real *vv, real *ww, bbb_geom G, real dt_rho)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int k = blockIdx.z + 1;
  double ddx = 1. / G.dx, ddy = 1. / G.dy, ddz = 1. / G.dz;
  if(j > G.ny + 1 || i > G.nx + 1) return;
  long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
  if(j <= G.ny && k <= G.nz) {
    long long C = i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
    double gp = abs(fu[C]) * ddx * (ph[cc] - ph[cc - 1]);
    uu[C] = us[C] - dt_rho * gp;
  }
  if(i <= G.nx && k <= G.nz) {
    long long C = i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2;
    double gp = abs(fv[C]) * ddy * (ph[cc] - ph[cc - G.cc_s1]);
    vv[C] = vs[C] - dt_rho * gp;
  }
  if(i <= G.nx && j <= G.ny) {
    long long C = i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2;
    double gp = abs(fw[C]) * ddz * (ph[cc] - ph[cc - G.cc_s2]);
    ww[C] = ws[C] - dt_rho * gp;
  }
}

extern "C" void cuda_project(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  bbb_geom G = bbb_make_geom();
  dim3 blk(32, 8), grd((G.nx + 1 + 31) / 32, (G.ny + 1 + 7) / 8, G.nz + 1);
  k_project<<<grd, blk, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws,
    g_dev.phi, g_dev.flag_u, g_dev.flag_v, g_dev.flag_w, g_dev.u, g_dev.v,
    g_dev.w, G, dt / rho_f);
  BBB_LAUNCHED();
}

/* ------------------------------------------------ pressure update
 * src/cuda_bluebottle.cu:3616-3671: p = (phase < 0)(p0 + phi) on interior
 * cells, then the interior mean is subtracted along every interior row,
 * ghost columns included: the cells forcing_add_c_const
 * (src/bluebottle_kernel.cu:2042) reaches under its launch shape when the
 * row and plane counts are multiples of 16.  Ghosts are rewritten by
 * cuda_dom_BC_p before any read.  The mean is reduced on the device. */
__global__ void k_update_p(const real *pp0, real *pp, const real *ph,
  const int *phs, bbb_geom G, double *partials, unsigned int *ticket,
  double *mean_out)
{
  __shared__ double sh[32];
  double v[1] = {0.};
  long long n = (long long)G.nx * G.ny * G.nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long r = t / G.nx;
    int j = (int)(r % G.ny) + 1, k = (int)(r / G.ny) + 1;
    long long C = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    double val = (phs[C] < 0) * (pp0[C] + ph[C]);
    pp[C] = val;
    v[0] += val;
  }
  if(bbb_grid_partial<1>(v, partials, ticket, sh)) {
    bbb_grid_finish_sum<1>(v, partials, ticket, sh);
    if(threadIdx.x == 0) *mean_out = v[0] / n;
  }
}

__global__ void k_add_const_cc(real *pp, bbb_geom G, int jmax, const double *val)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int k = blockIdx.z + 1;
  if(i > G.nx + 1 || j > jmax) return;
  double c = -*val;
  pp[i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2] += c;
}

/* rows (or planes) 1 .. the returned index that forcing_add_c_const
 * (src/bluebottle_kernel.cu:2042) reaches under the reference's launch
 * shape (src/cuda_bluebottle.cu:3629-3644: min(n, 16) threads,
 * ceil(n / threads) blocks, one ghost layer of offset, bounded by the
 * ghosted count): the interior, plus the far ghost row when n > 16 is not
 * a multiple of 16 */
static int add_const_cover(int n)
{
  int r = n < 16 ? n : (n + 15) / 16 * 16;
  return r < n + 1 ? r : n + 1;
}

extern "C" void cuda_update_p(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  bbb_geom G = bbb_make_geom();
  k_update_p<<<592, 256, 0, g_dev.stream>>>(g_dev.p0, g_dev.p, g_dev.phi,
    g_dev.phase, G, g_dev.partials, g_dev.red_ticket, g_dev.red_dev + 8);
  BBB_LAUNCHED();
  int jmax = add_const_cover(G.ny), kmax = add_const_cover(G.nz);
  dim3 blk(32, 8), grd((G.nx + 2 + 31) / 32, (jmax + 7) / 8, kmax);
  k_add_const_cc<<<grd, blk, 0, g_dev.stream>>>(g_dev.p, G, jmax, g_dev.red_dev + 8);
  BBB_LAUNCHED();
}

/* ------------------------------------------------ history store
 * src/cuda_bluebottle.cu:3580-3613 */
static void d2d(void *dst, const void *src, size_t n)
{
  BBB_CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, g_dev.stream));
}

extern "C" void cuda_store_u(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  const dom_struct *d = &Dom;
  size_t fx = sizeof(real) * d->Gfx.s3b, fy = sizeof(real) * d->Gfy.s3b,
         fz = sizeof(real) * d->Gfz.s3b;
  d2d(g_dev.conv0_u, g_dev.conv_u, fx);
  d2d(g_dev.conv0_v, g_dev.conv_v, fy);
  d2d(g_dev.conv0_w, g_dev.conv_w, fz);
  if(!g_opt.implicit) {
    d2d(g_dev.diff0_u, g_dev.diff_u, fx);
    d2d(g_dev.diff0_v, g_dev.diff_v, fy);
    d2d(g_dev.diff0_w, g_dev.diff_w, fz);
  }
  d2d(g_dev.p0, g_dev.p, sizeof(real) * d->Gcc.s3b);
  bbb_learn_step_boundary();
  d2d(g_dev.u0, g_dev.u, fx);
  d2d(g_dev.v0, g_dev.v, fy);
  d2d(g_dev.w0, g_dev.w, fz);
}

/* ------------------------------------------------ CFL time step
 * src/cuda_bluebottle.cu:3500-3577: maximum (not maximum magnitude, as in
 * the reference) of u, v, w over the full ghosted arrays, from 0. */
__global__ void k_max3(const real *a, long long na, const real *b,
  long long nb_, const real *c, long long nc, double *partials,
  unsigned int *ticket, double *out)
{
  __shared__ double sh[32 * 3];
  double v[3] = {0., 0., 0.};
  long long st = (long long)gridDim.x * blockDim.x;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < na; t += st)
    v[0] = fmax(v[0], a[t]);
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb_; t += st)
    v[1] = fmax(v[1], b[t]);
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nc; t += st)
    v[2] = fmax(v[2], c[t]);
  bbb_block_max<3>(v, sh);
  long long bid = blockIdx.x;
  __shared__ unsigned int s_last;
  if(threadIdx.x == 0) {
    for(int q = 0; q < 3; q++) partials[bid * 3 + q] = v[q];
    __threadfence();
    unsigned int tk = atomicAdd(ticket, 1u);
    s_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if(!s_last) return;
  __threadfence();
  double m[3] = {0., 0., 0.};
  for(long long q = threadIdx.x; q < gridDim.x; q += blockDim.x)
    for(int z = 0; z < 3; z++) m[z] = fmax(m[z], ((volatile double *)partials)[q * 3 + z]);
  bbb_block_max<3>(m, sh);
  if(threadIdx.x == 0) {
    out[0] = m[0]; out[1] = m[1]; out[2] = m[2];
    *ticket = 0u;
  }
}

extern "C" real cuda_find_dt(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return dt;
  const dom_struct *d = &Dom;
  k_max3<<<592, 256, 0, g_dev.stream>>>(g_dev.u, d->Gfx.s3b, g_dev.v,
    d->Gfy.s3b, g_dev.w, d->Gfz.s3b, g_dev.partials, g_dev.red_ticket,
    g_dev.red_dev + 16);
  BBB_LAUNCHED();
  d2h(g_dev.red_host, g_dev.red_dev + 16, 3 * sizeof(double));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  real umax = g_dev.red_host[0], vmax = g_dev.red_host[1], wmax = g_dev.red_host[2];
  g_stats.cfl_adv = g_stats.step_dt
    * (umax / d->dx + vmax / d->dy + wmax / d->dz);
  real tmp;
  if(!g_opt.implicit) {
    tmp = umax / d->dx + 2. * nu / d->dx / d->dx;
    tmp += vmax / d->dy + 2. * nu / d->dy / d->dy;
    tmp += wmax / d->dz + 2. * nu / d->dz / d->dz;
  } else {
    tmp = umax / d->dx;
    tmp += vmax / d->dy;
    tmp += wmax / d->dz;
  }
  real dtn = CFL / tmp;
  if(dtn > FLT_MAX) dtn = FLT_MAX;
  if(g_opt.implicit && dtn > 1.1 * dt) dtn = 1.1 * dt;
  if(g_opt.fixed_dt > 0) dtn = g_opt.fixed_dt;
  return dtn;
}

/* ------------------------------------------------ diagnostics */

/* kinetic energy 0.5 sum u^2 dV over the faces of each component (the
 * duplicated periodic face counted once) and divergence norms */
__global__ void k_energy_div(const real *uu, const real *vv, const real *ww,
  const int *phs, bbb_geom G, double *partials, unsigned int *ticket,
  double *out)
{
  __shared__ double sh[32 * 3];
  double v[3] = {0., 0., 0.};
  double mx[1] = {0.};
  long long n = (long long)G.nx * G.ny * G.nz;
  double ddx = 1. / G.dx, ddy = 1. / G.dy, ddz = 1. / G.dz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long r = t / G.nx;
    int j = (int)(r % G.ny) + 1, k = (int)(r / G.ny) + 1;
    long long cu = i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
    long long cv = i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2;
    long long cw = i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2;
    /* the reference's energy: face pairs averaged to the cell centre
     * (colocate_Gf?, src/bluebottle_kernel.cu:3849-3890), squares summed
     * u, v, w (energy_multiply :3891) */
    double uc = 0.5 * (uu[cu] + uu[cu + 1]);
    double vc = 0.5 * (vv[cv] + vv[cv + G.fy_s1]);
    double wc = 0.5 * (ww[cw] + ww[cw + G.fz_s2]);
    v[0] += uc * uc + vc * vc + wc * wc;
    long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    if(phs[cc] < 0) {
      double s = (uu[cu + 1] - uu[cu]) * ddx + (vv[cv + G.fy_s1] - vv[cv]) * ddy
        + (ww[cw + G.fz_s2] - ww[cw]) * ddz;
      v[1] += s * s;
      mx[0] = fmax(mx[0], fabs(s));
    }
  }
  bbb_block_max<1>(mx, sh + 64);
  v[2] = 0.;
  __shared__ double s_mx;
  if(threadIdx.x == 0) s_mx = mx[0];
  __syncthreads();
  if(bbb_grid_partial<3>(v, partials, ticket + 1, sh)) {
    bbb_grid_finish_sum<3>(v, partials, ticket + 1, sh);
    if(threadIdx.x == 0) {
      out[0] = v[0] / (double)n * 0.5;
      out[1] = sqrt(v[1]);
    }
  }
  if(threadIdx.x == 0) {
    unsigned long long *om = (unsigned long long *)(out + 2);
    atomicMax(om, (unsigned long long)__double_as_longlong(s_mx));
  }
}

static void energy_div(double *e, double *dl2, double *dmax)
{
  bbb_geom G = bbb_make_geom();
  BBB_CK(cudaMemsetAsync(g_dev.red_dev + 24, 0, 3 * sizeof(double), g_dev.stream));
  k_energy_div<<<592, 256, 0, g_dev.stream>>>(g_dev.u, g_dev.v, g_dev.w,
    g_dev.phase, G, g_dev.partials, g_dev.red_ticket + 4, g_dev.red_dev + 24);
  BBB_LAUNCHED();
  d2h(g_dev.red_host, g_dev.red_dev + 24, 3 * sizeof(double));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  *e = g_dev.red_host[0];
  *dl2 = g_dev.red_host[1];
  *dmax = g_dev.red_host[2];
}

/* src/cuda_bluebottle.cu:3944: half the mean over the cells of the
 * cell-centred |u|^2 */
extern "C" real cuda_compute_energy(void)
{
  bbb_dev_require();
  if(!g_dev.ready) return 0.;
  double e, l2, mx;
  energy_div(&e, &l2, &mx);
  return e;
}

extern "C" void bbb_divergence(real *max_abs, real *l2)
{
  bbb_dev_require();
  if(!g_dev.ready) { *max_abs = 0; *l2 = 0; return; }
  double e, dl2, mx;
  energy_div(&e, &dl2, &mx);
  *max_abs = mx;
  *l2 = dl2;
}

extern "C" void cuda_div_U(void) {}

/* precursor-only entry points (out of scope) */
extern "C" void cuda_dom_turb_planes_push(int *bc_configs)
{ (void)bc_configs; bbb_set_status(BBB_ERR_UNSUPPORTED, "turbulence precursor"); }
extern "C" void cuda_dom_turb_planes_pull(int *bc_configs)
{ (void)bc_configs; bbb_set_status(BBB_ERR_UNSUPPORTED, "turbulence precursor"); }
extern "C" void cuda_compute_turb_forcing(void)
{ bbb_set_status(BBB_ERR_UNSUPPORTED, "turbulence precursor"); }
extern "C" void cuda_yank_turb_planes(int *a, real *b, real *c)
{ (void)a; (void)b; (void)c; bbb_set_status(BBB_ERR_UNSUPPORTED, "turbulence precursor"); }
