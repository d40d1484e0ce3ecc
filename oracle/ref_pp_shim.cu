/* ref_pp_shim.cu -- test infrastructure (linked into oracle/_ref/libref_gpu.so
 * with the reference's own kernels; never part of the library).
 *
 * The reference assembles its pressure-Poisson system inside
 * cuda_PP_bicgstab (src/cuda_bicgstab.cu:715-1073), which cannot be built
 * here because the same function calls CUSP.  This file restates only the
 * assembly part of it -- the right-hand side (cuda_PP_rhs,
 * src/cuda_bicgstab.cu:1178-1202), the particle rewrite cuda_part_BC_p,
 * and the 13-diagonal matrix (src/cuda_bicgstab.cu:729-815) -- launching
 * the reference's own kernels from src/bicgstab_kernel.cu with the launch
 * shapes those lines use, and hands the system to the caller, so a test
 * can verify that this library's solve satisfies the reference's own
 * system.
 *
 * The matrix is returned in the layout of CUSP's dia_matrix values: column
 * d of a pitched array, A[d * pitch + row], with the diagonal offsets of
 * src/cuda_bicgstab.cu:733-745. */
#include "cuda_bicgstab.h"

/* rows of the system (un-ghosted Gcc cells) */
extern "C" int refshim_pp_rows(void)
{
  return dom[0].Gcc._s3;
}

/* the offsets of the 13 diagonals, src/cuda_bicgstab.cu:733-745 */
extern "C" void refshim_pp_offsets(int *off)
{
  const grid_info &G = dom[0].Gcc;
  int o[13] = {-G._s3 + G._s2, -G._s2, -G._s2 + G._s1, -G._s1, -G._s1 + 1, -1,
               0, 1, G._s1 - 1, G._s1, G._s2 - G._s1, G._s2, G._s3 - G._s2};
  for(int d = 0; d < 13; d++) off[d] = o[d];
}

/* A: 13 * rows reals (pitch = rows), b: rows reals.  Runs on the current
 * device state (push first).  Returns the CUDA status. */
extern "C" int refshim_pp_system(real *A, real *b)
{
  const int dev = 0;
  cudaSetDevice(dev + dev_start);

  /* right-hand side: src/cuda_bicgstab.cu:1180-1201 */
  {
    int tx = dom[dev].Gcc.inb < MAX_THREADS_DIM ? dom[dev].Gcc.inb + 2 : MAX_THREADS_DIM;
    int ty = dom[dev].Gcc.jnb < MAX_THREADS_DIM ? dom[dev].Gcc.jnb + 2 : MAX_THREADS_DIM;
    int bx = (int)ceil((real)dom[dev].Gcc.inb / (real)(tx - 2));
    int by = (int)ceil((real)dom[dev].Gcc.jnb / (real)(ty - 2));
    PP_rhs<<<dim3(bx, by), dim3(tx, ty)>>>(rho_f, _u_star[dev], _v_star[dev],
      _w_star[dev], _rhs_p[dev], _dom[dev], dt);
  }
  if(nparts > 0) cuda_part_BC_p(dev);

  /* matrix: src/cuda_bicgstab.cu:747-815 */
  const int rows = dom[dev].Gcc._s3, pitch = rows;
  real *vals = NULL;
  if(cudaMalloc((void **)&vals, sizeof(real) * 13 * (size_t)pitch) != cudaSuccess)
    return (int)cudaErrorMemoryAllocation;
  cudaMemset(vals, 0, sizeof(real) * 13 * (size_t)pitch);
  int tx = dom[dev].Gcc._in < MAX_THREADS_DIM ? dom[dev].Gcc._in : MAX_THREADS_DIM;
  int ty = dom[dev].Gcc._jn < MAX_THREADS_DIM ? dom[dev].Gcc._jn : MAX_THREADS_DIM;
  int tz = dom[dev].Gcc._kn < MAX_THREADS_DIM ? dom[dev].Gcc._kn : MAX_THREADS_DIM;
  int bx = (int)ceil((real)dom[dev].Gcc._in / (real)tx);
  int by = (int)ceil((real)dom[dev].Gcc._jn / (real)ty);
  int bz = (int)ceil((real)dom[dev].Gcc._kn / (real)tz);
  dim3 tX(ty, tz), gX(by, bz), tY(tz, tx), gY(bz, bx), tZ(tx, ty), gZ(bx, by);
  coeffs_init<<<gX, tX>>>(_dom[dev], pitch, vals);
  coeffs<<<gX, tX>>>(_dom[dev], _flag_u[dev], _flag_v[dev], _flag_w[dev], pitch, vals);
  if(bc.pW == PERIODIC) coeffs_periodic_W<<<gX, tX>>>(_dom[dev], pitch, vals, _flag_u[dev]);
  if(bc.pE == PERIODIC) coeffs_periodic_E<<<gX, tX>>>(_dom[dev], pitch, vals, _flag_u[dev]);
  if(bc.pS == PERIODIC) coeffs_periodic_S<<<gY, tY>>>(_dom[dev], pitch, vals, _flag_v[dev]);
  if(bc.pN == PERIODIC) coeffs_periodic_N<<<gY, tY>>>(_dom[dev], pitch, vals, _flag_v[dev]);
  if(bc.pB == PERIODIC) coeffs_periodic_B<<<gZ, tZ>>>(_dom[dev], pitch, vals, _flag_w[dev]);
  if(bc.pT == PERIODIC) coeffs_periodic_T<<<gZ, tZ>>>(_dom[dev], pitch, vals, _flag_w[dev]);
  coeffs_particle<<<gX, tX>>>(_dom[dev], pitch, vals, _phase[dev]);

  cudaError_t st = cudaDeviceSynchronize();
  if(st == cudaSuccess)
    st = cudaMemcpy(A, vals, sizeof(real) * 13 * (size_t)pitch, cudaMemcpyDeviceToHost);
  if(st == cudaSuccess)
    st = cudaMemcpy(b, _rhs_p[dev], sizeof(real) * (size_t)rows, cudaMemcpyDeviceToHost);
  cudaFree(vals);
  return (int)st;
}

/* ------------------------------------------------ Crank-Nicolson Helmholtz
 * The assembly half of cuda_{u,v,w}star_helmholtz (src/cuda_bicgstab.cu:
 * 44-318, 319-516, 517-712; the other half is CUSP's CG): the right-hand
 * side kernels with the launch shapes of cuda_{u,v,w}star_rhs
 * (:1091-1177, the v launch sizing its threads from Gfx as there), the
 * star boundary conditions, the un-ghosted copy that becomes the CG
 * right-hand side, and the 13-diagonal matrix with its per-face periodic or
 * Dirichlet kernels and the particle rows. */
#include "cuda_bluebottle.h"

struct refshim_dims { dim3 tX, gX, tY, gY, tZ, gZ; };

static refshim_dims refshim_face_dims(const grid_info &G)
{
  int tx = G._in < MAX_THREADS_DIM ? G._in : MAX_THREADS_DIM;
  int ty = G._jn < MAX_THREADS_DIM ? G._jn : MAX_THREADS_DIM;
  int tz = G._kn < MAX_THREADS_DIM ? G._kn : MAX_THREADS_DIM;
  int bx = (int)ceil((real)G._in / (real)tx);
  int by = (int)ceil((real)G._jn / (real)ty);
  int bz = (int)ceil((real)G._kn / (real)tz);
  refshim_dims d;
  d.tX = dim3(ty, tz); d.gX = dim3(by, bz);
  d.tY = dim3(tz, tx); d.gY = dim3(bz, bx);
  d.tZ = dim3(tx, ty); d.gZ = dim3(bx, by);
  return d;
}

/* the matrix kernels of one component: P the kernel prefix, STAR the star
 * array, c the lower-case component letter of the BC fields, OWN the
 * launch dims of the component's own kernels */
#define REFSHIM_FACE(P, STAR, c, F, FD, DIMT, DIMG)                           \
  if(bc.c##F == PERIODIC)                                                      \
    P##_coeffs_periodic_##F<<<D.DIMG, D.DIMT>>>(nu, dt, _dom[dev], pitch, vals); \
  else if(bc.c##F == DIRICHLET)                                                \
    P##_coeffs_dirichlet_##F<<<D.DIMG, D.DIMT>>>(bc.c##FD, STAR[dev], _dom[dev], \
      pitch, vals);
#define REFSHIM_MATRIX(P, STAR, c, FLAG, OWNT, OWNG)                           \
  P##_coeffs_init<<<D.OWNG, D.OWNT>>>(_dom[dev], pitch, vals);                 \
  P##_coeffs<<<D.OWNG, D.OWNT>>>(nu, dt, _dom[dev], pitch, vals, _flag_u[dev], \
    _flag_v[dev], _flag_w[dev]);                                               \
  REFSHIM_FACE(P, STAR, c, W, WD, tX, gX)                                         \
  REFSHIM_FACE(P, STAR, c, E, ED, tX, gX)                                         \
  REFSHIM_FACE(P, STAR, c, S, SD, tY, gY)                                         \
  REFSHIM_FACE(P, STAR, c, N, ND, tY, gY)                                         \
  REFSHIM_FACE(P, STAR, c, B, BD, tZ, gZ)                                         \
  REFSHIM_FACE(P, STAR, c, T, TD, tZ, gZ)                                         \
  P##_coeffs_particles<<<D.OWNG, D.OWNT>>>(_dom[dev], pitch, vals, FLAG[dev]);

/* rows of component comp's system (0 u, 1 v, 2 w) and its 13 offsets
 * (src/cuda_bicgstab.cu:65-77, 343-355, 541-553) */
extern "C" int refshim_helm_rows(int comp)
{
  const grid_info &G = comp == 0 ? dom[0].Gfx : comp == 1 ? dom[0].Gfy : dom[0].Gfz;
  return G._s3;
}

extern "C" void refshim_helm_offsets(int comp, int *off)
{
  const grid_info &G = comp == 0 ? dom[0].Gfx : comp == 1 ? dom[0].Gfy : dom[0].Gfz;
  int a4 = comp == 0 ? -G._s1 + 2 : -G._s1 + 1;
  int a8 = comp == 0 ? G._s1 - 2 : G._s1 - 1;
  int a2 = comp == 1 ? -G._s2 + 2 * G._s1 : -G._s2 + G._s1;
  int a10 = comp == 1 ? G._s2 - 2 * G._s1 : G._s2 - G._s1;
  int a0 = comp == 2 ? -G._s3 + 2 * G._s2 : -G._s3 + G._s2;
  int a12 = comp == 2 ? G._s3 - 2 * G._s2 : G._s3 - G._s2;
  int o[13] = {a0, -G._s2, a2, -G._s1, a4, -1, 0, 1, a8, G._s1, a10, G._s2, a12};
  for(int d = 0; d < 13; d++) off[d] = o[d];
}

/* A: 13 * rows reals (pitch = rows), b: rows reals, for component comp.
 * Runs on the current device state (push first); leaves the star array
 * holding the right-hand side, as the reference does before its solve. */
extern "C" int refshim_helm_system(int comp, real *A, real *b)
{
  const int dev = 0;
  cudaSetDevice(dev + dev_start);
  const grid_info &G = comp == 0 ? dom[dev].Gfx : comp == 1 ? dom[dev].Gfy : dom[dev].Gfz;
  if(comp == 0) {              /* src/cuda_bicgstab.cu:1091-1117 */
    int ty = dom[dev].Gfx.jnb < MAX_THREADS_DIM ? dom[dev].Gfx.jnb + 2 : MAX_THREADS_DIM;
    int tz = dom[dev].Gfx.knb < MAX_THREADS_DIM ? dom[dev].Gfx.knb + 2 : MAX_THREADS_DIM;
    int by = (int)ceil((real)dom[dev].Gfx.jnb / (real)(ty - 2));
    int bz = (int)ceil((real)dom[dev].Gfx.knb / (real)(tz - 2));
    ustar_rhs<<<dim3(by, bz), dim3(ty, tz)>>>(rho_f, nu, _u0[dev], _v0[dev], _w0[dev],
      _p0[dev], _f_x[dev], _conv0_u[dev], _conv_u[dev], _u_star[dev], _dom[dev], dt, dt0);
  } else if(comp == 1) {       /* :1119-1145 */
    int tz = dom[dev].Gfy.knb < MAX_THREADS_DIM ? dom[dev].Gfx.knb + 2 : MAX_THREADS_DIM;
    int tx = dom[dev].Gfy.inb < MAX_THREADS_DIM ? dom[dev].Gfx.inb + 2 : MAX_THREADS_DIM;
    int bz = (int)ceil((real)dom[dev].Gfy.knb / (real)(tz - 2));
    int bx = (int)ceil((real)dom[dev].Gfy.inb / (real)(tx - 2));
    vstar_rhs<<<dim3(bz, bx), dim3(tz, tx)>>>(rho_f, nu, _u0[dev], _v0[dev], _w0[dev],
      _p0[dev], _f_y[dev], _conv0_v[dev], _conv_v[dev], _v_star[dev], _dom[dev], dt, dt0);
  } else {                     /* :1147-1173 */
    int tx = dom[dev].Gfz.inb < MAX_THREADS_DIM ? dom[dev].Gfz.inb + 2 : MAX_THREADS_DIM;
    int ty = dom[dev].Gfz.jnb < MAX_THREADS_DIM ? dom[dev].Gfz.jnb + 2 : MAX_THREADS_DIM;
    int bx = (int)ceil((real)dom[dev].Gfz.inb / (real)(tx - 2));
    int by = (int)ceil((real)dom[dev].Gfz.jnb / (real)(ty - 2));
    wstar_rhs<<<dim3(bx, by), dim3(tx, ty)>>>(rho_f, nu, _u0[dev], _v0[dev], _w0[dev],
      _p0[dev], _f_z[dev], _conv0_w[dev], _conv_w[dev], _w_star[dev], _dom[dev], dt, dt0);
  }
  cuda_dom_BC_star();
  if(nparts > 0) cuda_part_BC_star();

  const int rows = G._s3, pitch = rows;
  real *vals = NULL, *rhs = NULL;
  if(cudaMalloc((void **)&vals, sizeof(real) * 13 * (size_t)pitch) != cudaSuccess)
    return (int)cudaErrorMemoryAllocation;
  if(cudaMalloc((void **)&rhs, sizeof(real) * (size_t)G.s3) != cudaSuccess) {
    cudaFree(vals);
    return (int)cudaErrorMemoryAllocation;
  }
  cudaMemset(vals, 0, sizeof(real) * 13 * (size_t)pitch);
  refshim_dims D = refshim_face_dims(G);
  if(comp == 0) {
    copy_u_noghost<<<D.gX, D.tX>>>(rhs, _u_star[dev], _dom[dev]);
    REFSHIM_MATRIX(ustar, _u_star, u, _flag_u, tX, gX)
  } else if(comp == 1) {
    copy_v_noghost<<<D.gY, D.tY>>>(rhs, _v_star[dev], _dom[dev]);
    REFSHIM_MATRIX(vstar, _v_star, v, _flag_v, tY, gY)
  } else {
    copy_w_noghost<<<D.gZ, D.tZ>>>(rhs, _w_star[dev], _dom[dev]);
    REFSHIM_MATRIX(wstar, _w_star, w, _flag_w, tZ, gZ)
  }
  cudaError_t st = cudaDeviceSynchronize();
  if(st == cudaSuccess)
    st = cudaMemcpy(A, vals, sizeof(real) * 13 * (size_t)pitch, cudaMemcpyDeviceToHost);
  if(st == cudaSuccess)
    st = cudaMemcpy(b, rhs, sizeof(real) * (size_t)rows, cudaMemcpyDeviceToHost);
  cudaFree(vals);
  cudaFree(rhs);
  return (int)st;
}
