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
 * shapes those lines use, and hands the system to the caller: the checker
 * that this library's solve satisfies the reference's own system.
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
