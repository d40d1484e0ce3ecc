/* bbb_reduce.cuh -- deterministic grid-wide reductions.
 *
 * Every block reduces its values with warp shuffles and shared memory and
 * writes one partial per value; the last block to finish (elected through
 * an atomic ticket) sums the partials in a fixed order and runs a
 * finaliser.  For a fixed launch shape the result is bit-reproducible, and
 * no host round trip is needed between producer and consumer kernels.
 */
#ifndef BBB_REDUCE_CUH
#define BBB_REDUCE_CUH

#include <cuda_runtime.h>

__device__ __forceinline__ double bbb_warp_sum(double v)
{
  for(int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double bbb_warp_max(double v)
{
  for(int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

/* Block-wide sum of NV values; the result is valid in thread 0.
 * `sh` must hold 32*NV doubles. */
template <int NV>
__device__ __forceinline__ void bbb_block_sum(double (&v)[NV], double *sh)
{
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nthr = blockDim.x * blockDim.y * blockDim.z;
  int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
  for(int a = 0; a < NV; a++) {
    double s = bbb_warp_sum(v[a]);
    if(lane == 0) sh[a * 32 + wid] = s;
  }
  __syncthreads();
  if(wid == 0) {
#pragma unroll
    for(int a = 0; a < NV; a++) {
      double s = lane < nw ? sh[a * 32 + lane] : 0.;
      s = bbb_warp_sum(s);
      if(lane == 0) v[a] = s;
    }
  }
  __syncthreads();
}

template <int NV>
__device__ __forceinline__ void bbb_block_max(double (&v)[NV], double *sh)
{
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nthr = blockDim.x * blockDim.y * blockDim.z;
  int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
  for(int a = 0; a < NV; a++) {
    double s = bbb_warp_max(v[a]);
    if(lane == 0) sh[a * 32 + wid] = s;
  }
  __syncthreads();
  if(wid == 0) {
#pragma unroll
    for(int a = 0; a < NV; a++) {
      double s = lane < nw ? sh[a * 32 + lane] : -1.7976931348623157e308;
      s = bbb_warp_max(s);
      if(lane == 0) v[a] = s;
    }
  }
  __syncthreads();
}

/* Write this block's NV partial sums and report whether this block is the
 * last one to arrive.  The caller then calls bbb_grid_finish_sum. */
template <int NV>
__device__ __forceinline__ bool bbb_grid_partial(double (&v)[NV],
  double *partials, unsigned int *ticket, double *sh)
{
  bbb_block_sum<NV>(v, sh);
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y
    + (long long)gridDim.y * blockIdx.z);
  __shared__ unsigned int s_last;
  if(tid == 0) {
#pragma unroll
    for(int a = 0; a < NV; a++) partials[bid * NV + a] = v[a];
    __threadfence();
    unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  return s_last != 0;
}

/* In the last block: fixed-order sum of all partials; result in v (all
 * threads); resets the ticket. */
template <int NV>
__device__ __forceinline__ void bbb_grid_finish_sum(double (&v)[NV],
  const double *partials, unsigned int *ticket, double *sh)
{
  __threadfence();
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nthr = blockDim.x * blockDim.y * blockDim.z;
  long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
#pragma unroll
  for(int a = 0; a < NV; a++) v[a] = 0.;
  for(long long b = tid; b < nb; b += nthr) {
#pragma unroll
    for(int a = 0; a < NV; a++) v[a] += ((volatile const double *)partials)[b * NV + a];
  }
  bbb_block_sum<NV>(v, sh);
  __shared__ double s_res[NV > 0 ? NV : 1];
  if(tid == 0) {
#pragma unroll
    for(int a = 0; a < NV; a++) s_res[a] = v[a];
    *ticket = 0u;
  }
  __syncthreads();
#pragma unroll
  for(int a = 0; a < NV; a++) v[a] = s_res[a];
}

#endif
