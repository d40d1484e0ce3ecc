/* bbb_learn.cu -- learned initial guess for the pressure-Poisson solve.
 *
 * No reference counterpart: the reference starts every solve from the
 * previous correction, x0 = phi (src/cuda_bicgstab.cu:971-979), which is the
 * linear extrapolation of the pressure, p_{n-1} - p_{n-2}.  Here a small 3-D
 * convolutional net predicts a correction to that extrapolation:
 *
 *   features (per cell, scaled): b h^2 / S, phi_prev / S, p_{n-1} / S_p,
 *                                solid mask            (4 of 16 channels)
 *   4 layers of 3x3x3 convolution, 16 channels, GELU after layers 1-3
 *   phi_0 = phi_prev + S * out    (fluid cells; solids keep phi_prev)
 *
 * S = rms(phi_prev) over fluid cells (or rms(b h^2) when phi_prev = 0),
 * S_p = rms(p_{n-1}).  The guess is used only when its FP64 residual
 * ||b - A phi_0|| is below that of the extrapolation; otherwise the solve
 * starts from phi_prev exactly as the reference does.
 *
 * Data layout: activations channels-last BF16, 16 channels = 32 bytes per
 * cell, x fastest.  Convolutions are implicit GEMMs on the 5th-generation
 * tensor cores: a tile is 128 consecutive cells of one x-row (M = 128), K =
 * 16 input channels, FP32 accumulators in TMEM.  A block marches along z
 * over a tile of LG_TY rows; the rows of each plane (+1 halo cell each
 * side, +1 halo row each side) are staged once in shared memory in the
 * no-swizzle K-major core-matrix layout, so a dx shift is the same rows at
 * a 16-byte shifted start address.  Each staged row meets the weights of
 * its three dy taps in one N = 48 MMA that adds into three output rows'
 * accumulators; one thread issues the MMAs, tcgen05.commit signals an
 * mbarrier, and eight warps read the accumulators back with tcgen05.ld for
 * the fused bias + GELU epilogue.
 * The backward data gradient is the same kernel with the taps flipped and
 * the channel roles swapped; the weight gradient (a reduction over cells
 * of outer products, M = 16) runs on the CUDA cores in FP32.
 * Training: Adam on MSE against recorded solver tuples (random crops of the
 * features and the converged correction), crops stacked along z, loss on
 * cells at least 4 cells (the receptive-field radius) from crop faces.
 */
#include <cuda_bf16.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "bbb_internal.h"
#include "bbb_reduce.cuh"

#define LG_C 16                   /* channels (padded)                 */
#define LG_L 4                    /* layers                            */
#define LG_T 27                   /* taps                              */
#define LG_M 128                  /* cells per tile (MMA M)            */
#define LG_RC (LG_M + 2)          /* staged cells per row              */
#define LG_HALF (LG_RC * 16)      /* bytes between the two K halves    */
#define LG_ROWB (2 * LG_HALF)     /* bytes per staged row              */
#define LG_WGRP 1536              /* bytes of one (dz, dx) weight group */
#define LG_WLAYER (9 * LG_WGRP)
#define LG_NWL (LG_T * LG_C * LG_C)   /* weights per layer ([t][cout][cin]) */
#define LG_NW (LG_L * LG_NWL)
#define LG_NP (LG_NW + LG_L * LG_C)   /* weights + biases                */
#define LG_EPI 256                /* staging + epilogue threads        */
#define LG_THREADS (LG_EPI + 32)  /* + one warp that issues the MMAs   */
#define LG_NIN 4                  /* live input channels              */
#define NPW_LG 1184

typedef __nv_bfloat16 bf16;

struct lg_box {
  int nx, ny, nz;
  int px, py, pz;                 /* periodic along each axis          */
  int ntx;                        /* tiles along x                     */
  long long ntiles;
};

static lg_box make_lg_box(int nx, int ny, int nz, int px, int py, int pz)
{
  lg_box b;
  b.nx = nx; b.ny = ny; b.nz = nz; b.px = px; b.py = py; b.pz = pz;
  b.ntx = (nx + LG_M - 1) / LG_M;
  b.ntiles = (long long)b.ntx * ny * nz;
  return b;
}

/* ------------------------------------------------ tcgen05 helpers */
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{ return (uint32_t)__cvta_generic_to_shared(p); }

/* shared-memory matrix descriptor: no swizzle, K-major canonical layout
 * ((8, m), 2) : ((16 B, sbo), lbo) */
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo,
  uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;                      /* descriptor version */
  return d;
}

/* instruction descriptor, kind::f16: D F32, A and B BF16, both K-major,
 * M = 128, N = 48 (three output rows of 16 channels) */
#define LG_IDESC ((1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(48 >> 3) << 17) \
                  | ((uint32_t)(LG_M >> 4) << 24))

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a,
  uint64_t b, uint32_t acc)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
               :: "r"(tmem_d), "l"(a), "l"(b), "r"((uint32_t)LG_IDESC), "r"(acc)
               : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/* bounded wait for the phase of parity `par`; false when the limit ran out */
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t par)
{
  for(int it = 0; it < (1 << 22); it++) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok) : "r"(mbar), "r"(par) : "memory");
    if(ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_after(void)
{ asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before(void)
{ asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
                 "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
                 "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                 "=r"(r[14]), "=r"(r[15])
               : "r"(taddr) : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for(int a = 0; a < 16; a++) v[a] = __uint_as_float(r[a]);
}

/* GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear
 * Units", 2016): gelu(z) = z/2 (1 + tanh(k (z + c z^3))), k = sqrt(2/pi),
 * c = 0.044715, with the tanh of the hardware's special-function unit
 * (PTX tanh.approx.f32, relative error about 2^-11, below the BF16
 * rounding of the activations it feeds).  gelu_d is its derivative. */
__device__ __forceinline__ float lg_tanh(float x)
{
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

#define LG_GELU_K 0.7978845608028654f
#define LG_GELU_C 0.044715f

__device__ __forceinline__ float gelu(float z)
{
  float t = lg_tanh(LG_GELU_K * (z + LG_GELU_C * z * z * z));
  return 0.5f * z * (1.f + t);
}

__device__ __forceinline__ float gelu_d(float z)
{
  float t = lg_tanh(LG_GELU_K * (z + LG_GELU_C * z * z * z));
  return 0.5f * (1.f + t)
    + 0.5f * z * (1.f - t * t) * LG_GELU_K * (1.f + 3.f * LG_GELU_C * z * z);
}

__device__ __forceinline__ int wrap_or(int g, int n, int per)
{
  if(g >= 0 && g < n) return g;
  if(!per) return -1;
  g %= n;
  return g < 0 ? g + n : g;
}

/* ------------------------------------------------ convolution (tcgen05)
 * MODE 0: hidden layer: z = conv + bias -> pre (FP32, optional), act =
 *         bf16(gelu(z)).
 * MODE 1: output layer: out32[cell] = conv[0] + bias[0].
 * MODE 2: backward data gradient: g = conv (flipped, transposed weights,
 *         no bias) -> act = bf16(g * gelu'(pre)) with pre the previous
 *         layer's pre-activation.
 *
 * A block owns a tile of 128 cells (the MMA's M) x LG_TY rows and marches
 * along z through a run of planes.  Each plane's LG_TY + 2 staged rows stay
 * in a ring of four plane slots, so a plane is read from global memory once
 * per tile.  The GEMM is organised around the staged rows: staged row r of
 * input plane k - 1 + dz, shifted by dx cells, feeds output rows r - 2,
 * r - 1 and r at once -- one M = 128, N = 48, K = 16 tcgen05.mma whose B
 * holds the three dy taps of (dz, dx) and whose D is the 48-column window
 * of the output plane's accumulator rows in TMEM.  9 (dz, dx) groups x
 * (LG_TY + 2) rows = 54 MMAs per plane instead of 27 per output row, so
 * each staged row is read from shared memory 9 times instead of 27.  The
 * accumulator holds LG_TY + 4 rows (-2 .. LG_TY + 1, the four outside the
 * tile are never read) in two sets: while one thread issues plane k's MMAs
 * into one set, the eight warps stream plane k + 2 into the free ring slot
 * with cp.async and run plane k - 1's epilogue from the other set. */
#define LG_TY 4
#define LG_SLOTB ((LG_TY + 2) * LG_ROWB)
#define LG_ACC ((LG_TY + 4) * LG_C)   /* TMEM columns of one accumulator set */
#define LG_ZSMEM (4 * LG_SLOTB + LG_WLAYER + 64)   /* 2 barriers, TMEM slot */

struct lg_zbox {
  lg_box b;
  int nty;                        /* row groups along y                */
  long long units, q, r;          /* (tile, plane) units, split evenly */
  int nblk;                       /* blocks: one wave                  */
};

static lg_zbox make_lg_zbox(const lg_box &b, int nblk_max)
{
  lg_zbox z;
  z.b = b;
  z.nty = (b.ny + LG_TY - 1) / LG_TY;
  z.units = (long long)b.ntx * z.nty * b.nz;
  long long nb = z.units / 4 < nblk_max ? z.units / 4 : nblk_max;
  if(nb < 1) nb = 1;
  z.nblk = (int)nb;
  z.q = z.units / nb;
  z.r = z.units % nb;
  return z;
}

__device__ __forceinline__ void lg_cp16(uint32_t dst, const void *src, int bytes)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
               :: "r"(dst), "l"(src), "r"(bytes) : "memory");
}

/* The 16-byte copies that stage one plane of a tile: (LG_TY + 2) rows x
 * LG_RC cells x 2 channel halves, copy q = ry * 2 LG_RC + 2 c + h going
 * to row ry, cell c, half h of the slot.  Thread t issues copies t, t +
 * LG_EPI, ..: LG_NQ of them. */
#define LG_NCOPY ((LG_TY + 2) * LG_RC * 2)
#define LG_NQ ((LG_NCOPY + LG_EPI - 1) / LG_EPI)

/* this thread's copies of tile (i0, j0): the source of each inside a
 * plane in 16-byte units (cell (gi, gj) wrapped on periodic axes, x
 * fastest), -1 where the cell lies outside a non-periodic box (zero
 * fill); plane-independent, so computed once per run of planes */
__device__ __forceinline__ void lg_stage_map(const lg_box &B, int i0, int j0,
  int (&src)[LG_NQ])
{
#pragma unroll
  for(int n = 0; n < LG_NQ; n++) {
    const int q = threadIdx.x + n * LG_EPI;
    src[n] = -1;
    if(q < LG_NCOPY) {
      const int ry = q / (LG_RC * 2), rem = q - ry * (LG_RC * 2);
      const int c = rem >> 1, h = rem & 1;
      const int gi = wrap_or(i0 - 1 + c, B.nx, B.px);
      const int gj = wrap_or(j0 - 1 + ry, B.ny, B.py);
      if(gi >= 0 && gj >= 0) src[n] = (gi + B.nx * gj) * 2 + h;
    }
  }
}

/* stage plane kk of the tile whose copies lg_stage_map listed into the
 * ring slot */
__device__ __forceinline__ void lg_stage_plane(const lg_box &B, const bf16 *in,
  uint32_t slot, const int (&src)[LG_NQ], int kk)
{
  const int gk = wrap_or(kk, B.nz, B.pz);
  const uint4 *base = reinterpret_cast<const uint4 *>(in)
    + (gk >= 0 ? (long long)gk * B.nx * B.ny * 2 : 0LL);
#pragma unroll
  for(int n = 0; n < LG_NQ; n++) {
    const int q = threadIdx.x + n * LG_EPI;
    if(q < LG_NCOPY) {
      const int ry = q / (LG_RC * 2), rem = q - ry * (LG_RC * 2);
      const bool live = src[n] >= 0 && gk >= 0;
      lg_cp16(slot + ry * LG_ROWB + (rem & 1) * LG_HALF + (rem >> 1) * 16,
        live ? base + src[n] : reinterpret_cast<const uint4 *>(in), live ? 16 : 0);
    }
  }
}

/* the 9 x (LG_TY + 2) MMAs of one plane: A rows from the three ring slots
 * (planes k - 1, k, k + 1, descriptors da[0..2] of their first staged row),
 * B from the layer's packed (dz, dx) groups (descriptor db of group 0), D
 * the window of accumulator rows r - 2 .. r at TMEM columns d + 16 r.  The
 * first group's windows r = 0, 3, 6, .. start their rows from zero and go
 * first; every other MMA accumulates.  Fully unrolled: every operand is a
 * base descriptor plus a constant (the start address lives in the
 * descriptor's low 14 bits, in 16-byte units). */
__device__ __forceinline__ void lg_issue_plane(uint32_t d, const uint64_t (&da)[3],
  uint64_t db)
{
#pragma unroll
  for(int g = 0; g < 9; g++) {
    const int dz = g / 3, dx = g % 3;
#pragma unroll
    for(int o = 0; o < LG_TY + 2; o++) {
      /* group 0: rows 0, 3, .. first (fresh), then the rest */
      const int n3 = (LG_TY + 2 + 2) / 3;
      const int r = g > 0 ? o : (o < n3 ? 3 * o : (o - n3) + (o - n3) / 2 + 1);
      uint64_t a = da[dz] + (uint64_t)((r * LG_ROWB + dx * 16) >> 4);
      uint64_t b = db + (uint64_t)((g * LG_WGRP) >> 4);
      umma_bf16(d + (uint32_t)(r * LG_C), a, b, (g == 0 && o < n3) ? 0u : 1u);
    }
  }
}

/* the epilogue of one plane from the accumulator set at TMEM column d:
 * bias, activation, stores.  Warp w reads TMEM lanes 32 (w % 4) .. + 31
 * (cells 32 (w % 4) .. of the tile, the lanes its warpgroup position may
 * access) of rows y = w / 4, w / 4 + 2, .. (row y at columns d + 16 (y + 2)) */
template <int MODE>
__device__ __forceinline__ void lg_epilogue(const lg_box &B, uint32_t d, int i0,
  int j0, int k, const float (&bv)[16], float *pre, bf16 *act, float *out32)
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;
  const int i = i0 + quad * 32 + lane;
#pragma unroll 1
  for(int y = warp >> 2; y < LG_TY; y += LG_EPI / 128) {
    float v[16];
    tmem_ld16(d + ((uint32_t)(quad * 32) << 16) + (uint32_t)((y + 2) * LG_C), v);
    int j = j0 + y;
    if(i >= B.nx || j >= B.ny) continue;
    long long cell = i + (long long)B.nx * (j + (long long)B.ny * k);
    if(MODE == 1) {
      out32[cell] = v[0] + bv[0];
    } else {
      float o[16];
      if(MODE == 0) {
#pragma unroll
        for(int a = 0; a < 16; a++) {
          float z = v[a] + bv[a];
          if(pre) pre[cell * 16 + a] = z;
          o[a] = gelu(z);
        }
      } else {
#pragma unroll
        for(int a = 0; a < 16; a++) o[a] = v[a] * gelu_d(pre[cell * 16 + a]);
      }
      uint4 w0, w1;
      uint32_t *p0 = &w0.x, *p1 = &w1.x;
#pragma unroll
      for(int a = 0; a < 4; a++) {
        __nv_bfloat162 lo = __floats2bfloat162_rn(o[2 * a], o[2 * a + 1]);
        __nv_bfloat162 hi = __floats2bfloat162_rn(o[8 + 2 * a], o[8 + 2 * a + 1]);
        p0[a] = *reinterpret_cast<uint32_t *>(&lo);
        p1[a] = *reinterpret_cast<uint32_t *>(&hi);
      }
      reinterpret_cast<uint4 *>(act)[cell * 2] = w0;
      reinterpret_cast<uint4 *>(act)[cell * 2 + 1] = w1;
    }
  }
}

/* Pipeline per plane k of a run: one thread of the ninth warp issues plane
 * k's MMAs into accumulator set k & 1 while the eight other warps stream
 * plane k + 2 into the slot plane k - 2 left and run plane k - 1's
 * epilogue from the other set; then the block waits for plane k's MMAs.
 * The issuing warp takes no part in the epilogue, so the epilogue never
 * waits behind the MMA issue. */
template <int MODE>
__global__ void __launch_bounds__(LG_THREADS, 2) k_conv_z(lg_zbox Z,
  const bf16 *__restrict__ in, const uint8_t *__restrict__ wpack,
  const float *__restrict__ bias, float *pre, bf16 *act, float *out32,
  int *err)
{
  extern __shared__ __align__(1024) uint8_t lg_sm[];
  const lg_box &B = Z.b;
  uint8_t *ring = lg_sm;
  uint8_t *wsm = lg_sm + 4 * LG_SLOTB;
  uint64_t *mbar = (uint64_t *)(wsm + LG_WLAYER);      /* two barriers */
  uint32_t *tslot = (uint32_t *)(wsm + LG_WLAYER + 16);
  int tid = threadIdx.x, warp = tid >> 5;

  for(int q = tid; q < LG_WLAYER / 16; q += LG_THREADS)
    reinterpret_cast<uint4 *>(wsm)[q] = reinterpret_cast<const uint4 *>(wpack)[q];
  if(tid == 0) { mbar_init(smem_u32(&mbar[0]), 1); mbar_init(smem_u32(&mbar[1]), 1); }
  if(warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tslot)), "n"(2 * LG_ACC) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  float bv[16];
#pragma unroll
  for(int a = 0; a < 16; a++) bv[a] = (MODE == 2 || bias == nullptr) ? 0.f : bias[a];
  const uint32_t rbase = smem_u32(ring);
  const uint64_t db = umma_desc(smem_u32(wsm), LG_WGRP / 2, 128);

  uint32_t ph[2] = {0u, 0u};
  bool ok = true;
  long long bxl = blockIdx.x;
  long long u0 = bxl * Z.q + (bxl < Z.r ? bxl : Z.r);
  const long long u1 = u0 + Z.q + (bxl < Z.r ? 1 : 0);
  while(u0 < u1 && ok) {
    long long tile = u0 / B.nz;
    int k0 = (int)(u0 - tile * B.nz);
    long long left_ = u1 - u0;
    int k1 = left_ < (long long)(B.nz - k0) ? k0 + (int)left_ : B.nz;
    int i0 = (int)(tile % B.ntx) * LG_M;
    int j0 = (int)(tile / B.ntx) * LG_TY;
    int srcm[LG_NQ];
    lg_stage_map(B, i0, j0, srcm);
    if(tid < LG_EPI) {
      for(int kk = k0 - 1; kk <= k0 + 1; kk++)
        lg_stage_plane(B, in, rbase + ((kk + 4) & 3) * LG_SLOTB, srcm, kk);
      asm volatile("cp.async.wait_all;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    for(int k = k0; k < k1; k++) {
      const int buf = k & 1;
      if(tid == LG_EPI) {
        /* planes k - 1 .. k + 1 are staged and set buf is free (plane
         * k - 2's epilogue is done): plane k's MMAs */
        tc_fence_after();
        uint64_t da[3];
#pragma unroll
        for(int dz = 0; dz < 3; dz++)
          da[dz] = umma_desc(rbase + ((k - 1 + dz + 4) & 3) * LG_SLOTB, LG_HALF, 128);
        lg_issue_plane(tmem + (uint32_t)(buf * LG_ACC), da, db);
        umma_commit(smem_u32(&mbar[buf]));
      } else if(tid < LG_EPI) {
        /* meanwhile: plane k + 2 into the slot plane k - 2 left (its last
         * reader, plane k - 1's MMAs, completed), plane k - 1's epilogue
         * from the other accumulator set */
        if(k + 1 < k1)
          lg_stage_plane(B, in, rbase + ((k + 2 + 4) & 3) * LG_SLOTB, srcm, k + 2);
        if(k > k0)
          lg_epilogue<MODE>(B, tmem + (uint32_t)((buf ^ 1) * LG_ACC), i0, j0,
            k - 1, bv, pre, act, out32);
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      tc_fence_before();
      ok = __syncthreads_and(mbar_wait(smem_u32(&mbar[buf]), ph[buf]) ? 1 : 0) != 0;
      ph[buf] ^= 1u;
      tc_fence_after();
      if(!ok) break;
    }
    /* the run's last plane */
    if(ok) {
      const int buf = (k1 - 1) & 1;
      if(tid < LG_EPI)
        lg_epilogue<MODE>(B, tmem + (uint32_t)(buf * LG_ACC), i0, j0, k1 - 1,
          bv, pre, act, out32);
      tc_fence_before();
      __syncthreads();
    }
    if(!ok && tid == 0) atomicExch(err, 1);
    u0 += k1 - k0;
  }
  /* copies are waited for above; MMAs whose wait ran out get a bounded
   * second chance before the accumulators are released */
  asm volatile("cp.async.wait_all;" ::: "memory");
  if(!ok) {
    mbar_wait(smem_u32(&mbar[0]), ph[0]);
    mbar_wait(smem_u32(&mbar[1]), ph[1]);
  }
  tc_fence_after();
  __syncthreads();
  if(warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "n"(2 * LG_ACC) : "memory");
}

/* ------------------------------------------------ reference convolution
 * The same three modes on the CUDA cores in FP32 (one thread per cell and
 * output channel group): the FP32 result the tests hold the tensor-core
 * path to, and the path for boxes where a 128-cell tile does not fit. */
template <int MODE>
__global__ void k_conv_ref(lg_box B, const bf16 *__restrict__ in,
  const float *__restrict__ w, const float *__restrict__ bias, float *pre,
  bf16 *act, float *out32)
{
  long long n = (long long)B.nx * B.ny * B.nz;
  for(long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
      cell < n; cell += (long long)gridDim.x * blockDim.x) {
    int i = (int)(cell % B.nx);
    long long rr = cell / B.nx;
    int j = (int)(rr % B.ny), k = (int)(rr / B.ny);
    float acc[16];
#pragma unroll
    for(int a = 0; a < 16; a++) acc[a] = 0.f;
    for(int t = 0; t < LG_T; t++) {
      int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
      int gi = wrap_or(i + dx, B.nx, B.px), gj = wrap_or(j + dy, B.ny, B.py),
          gk = wrap_or(k + dz, B.nz, B.pz);
      if(gi < 0 || gj < 0 || gk < 0) continue;
      long long src = gi + (long long)B.nx * (gj + (long long)B.ny * gk);
      float x[16];
#pragma unroll
      for(int c = 0; c < 16; c++) x[c] = __bfloat162float(in[src * 16 + c]);
      const float *wt = w + t * 256;
#pragma unroll 4
      for(int o = 0; o < 16; o++) {
        float s = 0.f;
#pragma unroll
        for(int c = 0; c < 16; c++) s += wt[o * 16 + c] * x[c];
        acc[o] += s;
      }
    }
    if constexpr(MODE == 1) {
      out32[cell] = acc[0] + bias[0];
    } else {
#pragma unroll
      for(int a = 0; a < 16; a++) {
        float o;
        if(MODE == 0) {
          float z = acc[a] + bias[a];
          if(pre) pre[cell * 16 + a] = z;
          o = gelu(z);
        } else {
          o = acc[a] * gelu_d(pre[cell * 16 + a]);
        }
        act[cell * 16 + a] = __float2bfloat16_rn(o);
      }
    }
  }
}

/* ------------------------------------------------ weight gradient
 * dW[t][cout][cin] = sum_cells X[cell + off(t)][cin] dZ[cell][cout],
 * db[cout] = sum_cells dZ[cell][cout].  Block: 432 threads = 27 taps x 4
 * cout groups x 4 cin groups, 16 FP32 accumulators each; the block walks
 * tiles of 128 cells with the 9 neighbouring rows staged in shared memory;
 * per-block partials are summed in block order by k_dw_reduce. */
#define LG_DW_THREADS 432
__global__ void __launch_bounds__(LG_DW_THREADS) k_dw(lg_box B,
  const bf16 *__restrict__ X, const bf16 *__restrict__ dZ, float *partials)
{
  __shared__ __align__(16) bf16 xs[9][LG_RC][16];
  __shared__ __align__(16) bf16 zs[LG_M][16];
  int tid = threadIdx.x;
  int t = tid / 16, cg = (tid / 4) % 4, ig = tid % 4;
  int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
  int r = (dz + 1) * 3 + (dy + 1);
  float acc[4][4], db[4];
#pragma unroll
  for(int a = 0; a < 4; a++) {
    db[a] = 0.f;
#pragma unroll
    for(int b = 0; b < 4; b++) acc[a][b] = 0.f;
  }
  for(long long tile = blockIdx.x; tile < B.ntiles; tile += gridDim.x) {
    int itx = (int)(tile % B.ntx);
    long long rest = tile / B.ntx;
    int j = (int)(rest % B.ny), k = (int)(rest / B.ny);
    int i0 = itx * LG_M;
    __syncthreads();
    for(int q = tid; q < 9 * LG_RC * 2; q += LG_DW_THREADS) {
      int rr = q / (LG_RC * 2), rem = q - rr * (LG_RC * 2);
      int c = rem >> 1, h = rem & 1;
      int ddz = rr / 3 - 1, ddy = rr % 3 - 1;
      int gi = wrap_or(i0 - 1 + c, B.nx, B.px);
      int gj = wrap_or(j + ddy, B.ny, B.py);
      int gk = wrap_or(k + ddz, B.nz, B.pz);
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if(gi >= 0 && gj >= 0 && gk >= 0) {
        long long cell = gi + (long long)B.nx * (gj + (long long)B.ny * gk);
        v = reinterpret_cast<const uint4 *>(X)[cell * 2 + h];
      }
      *reinterpret_cast<uint4 *>(&xs[rr][c][h * 8]) = v;
    }
    for(int q = tid; q < LG_M * 2; q += LG_DW_THREADS) {
      int m = q >> 1, h = q & 1;
      int i = i0 + m;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if(i < B.nx) {
        long long cell = i + (long long)B.nx * (j + (long long)B.ny * k);
        v = reinterpret_cast<const uint4 *>(dZ)[cell * 2 + h];
      }
      *reinterpret_cast<uint4 *>(&zs[m][h * 8]) = v;
    }
    __syncthreads();
    int mmax = min(LG_M, B.nx - i0);
    for(int m = 0; m < mmax; m++) {
      float xv[4], zv[4];
#pragma unroll
      for(int b = 0; b < 4; b++) xv[b] = __bfloat162float(xs[r][m + dx + 1][ig * 4 + b]);
#pragma unroll
      for(int a = 0; a < 4; a++) zv[a] = __bfloat162float(zs[m][cg * 4 + a]);
#pragma unroll
      for(int a = 0; a < 4; a++) {
#pragma unroll
        for(int b = 0; b < 4; b++) acc[a][b] += zv[a] * xv[b];
        db[a] += zv[a];
      }
    }
  }
  float *pb = partials + (long long)blockIdx.x * (LG_NWL + LG_C);
#pragma unroll
  for(int a = 0; a < 4; a++)
#pragma unroll
    for(int b = 0; b < 4; b++)
      pb[t * 256 + (cg * 4 + a) * 16 + ig * 4 + b] = acc[a][b];
  if(t == 0 && ig == 0)
#pragma unroll
    for(int a = 0; a < 4; a++) pb[LG_NWL + cg * 4 + a] = db[a];
}

__global__ void k_dw_reduce(const float *partials, int nblk, float *gw,
  float *gb)
{
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if(q >= LG_NWL + LG_C) return;
  float s = 0.f;
  for(int b = 0; b < nblk; b++) s += partials[(long long)b * (LG_NWL + LG_C) + q];
  if(q < LG_NWL) gw[q] = s;
  else gb[q - LG_NWL] = s;
}

/* ------------------------------------------------ parameters
 * FP32 master weights [layer][tap][cout][cin] (tap t = 9 dz + 3 dy + dx,
 * offsets dz - 1, dy - 1, dx - 1) and biases [layer][cout]; BF16 packs per
 * layer in the UMMA B layout of the convolution's (dz, dx) groups: group
 * g = 3 dz + dx at g * LG_WGRP bytes holds N = 48 rows n = 16 j + cout for
 * the taps dy = 2 - j, K = cin, at byte (cin / 8) * 768 + n * 16 +
 * (cin % 8) * 2.  The transposed pack of the data gradient swaps cout and
 * cin and flips the tap (26 - t). */
__device__ __forceinline__ int lg_pack_off(int t, int o, int c)
{
  int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
  int n = (2 - dy) * 16 + o;
  return (dz * 3 + dx) * LG_WGRP + (c / 8) * (LG_WGRP / 2) + n * 16 + (c % 8) * 2;
}

__global__ void k_pack(const float *w, uint8_t *pack, uint8_t *packT)
{
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if(q >= LG_NW) return;
  int l = q / LG_NWL, rem = q % LG_NWL;
  int t = rem / 256, o = (rem / 16) % 16, c = rem % 16;
  bf16 v = __float2bfloat16_rn(w[q]);
  uint8_t *P = pack + (long long)l * LG_WLAYER;
  uint8_t *PT = packT + (long long)l * LG_WLAYER;
  *reinterpret_cast<bf16 *>(P + lg_pack_off(t, o, c)) = v;
  *reinterpret_cast<bf16 *>(PT + lg_pack_off(26 - t, c, o)) = v;
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int n,
  float lr, float b1, float b2, float eps, float c1, float c2, const int *live)
{
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if(q >= n) return;
  if(!live[q]) { p[q] = 0.f; return; }
  float gq = g[q];
  float mq = b1 * m[q] + (1.f - b1) * gq;
  float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

/* ------------------------------------------------ features and targets */

/* rms sums over fluid cells: (phi_prev^2, (b h^2)^2, p0^2, count) */
__global__ void k_feat_stats(const real *phi, const double *b, const real *p0,
  const int *phase, bbb_geom G, double h2, double *partials,
  unsigned int *ticket, double *out)
{
  __shared__ double sh[32 * 4];
  double v[4] = {0., 0., 0., 0.};
  long long n = (long long)G.nx * G.ny * G.nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    if(phase[cc] > -1) continue;
    double f = phi[cc], bb = b[t] * h2, pp = p0[cc];
    v[0] += f * f; v[1] += bb * bb; v[2] += pp * pp; v[3] += 1.;
  }
  if(bbb_grid_partial<4>(v, partials, ticket, sh)) {
    bbb_grid_finish_sum<4>(v, partials, ticket, sh);
    if(threadIdx.x == 0) {
      double cnt = v[3] > 0 ? v[3] : 1.;
      double s = sqrt(v[0] / cnt), sb = sqrt(v[1] / cnt), sp = sqrt(v[2] / cnt);
      double S = s > 0 ? s : (sb > 0 ? sb : 1.);
      out[0] = S;
      out[1] = sp > 0 ? sp : 1.;
      out[2] = s;
    }
  }
}

/* features on the dense pressure grid, channels-last BF16 (16 channels,
 * 4 live); optionally phi_prev as FP32 for the recorded target */
__global__ void k_features(const real *phi, const double *b, const real *p0,
  const int *phase, bbb_geom G, double h2, const double *scales, bf16 *feat,
  float *phiprev)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  double S = scales[0], Sp = scales[1];
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    bool solid = phase[cc] > -1;
    float f[4];
    f[0] = (float)(b[t] * h2 / S);
    f[1] = (float)(phi[cc] / S);
    f[2] = (float)(p0[cc] / Sp);
    f[3] = solid ? 1.f : 0.f;
    uint4 w0, w1 = make_uint4(0u, 0u, 0u, 0u);
    __nv_bfloat162 a = __floats2bfloat162_rn(f[0], f[1]);
    __nv_bfloat162 c = __floats2bfloat162_rn(f[2], f[3]);
    w0.x = *reinterpret_cast<uint32_t *>(&a);
    w0.y = *reinterpret_cast<uint32_t *>(&c);
    w0.z = 0u; w0.w = 0u;
    reinterpret_cast<uint4 *>(feat)[t * 2] = w0;
    reinterpret_cast<uint4 *>(feat)[t * 2 + 1] = w1;
    if(phiprev) phiprev[t] = (float)phi[cc];
  }
}

/* candidate x = phi_prev + S out in fluid cells, phi_prev in solids */
__global__ void k_guess(const real *phi, const float *out, const int *phase,
  bbb_geom G, const double *scales, double *x)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  double S = scales[0];
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    double v = phi[cc];
    if(phase[cc] <= -1) v += S * (double)out[t];
    x[t] = v;
  }
}

/* crop gather: box of cx*cy*cz cells at (ox, oy, oz) of the full grid
 * (wrapping), features and target (phi_new - phi_prev) / S into slot `s`
 * of the crop store */
__global__ void k_crop(const bf16 *feat, const real *phi_new,
  const float *phiprev, bbb_geom G, const double *scales, int ox, int oy,
  int oz, int cx, int cy, int cz, bf16 *cfeat, float *ctgt)
{
  long long n = (long long)cx * cy * cz;
  double S = scales[0];
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int a = (int)(t % cx);
    long long rr = t / cx;
    int bq = (int)(rr % cy), c = (int)(rr / cy);
    int i = (ox + a) % G.nx, j = (oy + bq) % G.ny, k = (oz + c) % G.nz;
    long long d = i + (long long)G.nx * (j + (long long)G.ny * k);
    long long cc = (i + 1) + (long long)(j + 1) * G.cc_s1 + (long long)(k + 1) * G.cc_s2;
    reinterpret_cast<uint4 *>(cfeat)[t * 2] = reinterpret_cast<const uint4 *>(feat)[d * 2];
    reinterpret_cast<uint4 *>(cfeat)[t * 2 + 1] = reinterpret_cast<const uint4 *>(feat)[d * 2 + 1];
    ctgt[t] = (float)((phi_new[cc] - (double)phiprev[d]) / S);
  }
}

/* loss and output gradient on the stacked-crop batch: cells at least
 * `margin` from every crop face */
__global__ void k_loss(const float *out, const float *tgt, int cx, int cy,
  int cz, int ncrop, int margin, double inv_n, bf16 *dz, double *partials,
  unsigned int *ticket, double *loss)
{
  __shared__ double sh[32 * 2];
  double v[2] = {0., 0.};
  long long n = (long long)cx * cy * cz * ncrop;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int a = (int)(t % cx);
    long long rr = t / cx;
    int bq = (int)(rr % cy), c = (int)((rr / cy) % cz);
    bool in = a >= margin && a < cx - margin && bq >= margin && bq < cy - margin
      && c >= margin && c < cz - margin;
    float g = 0.f;
    if(in) {
      float d = out[t] - tgt[t];
      v[0] += (double)d * d;
      v[1] += (double)tgt[t] * tgt[t];
      g = (float)(2.0 * inv_n) * d;
    }
    uint4 w0 = make_uint4(0u, 0u, 0u, 0u), w1 = w0;
    bf16 gb = __float2bfloat16_rn(g);
    w0.x = (uint32_t)(*reinterpret_cast<unsigned short *>(&gb));
    reinterpret_cast<uint4 *>(dz)[t * 2] = w0;
    reinterpret_cast<uint4 *>(dz)[t * 2 + 1] = w1;
  }
  if(bbb_grid_partial<2>(v, partials, ticket, sh)) {
    bbb_grid_finish_sum<2>(v, partials, ticket, sh);
    if(threadIdx.x == 0) { loss[0] = v[0] * inv_n; loss[1] = v[1] * inv_n; }
  }
}

/* ------------------------------------------------ host state */
static struct {
  int init;
  int mode;                       /* bit 0 record, bit 1 use the guess  */
  int first_pending;              /* next solve is the first of a step  */
  unsigned long long rng;
  long long steps_recorded;
  /* parameters */
  float *w, *g, *m, *v;           /* LG_NP each (weights then biases)   */
  int *live;
  uint8_t *pack, *packT;
  long long adam_t;
  /* full-grid buffers */
  long long n;
  bf16 *feat, *act[2];
  float *out, *phiprev;
  double *xc, *scales;
  /* crop store */
  int cx, cy, cz, cap, ncrop, next;
  bf16 *cfeat;
  float *ctgt;
  /* training batch */
  int bcrops;
  bf16 *bfeat;
  float *btgt;
  int *err;
  int pending_record;
  double last_loss;
  /* cost gate (mode bit 4) */
  cudaEvent_t ev[4];              /* guess start/end, solve start/end   */
  int timing;                     /* the solve after an evaluation runs */
  double t_guess, r_ext, r_start;
  int gate_fail, gate_skip;
} L;

template <typename T>
static T *lg_alloc(long long n)
{
  T *p = NULL;
  if(n <= 0) n = 1;
  if(cudaMalloc((void **)&p, sizeof(T) * (size_t)n) != cudaSuccess) {
    bbb_set_status(BBB_ERR_CUDA, "cudaMalloc (learned guess)");
    return NULL;
  }
  cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, g_dev.stream);
  return p;
}

static void lg_free_all(void)
{
  void *ps[] = {L.w, L.g, L.m, L.v, L.live, L.pack, L.packT, L.feat, L.act[0],
    L.act[1], L.out, L.phiprev, L.xc, L.scales, L.cfeat, L.ctgt,
    L.bfeat, L.btgt, L.err};
  for(size_t a = 0; a < sizeof(ps) / sizeof(ps[0]); a++) if(ps[a]) cudaFree(ps[a]);
  int mode = L.mode;
  memset(&L, 0, sizeof(L));
  L.mode = mode;
}

static uint64_t lg_rand(void)
{
  uint64_t z = (L.rng += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static double lg_urand(void) { return (lg_rand() >> 11) * (1.0 / 9007199254740992.0); }

/* Glorot-style init, last layer zero (the net starts as the extrapolation) */
static void lg_init_params(void)
{
  float *h = (float *)calloc(LG_NP, sizeof(float));
  int *live = (int *)calloc(LG_NP, sizeof(int));
  for(int l = 0; l < LG_L; l++) {
    int cin = l == 0 ? LG_NIN : LG_C, cout = l == LG_L - 1 ? 1 : LG_C;
    double sc = sqrt(6.0 / (27.0 * (cin + cout)));
    for(int t = 0; t < LG_T; t++)
      for(int o = 0; o < cout; o++)
        for(int c = 0; c < cin; c++) {
          long long q = (long long)l * LG_NWL + t * 256 + o * 16 + c;
          live[q] = 1;
          h[q] = l == LG_L - 1 ? 0.f : (float)((2.0 * lg_urand() - 1.0) * sc);
        }
    for(int o = 0; o < cout; o++) live[LG_NW + l * LG_C + o] = 1;
  }
  cudaMemcpyAsync(L.w, h, sizeof(float) * LG_NP, cudaMemcpyHostToDevice, g_dev.stream);
  cudaMemcpyAsync(L.live, live, sizeof(int) * LG_NP, cudaMemcpyHostToDevice, g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  free(h);
  free(live);
  cudaMemsetAsync(L.m, 0, sizeof(float) * LG_NP, g_dev.stream);
  cudaMemsetAsync(L.v, 0, sizeof(float) * LG_NP, g_dev.stream);
  L.adam_t = 0;
}

static void lg_repack(void)
{
  k_pack<<<(LG_NW + 255) / 256, 256, 0, g_dev.stream>>>(L.w, L.pack, L.packT);
  BBB_LAUNCHED();
}

static int lg_setup(void)
{
  if(L.init) return 0;
  bbb_dev_require();
  if(!g_dev.ready) return -1;
  static int attr = 0;
  if(!attr) {
    cudaFuncSetAttribute(k_conv_z<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, LG_ZSMEM);
    cudaFuncSetAttribute(k_conv_z<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, LG_ZSMEM);
    cudaFuncSetAttribute(k_conv_z<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, LG_ZSMEM);
    attr = 1;
  }
  if(!L.rng) L.rng = 0x5DEECE66DULL;
  for(int a = 0; a < 4; a++) cudaEventCreate(&L.ev[a]);
  L.w = lg_alloc<float>(LG_NP); L.g = lg_alloc<float>(LG_NP);
  L.m = lg_alloc<float>(LG_NP); L.v = lg_alloc<float>(LG_NP);
  L.live = lg_alloc<int>(LG_NP);
  L.pack = lg_alloc<uint8_t>(LG_L * LG_WLAYER);
  L.packT = lg_alloc<uint8_t>(LG_L * LG_WLAYER);
  L.scales = lg_alloc<double>(8);
  L.err = lg_alloc<int>(4);
  bbb_geom G = bbb_make_geom();
  L.n = (long long)G.nx * G.ny * G.nz;
  L.cx = G.nx < LG_M ? G.nx : LG_M;
  L.cy = G.ny < 32 ? G.ny : 32;
  L.cz = G.nz < 32 ? G.nz : 32;
  L.bcrops = 8;
  lg_init_params();
  lg_repack();
  L.init = 1;
  return bbb_last_status() == BBB_ERR_CUDA ? -1 : 0;
}

static void lg_full_buffers(void)
{
  if(L.feat) return;
  L.feat = lg_alloc<bf16>(L.n * LG_C);
  L.act[0] = lg_alloc<bf16>(L.n * LG_C);
  L.act[1] = lg_alloc<bf16>(L.n * LG_C);
  L.out = lg_alloc<float>(L.n);
  L.phiprev = lg_alloc<float>(L.n);
  L.xc = lg_alloc<double>(L.n);
}

static void lg_crop_store(void)
{
  if(L.cfeat) return;
  L.cap = 256;
  long long cc = (long long)L.cx * L.cy * L.cz;
  L.cfeat = lg_alloc<bf16>(cc * L.cap * LG_C);
  L.ctgt = lg_alloc<float>(cc * L.cap);
}

/* one convolution layer on box B (tensor cores, or the FP32 reference
 * when `ref`) */
static int g_lg_ref = 0;
/* crops recorded per recorded step (bbb_learn_set_crops_per_step) */
static int g_lg_per_step = 8;
static void lg_conv(int mode, const lg_box &B, const bf16 *in, int layer,
  int transposed, float *pre, bf16 *act, float *out32)
{
  const float *bias = L.w + LG_NW + layer * LG_C;
  if(!g_lg_ref) {
    const uint8_t *wp = (transposed ? L.packT : L.pack) + (long long)layer * LG_WLAYER;
    lg_zbox Z = make_lg_zbox(B, 148 * 2);
    if(mode == 0) k_conv_z<0><<<Z.nblk, LG_THREADS, LG_ZSMEM, g_dev.stream>>>(Z, in, wp, bias, pre, act, out32, L.err);
    else if(mode == 1) k_conv_z<1><<<Z.nblk, LG_THREADS, LG_ZSMEM, g_dev.stream>>>(Z, in, wp, bias, pre, act, out32, L.err);
    else k_conv_z<2><<<Z.nblk, LG_THREADS, LG_ZSMEM, g_dev.stream>>>(Z, in, wp, bias, pre, act, out32, L.err);
  } else {
    /* FP32 weights: the transposed form is built on the fly by the host
     * into the gradient buffer's spare space */
    const float *w = L.w + (long long)layer * LG_NWL;
    if(transposed) {
      static float *wt = NULL;
      if(!wt) cudaMalloc((void **)&wt, sizeof(float) * LG_NWL);
      float hw[LG_NWL], ht[LG_NWL];
      cudaMemcpyAsync(hw, w, sizeof(hw), cudaMemcpyDeviceToHost, g_dev.stream);
      cudaStreamSynchronize(g_dev.stream);
      for(int t = 0; t < LG_T; t++)
        for(int o = 0; o < 16; o++)
          for(int c = 0; c < 16; c++) ht[(26 - t) * 256 + c * 16 + o] = hw[t * 256 + o * 16 + c];
      cudaMemcpyAsync(wt, ht, sizeof(ht), cudaMemcpyHostToDevice, g_dev.stream);
      cudaStreamSynchronize(g_dev.stream);
      w = wt;
    }
    if(mode == 0) k_conv_ref<0><<<1184, 128, 0, g_dev.stream>>>(B, in, w, bias, pre, act, out32);
    else if(mode == 1) k_conv_ref<1><<<1184, 128, 0, g_dev.stream>>>(B, in, w, bias, pre, act, out32);
    else k_conv_ref<2><<<1184, 128, 0, g_dev.stream>>>(B, in, w, bias, pre, act, out32);
  }
  BBB_LAUNCHED();
}

/* forward of the 4 layers: in -> out32; pre-activations saved when `pre` */
static void lg_forward(const lg_box &B, const bf16 *in, bf16 *a0, bf16 *a1,
  bf16 *a2, float **pre, float *out32)
{
  bf16 *acts[3] = {a0, a1, a2};
  const bf16 *x = in;
  for(int l = 0; l < 3; l++) {
    lg_conv(0, B, x, l, 0, pre ? pre[l] : NULL, acts[l], NULL);
    x = acts[l];
  }
  lg_conv(1, B, x, 3, 0, NULL, NULL, out32);
}

/* ------------------------------------------------ C ABI */

extern "C" int bbb_learn_enable(int mode)
{
  L.mode = mode;
  if(mode && lg_setup() != 0) return bbb_last_status() ? bbb_last_status() : BBB_ERR_CUDA;
  L.first_pending = 1;
  return BBB_OK;
}

extern "C" void bbb_learn_use_reference_conv(int on) { g_lg_ref = on; }

extern "C" int bbb_learn_set_crops_per_step(int n)
{
  if(n < 1 || n > 64) return BBB_ERR_CONFIG;
  g_lg_per_step = n;
  return BBB_OK;
}

/* the solve that follows is the first of a time step (called by
 * cuda_store_u, the last call of the reference's step) */
void bbb_learn_step_boundary(void)
{
  L.first_pending = 1;
}

/* The cost gate's decision after an evaluated solve.  The guess saved
 * about ln(r_ext / r_start) / ln(r_start / r_final) of the solve's
 * Krylov work (the solve reduces its residual geometrically from r_start
 * to r_final; starting from the extrapolation it would have had the
 * extra factor r_ext / r_start to remove), so its benefit in time is that
 * fraction of t_solve_ms.  When the benefit does not exceed the cost of
 * evaluating the guess (features, net, the two residual norms), the next
 * evaluations are skipped: 8 steps after the first such solve, doubling
 * per consecutive one up to 256; a paying evaluation resets the count.
 * Returns the number of steps to skip; *benefit_ms gets the estimate. */
extern "C" int bbb_learn_gate_decide(double t_guess_ms, double t_solve_ms,
  double r_ext, double r_start, double r_final, int *fails, double *benefit_ms)
{
  double benefit = 0.;
  if(r_start < r_ext && r_final > 0. && r_start > r_final && t_solve_ms > 0.)
    benefit = t_solve_ms * log(r_ext / r_start) / log(r_start / r_final);
  if(benefit_ms) *benefit_ms = benefit;
  if(benefit > t_guess_ms) {
    *fails = 0;
    return 0;
  }
  int f = ++*fails;
  return 8 << (f - 1 < 5 ? f - 1 : 5);
}

/* called after b (kb), x = phi_prev (kx) are set: features, the guess and
 * the gate.  Returns 1 when the guess replaced x.  With mode bit 4 the
 * evaluation itself is gated on its measured cost (bbb_learn_gate_decide):
 * the evaluation and the solve after it are timed with CUDA events. */
int bbb_learn_pre_solve(void)
{
  L.pending_record = 0;
  if(!L.mode || !L.first_pending) return 0;
  L.first_pending = 0;
  int record = (L.mode & 1) != 0;
  int use = (L.mode & 2) != 0;
  if(use && (L.mode & 4) && L.gate_skip > 0) {
    L.gate_skip--;
    use = 0;
  }
  if(!record && !use) return 0;
  if(lg_setup() != 0) return 0;
  lg_full_buffers();
  bbb_geom G = bbb_make_geom();
  double h2 = G.dx * G.dx;
  if(use) cudaEventRecord(L.ev[0], g_dev.stream);
  k_feat_stats<<<NPW_LG, 256, 0, g_dev.stream>>>(g_dev.phi, g_dev.kb, g_dev.p0,
    g_dev.phase, G, h2, g_dev.partials, g_dev.red_ticket + 8, L.scales);
  BBB_LAUNCHED();
  k_features<<<NPW_LG, 256, 0, g_dev.stream>>>(g_dev.phi, g_dev.kb, g_dev.p0,
    g_dev.phase, G, h2, L.scales, L.feat, record ? L.phiprev : NULL);
  BBB_LAUNCHED();
  L.pending_record = record;
  int used = 0;
  if(use) {
    lg_box B = make_lg_box(G.nx, G.ny, G.nz, bc.pW == BBB_PERIODIC,
      bc.pS == BBB_PERIODIC, bc.pB == BBB_PERIODIC);
    lg_forward(B, L.feat, L.act[0], L.act[1], L.act[0], NULL, L.out);
    k_guess<<<NPW_LG, 256, 0, g_dev.stream>>>(g_dev.phi, L.out, g_dev.phase, G,
      L.scales, L.xc);
    BBB_LAUNCHED();
    double r_ext = bbb_poisson_resid_norm(g_dev.kx);
    double r_gs = bbb_poisson_resid_norm(L.xc);
    cudaEventRecord(L.ev[1], g_dev.stream);
    g_stats.extrap_r0 = r_ext;
    g_stats.guess_r0 = r_gs;
    int err = 0;
    cudaMemcpyAsync(&err, L.err, sizeof(int), cudaMemcpyDeviceToHost, g_dev.stream);
    cudaStreamSynchronize(g_dev.stream);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, L.ev[0], L.ev[1]);
    g_stats.guess_evaluated = 1;
    g_stats.guess_cost_ms = ms;
    g_stats.guess_benefit_ms = 0.;
    if(err) bbb_set_status(BBB_ERR_CUDA, "learned guess: tensor-core wait ran out");
    if(!err && isfinite(r_gs) && r_gs < r_ext) {
      BBB_CK(cudaMemcpyAsync(g_dev.kx, L.xc, sizeof(double) * L.n,
        cudaMemcpyDeviceToDevice, g_dev.stream));
      g_stats.guess_used++;
      used = 1;
    }
    if(L.mode & 4) {
      L.timing = 1;
      L.t_guess = ms;
      L.r_ext = r_ext;
      L.r_start = used ? r_gs : r_ext;
      cudaEventRecord(L.ev[2], g_dev.stream);
    }
  }
  return used;
}

/* called once a solve's final residual norm r_final is on the host: the
 * gate's decision after an evaluated solve */
void bbb_learn_solve_done(double r_final)
{
  if(!L.timing) return;
  L.timing = 0;
  cudaEventRecord(L.ev[3], g_dev.stream);
  cudaEventSynchronize(L.ev[3]);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, L.ev[2], L.ev[3]);
  double benefit = 0.;
  L.gate_skip = bbb_learn_gate_decide(L.t_guess, ms, L.r_ext, L.r_start, r_final,
    &L.gate_fail, &benefit);
  g_stats.guess_benefit_ms = benefit;
}

/* called after the solve wrote phi: record crops of (features, target) */
void bbb_learn_post_solve(void)
{
  if(!L.pending_record) return;
  L.pending_record = 0;
  lg_crop_store();
  bbb_geom G = bbb_make_geom();
  long long cc = (long long)L.cx * L.cy * L.cz;
  for(int q = 0; q < g_lg_per_step; q++) {
    int slot = L.next;
    L.next = (L.next + 1) % L.cap;
    if(L.ncrop < L.cap) L.ncrop++;
    int ox = (int)(lg_rand() % (uint64_t)G.nx);
    int oy = (int)(lg_rand() % (uint64_t)G.ny);
    int oz = (int)(lg_rand() % (uint64_t)G.nz);
    k_crop<<<256, 256, 0, g_dev.stream>>>(L.feat, g_dev.phi, L.phiprev, G,
      L.scales, ox, oy, oz, L.cx, L.cy, L.cz, L.cfeat + slot * cc * LG_C,
      L.ctgt + slot * cc);
    BBB_LAUNCHED();
  }
  L.steps_recorded++;
}

/* work buffers of one gradient evaluation on an nb-crop box */
struct lg_work {
  bf16 *act[3], *dz[2];
  float *pre[3], *out, *part;
  double *loss;
};

static void lg_work_alloc(lg_work &W, long long n)
{
  for(int a = 0; a < 3; a++) {
    W.act[a] = lg_alloc<bf16>(n * LG_C);
    W.pre[a] = lg_alloc<float>(n * LG_C);
  }
  W.dz[0] = lg_alloc<bf16>(n * LG_C);
  W.dz[1] = lg_alloc<bf16>(n * LG_C);
  W.out = lg_alloc<float>(n);
  W.part = lg_alloc<float>((long long)296 * (LG_NWL + LG_C));
  W.loss = lg_alloc<double>(4);
}

static void lg_work_free(lg_work &W)
{
  void *ps[] = {W.act[0], W.act[1], W.act[2], W.dz[0], W.dz[1], W.pre[0],
    W.pre[1], W.pre[2], W.out, W.part, W.loss};
  for(size_t a = 0; a < sizeof(ps) / sizeof(ps[0]); a++) if(ps[a]) cudaFree(ps[a]);
  memset(&W, 0, sizeof(W));
}

static lg_work g_train_w;

/* loss (MSE over cells at least `margin` from the faces of every crop of
 * cx*cy*cz cells, nb crops stacked along z) and its gradient into L.g */
static void lg_grad(const bf16 *feat, const float *tgt, int cx, int cy,
  int cz, int nb, int margin, lg_work &W)
{
  lg_box B = make_lg_box(cx, cy, cz * nb, 0, 0, 0);
  long long nin = (long long)(cx - 2 * margin) * (cy - 2 * margin)
    * (cz - 2 * margin) * nb;
  double inv_n = nin > 0 ? 1.0 / (double)nin : 0.;
  lg_forward(B, feat, W.act[0], W.act[1], W.act[2], W.pre, W.out);
  k_loss<<<NPW_LG, 256, 0, g_dev.stream>>>(W.out, tgt, cx, cy, cz, nb, margin,
    inv_n, W.dz[0], g_dev.partials, g_dev.red_ticket + 9, W.loss);
  BBB_LAUNCHED();
  /* backward: layer 4 .. 1 */
  const bf16 *xin[4] = {feat, W.act[0], W.act[1], W.act[2]};
  int cur = 0;
  for(int l = LG_L - 1; l >= 0; l--) {
    int blocks = (int)(B.ntiles < 296 ? B.ntiles : 296);
    k_dw<<<blocks, LG_DW_THREADS, 0, g_dev.stream>>>(B, xin[l], W.dz[cur], W.part);
    BBB_LAUNCHED();
    k_dw_reduce<<<(LG_NWL + LG_C + 255) / 256, 256, 0, g_dev.stream>>>(W.part,
      blocks, L.g + (long long)l * LG_NWL, L.g + LG_NW + l * LG_C);
    BBB_LAUNCHED();
    if(l > 0) {
      lg_conv(2, B, W.dz[cur], l, 1, W.pre[l - 1], W.dz[cur ^ 1], NULL);
      cur ^= 1;
    }
  }
}

static double lg_check_err(void)
{
  int err = 0;
  cudaMemcpyAsync(&err, L.err, sizeof(int), cudaMemcpyDeviceToHost, g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  if(err) bbb_set_status(BBB_ERR_CUDA, "learned guess: tensor-core wait ran out");
  return err;
}

/* `iters` Adam steps on batches of recorded crops; returns the last
 * relative loss (MSE / mean target^2), or -1 without data */
extern "C" double bbb_learn_train(int iters, double lr)
{
  if(lg_setup() != 0 || L.ncrop == 0) return -1.;
  long long cc = (long long)L.cx * L.cy * L.cz;
  int nb = L.bcrops;
  lg_work &W = g_train_w;
  if(!L.bfeat) {
    L.bfeat = lg_alloc<bf16>(cc * nb * LG_C);
    L.btgt = lg_alloc<float>(cc * nb);
    lg_work_alloc(W, cc * nb);
  }
  cudaMemsetAsync(L.err, 0, sizeof(int), g_dev.stream);
  double hl[2] = {0., 0.};
  for(int it = 0; it < iters; it++) {
    for(int q = 0; q < nb; q++) {
      int s = (int)(lg_rand() % (uint64_t)L.ncrop);
      BBB_CK(cudaMemcpyAsync(L.bfeat + q * cc * LG_C, L.cfeat + s * cc * LG_C,
        sizeof(bf16) * cc * LG_C, cudaMemcpyDeviceToDevice, g_dev.stream));
      BBB_CK(cudaMemcpyAsync(L.btgt + q * cc, L.ctgt + s * cc, sizeof(float) * cc,
        cudaMemcpyDeviceToDevice, g_dev.stream));
    }
    lg_grad(L.bfeat, L.btgt, L.cx, L.cy, L.cz, nb, 4, W);
    L.adam_t++;
    float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - powf(b1, (float)L.adam_t), c2 = 1.f - powf(b2, (float)L.adam_t);
    k_adam<<<(LG_NP + 255) / 256, 256, 0, g_dev.stream>>>(L.w, L.g, L.m, L.v,
      LG_NP, (float)lr, b1, b2, 1e-8f, c1, c2, L.live);
    BBB_LAUNCHED();
    lg_repack();
  }
  cudaMemcpyAsync(hl, W.loss, sizeof(hl), cudaMemcpyDeviceToHost, g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  lg_check_err();
  L.last_loss = hl[1] > 0 ? hl[0] / hl[1] : hl[0];
  return L.last_loss;
}

/* loss and parameter gradient on a caller's device batch (nb crops of
 * cx*cy*cz cells stacked along z, features channels-last BF16 16 channels,
 * FP32 targets) without updating the parameters; the gradient goes to
 * grad_host (bbb_learn_param_count floats).  Returns the MSE or -1. */
extern "C" double bbb_learn_grad(int cx, int cy, int cz, int nb, int margin,
  const void *feat_d, const float *tgt_d, float *grad_host)
{
  if(lg_setup() != 0) return -1.;
  lg_work W;
  memset(&W, 0, sizeof(W));
  lg_work_alloc(W, (long long)cx * cy * cz * nb);
  cudaMemsetAsync(L.err, 0, sizeof(int), g_dev.stream);
  lg_grad((const bf16 *)feat_d, tgt_d, cx, cy, cz, nb, margin, W);
  double hl[2] = {0., 0.};
  cudaMemcpyAsync(hl, W.loss, sizeof(hl), cudaMemcpyDeviceToHost, g_dev.stream);
  cudaMemcpyAsync(grad_host, L.g, sizeof(float) * LG_NP, cudaMemcpyDeviceToHost,
    g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  lg_work_free(W);
  if(lg_check_err()) return -1.;
  return hl[0];
}

extern "C" int bbb_learn_crops(void) { return L.ncrop; }

/* parameters as FP32 [layer][tap][cout][cin] then biases [layer][cout] */
extern "C" int bbb_learn_get_params(float *host, int n)
{
  if(!L.init || n < LG_NP) return BBB_ERR_STATE;
  cudaMemcpyAsync(host, L.w, sizeof(float) * LG_NP, cudaMemcpyDeviceToHost, g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  return BBB_OK;
}

extern "C" int bbb_learn_set_params(const float *host, int n)
{
  if(lg_setup() != 0) return BBB_ERR_CUDA;
  if(n < LG_NP) return BBB_ERR_CONFIG;
  cudaMemcpyAsync(L.w, host, sizeof(float) * LG_NP, cudaMemcpyHostToDevice, g_dev.stream);
  lg_repack();
  cudaStreamSynchronize(g_dev.stream);
  return BBB_OK;
}

extern "C" int bbb_learn_param_count(void) { return LG_NP; }

/* run the 4-layer net on a caller-supplied box of features (device
 * pointers; channels-last BF16 16 channels in, FP32 out) -- the tensor-core
 * path, or the FP32 CUDA-core reference when `ref` */
extern "C" int bbb_learn_forward(int nx, int ny, int nz, int px, int py,
  int pz, const void *feat_d, float *out_d, int ref)
{
  if(lg_setup() != 0) return BBB_ERR_CUDA;
  long long n = (long long)nx * ny * nz;
  bf16 *a0 = NULL, *a1 = NULL;
  if(cudaMalloc((void **)&a0, sizeof(bf16) * n * LG_C) != cudaSuccess ||
     cudaMalloc((void **)&a1, sizeof(bf16) * n * LG_C) != cudaSuccess) {
    if(a0) cudaFree(a0);
    return BBB_ERR_CUDA;
  }
  lg_box B = make_lg_box(nx, ny, nz, px, py, pz);
  int save = g_lg_ref;
  g_lg_ref = ref;
  cudaMemsetAsync(L.err, 0, sizeof(int), g_dev.stream);
  lg_forward(B, (const bf16 *)feat_d, a0, a1, a0, NULL, out_d);
  g_lg_ref = save;
  int err = 0;
  cudaMemcpyAsync(&err, L.err, sizeof(int), cudaMemcpyDeviceToHost, g_dev.stream);
  cudaStreamSynchronize(g_dev.stream);
  cudaFree(a0);
  cudaFree(a1);
  if(err) return BBB_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? BBB_OK : BBB_ERR_CUDA;
}

void bbb_learn_release(void)
{
  lg_work_free(g_train_w);
  lg_free_all();
}
