/*
 * Wake network: a 1-D convolutional surrogate of the CSR wake integral,
 * trained and evaluated with hand-written tcgen05 (UMMA) kernels, BF16
 * operands and FP32 accumulation in tensor memory.
 *
 * Tensors are channels-last: an activation is [n_profiles][n_bins][64] BF16,
 * one 128-byte row per bin, so one TMA box of 128 rows x 64 channels is one
 * UMMA operand tile in the 128-byte-swizzled layout.  A dilated convolution
 * with 5 taps is an implicit GEMM: for tap t the A tile is the same box
 * shifted by (t-2)*dilation rows, with rows outside the profile read as zero
 * by the TMA unit.
 *
 * Layers: 6 convolutions of 64 channels, 5 taps, dilations set per layer,
 * GELU between them.  The input has 4 live channels (density, derivative,
 * slippage code, density shifted by the slippage) and the output 1 live channel; both are carried in 64-wide
 * tensors with zero channels, so every layer runs the same kernels.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>
#include "b2e_tmap.h"
#include "b2e_umma.cuh"
#include "b2e_wakenet.h"
#include "elegant_b200.h"

namespace b2e {
using namespace umma;

/* ------------------------------------------------------------------ self-test
 * mode 0 (K-major):  D[128][64] = A[128][64] . B[64][64]^T  (K = 64)
 * mode 1 (MN-major): D[m][n] = sum_k A[m/64][k][m%64] * B[k][n], A two blocks
 *                    [2][128][64], B [128][64]  (K = 128)
 * mode 2 (timeout drill): the same kernel, but thread 0 issues no load and
 *                    waits on the load barrier, which nothing completes,
 *                    for `spin_limit` polls; it then takes the kernel's
 *                    timeout path (status ST_TIMEOUT_TMA, the epilogue
 *                    released without an MMA, TMEM freed) and returns.
 * One CTA of 128 threads; thread 0 issues TMA and MMA, all four warps read
 * TMEM. */
__global__ void __launch_bounds__(128, 1)
    umma_selftest_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int mode,
                         float *D, unsigned int *status, uint32_t spin_limit) {
  extern __shared__ __align__(1024) unsigned char dsmem[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)dsmem + 1023) & ~(uintptr_t)1023);
  unsigned char *sa = smem;           /* 32 KB: A (mode 0: 16 KB) */
  unsigned char *sb = smem + 32768;   /* 16 KB: B */
  __shared__ __align__(8) uint64_t bar_load, bar_mma;
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5;

  if (threadIdx.x == 0) {
    mbar_init(&bar_load, 1);
    mbar_init(&bar_mma, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(&tmem_base, 64);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (threadIdx.x == 0) {
    if (mode == 0) {
      mbar_expect_tx(&bar_load, 16384 + 8192);
      tma_load_3d(sa, &ta, &bar_load, 0, 0, 0);
      tma_load_3d(sb, &tb, &bar_load, 0, 0, 0);
    } else if (mode == 1) {
      mbar_expect_tx(&bar_load, 16384 * 2 + 16384);
      tma_load_3d(sa, &ta, &bar_load, 0, 0, 0);
      tma_load_3d(sa + 16384, &ta, &bar_load, 0, 0, 1);
      tma_load_3d(sb, &tb, &bar_load, 0, 0, 0);
    } /* mode 2: nothing will arrive on bar_load */
    if (mbar_wait(&bar_load, 0, status, ST_TIMEOUT_TMA, spin_limit)) {
      tc_fence_after();
      if (mode == 0) {
        const uint32_t id = idesc_bf16(128, 64, false, false);
        for (int k = 0; k < 4; k++) {
          uint64_t da = sw128_desc(smem_u32(sa) + 32 * k, 16, 1024);
          uint64_t db = sw128_desc(smem_u32(sb) + 32 * k, 16, 1024);
          mma_bf16(tmem, da, db, id, k > 0);
        }
      } else {
        const uint32_t id = idesc_bf16(128, 64, true, true);
        for (int k = 0; k < 8; k++) {
          uint64_t da = sw128_desc(smem_u32(sa) + 2048 * k, 16384, 1024);
          uint64_t db = sw128_desc(smem_u32(sb) + 2048 * k, 16384, 1024);
          mma_bf16(tmem, da, db, id, k > 0);
        }
      }
      mma_commit(&bar_mma);
    } else {
      /* no MMA issued: release the epilogue */
      mbar_arrive(&bar_mma);
    }
  }
  __syncwarp();
  const bool ok = mbar_wait(&bar_mma, 0, status, ST_TIMEOUT_MMA, spin_limit);
  tc_fence_after();
  if (ok && *(volatile unsigned int *)status == ST_OK) {
    const int row = warp * 32 + (threadIdx.x & 31);
    for (int c = 0; c < 64; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
      tmem_wait_ld();
      for (int i = 0; i < 16; i++)
        D[row * 64 + c + i] = v[i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 64);
  }
}


/* ------------------------------------------------------------ conv kernel
 * Persistent, warp-specialised implicit-GEMM convolution, one 128-bin tile
 * of one profile per accumulator:
 *   warp 0   TMA producer: the 5 weight taps once, then per tile the 5
 *            shifted 128x64 activation boxes through a WN_STAGES-deep ring;
 *   warp 1   one thread issues UMMA 128x64x16 (4 per tap, 20 per tile) into
 *            one of two TMEM accumulators and commits to free the stage;
 *   warps 2-9 epilogue: TMEM -> registers (warp w reads lanes 32*(w%4)..;
 *            warps 2-5 take channels 0-31, warps 6-9 channels 32-63),
 *            bias + GELU (hidden), output channel 0 (output), or times
 *            GELU'(z) of the previous layer (backward data), BF16 stores.
 *            The erf/exp of GELU and GELU' bound the epilogue, hence two
 *            warps per lane quadrant; launch bounds of two CTAs per SM
 *            (96 registers, no spills) keep 16 epilogue warps per SM.
 * Bounded waits everywhere; a timeout sets the status word and every role
 * leaves its loop. */
constexpr int CONV_EPI_WARPS = 8;
constexpr int CONV_THREADS = 64 + 32 * CONV_EPI_WARPS;
constexpr int WG_THREADS = 192;
constexpr size_t CONV_W_BYTES = (size_t)WN_TAPS * 64 * 128;  /* 40 KB */
constexpr size_t CONV_STAGE_BYTES = 128 * 128;               /* 16 KB */
constexpr size_t CONV_SMEM = 1024 + CONV_W_BYTES + WN_STAGES * CONV_STAGE_BYTES;

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

template <int EPI>
__global__ void __launch_bounds__(CONV_THREADS, 2)
    conv_kernel(const __grid_constant__ CUtensorMap t_in, const __grid_constant__ CUtensorMap t_w, ConvArgs a) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  unsigned char *sm = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  unsigned char *sw = sm;
  unsigned char *sa = sm + CONV_W_BYTES;
  __shared__ __align__(8) uint64_t full[WN_STAGES], empty[WN_STAGES], tfull[2], tempty[2], wbar;
  __shared__ uint32_t tmem_base;
  __shared__ float sbias[64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tpp = a.L >> 7, n_tiles = a.n_prof * tpp;
  constexpr int N = EPI == EPI_OUTPUT ? 16 : 64;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, N, false, false);

  if (threadIdx.x == 0) {
    for (int i = 0; i < WN_STAGES; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], CONV_EPI_WARPS);
    }
    mbar_init(&wbar, 1);
    fence_barrier_init();
  }
  if (threadIdx.x < 64)
    sbias[threadIdx.x] = (EPI != EPI_BWD && a.bias) ? a.bias[threadIdx.x] : 0.f;
  if (warp == 0) {
    tmem_alloc(&tmem_base, 128);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&t_in);
      prefetch_tmap(&t_w);
      mbar_expect_tx(&wbar, (uint32_t)CONV_W_BYTES);
      for (int t = 0; t < WN_TAPS; t++)
        tma_load_3d(sw + t * 8192, &t_w, &wbar, 0, t * 64, 0);
      uint32_t it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const int b = tile / tpp, l0 = (tile - b * tpp) << 7;
        for (int t = 0; t < WN_TAPS; t++, it++) {
          const int s = it % WN_STAGES;
          if (!mbar_wait(&empty[s], ((it / WN_STAGES) & 1) ^ 1, a.status, ST_TIMEOUT_TMA)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], (uint32_t)CONV_STAGE_BYTES);
          tma_load_3d(sa + s * CONV_STAGE_BYTES, &t_in, &full[s], 0, l0 + a.sign * (t - 2) * a.dilation, b);
        }
      }
      /* let the copies still in flight land before the block can exit */
      for (uint32_t k = it > WN_STAGES ? it - WN_STAGES : 0; k < it; k++)
        mbar_wait(&full[k % WN_STAGES], (k / WN_STAGES) & 1, nullptr, 0);
      mbar_wait(&wbar, 0, nullptr, 0);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = mbar_wait(&wbar, 0, a.status, ST_TIMEOUT_WEIGHTS);
      tc_fence_after();
      uint32_t it = 0, j = 0;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x, j++) {
        const uint32_t acc = j & 1;
        if (!mbar_wait(&tempty[acc], ((j >> 1) & 1) ^ 1, a.status, ST_TIMEOUT_MMA)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + acc * 64;
        for (int t = 0; t < WN_TAPS; t++, it++) {
          const int s = it % WN_STAGES;
          if (!mbar_wait(&full[s], (it / WN_STAGES) & 1, a.status, ST_TIMEOUT_MMA)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sa + s * CONV_STAGE_BYTES), b0 = smem_u32(sw + t * 8192);
          for (int k = 0; k < 4; k++)
            mma_bf16(d, sw128_desc(a0 + 32 * k, 16, 1024), sw128_desc(b0 + 32 * k, 16, 1024), IDESC,
                     (t | k) != 0);
          mma_commit(&empty[s]);
        }
        if (!ok)
          break;
        mma_commit(&tfull[acc]);
      }
    }
  } else {
    const int q = warp & 3;               /* the TMEM lane quadrant this warp may read */
    const int half = (warp - 2) >> 2;     /* channels [32 half, 32 half + 32) */
    constexpr int NC = N == 64 ? 32 : N;  /* channels per thread */
    const int c0 = N == 64 ? 32 * half : 0;
    const bool works = N == 64 || half == 0; /* the output layer's channel 0: one warp per quadrant */
    const int r = q * 32 + lane;           /* row of the tile this thread owns */
    uint32_t j = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, j++) {
      const uint32_t acc = j & 1;
      if (!mbar_wait(&tfull[acc], (j >> 1) & 1, a.status, ST_TIMEOUT_EPI))
        break;
      tc_fence_after();
      float v[NC];
      if (works) {
        const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + acc * 64 + c0;
#pragma unroll
        for (int c = 0; c < NC; c += 16)
          tmem_ld16(base + c, v + c);
        tmem_wait_ld();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0)
        mbar_arrive(&tempty[acc]);
      if (!works)
        continue;
      const int b = tile / tpp, l0 = (tile - b * tpp) << 7;
      const size_t row = (size_t)b * a.L + l0 + r;
      if (EPI == EPI_OUTPUT) {
        a.y_out[row] = v[0] + sbias[0];
      } else if (EPI == EPI_HIDDEN) {
        uint4 *zo = a.z_out ? reinterpret_cast<uint4 *>(a.z_out + row * 64 + c0) : nullptr;
        uint4 *ao = reinterpret_cast<uint4 *>(a.a_out + row * 64 + c0);
#pragma unroll
        for (int c = 0; c < NC; c += 8) {
          float z[8];
#pragma unroll
          for (int i = 0; i < 8; i++)
            z[i] = v[c + i] + sbias[c0 + c + i];
          if (zo)
            zo[c / 8] = make_uint4(pack_bf16(z[0], z[1]), pack_bf16(z[2], z[3]), pack_bf16(z[4], z[5]),
                                   pack_bf16(z[6], z[7]));
          ao[c / 8] = make_uint4(pack_bf16(gelu_f(z[0]), gelu_f(z[1])), pack_bf16(gelu_f(z[2]), gelu_f(z[3])),
                                 pack_bf16(gelu_f(z[4]), gelu_f(z[5])), pack_bf16(gelu_f(z[6]), gelu_f(z[7])));
        }
      } else {
        const uint4 *zp = reinterpret_cast<const uint4 *>(a.z_prev + row * 64 + c0);
        uint4 *go = reinterpret_cast<uint4 *>(a.a_out + row * 64 + c0);
#pragma unroll
        for (int c = 0; c < NC; c += 8) {
          uint4 zz = zp[c / 8];
          const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&zz);
          float g[8];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            float2 f = __bfloat1622float2(h[i]);
            g[2 * i] = v[c + 2 * i] * gelu_grad_f(f.x);
            g[2 * i + 1] = v[c + 2 * i + 1] * gelu_grad_f(f.y);
          }
          go[c / 8] = make_uint4(pack_bf16(g[0], g[1]), pack_bf16(g[2], g[3]), pack_bf16(g[4], g[5]),
                                 pack_bf16(g[6], g[7]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
}

/* ---------------------------------------------------------- weight gradient
 * dW[t][co][ci] = sum over bins of dZ[bin][co] * X[bin + (t-2) d][ci].
 * Per 128-bin tile the producer loads the dZ box and the 5 shifted input
 * boxes (96 KB, two stages).  The MMA thread treats the input boxes as
 * MN-major A operands (M = ci of two taps stacked: taps (0,1), (2,3), (4,-))
 * and the dZ box as an MN-major B operand (N = co), K = the 128 bins in
 * steps of 16, accumulating three 128x64 FP32 tiles in TMEM over all tiles
 * of the block.  The epilogue writes the block's partial sums
 * [5][64 ci][64 co]. */
constexpr int WG_STAGES = 2;
constexpr size_t WG_STAGE_BYTES = 6 * CONV_STAGE_BYTES; /* 96 KB */
constexpr size_t WG_SMEM = 1024 + WG_STAGES * WG_STAGE_BYTES;

__global__ void __launch_bounds__(WG_THREADS, 1)
    wgrad_kernel(const __grid_constant__ CUtensorMap t_in, const __grid_constant__ CUtensorMap t_dz, WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  unsigned char *sm = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[WG_STAGES], empty[WG_STAGES], done;
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tpp = a.L >> 7, n_tiles = a.n_prof * tpp;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, 64, true, true);

  if (threadIdx.x == 0) {
    for (int i = 0; i < WG_STAGES; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(&tmem_base, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  bool any = false;

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&t_in);
      prefetch_tmap(&t_dz);
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, it++) {
        const int b = tile / tpp, l0 = (tile - b * tpp) << 7;
        const int s = it % WG_STAGES;
        if (!mbar_wait(&empty[s], ((it / WG_STAGES) & 1) ^ 1, a.status, ST_TIMEOUT_TMA))
          break;
        unsigned char *st = sm + s * WG_STAGE_BYTES;
        mbar_expect_tx(&full[s], (uint32_t)WG_STAGE_BYTES);
        for (int t = 0; t < WN_TAPS; t++)
          tma_load_3d(st + t * CONV_STAGE_BYTES, &t_in, &full[s], 0, l0 + (t - 2) * a.dilation, b);
        tma_load_3d(st + 5 * CONV_STAGE_BYTES, &t_dz, &full[s], 0, l0, b);
      }
      for (uint32_t k = it > WG_STAGES ? it - WG_STAGES : 0; k < it; k++)
        mbar_wait(&full[k % WG_STAGES], (k / WG_STAGES) & 1, nullptr, 0);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, it++) {
        const int s = it % WG_STAGES;
        if (!mbar_wait(&full[s], (it / WG_STAGES) & 1, a.status, ST_TIMEOUT_MMA)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t st = smem_u32(sm + s * WG_STAGE_BYTES);
        const uint32_t bz = st + 5 * (uint32_t)CONV_STAGE_BYTES;
        for (int p = 0; p < 3; p++) {
          const uint32_t ax = st + 2 * p * (uint32_t)CONV_STAGE_BYTES;
          for (int k = 0; k < 8; k++)
            mma_bf16(tmem + 64 * p, sw128_desc(ax + 2048 * k, (uint32_t)CONV_STAGE_BYTES, 1024),
                     sw128_desc(bz + 2048 * k, (uint32_t)CONV_STAGE_BYTES, 1024), IDESC, it > 0 || k > 0);
        }
        mma_commit(&empty[s]);
      }
      if (ok && it > 0)
        mma_commit(&done);
      else
        mbar_arrive(&done);
    }
  }
  any = blockIdx.x < n_tiles;
  if (warp >= 2) {
    const int q = warp & 3;
    const int m = q * 32 + lane; /* accumulator row */
    const bool ok = mbar_wait(&done, 0, a.status, ST_TIMEOUT_EPI);
    tc_fence_after();
    for (int p = 0; p < 3; p++) {
      const int t = 2 * p + (m >> 6), ci = m & 63;
      float v[64];
      if (ok && any && *(volatile unsigned int *)a.status == ST_OK) {
#pragma unroll
        for (int c = 0; c < 64; c += 16)
          tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + 64 * p + c, v + c);
        tmem_wait_ld();
      } else {
#pragma unroll
        for (int c = 0; c < 64; c++)
          v[c] = 0.f;
      }
      if (t < WN_TAPS) {
        float4 *o = reinterpret_cast<float4 *>(a.partial + (((size_t)blockIdx.x * WN_TAPS + t) * 64 + ci) * 64);
#pragma unroll
        for (int c = 0; c < 64; c += 4)
          o[c / 4] = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

cudaError_t launch_conv(int epi, const CUtensorMap &t_in, const CUtensorMap &t_w, const ConvArgs &a, int grid,
                        cudaStream_t s) {
  cudaError_t e;
  switch (epi) {
  case EPI_HIDDEN:
    e = cudaFuncSetAttribute(conv_kernel<EPI_HIDDEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
    if (e == cudaSuccess)
      conv_kernel<EPI_HIDDEN><<<grid, CONV_THREADS, CONV_SMEM, s>>>(t_in, t_w, a);
    break;
  case EPI_OUTPUT:
    e = cudaFuncSetAttribute(conv_kernel<EPI_OUTPUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
    if (e == cudaSuccess)
      conv_kernel<EPI_OUTPUT><<<grid, CONV_THREADS, CONV_SMEM, s>>>(t_in, t_w, a);
    break;
  default:
    e = cudaFuncSetAttribute(conv_kernel<EPI_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
    if (e == cudaSuccess)
      conv_kernel<EPI_BWD><<<grid, CONV_THREADS, CONV_SMEM, s>>>(t_in, t_w, a);
    break;
  }
  return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t launch_wgrad(const CUtensorMap &t_in, const CUtensorMap &t_dz, const WgradArgs &a, int grid,
                         cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WG_SMEM);
  if (e != cudaSuccess)
    return e;
  wgrad_kernel<<<grid, WG_THREADS, WG_SMEM, s>>>(t_in, t_dz, a);
  return cudaGetLastError();
}

} // namespace b2e

using namespace b2e;

extern "C" int b2e_umma_selftest(int mode, const void *dev_a, const void *dev_b, float *dev_d, void *stream) {
  if (mode < 0 || mode > 2 || (mode < 2 && (!dev_a || !dev_b || !dev_d)))
    return B2E_ERR_ARG;
  CUtensorMap ta, tb;
  memset(&ta, 0, sizeof(ta));
  memset(&tb, 0, sizeof(tb));
  cudaError_t e = cudaSuccess;
  if (mode == 2) {
    /* the drill loads nothing: no tensor maps */
  } else if (mode == 0) {
    e = make_tmap_rows64(&ta, dev_a, 128, 1, 128);
    if (e == cudaSuccess)
      e = make_tmap_rows64(&tb, dev_b, 64, 1, 64);
  } else {
    e = make_tmap_rows64(&ta, dev_a, 128, 2, 128);
    if (e == cudaSuccess)
      e = make_tmap_rows64(&tb, dev_b, 128, 1, 128);
  }
  if (e != cudaSuccess)
    return B2E_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int *status = nullptr;
  if (cudaMallocAsync((void **)&status, sizeof(unsigned int), s) != cudaSuccess)
    return B2E_ERR_NOMEM;
  cudaMemsetAsync(status, 0, sizeof(unsigned int), s);
  const size_t smem = 32768 + 16384 + 1024;
  cudaFuncSetAttribute(umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  /* the drill's wait gives up after 4096 polls instead of the kernels' limit */
  umma_selftest_kernel<<<1, 128, smem, s>>>(ta, tb, mode, dev_d, status, mode == 2 ? 4096u : B2E_SPIN_LIMIT);
  e = cudaGetLastError();
  unsigned int st = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&st, status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  cudaFreeAsync(status, s);
  if (e != cudaSuccess)
    return B2E_ERR_CUDA;
  return st ? B2E_ERR_TIMEOUT : B2E_OK;
}

/* ======================================================== network context */
namespace b2e {

/* inputs [n][WN_IN][L] FP32 -> X0 [n][L][64] BF16 (channels WN_IN..63 zero) */
__global__ void wn_pack_kernel(const float *in, int L, int64_t rows, __nv_bfloat16 *x0) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= rows)
    return;
  const int64_t p = r / L, i = r - p * L;
  const float *src = in + p * WN_IN * L + i;
  uint4 *dst = reinterpret_cast<uint4 *>(x0 + r * 64);
  dst[0] = make_uint4(pack_bf16(src[0], src[L]), pack_bf16(src[2 * L], src[3 * L]), 0u, 0u);
  for (int c = 1; c < 8; c++)
    dst[c] = make_uint4(0u, 0u, 0u, 0u);
}

/* residual y - target into channel 0 of dZ6; per-block sums of squares */
__global__ void wn_loss_kernel(const float *y, const float *target, int64_t rows, __nv_bfloat16 *dz6, double *partial) {
  __shared__ double red[256];
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double sq = 0;
  if (r < rows) {
    const float d = y[r] - target[r];
    sq = (double)d * d;
    uint4 *dst = reinterpret_cast<uint4 *>(dz6 + r * 64);
    dst[0] = make_uint4(pack_bf16(d, 0.f), 0u, 0u, 0u);
    for (int c = 1; c < 8; c++)
      dst[c] = make_uint4(0u, 0u, 0u, 0u);
  }
  red[threadIdx.x] = sq;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    partial[blockIdx.x] = red[0];
}

/* per-block channel sums of dZ [rows][64]: thread (chunk of 8 channels, row lane) */
__global__ void wn_bias_grad_kernel(const __nv_bfloat16 *dz, int64_t rows, float *partial) {
  __shared__ float red[32][65];
  const int chunk = threadIdx.x & 7, lane = threadIdx.x >> 3; /* 8 x 32 */
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t r = blockIdx.x * 32 + lane; r < rows; r += (int64_t)gridDim.x * 32) {
    uint4 v = reinterpret_cast<const uint4 *>(dz + r * 64)[chunk];
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
    for (int i = 0; i < 4; i++) {
      float2 f = __bfloat1622float2(h[i]);
      acc[2 * i] += f.x;
      acc[2 * i + 1] += f.y;
    }
  }
  for (int i = 0; i < 8; i++)
    red[lane][chunk * 8 + i] = acc[i];
  __syncthreads();
  if (threadIdx.x < 64) {
    float s = 0;
    for (int l = 0; l < 32; l++)
      s += red[l][threadIdx.x];
    partial[blockIdx.x * 64 + threadIdx.x] = s;
  }
}

/* grad[t][co][ci] = scale * sum_block wpart[block][t][ci][co]; grad_b[co] likewise */
__global__ void wn_reduce_kernel(const float *wpart, int n_wblocks, const float *bpart, int n_bblocks, float scale,
                                 float *grad_w, float *grad_b) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < WN_WSIZE) {
    const int co = idx & 63, ci = (idx >> 6) & 63, t = idx >> 12; /* idx = (t, ci, co) */
    float s = 0;
    for (int b = 0; b < n_wblocks; b++)
      s += wpart[(size_t)b * WN_WSIZE + idx];
    grad_w[(t * 64 + co) * 64 + ci] = s * scale;
  } else if (idx < WN_WSIZE + 64) {
    const int co = idx - WN_WSIZE;
    float s = 0;
    for (int b = 0; b < n_bblocks; b++)
      s += bpart[b * 64 + co];
    grad_b[co] = s * scale;
  }
}

/* Adam (Kingma & Ba 2015) on the flat FP32 parameters, then the BF16 weight
 * copies: wk[l][t][co][ci] and the transposed wt[l][t][ci][co]. */
__global__ void wn_adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2,
                               float eps, float bc1, float bc2, __nv_bfloat16 *wk, __nv_bfloat16 *wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  if (lr != 0.f) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
  if (i < WN_LAYERS * WN_WSIZE) {
    const int l = i / WN_WSIZE, r = i - l * WN_WSIZE;
    const int t = r >> 12, co = (r >> 6) & 63, ci = r & 63;
    const __nv_bfloat16 h = __float2bfloat16_rn(p[i]);
    wk[i] = h;
    wt[(size_t)l * WN_WSIZE + (t * 64 + ci) * 64 + co] = h;
  }
}

} // namespace b2e

struct b2e_wakenet {
  int device = 0, L = 0, max_batch = 0;
  int dil[WN_LAYERS];
  int64_t step = 0;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  __nv_bfloat16 *wk = nullptr, *wt = nullptr;
  __nv_bfloat16 *x0 = nullptr, *z[WN_LAYERS] = {}, *act[WN_LAYERS] = {}, *dz[WN_LAYERS] = {};
  float *y = nullptr, *wpart = nullptr, *bpart = nullptr;
  double *lpart = nullptr;
  unsigned int *status = nullptr;
  CUtensorMap t_x0, t_act[WN_LAYERS], t_dz[WN_LAYERS], t_wk[WN_LAYERS], t_wt[WN_LAYERS];
  int conv_grid_max = 296, wgrad_grid_max = 148, bias_blocks = 148;
  std::string err;
};

namespace {

int wn_fail(b2e_wakenet *n, int code, const char *msg) {
  if (n)
    n->err = msg;
  return code;
}

#define WN_TRY(net, call)                                                                                         \
  do {                                                                                                           \
    cudaError_t e_ = (call);                                                                                     \
    if (e_ != cudaSuccess)                                                                                       \
      return wn_fail(net, e_ == cudaErrorMemoryAllocation ? B2E_ERR_NOMEM : B2E_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

template <typename T> cudaError_t dalloc(T **p, size_t n) { return cudaMalloc((void **)p, sizeof(T) * n); }

/* bf16 weight copies from the FP32 parameters (Adam kernel with lr = 0) */
cudaError_t refresh_weights(b2e_wakenet *n, cudaStream_t s) {
  wn_adam_kernel<<<(WN_NPARAM + 255) / 256, 256, 0, s>>>(n->params, n->grads, n->adam_m, n->adam_v, WN_NPARAM, 0.f,
                                                          0.9f, 0.999f, 1e-8f, 1.f, 1.f, n->wk, n->wt);
  return cudaGetLastError();
}

/* forward pass of n_prof profiles; keeps the pre-activations when train;
 * the output goes to y_out (the network's own buffer when null) */
int forward(b2e_wakenet *n, const float *inputs, int n_prof, bool train, cudaStream_t s, float *y_out = nullptr) {
  const int64_t rows = (int64_t)n_prof * n->L;
  wn_pack_kernel<<<(int)((rows + 255) / 256), 256, 0, s>>>(inputs, n->L, rows, n->x0);
  WN_TRY(n, cudaGetLastError());
  const int tiles = n_prof * (n->L / 128);
  const int grid = std::min(tiles, n->conv_grid_max);
  for (int l = 0; l < WN_LAYERS; l++) {
    ConvArgs a{};
    a.L = n->L;
    a.n_prof = n_prof;
    a.dilation = n->dil[l];
    a.sign = 1;
    a.bias = n->params + WN_LAYERS * WN_WSIZE + l * WN_CH;
    a.status = n->status;
    const CUtensorMap &tin = l == 0 ? n->t_x0 : n->t_act[l - 1];
    if (l < WN_LAYERS - 1) {
      a.z_out = train ? n->z[l] : nullptr;
      a.a_out = n->act[l];
      WN_TRY(n, launch_conv(EPI_HIDDEN, tin, n->t_wk[l], a, grid, s));
    } else {
      a.y_out = y_out ? y_out : n->y;
      WN_TRY(n, launch_conv(EPI_OUTPUT, tin, n->t_wk[l], a, grid, s));
    }
  }
  return B2E_OK;
}

/* loss, backward pass and gradients (scaled to d(mean squared error)) */
int backward(b2e_wakenet *n, const float *targets, int n_prof, double *loss, cudaStream_t s) {
  const int64_t rows = (int64_t)n_prof * n->L;
  const int lb = (int)((rows + 255) / 256);
  wn_loss_kernel<<<lb, 256, 0, s>>>(n->y, targets, rows, n->dz[WN_LAYERS - 1], n->lpart);
  WN_TRY(n, cudaGetLastError());
  const int tiles = n_prof * (n->L / 128);
  const int cgrid = std::min(tiles, n->conv_grid_max), wgrid = std::min(tiles, n->wgrad_grid_max);
  const float scale = (float)(2.0 / (double)rows);
  for (int l = WN_LAYERS - 1; l >= 0; l--) {
    WgradArgs w{};
    w.L = n->L;
    w.n_prof = n_prof;
    w.dilation = n->dil[l];
    w.partial = n->wpart;
    w.status = n->status;
    WN_TRY(n, launch_wgrad(l == 0 ? n->t_x0 : n->t_act[l - 1], n->t_dz[l], w, wgrid, s));
    wn_bias_grad_kernel<<<n->bias_blocks, 256, 0, s>>>(n->dz[l], rows, n->bpart);
    WN_TRY(n, cudaGetLastError());
    wn_reduce_kernel<<<(WN_WSIZE + 64 + 255) / 256, 256, 0, s>>>(
        n->wpart, wgrid, n->bpart, n->bias_blocks, scale, n->grads + l * WN_WSIZE,
        n->grads + WN_LAYERS * WN_WSIZE + l * WN_CH);
    WN_TRY(n, cudaGetLastError());
    if (l > 0) {
      ConvArgs a{};
      a.L = n->L;
      a.n_prof = n_prof;
      a.dilation = n->dil[l];
      a.sign = -1;
      a.z_prev = n->z[l - 1];
      a.a_out = n->dz[l - 1];
      a.status = n->status;
      WN_TRY(n, launch_conv(EPI_BWD, n->t_dz[l], n->t_wt[l], a, cgrid, s));
    }
  }
  if (loss) {
    std::vector<double> lp(lb);
    WN_TRY(n, cudaMemcpyAsync(lp.data(), n->lpart, sizeof(double) * lb, cudaMemcpyDeviceToHost, s));
    WN_TRY(n, cudaStreamSynchronize(s));
    double sum = 0;
    for (double v : lp)
      sum += v;
    *loss = sum / (double)rows;
  }
  return B2E_OK;
}

int check_status(b2e_wakenet *n, cudaStream_t s) {
  unsigned int st = 0;
  WN_TRY(n, cudaMemcpyAsync(&st, n->status, sizeof(st), cudaMemcpyDeviceToHost, s));
  WN_TRY(n, cudaStreamSynchronize(s));
  if (st) {
    cudaMemsetAsync(n->status, 0, sizeof(unsigned int), s);
    return wn_fail(n, B2E_ERR_TIMEOUT, "wake network: a bounded device wait gave up");
  }
  return B2E_OK;
}

} // namespace

namespace b2e {
int wakenet_infer(b2e_wakenet *net, const float *dev_inputs, int n_prof, float *dev_out, cudaStream_t s) {
  if (!net || n_prof < 0 || n_prof > net->max_batch)
    return B2E_ERR_ARG;
  return n_prof ? forward(net, dev_inputs, n_prof, false, s, dev_out) : B2E_OK;
}
int wakenet_bins(const b2e_wakenet *net) { return net ? net->L : 0; }
int wakenet_max_batch(const b2e_wakenet *net) { return net ? net->max_batch : 0; }
unsigned int wakenet_take_status(b2e_wakenet *net, cudaStream_t s) {
  unsigned int st = 0;
  if (cudaMemcpyAsync(&st, net->status, sizeof(st), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ~0u;
  if (st)
    cudaMemsetAsync(net->status, 0, sizeof(unsigned int), s);
  return st;
}
} // namespace b2e

extern "C" int b2e_wakenet_create(b2e_wakenet **out, int32_t bins, int32_t max_batch, const int32_t *dilations,
                                  int32_t device) {
  if (!out || bins < 128 || bins % 128 || max_batch < 1 || !dilations)
    return B2E_ERR_ARG;
  *out = nullptr;
  for (int l = 0; l < WN_LAYERS; l++)
    if (dilations[l] < 1 || dilations[l] > 4096)
      return B2E_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess)
    return B2E_ERR_CUDA;
  b2e_wakenet *n = new b2e_wakenet();
  n->device = device;
  n->L = bins;
  n->max_batch = max_batch;
  for (int l = 0; l < WN_LAYERS; l++)
    n->dil[l] = dilations[l];
  const size_t act = (size_t)max_batch * bins * 64;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess)
      e = r;
  };
  ok(dalloc(&n->params, WN_NPARAM));
  ok(dalloc(&n->grads, WN_NPARAM));
  ok(dalloc(&n->adam_m, WN_NPARAM));
  ok(dalloc(&n->adam_v, WN_NPARAM));
  ok(dalloc(&n->wk, (size_t)WN_LAYERS * WN_WSIZE));
  ok(dalloc(&n->wt, (size_t)WN_LAYERS * WN_WSIZE));
  ok(dalloc(&n->x0, act));
  for (int l = 0; l < WN_LAYERS; l++) {
    ok(dalloc(&n->dz[l], act));
    if (l < WN_LAYERS - 1) {
      ok(dalloc(&n->z[l], act));
      ok(dalloc(&n->act[l], act));
    }
  }
  ok(dalloc(&n->y, (size_t)max_batch * bins));
  ok(dalloc(&n->wpart, (size_t)n->wgrad_grid_max * WN_WSIZE));
  ok(dalloc(&n->bpart, (size_t)n->bias_blocks * 64));
  ok(dalloc(&n->lpart, (size_t)((int64_t)max_batch * bins + 255) / 256));
  ok(dalloc(&n->status, 1));
  if (e == cudaSuccess) {
    ok(cudaMemset(n->params, 0, sizeof(float) * WN_NPARAM));
    ok(cudaMemset(n->grads, 0, sizeof(float) * WN_NPARAM));
    ok(cudaMemset(n->adam_m, 0, sizeof(float) * WN_NPARAM));
    ok(cudaMemset(n->adam_v, 0, sizeof(float) * WN_NPARAM));
    ok(cudaMemset(n->status, 0, sizeof(unsigned int)));
  }
  if (e == cudaSuccess) {
    ok(make_tmap_rows64(&n->t_x0, n->x0, bins, max_batch, 128));
    for (int l = 0; l < WN_LAYERS; l++) {
      ok(make_tmap_rows64(&n->t_dz[l], n->dz[l], bins, max_batch, 128));
      if (l < WN_LAYERS - 1)
        ok(make_tmap_rows64(&n->t_act[l], n->act[l], bins, max_batch, 128));
      ok(make_tmap_rows64(&n->t_wk[l], n->wk + (size_t)l * WN_WSIZE, WN_TAPS * 64, 1, 64));
      ok(make_tmap_rows64(&n->t_wt[l], n->wt + (size_t)l * WN_WSIZE, WN_TAPS * 64, 1, 64));
    }
  }
  if (e == cudaSuccess)
    ok(refresh_weights(n, 0));
  if (e == cudaSuccess)
    ok(cudaDeviceSynchronize());
  if (e != cudaSuccess) {
    b2e_wakenet_destroy(n);
    return e == cudaErrorMemoryAllocation ? B2E_ERR_NOMEM : B2E_ERR_CUDA;
  }
  *out = n;
  return B2E_OK;
}

extern "C" int b2e_wakenet_destroy(b2e_wakenet *n) {
  if (!n)
    return B2E_ERR_ARG;
  cudaSetDevice(n->device);
  cudaDeviceSynchronize();
  void *ptrs[] = {n->params, n->grads, n->adam_m, n->adam_v, n->wk, n->wt, n->x0, n->y, n->wpart, n->bpart,
                  n->lpart, n->status};
  for (void *p : ptrs)
    if (p)
      cudaFree(p);
  for (int l = 0; l < WN_LAYERS; l++) {
    if (n->z[l])
      cudaFree(n->z[l]);
    if (n->act[l])
      cudaFree(n->act[l]);
    if (n->dz[l])
      cudaFree(n->dz[l]);
  }
  delete n;
  return B2E_OK;
}

extern "C" const char *b2e_wakenet_last_error(const b2e_wakenet *n) { return n ? n->err.c_str() : "null network"; }

extern "C" int64_t b2e_wakenet_param_count(void) { return WN_NPARAM; }

extern "C" int b2e_wakenet_set_params(b2e_wakenet *n, const float *host_params) {
  if (!n || !host_params)
    return B2E_ERR_ARG;
  cudaSetDevice(n->device);
  WN_TRY(n, cudaMemcpy(n->params, host_params, sizeof(float) * WN_NPARAM, cudaMemcpyHostToDevice));
  WN_TRY(n, cudaMemset(n->adam_m, 0, sizeof(float) * WN_NPARAM));
  WN_TRY(n, cudaMemset(n->adam_v, 0, sizeof(float) * WN_NPARAM));
  n->step = 0;
  WN_TRY(n, refresh_weights(n, 0));
  WN_TRY(n, cudaDeviceSynchronize());
  return B2E_OK;
}

extern "C" int b2e_wakenet_get_params(b2e_wakenet *n, float *host_params, float *host_grads) {
  if (!n)
    return B2E_ERR_ARG;
  cudaSetDevice(n->device);
  WN_TRY(n, cudaDeviceSynchronize());
  if (host_params)
    WN_TRY(n, cudaMemcpy(host_params, n->params, sizeof(float) * WN_NPARAM, cudaMemcpyDeviceToHost));
  if (host_grads)
    WN_TRY(n, cudaMemcpy(host_grads, n->grads, sizeof(float) * WN_NPARAM, cudaMemcpyDeviceToHost));
  return B2E_OK;
}

extern "C" int b2e_wakenet_forward(b2e_wakenet *n, const float *dev_inputs, int32_t n_prof, float *dev_out,
                                   void *stream) {
  if (!n || !dev_inputs || !dev_out || n_prof < 0 || n_prof > n->max_batch)
    return B2E_ERR_ARG;
  if (n_prof == 0)
    return B2E_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = forward(n, dev_inputs, n_prof, false, s);
  if (rc)
    return rc;
  WN_TRY(n, cudaMemcpyAsync(dev_out, n->y, sizeof(float) * (size_t)n_prof * n->L, cudaMemcpyDeviceToDevice, s));
  return check_status(n, s);
}

extern "C" int b2e_wakenet_gradients(b2e_wakenet *n, const float *dev_inputs, const float *dev_targets,
                                     int32_t n_prof, double *loss, void *stream) {
  if (!n || !dev_inputs || !dev_targets || n_prof < 1 || n_prof > n->max_batch)
    return B2E_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = forward(n, dev_inputs, n_prof, true, s);
  if (!rc)
    rc = backward(n, dev_targets, n_prof, loss, s);
  if (rc)
    return rc;
  return check_status(n, s);
}

extern "C" int b2e_wakenet_train_step(b2e_wakenet *n, const float *dev_inputs, const float *dev_targets,
                                      int32_t n_prof, float lr, double *loss, void *stream) {
  if (!n || !dev_inputs || !dev_targets || n_prof < 1 || n_prof > n->max_batch || !(lr >= 0))
    return B2E_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = forward(n, dev_inputs, n_prof, true, s);
  if (!rc)
    rc = backward(n, dev_targets, n_prof, loss, s);
  if (rc)
    return rc;
  n->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - powf(b1, (float)n->step), bc2 = 1.f - powf(b2, (float)n->step);
  wn_adam_kernel<<<(WN_NPARAM + 255) / 256, 256, 0, s>>>(n->params, n->grads, n->adam_m, n->adam_v, WN_NPARAM, lr,
                                                          b1, b2, 1e-8f, bc1, bc2, n->wk, n->wt);
  WN_TRY(n, cudaGetLastError());
  return loss ? check_status(n, s) : B2E_OK;
}
