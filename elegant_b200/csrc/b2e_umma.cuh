/*
 * Thin wrappers over the sm_100a instructions used by the wake-network
 * kernels: mbarriers with bounded waits, TMA tiled loads (no multicast),
 * tcgen05 TMEM allocation, UMMA (kind::f16, BF16 x BF16 -> FP32), commit and
 * TMEM loads.  Shared-memory operand tiles use the 128-byte swizzle: rows of
 * 64 BF16 values (128 B), 16-byte chunk c of row r stored at chunk c ^ (r & 7),
 * 8-row atoms of 1024 B.  This is the layout a TMA load with
 * CU_TENSOR_MAP_SWIZZLE_128B writes.
 *
 * Every wait is bounded: after B2E_SPIN_LIMIT polls it records an error code
 * and returns false, so a kernel can release its TMEM and exit instead of
 * hanging the GPU.
 */
#ifndef B2E_UMMA_CUH
#define B2E_UMMA_CUH
#include <cuda_runtime.h>
#include <stdint.h>

namespace b2e {
namespace umma {

#ifndef B2E_SPIN_LIMIT
#define B2E_SPIN_LIMIT (1u << 24)
#endif

/* error codes written to the kernel's status word */
enum : unsigned int { ST_OK = 0, ST_TIMEOUT_TMA = 1, ST_TIMEOUT_MMA = 2, ST_TIMEOUT_EPI = 4, ST_TIMEOUT_WEIGHTS = 8 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

/* Wait for the phase with the given parity to complete; false after `limit`
 * polls (the status word gets `code`). */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned int *status, unsigned int code,
                                          uint32_t limit = B2E_SPIN_LIMIT) {
  for (uint32_t i = 0; i < limit; i++) {
    if (mbar_try_wait(bar, parity))
      return true;
    if (status && (i & 1023u) == 1023u && *(volatile unsigned int *)status != ST_OK)
      return false; /* another role already gave up */
  }
  if (status)
    atomicOr(status, code);
  return false;
}

/* 3-D tiled TMA load (no multicast) into shared memory, completing on bar. */
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const void *tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

/* ---- TMEM ---- */
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* D[tmem] (+)= A[smem] x B[smem]^T, one instruction, issued by one thread. */
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

/* Arrive on bar once every previously issued MMA of this thread completes. */
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

/* 32 lanes x 32 bit, 16 consecutive columns: thread i of the warp gets lane
 * (base lane + i), columns [col, col+16). */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
               "%14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  for (int i = 0; i < 16; i++)
    v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

/* ---- descriptors ---- */

/* Shared-memory matrix descriptor, 128-byte swizzle (layout type 2), sm_100
 * descriptor version 1.  lbo/sbo in bytes. */
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46; /* version */
  d |= (uint64_t)2 << 61; /* SWIZZLE_128B */
  return d;
}

/* Instruction descriptor: BF16 A and B, FP32 accumulator, dense. a_mn / b_mn
 * select MN-major operands. */
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4)                       /* D format F32 */
         | (1u << 7)                     /* A BF16 */
         | (1u << 10)                    /* B BF16 */
         | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

} // namespace umma
} // namespace b2e
#endif
