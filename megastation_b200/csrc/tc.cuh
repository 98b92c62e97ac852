// tc.cuh -- sm_100a tensor-core plumbing: mbarriers with bounded waits,
// TMEM allocation, tcgen05.mma / commit / ld, and the shared-memory matrix
// and instruction descriptors (PTX ISA "tcgen05" matrix descriptor and
// instruction descriptor formats for kind::f16).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace mb {
namespace tc {

// error bits OR-ed into the device error word
enum : int { kErrTimeout = 1, kErrTmem = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait that may suspend the thread until the phase completes or
// hint_ns have passed, whichever comes first (fewer polling instructions
// for warps that wait long)
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t *bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Waits for completion of the phase with the given parity; gives up after
// limit_ns of wall time and returns false (the caller records an error).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          uint64_t limit_ns = 1000000000ull) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer() - t0 > limit_ns) return false;
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// whole warp: allocate ncols TMEM columns (power of two >= 32); the address
// is written to *slot in shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// D[tmem] (+)= A[smem desc] * B[smem desc], kind::f16 (BF16/FP16 in, FP32 acc)
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the mbarrier arrives once every tcgen05.mma issued so far by this thread
// has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp-collective)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive fp32 columns at each of two TMEM addresses of this thread's
// lane, one wait for both (warp-collective)
__device__ __forceinline__ void tmem_ld8x2(uint32_t ta, float *va, uint32_t tb, float *vb) {
  uint32_t a[8], b[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7])
               : "r"(ta));
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7])
               : "r"(tb));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}

// Shared-memory matrix descriptor, no swizzle ("interleave") canonical
// layouts built from 8x16-byte core matrices:
//   K-major : core matrix = 8 rows x 8 K-elements; lbo = byte step between
//             the two K core matrices of one MMA, sbo = byte step between
//             8-row groups along M/N.
//   MN-major: core matrix = 8 K-rows x 8 MN-elements; lbo = byte step
//             between 8-row K groups, sbo = byte step between 8-element
//             MN chunks.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// Shared-memory matrix descriptor of an MN-major operand in the 32-byte
// swizzle canonical layout: atoms of 16 MN elements (32 bytes) by 8 K rows
// (256 bytes, as a 32-byte-swizzled TMA box row group stores them: the two
// 16-byte halves of rows 4-7 swapped); lbo = byte step between atoms along
// MN, sbo = byte step between 8-row K groups; start 256-byte aligned.
__device__ __forceinline__ uint64_t smem_desc_mn_sw32(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return smem_desc(saddr, lbo, sbo) | ((uint64_t)6 << 61);  // layout type 6: 32-byte swizzle
}

// Instruction descriptor, kind::f16: FP32 accumulate, BF16 A and B.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, bool a_mn_major,
                                                  bool b_mn_major) {
  return (1u << 4)                          // D format F32
         | (1u << 7)                        // A format BF16
         | (1u << 10)                       // B format BF16
         | ((a_mn_major ? 1u : 0u) << 15)   // A major
         | ((b_mn_major ? 1u : 0u) << 16)   // B major
         | ((N >> 3) << 17)                 // N / 8
         | ((M >> 4) << 24);                // M / 16
}

// Instruction descriptor, kind::f16: FP32 accumulate, FP16 A and B.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t M, uint32_t N, bool a_mn_major,
                                                 bool b_mn_major) {
  return (1u << 4)                          // D format F32; A, B format F16 (0)
         | ((a_mn_major ? 1u : 0u) << 15)   // A major
         | ((b_mn_major ? 1u : 0u) << 16)   // B major
         | ((N >> 3) << 17)                 // N / 8
         | ((M >> 4) << 24);                // M / 16
}

}  // namespace tc
}  // namespace mb

#include <cuda.h>

namespace mb {
namespace tc {

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared, completion counted on the mbarrier
// (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 2-D tiled tensor copy global -> shared (box from the tensor map) into
// this CTA's own shared memory; x must be a multiple of 16 bytes / element size
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int32_t x, int32_t y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tc

// Host: a 2-D BF16 tensor map over rows of `pitch_elems` elements (row pitch
// a multiple of 16 bytes), box = box_x elements by box_y rows; no swizzle,
// or with sw32 (box_x = 16) the 32-byte swizzle: box row y's two 16-byte
// halves swap places when y % 8 >= 4 (boxes 256-byte aligned).
mb_status make_tmap_2d_bf16(CUtensorMap *map, const void *base, uint64_t width, uint64_t rows,
                            uint64_t pitch_elems, uint32_t box_x, uint32_t box_y, bool sw32 = false);
// Host: a 2-D byte tensor map, 128-byte boxes of box_y rows, 128-byte
// swizzle in shared memory.
mb_status make_tmap_2d_u8_sw128(CUtensorMap *map, const void *base, uint64_t width, uint64_t rows,
                                uint64_t pitch, uint32_t box_y);

}  // namespace mb
