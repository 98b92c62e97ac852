// eq_common.cuh -- demap + LLR placement + descrambled hard bits for one
// equalized symbol, shared by the SIMT and tensor-core equalizers.  All
// index arithmetic is 32-bit (equalize_prepare checks the ranges) and the
// scrambler index advances incrementally, so the per-symbol cost is the
// demapper itself plus a handful of integer operations.
#pragma once
#include "demod.cuh"
#include "sgemv.cuh"

namespace mb {

// Stores the Qm LLRs lv of the subcarrier whose first stream bit is t0 in
// llr_row (the (symbol, user) row), by the placement of
// equalize_kernel.cuh:272-287: code block cb = t0 / cb_size, offset
// cb * cb_stride + zeros + t0 - cb * cb_size; blocks past cb_blocks and
// positions past the row are dropped.
__device__ __forceinline__ void eq_store_llr(const EqParams &p, __half *llr_row, uint32_t cb,
                                             uint32_t base, const __half *lv) {
  if (cb >= p.cb_blocks) return;
  const uint32_t Qm = p.Qm;
  __half *dst = llr_row + base;
  if (base + Qm <= p.row_len32 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
#pragma unroll
    for (int q = 0; q < 8; q += 2)
      if (q < (int)Qm) reinterpret_cast<__half2 *>(dst)[q / 2] = __halves2half2(lv[q], lv[q + 1]);
  } else {
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (q < (int)Qm && base + q < p.row_len32) dst[q] = lv[q];
  }
}

// the Qm hard decisions (llr < 0) of the subcarrier whose first stream bit
// is t0, first stream bit most significant; bits of stream positions >=
// n_valid are 0
__device__ __forceinline__ uint32_t eq_hard_bits(const EqParams &p, uint32_t t0, const __half *lv) {
  const __half zero = __float2half_rn(0.f);
  uint32_t hb = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    if (q >= (int)p.Qm) break;
    const uint32_t h = (t0 + q < p.n_valid32 && __hlt(lv[q], zero)) ? 1u : 0u;
    hb = (hb << 1) | h;
  }
  return hb;
}

// Demaps x of subcarrier s, stores its Qm LLRs in llr_row and returns the Qm
// hard decisions (0 without a hard-bit output).  Descrambling is applied per
// byte by the caller (eq_seq_byte).
__device__ __forceinline__ uint32_t eq_demap_store(const EqParams &p, __half *llr_row,
                                                   uint32_t s, float2 x) {
  __half lv[8];
  demod(p.Qm, x, lv);
  const uint32_t t0 = s * p.Qm;
  const uint32_t cb = t0 / p.cb_size32;
  eq_store_llr(p, llr_row, cb, cb * p.cb_stride32 + p.zeros32 + (t0 - cb * p.cb_size32), lv);
  return p.hard ? eq_hard_bits(p, t0, lv) : 0u;
}

// descrambling byte for output byte gb of user u's hard-bit row, with the
// bits past n_valid cleared so the row's padding stays zero
__device__ __forceinline__ uint8_t eq_seq_byte(const EqParams &p, uint32_t u, uint32_t gb) {
  if (!p.seqb) return 0;
  uint8_t v = __ldg(p.seqb + (uint64_t)u * p.seq_row_bytes + gb);
  const uint32_t end = p.n_valid32 - gb * 8;  // > 0 for every written byte
  if (end < 8) v &= (uint8_t)(0xFF00u >> end);
  return v;
}

}  // namespace mb
