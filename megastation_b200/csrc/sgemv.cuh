// sgemv.cuh -- internal parameters of the equalize / precode kernels.
#pragma once
#include <vector>

#include "common.cuh"

namespace mb {

struct EqParams {
  const float2 *W;   // [G][M][K]
  const float2 *y;   // [n_sym][M][S]
  uint16_t *llr;     // [n_sym][K][row_len] fp16 bits
  uint8_t *hard;     // [n_sym][K][hrow] or null
  float2 *x;         // [n_sym][K][S] equalized symbols or null
  const uint8_t *seqb;     // descrambling sequence, MSB-first bytes, or null
  uint64_t seq_row_bytes;  // byte stride between users' sequences (0: shared)
  uint32_t K, M, S, sg, n_sym, Qm;
  uint64_t cb_size, cb_stride, zeros;
  uint32_t cb_blocks;
  uint64_t row_len, n_valid, hrow;
  uint32_t hw_words;  // 32-bit words of hard bits per (symbol, user) in a group
  uint32_t L;         // symbols per CTA
  // 32-bit copies for the epilogue (ranges checked by equalize_prepare)
  uint32_t cb_size32, cb_stride32, zeros32, row_len32, n_valid32;
};

const uint8_t *scrambler_bytes(const mb_scrambler *s, uint64_t *nbits,
                               uint64_t *row_bytes);
mb_status equalize_prepare(EqParams &p, const mb_c32 *W, const mb_c32 *y,
                           uint32_t K, uint32_t M, uint32_t S, uint32_t sg,
                           uint32_t n_sym, uint32_t Qm, uint64_t cb_size,
                           uint64_t cb_stride, uint64_t zeros,
                           uint32_t cb_blocks, uint16_t *llr, uint8_t *hard,
                           const mb_scrambler *scr);
mb_status equalize_fp32(EqParams p, cudaStream_t st);
mb_status precode_fp32(const float2 *P, const float2 *s, float2 *out,
                       uint32_t M, uint32_t K, uint32_t S, uint32_t sg,
                       uint32_t N, uint32_t start, uint32_t n_sym,
                       cudaStream_t st);

}  // namespace mb
