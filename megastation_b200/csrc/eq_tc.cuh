// eq_tc.cuh -- tensor-core equalizer interface.
#pragma once
#include <cuda_bf16.h>

#include "sgemv.cuh"

namespace mb {

struct EqTcParams {
  EqParams p;                 // shapes, layout and epilogue outputs
  const uint8_t *a_img;       // per-group detector images (BF16)
  const __nv_bfloat16 *y_lp;  // [nb][re|im][M][S_pad]
  uint32_t S_pad, Mp, nkt, N, l0, tmem_cols;
  uint32_t spc, nb;           // symbols per CTA, symbols in the launch
  uint32_t y16;               // 1: 16-subcarrier y boxes, 32-byte swizzle (sg % 16 == 0)
  int *err;
};

struct TcShape {
  uint32_t MM;               // MMA rows: 64 (K <= 32) or 128 (K <= 64)
  uint32_t Mp;               // antennas padded to the 64-wide k tile
  uint32_t nkt;              // k tiles: 2 * Mp / 64
  uint64_t img_group_bytes;  // detector image bytes per group
};

TcShape tc_shape(uint32_t M, uint32_t K);
bool equalize_tc_supported(uint32_t K, uint32_t sg, uint32_t nb);
// W [G][M][K] c32 -> detector images
mb_status w_image(const float2 *W, void *img, uint32_t G, uint32_t M, uint32_t K,
                  cudaStream_t st);
// equalize nb symbols (outputs at symbol offset l0 of p's outputs); a CTA
// takes the symbols of one group that fit in max_cols (<= 128, 0: 128)
// (symbol, subcarrier) columns
mb_status equalize_tc(const EqParams &p, const void *a_img, const void *y_lp, uint32_t S_pad,
                      uint32_t l0, uint32_t nb, int *err, cudaStream_t st, uint32_t max_cols = 0);
// error word of mb_equalize_tc_noalloc's kernels on the current device
// (0 when it has not run there), cleared when clear is set
mb_status noalloc_error_word(int *bits, bool clear);
// y [nb][M][S] c32 -> y_lp [nb][re|im][M][S_pad] BF16
mb_status y_to_lp(const float2 *y, void *y_lp, uint32_t nb, uint32_t M, uint32_t S,
                  uint32_t S_pad, cudaStream_t st);

}  // namespace mb
