// precode_tc.cuh -- tensor-core precoder interface (precode_tc.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace mb {

struct PcShape {
  uint32_t Kp;               // users padded to 32 (reduction 2 Kp, whole 64-wide k tiles)
  uint32_t H;                // halves of up to 128 antennas
  uint32_t nkt;              // k tiles: 2 Kp / 64
  uint64_t img_group_bytes;  // precoder image bytes per group
};

PcShape precode_tc_shape(uint32_t M, uint32_t K);
bool precode_tc_supported(uint32_t K, uint32_t sg);
// P [G][K][M] c32 (the scaled precoder) -> precoder images (BF16)
mb_status precoder_image(const float2 *P, void *img, uint32_t G, uint32_t M, uint32_t K, cudaStream_t st);
// z [D][M][N] FP16 (re, im) pairs at the data bins (s + start + N/2) mod N
// from the user symbols sym [D][K][S]; the other bins are left untouched
mb_status precode_tc(const void *img, const float2 *sym, void *z, uint32_t M, uint32_t K, uint32_t S, uint32_t sg,
                     uint32_t N, uint32_t start, uint32_t D, int *err, cudaStream_t st);

}  // namespace mb
