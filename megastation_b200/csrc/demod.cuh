// demod.cuh -- the reference soft demapper in FP16.
#pragma once
#include <cuda_fp16.h>

namespace mb {

// ---- soft demapper: demodulation.h:30-67, same operations in FP16 --------
__device__ __forceinline__ void demod(uint32_t Qm, float2 c, __half *l) {
  switch (Qm) {
    case 2:
      l[0] = __float2half_rn(c.x * -20.0f * sqrtf(2.f));
      l[1] = __float2half_rn(c.y * -20.0f * sqrtf(2.f));
      break;
    case 4: {
      const __half t = __float2half_rn(2 * 100 / sqrtf(10.f));
      l[0] = __float2half_rn(100 * c.x);
      l[1] = __float2half_rn(100 * c.y);
      l[2] = __hsub(t, __habs(l[0]));
      l[3] = __hsub(t, __habs(l[1]));
      break;
    }
    case 6: {
      const __half t1 = __float2half_rn(4 * 100 / sqrtf(42.f));
      const __half t2 = __float2half_rn(2 * 100 / sqrtf(42.f));
      l[0] = __float2half_rn(100 * c.x);
      l[1] = __float2half_rn(100 * c.y);
      l[2] = __hsub(t1, __habs(l[0]));
      l[3] = __hsub(t1, __habs(l[1]));
      l[4] = __hsub(t2, __habs(l[2]));
      l[5] = __hsub(t2, __habs(l[3]));
      break;
    }
    default: {
      const __half t1 = __float2half_rn(8 * 100 / sqrtf(170.f));
      const __half t2 = __float2half_rn(4 * 100 / sqrtf(170.f));
      const __half t3 = __float2half_rn(2 * 100 / sqrtf(170.f));
      l[0] = __float2half_rn(100 * c.x);
      l[1] = __float2half_rn(100 * c.y);
      l[2] = __hsub(t1, __habs(l[0]));
      l[3] = __hsub(t1, __habs(l[1]));
      l[4] = __hsub(t2, __habs(l[2]));
      l[5] = __hsub(t2, __habs(l[3]));
      l[6] = __hsub(t3, __habs(l[4]));
      l[7] = __hsub(t3, __habs(l[5]));
      break;
    }
  }
}

// demod() for a compile-time Qm on (Re, Im) pairs: lv[i] holds (l[2i],
// l[2i + 1]).  Each lane takes exactly the scalar form's operations (the
// same FP32 products rounded once to FP16, then FP16 subtractions of
// absolute values), so the LLRs are bit-identical to demod()'s.
template <int QM>
__device__ __forceinline__ void demod2(float2 c, __half2 (&lv)[QM / 2]) {
  if constexpr (QM == 2) {
    lv[0] = __floats2half2_rn(c.x * -20.0f * sqrtf(2.f), c.y * -20.0f * sqrtf(2.f));
  } else {
    lv[0] = __floats2half2_rn(100 * c.x, 100 * c.y);
    // thresholds 2^(QM/2 - i) * 100 / sqrt(norm), as in the scalar form
    const float d = QM == 4 ? sqrtf(10.f) : QM == 6 ? sqrtf(42.f) : sqrtf(170.f);
#pragma unroll
    for (int i = 1; i < QM / 2; i++) {
      const __half t = __float2half_rn((1 << (QM / 2 - i)) * 100 / d);
      lv[i] = __hsub2(__half2half2(t), __habs2(lv[i - 1]));
    }
  }
}

// The Qm hard decisions (l < 0, as __hlt(l, 0) gives them: false for -0
// and NaN) of demod2's output, l[0] the most significant bit.
template <int QM>
__device__ __forceinline__ uint32_t hard2(const __half2 (&lv)[QM / 2]) {
  const __half2 z = __float2half2_rn(0.f);
  uint32_t hb = 0;
#pragma unroll
  for (int i = 0; i < QM / 2; i++) {
    const uint32_t m = __hlt2_mask(lv[i], z);  // low 16 bits: l[2i] < 0, high 16 bits: l[2i + 1] < 0
    hb = (hb << 2) | (m & 2u) | (m >> 31);
  }
  return hb;
}

}  // namespace mb
