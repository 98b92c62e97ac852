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

}  // namespace mb
