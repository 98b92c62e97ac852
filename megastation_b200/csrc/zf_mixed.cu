// zf_mixed.cu -- mixed-precision zero forcing (BF16 Gram on tensor cores,
// FP32 inverse with Newton-Schulz refinement, FP64 fallback).
#include "zf.cuh"

namespace mb {

mb_status zf_mixed(float2 *csi, float2 *precoder, uint32_t groups, uint32_t M,
                   uint32_t K, const mb_zf_opts *opts, int32_t *status,
                   float *cond, cudaStream_t st) {
  (void)csi; (void)precoder; (void)groups; (void)M; (void)K; (void)opts;
  (void)status; (void)cond; (void)st;
  return MB_UNSUPPORTED;
}

}  // namespace mb
