// common.cuh -- shared device/host helpers of the sm_100a baseband library.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/megastation_b200.h"

namespace mb {

// On failure the runtime's sticky "last error" is cleared as well, so that a
// failed API call is reported once and not again by a later launch check.
#define MB_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) {                                \
      (void)cudaGetLastError();                             \
      return ::mb::record_error(_e);                        \
    }                                                       \
  } while (0)

#define MB_LAUNCH_CHECK() MB_CUDA_TRY(cudaGetLastError())

mb_status record_error(cudaError_t e);

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) {
  return make_float2(a.x, -a.y);
}
// acc += a * b
__device__ __forceinline__ void cfma(float2 &acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool is_pow2(uint64_t x) { return x && !(x & (x - 1)); }

inline int ilog2(uint64_t x) {
  int l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

// Per-device table registry (twiddles, scrambler bits).
struct DeviceTables {
  // Stockham twiddle tables per N = 2^l, l in [4, 13]: for each pass p >= 1
  // (radix R, Ns = product of earlier radices) the R x Ns block
  // exp(-2 pi i r k / (Ns R)) at [r][k], blocks concatenated by pass
  float2 *twiddle[14];
  uint32_t *lfsr127_bits;  // 127 bits packed LSB-first in 4 words
  int *err;                // device error word (mb_tc error bits)
};
// for the current device, built once per device under a lock (the QAM maps
// of the modulator are uploaded then too); nullptr on error
const DeviceTables *device_tables();
mb_status upload_mod_tables();  // modscr.cu: QAM maps to the current device

}  // namespace mb
