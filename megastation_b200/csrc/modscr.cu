// modscr.cu -- QAM modulation with DM-RS insertion and byte scrambling.
#include <algorithm>
#include <math.h>

#include "common.cuh"

namespace mb {

// modulation/modulation.cu:22-72: Gray maps, first stream bit = index MSB
__constant__ float2 c_mod_table[4][256];  // Qm = 2, 4, 6, 8

static void host_mod_table(int Qm, float2 *t) {
  if (Qm == 2) {
    float s = (float)(1 / sqrt(2.0));
    float v[2] = {-s, s};
    for (int i = 0; i < 4; i++) t[i] = make_float2(v[i / 2], v[i % 2]);
  } else if (Qm == 4) {
    float s = (float)(1 / sqrt(10.0));
    float v[4] = {1 * s, 3 * s, -1 * s, -3 * s};
    for (int i = 0; i < 16; i++) {
      int im = (((i >> 2) & 1) << 1) + (i & 1);
      int re = (((i >> 3) & 1) << 1) + ((i >> 1) & 1);
      t[i] = make_float2(v[re], v[im]);
    }
  } else if (Qm == 6) {
    float s = (float)(1 / sqrt(42.0));
    float v[8] = {3 * s, 1 * s, 5 * s, 7 * s, -3 * s, -1 * s, -5 * s, -7 * s};
    for (int i = 0; i < 64; i++) {
      int im = (((i >> 4) & 1) << 2) + (((i >> 2) & 1) << 1) + (i & 1);
      int re = (((i >> 5) & 1) << 2) + (((i >> 3) & 1) << 1) + ((i >> 1) & 1);
      t[i] = make_float2(v[re], v[im]);
    }
  } else {
    float s = (float)(1 / sqrt(170.0));
    float v[16] = {-15 * s, -13 * s, -9 * s, -11 * s, -1 * s, -3 * s,
                   -7 * s,  -5 * s,  15 * s, 13 * s,  9 * s,  11 * s,
                   1 * s,   3 * s,   7 * s,  5 * s};
    for (int i = 0; i < 256; i++) {
      int im = ((i & 0x40) >> 3) + ((i & 0x10) >> 2) + ((i & 0x4) >> 1) + (i & 0x1);
      int re = ((i & 0x80) >> 4) + ((i & 0x20) >> 3) + ((i & 0x8) >> 2) + ((i & 0x2) >> 1);
      t[i] = make_float2(v[re], v[im]);
    }
  }
}

// Uploads the QAM maps to the current device.  Called once per device by
// device_tables() under its lock, so concurrent first calls of mb_modulate
// cannot race on the upload.
mb_status upload_mod_tables() {
  float2 h[4][256];
  for (int q = 0; q < 4; q++) host_mod_table(2 * (q + 1), h[q]);
  MB_CUDA_TRY(cudaMemcpyToSymbol(c_mod_table, h, sizeof(h)));
  return MB_OK;
}

// modulation_kernel.cuh:37-68
__global__ void modulate_kernel(const uint8_t *in, float2 *out,
                                uint64_t in_bytes, uint64_t num_carriers,
                                uint64_t num_ues, uint32_t Qm,
                                uint32_t pilot_spacing, const float2 *pilots) {
  const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t u = blockIdx.y;
  if (c >= num_carriers || u >= num_ues) return;
  if (pilot_spacing && (c % pilot_spacing) == 0) {
    out[u * num_carriers + c] = pilots ? pilots[u * num_carriers + c] : make_float2(0.f, 0.f);
    return;
  }
  const uint64_t shrink = pilot_spacing ? c - ((c / pilot_spacing) + 1) : c;
  const uint8_t *src = in + u * in_bytes;
  uint32_t mb = 0;
  uint64_t idx = shrink * Qm;
  for (uint32_t i = 0; i < Qm && (idx / 8) < in_bytes; i++, idx++)
    mb = ((src[idx / 8] >> (idx % 8)) & 1u) | (mb << 1);
  out[u * num_carriers + c] = c_mod_table[Qm / 2 - 1][mb & ((1u << Qm) - 1)];
}

// scrambler_kernel.cuh:36-56, 16 bytes per thread
__global__ void scramble_kernel(uint8_t *out, const uint8_t *in,
                                uint64_t num_bytes, uint64_t batch,
                                const uint32_t *seq_words) {
  __shared__ uint8_t seq[127];
  if (threadIdx.x < 127) seq[threadIdx.x] = (seq_words[threadIdx.x / 32] >> (threadIdx.x % 32)) & 1u;
  __syncthreads();
  const uint64_t total = num_bytes * batch;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = e % num_bytes;
    uint32_t idx = (uint32_t)((j * 8) % 127);
    uint8_t sb = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      sb = (uint8_t)((sb << 1) | seq[idx]);
      idx = idx == 126 ? 0 : idx + 1;
    }
    out[e] = sb ^ in[e];
  }
}

}  // namespace mb

using namespace mb;

extern "C" mb_status mb_modulate(const uint8_t *in, mb_c32 *out,
                                 uint64_t in_bytes, uint64_t num_carriers,
                                 uint64_t num_ues, uint32_t Qm,
                                 uint32_t pilot_spacing,
                                 const mb_c32 *pilot_table, void *stream) {
  if (!in || !out) return MB_BAD_ARG;
  if (Qm != 2 && Qm != 4 && Qm != 6 && Qm != 8) return MB_BAD_ARG;
  if (pilot_spacing && !pilot_table) return MB_BAD_ARG;
  if (num_ues > 65535) return MB_BAD_SHAPE;
  if (num_carriers == 0 || num_ues == 0) return MB_OK;
  if (!device_tables()) return MB_CUDA_ERROR;  // the QAM maps are uploaded with the tables
  dim3 grid((unsigned)((num_carriers + 255) / 256), (unsigned)num_ues);
  modulate_kernel<<<grid, 256, 0, as_stream(stream)>>>(
      in, reinterpret_cast<float2 *>(out), in_bytes, num_carriers, num_ues, Qm,
      pilot_spacing, reinterpret_cast<const float2 *>(pilot_table));
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" mb_status mb_scramble(uint8_t *out, const uint8_t *in,
                                 uint64_t num_bytes, uint64_t batch,
                                 void *stream) {
  if (!out || !in) return MB_BAD_ARG;
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  uint64_t total = num_bytes * batch;
  if (total == 0) return MB_OK;
  unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148 * 16);
  scramble_kernel<<<blocks, 256, 0, as_stream(stream)>>>(out, in, num_bytes, batch,
                                                         tab->lfsr127_bits);
  MB_LAUNCH_CHECK();
  return MB_OK;
}
