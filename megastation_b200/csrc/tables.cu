// tables.cu -- status strings, per-device constant tables and host-side
// sequence generators of the C ABI.
#include <math.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "tc.cuh"
#include "eq_tc.cuh"

namespace mb {

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;

mb_status record_error(cudaError_t e) {
  g_last_cuda_error = e;
  return e == cudaErrorMemoryAllocation ? MB_NO_MEMORY : MB_CUDA_ERROR;
}

static std::mutex g_tables_mu;
static DeviceTables g_tables[64];
static bool g_tables_ready[64];

static mb_status build_tables(DeviceTables &t) {
  for (int l = 0; l < 14; l++) t.twiddle[l] = nullptr;
  t.lfsr127_bits = nullptr;
  for (int l = 4; l <= 13; l++) {
    // Stockham pass tables: pass p >= 1 (radix R, Ns = product of the
    // earlier radices) holds exp(-2 pi i r k / (Ns R)) at [r][k], so the
    // threads of a warp (consecutive k) read consecutive entries.
    std::vector<float2> h;
    uint32_t ns = 1;
    const int p16 = l / 4, rlast = 1 << (l % 4);
    const int passes = p16 + (rlast > 1 ? 1 : 0);
    for (int p = 0; p < passes; p++) {
      const uint32_t R = p < p16 ? 16 : rlast;
      if (p > 0)
        for (uint32_t r = 0; r < R; r++)
          for (uint32_t k = 0; k < ns; k++) {
            double a = -2.0 * M_PI * (double)(r * k) / (double)(ns * R);
            h.push_back(make_float2((float)cos(a), (float)sin(a)));
          }
      ns *= R;
    }
    if (h.empty()) h.push_back(make_float2(1.f, 0.f));
    MB_CUDA_TRY(cudaMalloc(&t.twiddle[l], sizeof(float2) * h.size()));
    MB_CUDA_TRY(cudaMemcpy(t.twiddle[l], h.data(), sizeof(float2) * h.size(),
                           cudaMemcpyHostToDevice));
  }
  // scrambler/scrambler.cu:22-31: x^7 + x^4 + 1 from 0x5D
  uint32_t words[4] = {0, 0, 0, 0};
  uint8_t s = 0x5D;
  for (int i = 0; i < 127; i++) {
    uint8_t fb = (s ^ (s >> 3)) & 1;
    words[i / 32] |= (uint32_t)fb << (i % 32);
    s >>= 1;
    s |= fb << 6;
  }
  MB_CUDA_TRY(cudaMalloc(&t.err, sizeof(int)));
  MB_CUDA_TRY(cudaMemset(t.err, 0, sizeof(int)));
  MB_CUDA_TRY(cudaMalloc(&t.lfsr127_bits, sizeof(words)));
  MB_CUDA_TRY(cudaMemcpy(t.lfsr127_bits, words, sizeof(words),
                         cudaMemcpyHostToDevice));
  return upload_mod_tables();
}

const DeviceTables *device_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_tables_mu);
  if (!g_tables_ready[dev]) {
    if (build_tables(g_tables[dev]) != MB_OK) return nullptr;
    g_tables_ready[dev] = true;
  }
  return &g_tables[dev];
}

// utils.h:54-75: Zadoff-Chu of the largest tabulated prime <= len (2039
// when len is larger or nothing matches), phase formed in double and
// rounded to float by sincosf's argument.
static void zadoff_chu(uint64_t seq_len, std::vector<float2> &out) {
  uint32_t len = 0;
  for (uint32_t p = 2; p <= 2039; p++) {
    bool prime = true;
    for (uint32_t d = 2; d * d <= p; d++)
      if (p % d == 0) { prime = false; break; }
    if (prime && p <= seq_len) len = p;
  }
  if (len == 0 || seq_len >= 2039) len = 2039;
  double root = floor(len * 2.0 / 31.0 + 0.5);
  out.resize(seq_len);
  for (uint64_t i = 0; i < seq_len; i++) {
    uint16_t m = (uint16_t)(i % len);
    float s, c;
    sincosf((float)(-M_PI * root * m * (m + 1) / len), &s, &c);
    out[i] = make_float2(c, s);
  }
}

// utils.h:77-95
static void cyclic_shift(std::vector<float2> &seq, const std::vector<float2> &in,
                         float alpha) {
  seq.resize(in.size());
  for (uint64_t i = 0; i < in.size(); i++) {
    float s, c;
    sincosf(alpha * (float)i, &s, &c);
    float2 v = in[i];
    seq[i] = make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

mb_status make_tmap_2d_bf16(CUtensorMap *map, const void *base, uint64_t width, uint64_t rows,
                            uint64_t pitch_elems, uint32_t box_x, uint32_t box_y, bool sw32) {
  static EncodeTiledFn fn = nullptr;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
      void *p = nullptr;
      cudaDriverEntryPointQueryResult q;
      MB_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
      if (q != cudaDriverEntryPointSuccess || !p) return MB_CUDA_ERROR;
      fn = reinterpret_cast<EncodeTiledFn>(p);
    }
  }
  if ((pitch_elems * 2) % 16 || (reinterpret_cast<uintptr_t>(base) % 16)) return MB_BAD_ARG;
  if (sw32 && box_x * 2 != 32) return MB_BAD_ARG;
  cuuint64_t dims[2] = {width, rows};
  cuuint64_t strides[1] = {pitch_elems * 2};
  cuuint32_t box[2] = {box_x, box_y};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  sw32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MB_OK : MB_BAD_ARG;
}

// Host: a 2-D byte tensor map over `rows` rows of `width` bytes (row pitch
// `pitch` bytes, a multiple of 16), box = 128 bytes by box_y rows, stored
// in shared memory with the 128-byte swizzle (16-byte chunk c of box row y
// at chunk c ^ (y % 8); boxes 1024-byte aligned).
mb_status make_tmap_2d_u8_sw128(CUtensorMap *map, const void *base, uint64_t width, uint64_t rows,
                                uint64_t pitch, uint32_t box_y) {
  static EncodeTiledFn fn = nullptr;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
      void *p = nullptr;
      cudaDriverEntryPointQueryResult q;
      MB_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
      if (q != cudaDriverEntryPointSuccess || !p) return MB_CUDA_ERROR;
      fn = reinterpret_cast<EncodeTiledFn>(p);
    }
  }
  if (pitch % 16 || (reinterpret_cast<uintptr_t>(base) % 16)) return MB_BAD_ARG;
  cuuint64_t dims[2] = {width, rows};
  cuuint64_t strides[1] = {pitch};
  cuuint32_t box[2] = {128, box_y};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MB_OK : MB_BAD_ARG;
}

// One warp waits on a shared-memory mbarrier of arrival count 1 through the
// same bounded wait as the tensor-core kernels.  With arm = 0 nothing ever
// arrives, so the wait runs out after limit_ns and the timeout bit lands in
// the device error word; with arm != 0 thread 0 arrives first and the wait
// completes at once.  Nothing else is in flight in the CTA, so giving up is
// a plain return.
__global__ void wait_selftest_kernel(uint64_t limit_ns, int arm, int *err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  __syncwarp();
  if (arm && threadIdx.x == 0) tc::mbar_arrive(&bar);
  __syncwarp();
  const bool ok = tc::mbar_wait(&bar, 0, limit_ns);
  if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicOr(err, tc::kErrTimeout);
}

}  // namespace mb

using namespace mb;

extern "C" mb_status mb_selftest_wait(uint64_t limit_ns, int arm, void *stream) {
  if (limit_ns == 0 || limit_ns > 1000000000ull) return MB_BAD_ARG;
  const DeviceTables *t = device_tables();
  if (!t) return MB_CUDA_ERROR;
  wait_selftest_kernel<<<1, 32, 0, as_stream(stream)>>>(limit_ns, arm, t->err);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" const char *mb_status_str(mb_status s) {
  switch (s) {
    case MB_OK: return "ok";
    case MB_BAD_SHAPE: return "bad shape";
    case MB_BAD_ARG: return "bad argument";
    case MB_NOT_PD: return "Gram matrix not positive definite";
    case MB_CUDA_ERROR: return cudaGetErrorString(g_last_cuda_error);
    case MB_TIMEOUT: return "device wait timed out";
    case MB_NO_MEMORY: return "out of device memory";
    case MB_UNSUPPORTED: return "unsupported";
    case MB_TOO_LARGE: return "request exceeds the fixed scratch of mb_equalize_tc_noalloc";
  }
  return "unknown status";
}

extern "C" const char *mb_version(void) { return "megastation_b200 0.1 sm_100a"; }

extern "C" mb_status mb_tables_init(int device) {
  int cur = 0;
  MB_CUDA_TRY(cudaGetDevice(&cur));
  if (device != cur) MB_CUDA_TRY(cudaSetDevice(device));
  const DeviceTables *t = device_tables();
  if (device != cur) MB_CUDA_TRY(cudaSetDevice(cur));
  return t ? MB_OK : MB_CUDA_ERROR;
}

extern "C" mb_status mb_device_error(int *out, int clear) {
  if (!out) return MB_BAD_ARG;
  const DeviceTables *t = device_tables();
  if (!t) return MB_CUDA_ERROR;
  MB_CUDA_TRY(cudaDeviceSynchronize());
  MB_CUDA_TRY(cudaMemcpy(out, t->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (clear) MB_CUDA_TRY(cudaMemset(t->err, 0, sizeof(int)));
  int na = 0;  // the fixed-scratch equalizer keeps its own word
  const mb_status s = noalloc_error_word(&na, clear != 0);
  if (s != MB_OK) return s;
  *out |= na;
  return MB_OK;
}

extern "C" mb_status mb_pilot_sign(uint64_t S, mb_c32 *out) {
  if (!out || S == 0) return MB_BAD_ARG;
  std::vector<float2> zc, sh;
  zadoff_chu(S, zc);
  cyclic_shift(sh, zc, (float)(M_PI / 4));
  for (uint64_t i = 0; i < S; i++) {
    float p2 = sh[i].x * sh[i].x + sh[i].y * sh[i].y;
    out[i].re = sh[i].x / p2;
    out[i].im = sh[i].y / p2;
  }
  return MB_OK;
}

extern "C" mb_status mb_dmrs_table(uint64_t S, uint64_t K, mb_c32 *out) {
  if (!out || S == 0) return MB_BAD_ARG;
  std::vector<float2> zc, sh;
  zadoff_chu(S, zc);
  for (uint64_t u = 0; u < K; u++) {
    cyclic_shift(sh, zc, (float)(u * M_PI / 6));
    for (uint64_t i = 0; i < S; i++) {
      out[u * S + i].re = sh[i].x;
      out[u * S + i].im = sh[i].y;
    }
  }
  return MB_OK;
}

extern "C" mb_status mb_ldpc_sizes(uint64_t S, uint32_t Qm, double rate,
                                   uint32_t bg, uint64_t pilot_spacing,
                                   int downlink, uint64_t *encoded,
                                   uint64_t *punctured, uint64_t *decoded) {
  if (!encoded || !punctured || !decoded || !(rate > 0) || (bg != 1 && bg != 2))
    return MB_BAD_ARG;
  static const uint64_t zc_set[] = {
      2,   4,   8,   16, 32, 64,  128, 256, 3,   6,   12,  24, 48,
      96,  192, 384, 5,  10, 20,  40,  80,  160, 320, 7,   14, 28,
      56,  112, 224, 9,  18, 36,  72,  144, 288, 11,  22,  44, 88,
      176, 352, 13,  26, 52, 104, 208, 15,  30,  60,  120, 240};
  std::vector<uint64_t> zc(zc_set, zc_set + sizeof(zc_set) / sizeof(zc_set[0]));
  std::sort(zc.begin(), zc.end());
  uint64_t kb = bg == 1 ? 22 : 10;
  uint64_t data = downlink && pilot_spacing ? S - S / pilot_spacing : S;
  uint64_t uncoded = (uint64_t)((double)(data * Qm) * rate);
  uint64_t z = zc.back();
  for (size_t i = 0; i + 1 < zc.size(); i++)
    if (kb * zc[i] <= uncoded && kb * zc[i + 1] > uncoded) {
      z = zc[i];
      break;
    }
  uint64_t rows = (uint64_t)llround(kb / rate) - (kb - 2);
  *encoded = (kb - 2 + rows) * z;
  *decoded = kb * z;
  *punctured = 2 * z;
  return MB_OK;
}
