// noalloc.cu -- the tensor-core equalize entry point for callers that must
// not allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they equalize: a
// real-time fronthaul thread that may not block on the driver's allocator,
// a process whose device memory is carved up and fixed at start-up, or an
// embedding framework that owns every allocation itself.  mb_equalize_tc
// asks such callers for two scratch buffers; this variant instead keeps its
// scratch (the BF16 detector images and the BF16 copy of the FFT output) in
// one fixed array compiled into the library, so a call needs nothing but
// its inputs and outputs.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "eq_tc.cuh"

namespace {

// Fixed scratch shared by every call on a device.  Each device that loads
// the library holds these bytes until the process exits.
constexpr uint64_t kNoAllocScratchBytes = 32ull << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];
// The error word of this entry point's kernels (bit 1: a bounded mbarrier
// wait gave up), kept beside the scratch because the library's own error
// word is allocated on first use.  mb_device_error reports and clears it
// together with that word.
static __device__ int g_noalloc_err;

// Device addresses of g_noalloc_scratch and g_noalloc_err per device, looked
// up once per device with that device current.  In host code the arrays'
// names are only handles for the runtime, not device addresses.  The cached
// addresses belong to the device's current context: after cudaDeviceReset
// they are stale, and this entry point must not be called again in that
// process (as with every other per-device table of the library).
std::mutex g_noalloc_mu;
void *g_noalloc_addr[64];
int *g_noalloc_err_addr[64];

}  // namespace

using namespace mb;

// Reads (and optionally clears) this entry point's error word on the current
// device; 0 when the entry point has not run there.
mb_status mb::noalloc_error_word(int *bits, bool clear) {
  *bits = 0;
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return MB_OK;
  int *addr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    addr = g_noalloc_err_addr[dev];
  }
  if (!addr) return MB_OK;
  MB_CUDA_TRY(cudaMemcpy(bits, addr, sizeof(int), cudaMemcpyDeviceToHost));
  if (clear) MB_CUDA_TRY(cudaMemset(addr, 0, sizeof(int)));
  return MB_OK;
}

extern "C" mb_status mb_equalize_tc_noalloc(const mb_c32 *W, const mb_c32 *y, uint32_t K,
                                            uint32_t M, uint32_t S, uint32_t sg,
                                            uint32_t n_sym, uint32_t Qm, uint64_t cb_size,
                                            uint64_t cb_stride, uint64_t zeros,
                                            uint32_t cb_blocks, uint16_t *llr, uint8_t *hard,
                                            const mb_scrambler *scr, mb_c32 *x, void *stream) {
  EqParams p;
  mb_status s = equalize_prepare(p, W, y, K, M, S, sg, n_sym, Qm, cb_size, cb_stride, zeros,
                                 cb_blocks, llr, hard, scr);
  if (s != MB_OK) return s;
  p.x = reinterpret_cast<float2 *>(x);
  if (n_sym == 0) return MB_OK;
  if (!equalize_tc_supported(K, sg, 1)) return MB_UNSUPPORTED;

  // scratch layout: detector images, then as many symbols of BF16 rows as fit
  const TcShape sh = tc_shape(M, K);
  const uint32_t G = (S + sg - 1) / sg;
  const uint32_t S_pad = (S + 7) / 8 * 8;
  const uint64_t img_bytes = ((uint64_t)G * sh.img_group_bytes + 255) / 256 * 256;
  const uint64_t sym_bytes = (uint64_t)2 * M * S_pad * 2;
  if (img_bytes + sym_bytes > kNoAllocScratchBytes) return MB_TOO_LARGE;
  const uint32_t sym_fit = (uint32_t)std::min<uint64_t>((kNoAllocScratchBytes - img_bytes) / sym_bytes, 1u << 20);

  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return MB_UNSUPPORTED;
  uint8_t *base = nullptr;
  int *err = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void *addr = nullptr, *eaddr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&eaddr, g_noalloc_err);
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return record_error(e);
      }
      g_noalloc_err_addr[dev] = reinterpret_cast<int *>(eaddr);
      g_noalloc_addr[dev] = addr;
    }
    base = reinterpret_cast<uint8_t *>(g_noalloc_addr[dev]);
    err = g_noalloc_err_addr[dev];
  }
  uint8_t *img = base;
  uint8_t *ylp = base + img_bytes;

  cudaStream_t st = as_stream(stream);
  s = w_image(reinterpret_cast<const float2 *>(W), img, G, M, K, st);
  if (s != MB_OK) return s;
  uint32_t nb_max = std::max<uint32_t>(1, 256 / sg);
  while (nb_max > 1 && !equalize_tc_supported(K, sg, nb_max)) nb_max--;
  for (uint32_t c0 = 0; c0 < n_sym; c0 += sym_fit) {
    const uint32_t nc = std::min(sym_fit, n_sym - c0);
    s = y_to_lp(reinterpret_cast<const float2 *>(y) + (uint64_t)c0 * M * S, ylp, nc, M, S, S_pad,
                st);
    if (s != MB_OK) return s;
    for (uint32_t j = 0; j < nc;) {
      uint32_t nb = std::min(nb_max, nc - j);
      while (nb > 1 && !equalize_tc_supported(K, sg, nb)) nb--;
      s = equalize_tc(p, img, ylp + (uint64_t)j * sym_bytes, S_pad, c0 + j, nb, err, st);
      if (s != MB_OK) return s;
      j += nb;
    }
  }
  return MB_OK;
}
