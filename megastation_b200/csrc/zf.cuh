// zf.cuh -- internal launchers of the zero-forcing kernels.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"
#include "sgemv.cuh"

namespace mb {

// copies users without a pilot in a short last group from group G-2
mb_status zf_fill_tail(float2 *csi, uint32_t groups, uint32_t S, uint32_t sg,
                       uint32_t M, uint32_t K, cudaStream_t st);
// Cholesky ZF in FP32 or FP64, W in place; optional fused precoder
mb_status zf_chol(float2 *csi, float2 *precoder, uint32_t groups, uint32_t M,
                  uint32_t K, bool dbl, int32_t *status, float *cond,
                  cudaStream_t st);
// mixed precision ZF (zf_mixed.cu): the detector images for the
// tensor-core equalizer in img_w (zf_mixed_scratch_bytes) and, with write_w,
// W in place (FP32) and its per-group max |W| in wmax (if not null);
// without write_w csi is left as scratch
uint64_t zf_mixed_scratch_bytes(uint32_t groups, uint32_t M, uint32_t K);

// Device view of the network of the learned polynomial initial iterate
// (an mb_mlp with kZfInitFeatures inputs and kZfInitCoeffs outputs): BF16
// weights W1 [n_in][width], W2 [width][width], W3 [width][n_out] and FP32
// biases, all device memory owned by the mb_mlp.
constexpr uint32_t kZfInitFeatures = 6, kZfInitCoeffs = 4, kZfInitMaxWidth = 256;
struct ZfNetView {
  const __nv_bfloat16 *w1, *w2, *w3;
  const float *b1, *b2, *b3;
  uint32_t width;
};
// fills v from an mb_mlp of the right shape (MB_BAD_SHAPE otherwise)
mb_status mlp_zf_init_view(const mb_mlp *n, ZfNetView *v);

// net (nullable) is used when opts->init == 1.  path: where the inverse's
// matrix products run for K <= 32 -- 0 the tensor cores for 16 < K and the
// CUDA cores below, 1 the CUDA cores, 2 the tensor cores
mb_status zf_mixed_run(float2 *csi, void *img_w, uint32_t groups, uint32_t M, uint32_t K,
                       const mb_zf_opts *opts, int32_t *status, float *cond, cudaStream_t st,
                       bool write_w = true, float *wmax = nullptr, const ZfNetView *net = nullptr,
                       uint32_t path = 0);
// the same ZF fused with the tensor-core equalizer: each CTA keeps its
// group's detector image in shared memory and equalizes the group's
// columns of nb symbols of planar BF16 samples y_lp [nb][re|im][M][S_pad]
// into p's outputs (symbols 0..nb-1); MB_UNSUPPORTED when the shapes do
// not allow it (K > 32, M > 256, sg % 16, more than one 128-column tile
// per group, i.e. nb sg > 128), the caller then runs zf_mixed_run and
// equalize_tc
mb_status zf_mixed_eq_run(float2 *csi, uint32_t groups, uint32_t M, uint32_t K, const mb_zf_opts *opts,
                          int32_t *status, float *cond, cudaStream_t st, bool write_w, float *wmax,
                          const ZfNetView *net, const EqParams &p, const void *y_lp, uint32_t S_pad,
                          uint32_t nb, uint32_t path = 0);
// precoder P[g][u][b] = W[g][b][u] / wmax[g] from a precomputed per-group max
mb_status precoder_scale(const float2 *W, float2 *P, const float *wmax, uint32_t M, uint32_t K,
                         uint32_t groups, cudaStream_t st);
mb_status precoder_launch(const float2 *W, float2 *P, uint32_t M, uint32_t K,
                          uint32_t groups, cudaStream_t st);
size_t zf_chol_smem(uint32_t M, uint32_t K, bool dbl);

}  // namespace mb
