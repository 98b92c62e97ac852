// fft.cuh -- internal FFT launchers.
#pragma once
#include "common.cuh"

namespace mb {

// uplink FFT writing planar BF16 rows [n_sym][re|im][M][S_pad] for the
// tensor-core equalizer
// max_ctas: CTAs of the tensor-core FFT launch (N = 4096), 0 for one per SM
mb_status fft_uplink_lp(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                        void *y_lp, uint32_t S_pad, cudaStream_t st, uint32_t max_ctas = 0);

// pilot FFT of n_sym comb-pilot symbols (ue_start 0) that also fills the
// short last group's users without a pilot from group G-2 (zf_fill_tail);
// tensor: the FP16 tensor-core FFT where it applies (mixed precision)
mb_status fft_pilot_fill(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym, mb_c32 *csi,
                         cudaStream_t st, bool tensor = false);

// the slot's P pilot symbols and first U uplink symbols (adjacent rows of
// iq) in one tensor-core launch: CSI with the tail fill, and planar BF16
// rows; fft_slot_tc_ok tells whether it applies (N = 4096, alignment)
bool fft_slot_tc_ok(mb_fft *f, const void *iq, uint32_t S_pad, const void *y_lp);
mb_status fft_slot_tc(mb_fft *f, const void *iq, int iq_dtype, uint32_t P, uint32_t U, mb_c32 *csi, void *y_lp,
                      uint32_t S_pad, cudaStream_t st, uint32_t max_ctas = 0);

// tensor-core FFT for N = 4096 (fft_tc.cu): a plan holds the DFT operands
// with the FFT shift of `start` folded in; null for other N
struct FftTcPlan;
FftTcPlan *fft_tc_plan_create(uint32_t N, uint32_t start);
void fft_tc_plan_destroy(FftTcPlan *plan);
bool fft_tc_lp_supported(const FftTcPlan *plan, const void *iq, uint32_t S_pad, const void *y_lp);
// rows = n_sym * M rows of 4096 samples -> planar BF16 rows as fft_uplink_lp;
// upc: units of two rows per CTA (0: default)
mb_status fft_tc_uplink_lp(const FftTcPlan *plan, const void *iq, int iq_dtype, uint32_t rows, uint32_t M,
                           uint32_t S, void *y_lp, uint32_t S_pad, int *err, cudaStream_t st,
                           uint32_t upc = 0);
// pilot FFT of n_sym comb-pilot symbols into csi [G][M][K] as mb_fft_pilot,
// with the short-last-group fill when tail_rem != 0 (fft_pilot_fill)
bool fft_tc_pilot_supported(const FftTcPlan *plan, const void *iq);
mb_status fft_tc_pilot(const FftTcPlan *plan, const void *iq, int iq_dtype, uint32_t n_sym, uint32_t M, uint32_t S,
                       uint32_t K, uint32_t sg, uint32_t ue_start, uint32_t tail_rem, const float2 *pilot,
                       float2 *csi, int *err, cudaStream_t st, uint32_t upc = 0);
// one launch for a slot's P comb-pilot symbols (CSI out, tail fill with
// tail_rem) followed by U uplink symbols (planar BF16 rows out)
mb_status fft_tc_slot(const FftTcPlan *plan, const void *iq, int iq_dtype, uint32_t P, uint32_t U, uint32_t M,
                      uint32_t S, uint32_t K, uint32_t sg, uint32_t tail_rem, const float2 *pilot, float2 *csi,
                      void *y_lp, uint32_t S_pad, int *err, cudaStream_t st, uint32_t upc = 0);
// units of two rows per CTA that spread `rows` over at most max_ctas CTAs
// (0 when max_ctas is 0: the launcher's one CTA per SM)
inline uint32_t fft_tc_upc(uint64_t rows, uint32_t max_ctas) {
  if (!max_ctas) return 0;
  const uint64_t units = (rows + 1) / 2;
  return (uint32_t)((units + max_ctas - 1) / max_ctas);
}

// inverse FFT on the tensor cores (N = 4096): rows of N spectrum samples
// (c32 or FP16 pairs) -> int16 / int8 quantised or FP16 time samples as
// mb_ifft_downlink (FP16 operands, FP32 accumulation)
bool fft_tc_inverse_supported(const FftTcPlan *plan, const void *in, int in_dtype, const void *out, int out_dtype);
mb_status fft_tc_inverse(const FftTcPlan *plan, const void *in, int in_dtype, uint32_t rows, void *out,
                         int out_dtype, int *err, cudaStream_t st);
// the same through an FFT handle: true when the handle's tensor-core plan
// takes these buffers
bool fft_ifft_tc_ok(mb_fft *f, const void *in, int in_dtype, const void *out, int out_dtype);
// n_sym symbols of FP16 spectra [n_sym][M][N] through the handle's
// tensor-core inverse FFT (fft_ifft_tc_ok must hold)
mb_status fft_tc_inverse_slot(mb_fft *f, const void *in, uint32_t n_sym, void *out, int out_dtype, cudaStream_t st);

}  // namespace mb
