// fft.cuh -- internal FFT launchers.
#pragma once
#include "common.cuh"

namespace mb {

// uplink FFT writing planar BF16 rows [n_sym][re|im][M][S_pad] for the
// tensor-core equalizer
mb_status fft_uplink_lp(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                        void *y_lp, uint32_t S_pad, cudaStream_t st);

// pilot FFT of n_sym comb-pilot symbols (ue_start 0) that also fills the
// short last group's users without a pilot from group G-2 (zf_fill_tail)
mb_status fft_pilot_fill(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym, mb_c32 *csi,
                         cudaStream_t st);

}  // namespace mb
