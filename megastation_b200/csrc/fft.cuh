// fft.cuh -- internal FFT launchers.
#pragma once
#include "common.cuh"

namespace mb {

// uplink FFT writing planar BF16 rows [n_sym][re|im][M][S_pad] for the
// tensor-core equalizer
mb_status fft_uplink_lp(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                        void *y_lp, uint32_t S_pad, cudaStream_t st);

}  // namespace mb
