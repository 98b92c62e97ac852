// slot.cuh -- internal hooks of the slot runner.
#pragma once
#include "common.cuh"

namespace mb {

// equalize one batch of nb uplink symbols with the cell's precision
mb_status slot_equalize(const mb_cell_desc &c, const float2 *W, const float2 *y,
                        void *y_lp, uint32_t nb, uint16_t *llr, uint8_t *hard,
                        const mb_scrambler *scr, cudaStream_t st);

}  // namespace mb
