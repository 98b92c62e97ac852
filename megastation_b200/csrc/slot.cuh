// slot.cuh -- internal interface of the slot runner (slot.cu) for the
// pipeline (pipe.cu).
#pragma once
#include "common.cuh"

namespace mb {

// bytes of one slot's samples ([P+U][M][N] of iq_dtype), FP16 LLRs
// ([U][K][cb_stride]) and hard bits ([U][K][hrow])
void slot_io_bytes(const mb_slot *s, uint64_t *iq, uint64_t *llr, uint64_t *hard);

}  // namespace mb
