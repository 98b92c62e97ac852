// ldpc.cuh -- the LDPC handle (ldpc.cu), for the slot's decode stage.
#pragma once
#include "common.cuh"

struct mb_ldpc {
  uint32_t kb, Z, mb, nnz, max_batch, words;  // words: 32-bit words of 4Z bits
  int dev;
  uint32_t *row_ptr;   // [mb + 1] device
  uint16_t *col, *sh;  // [nnz] device, rows < mb, by (row, col)
  uint32_t *binv;      // [4Z][words] device: B^-1 rows as bit words
  uint4 *state;        // [(max_batch + 1) / 2][mb][Z] device, per pair of blocks: min1, min2, signs + index
};
