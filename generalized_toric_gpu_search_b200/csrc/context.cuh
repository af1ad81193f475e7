// The opaque tg_context of the C ABI (shared by the host-side translation units).
#pragma once

#include <cstdint>

struct tg_context {
  int device;
  int sm_count;
  int is_toric;    // M is the toric evaluation matrix
  uint8_t* d_M;    // 49 x 49 matrix entries
  uint64_t* d_Mp;  // 49 rows x 3 bit planes of M (bit j of plane b: bit b of M[row][j])
  uint8_t* d_gl2;  // 2016 x 49 GL2(F7) point permutations
};
