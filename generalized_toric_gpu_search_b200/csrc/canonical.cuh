// Internal interface of canonical.cu.
#pragma once

#include "common.cuh"

namespace tg {

int run_canonical(int device, int sm_count, const uint8_t* d_gl2, const int32_t* d_sets,
                  const uint64_t* d_masks, int n, int k, uint64_t* d_out_mask,
                  uint64_t* d_lo, uint64_t* d_hi, int32_t* d_status, cudaStream_t s,
                  int expand = 0);
size_t compact_scratch_bytes(int n);
int run_compact(const uint64_t* d_masks, const uint8_t* d_flags, int n, int k, void* d_scratch,
                uint64_t* d_out_masks, int32_t* d_out_sets, int64_t* d_out_offsets,
                int32_t* d_count, cudaStream_t s);
size_t hashset_bytes(int64_t cap);
int run_hash_clear(void* table, int64_t cap, cudaStream_t s);
int run_hash_insert(void* table, int64_t cap, const uint64_t* d_keys, int n, uint32_t call_id,
                    uint8_t* d_is_new, int32_t* d_n_new, int32_t* d_status, cudaStream_t s);
int measure_int_pipes(int sm_count, void* d_scratch, double* out6);

}  // namespace tg
