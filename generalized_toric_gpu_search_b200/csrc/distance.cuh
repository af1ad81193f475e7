// Internal interface of the max_zeros kernels (distance.cu).
#pragma once

#include "common.cuh"

namespace tg {

// Workspace header (first 256 bytes of a distance workspace).
struct WsHeader {
  int32_t status;                 // TG_OK or a TG_ERR_* raised on the device
  int32_t pad0;
  unsigned long long counter;     // next unclaimed task
  unsigned long long total_tasks; // tasks of the run (after the scan)
  unsigned long long codewords;   // codewords the tasks cover
  double ref_messages;            // sum over exact sets of 8^k - 1
};

// Per-code descriptor written by the prep kernels.
struct CodeDesc {
  int32_t k;        // rows of the code
  int32_t R;        // tail rows walked inside one task
  int32_t H;        // head rows (k - R)
  int32_t n_pat;    // message patterns over the head
  int32_t tmax;     // 49 - target_distance
  int32_t flags;
  int32_t set_id;   // sampling id (the reference's blockIdx.x)
  int32_t pad;
  uint64_t n_tasks; // tasks of this code
};

struct WsLayout {
  size_t hdr, desc, task_off, abort, basis, pat_cum, pat_info, bitpat, total;
  int basis_stride, pat_stride, bitpat_stride;
};

struct DistArgs {
  const int32_t* idx;
  const int64_t* off;
  const int32_t* target;
  const int32_t* set_ids;
  int32_t* out;
  int n;
  int k_max;
  int R;
  int enumeration;   // TG_ENUM_PROJECTIVE or TG_ENUM_ORBIT
  int variant;       // TG_VARIANT_HISTOGRAM or TG_VARIANT_DIRECT
  int td_default;
  int64_t sample_count;
  uint64_t seed;
  WsHeader* hdr;
  CodeDesc* desc;
  uint64_t* task_off;
  int32_t* abort;
  V6* basis;
  uint64_t* pat_cum;
  uint32_t* pat_info;
  V6* bitpat;
  int basis_stride;
  int pat_stride;
  int bitpat_stride;
  DeviceTables tab;
};

int upload_field_tables(int device);
int max_patterns(int H);
int default_tail_rows(const tg_distance_params& p);
WsLayout ws_layout(const tg_distance_params& p);
int run_prepare(const DistArgs& args, cudaStream_t s);
int run_walk(const DistArgs& args, int sm_count, int blocks_per_sm, int tpb, cudaStream_t s);

}  // namespace tg
