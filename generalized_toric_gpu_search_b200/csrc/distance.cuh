// Internal interface of the max_zeros kernels (distance.cu).
#pragma once

#include "common.cuh"

namespace tg {

// Workspace header (first 256 bytes of a distance workspace).
struct WsHeader {
  int32_t status;                 // TG_OK or a TG_ERR_* raised on the device
  int32_t has_tasks;              // set by the prep kernels when some code has walk tasks
  unsigned long long counter;     // next unclaimed task
  unsigned long long total_tasks; // tasks of the run (after the scan)
  unsigned long long codewords;   // codewords the tasks cover
  double ref_messages;            // sum over exact sets of 8^k - 1
};

// Header of the information-set walk (one level at a time).
// Stages of the information-set walk: 0 = levels 1 to 3 (one launch), then
// 2 w + part - 1 for part 1 or 2 of level w >= 4.
constexpr int kIsStages = 2 * kMaxExactK + 2;

struct IsHeader {
  unsigned long long counter;    // next unclaimed task of the level being walked
  unsigned long long total;      // tasks of that level
  unsigned long long units;      // units (49-codeword blocks) per task of that level
  unsigned long long tasks_all;  // tasks over all levels walked
  unsigned long long codewords;  // codewords evaluated
  int32_t level;
  int32_t work;                  // set by plan_level_kernel when some set needs the level
  unsigned long long stage_codewords[kIsStages];  // codewords evaluated per stage
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
// Information-set codes reuse the descriptor: R = full sets, H = all sets,
// n_pat = rank deficit of the partial set (0 when there is none).

constexpr int32_t kDecidedFlag = 1;  // value known after preparation
constexpr int32_t kIsCodeFlag = 2;   // evaluated by information sets
constexpr int32_t kTorusBoundFlag = 4;  // one set, bound ceil(49 (L + 1) / k) (toric M)

constexpr int kIsMaxSets = 8;     // information sets per code
constexpr int kIsMaxRows = 64;    // sets x k per code
constexpr int kIsVecPerRow = 7;   // g and the deltas (alpha^v + alpha^(v+1)) g, v = 0..5
constexpr int kIsMaxDelta = 3;    // a partial set is kept when k - rank <= this

// Most information sets a code of k rows stores: the full ones that fit in
// 49 columns, plus a partial one when the leftover columns could give it a
// rank deficit <= kIsMaxDelta, within kIsMaxSets and kIsMaxRows.
__host__ __device__ constexpr int infoset_max_sets(int k) {
  const int cap = kIsMaxSets < kIsMaxRows / k ? kIsMaxSets : kIsMaxRows / k;
  const int full = cap < 49 / k ? cap : 49 / k;
  const int partial = (full < cap && 49 - full * k >= k - kIsMaxDelta && 49 - full * k > 0) ? 1 : 0;
  return full + partial;
}

struct WsLayout {
  size_t hdr, desc, task_off, abort, basis, pat_cum, pat_info, bitpat;
  size_t is_hdr, is_rows, is_units, is_off, is_best, is_perm, total;
  int basis_stride, pat_stride, bitpat_stride, is_stride, is_min_k;
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
  int enumeration;   // TG_ENUM_PROJECTIVE or TG_ENUM_ORBIT (codes with k < is_min_k)
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
  // Information-set path: codes with is_min_k <= k (is_min_k > k_max: none).
  int is_min_k;
  int is_toric;                  // M is the toric matrix (torus translations are automorphisms)
  int is_stride;                 // V6 per code in is_rows
  int is_lanes;                  // resident threads of the walk (task sizing)
  int is_blocks_per_sm;          // walk CTAs per SM
  int is_tasks_per_thread;       // tasks per resident thread a level is cut into
  int is_max_task_units;         // largest task, in blocks
  IsHeader* is_hdr;              // task queue of the information-set walk
  V6* is_rows;                   // per code and set: k rows x (g, 6 deltas)
  uint64_t* is_units;            // units of the current part per code position
  uint64_t* is_off;              // task offsets of the current level per code position (n + 1)
  int32_t* is_perm;              // code at each position (codes ordered by k)
  int32_t* is_best;              // smallest weight met per code
  // Witness pass only (NULL otherwise): per code and set the pivot columns
  // (kIsMaxSets words), the witness codewords (49 GF(8) symbols per code, in
  // the original column order) and one claim word per code.
  uint64_t* is_piv;
  uint8_t* witness;
  int32_t* wit_lock;
  DeviceTables tab;
};

// Internal enumeration of the witness pass: information sets for every
// k >= 1 (not a TG_ENUM_* value of the C ABI).
constexpr int kEnumInfosetAll = 16;

int upload_field_tables(int device);
int max_patterns(int H);
int default_tail_rows(const tg_distance_params& p);
int infoset_min_k(const tg_distance_params& p);
WsLayout ws_layout(const tg_distance_params& p);
int run_prepare(const DistArgs& args, cudaStream_t s);
int infoset_last_level(int k_max, int is_toric);
// parts: kWalkEnumeration (orbit / projective / sampled walk) and/or
// kWalkInfoset (information-set walk and its finalisation).
constexpr int kWalkEnumeration = 1;
constexpr int kWalkInfoset = 2;
int run_walk(const DistArgs& args, int sm_count, int blocks_per_sm, int tpb, cudaStream_t s,
             int parts = kWalkEnumeration | kWalkInfoset);
// Witness pass helpers: per-code targets 50 - out (the walk then stops at the
// first codeword with out zeros or more), and the copy of the pass's values
// into out with a check that every evaluated code got its witness (status
// into hdr1).
int run_witness_targets(const int32_t* out, const int64_t* off, int32_t* td, int n,
                        cudaStream_t s);
int run_witness_finish(const DistArgs& a2, int32_t* out, WsHeader* hdr1, cudaStream_t s);
size_t align_ws(size_t x);

}  // namespace tg
