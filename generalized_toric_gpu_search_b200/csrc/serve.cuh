// Device-resident serving loop of max_zeros requests: shared layouts of the
// host-mapped control area and the device arena (serve_kernel.cuh, server.cu).
//
// Host-mapped (page-locked, written by one side, read by the other):
//   SrvCtl      the host's publication counter and stop flag
//   pubq        publication ring: entry i = slot | (request id i) << 32
//   SrvInput    one per slot: the request as submitted
//   SrvResult   one per slot: the answer; `seq` = id + 1 is written last
// Device arena:
//   SrvDevHeader; S slots (request state and its information set: k rows of
//   g and six Gray deltas); the job ring; the canonical dedup table (keys,
//   values).
#pragma once

#include "common.cuh"

namespace tg {

constexpr int kSrvMaxK = kMaxExactK;
constexpr int kSrvTPB = 128;
constexpr int kSrvPerSm = 5;  // CTAs per SM: the walk's register and shared-memory budget
constexpr int kSrvDoorbellStride = 16;  // warp 0 of every 16th CTA reads host memory

enum : unsigned int { kSlotFree = 0, kSlotPrep = 1, kSlotRun = 2, kSlotWait = 3, kSlotDone = 4 };

// Dedup table value: state << 56 | max_zeros << 48 | leader id.
enum : unsigned int { kEntEmpty = 0, kEntInFlight = 1, kEntExact = 2, kEntAbort = 3 };

// A request's levels from 4 on run in two parts each (the supports that hold
// its last row, then the others); stage 2 w + part - 1 (>= 8) names part
// `part` of level w.  Claim word of a request: id << 32 | stage << 26 | next
// unclaimed task of that stage.  Done word: stage << 40 | tasks of that stage
// counted.
constexpr int kSrvFirstStage = 8;  // level 4, part 1
constexpr unsigned long long kSrvTaskMask = (1ull << 26) - 1ull;
constexpr unsigned long long kSrvMaxTasks = (1ull << 26) - (1ull << 20);
constexpr unsigned long long kSrvDoneMask = (1ull << 40) - 1ull;

struct SrvCtl {
  unsigned int published;  // requests 0..published-1 are in pubq/inputs
  unsigned int stop;       // nonzero: the loop exits
  unsigned int pad[14];
};

struct SrvInput {
  int32_t k;
  int32_t target_distance;
  uint32_t id;
  int32_t pad;
  int32_t idx[24];
};

struct SrvResult {
  int32_t max_zeros;
  int32_t flags;  // TG_RESULT_* bits
  uint32_t id;
  uint32_t seq;   // id + 1 once final
  uint64_t t_admit_ns;
  uint64_t t_done_ns;
};

// The words every warp polls or updates sit on cache lines of their own, so
// the claims and pops of busy warps do not queue behind the reads of idle
// ones.
struct alignas(128) SrvLine32 {
  unsigned int v;
  unsigned int pad[31];
};
struct alignas(128) SrvLine64 {
  unsigned long long v;
  unsigned long long pad[15];
};

struct SrvDevHeader {
  SrvLine32 prep_next;                // next published request to prepare
  SrvLine32 pub_mirror;               // device copy of SrvCtl::published
  SrvLine64 last_activity;            // globaltimer of the last useful step
  SrvLine32 job_head;                 // next job to serve
  SrvLine32 job_tail;                 // next free job position
  SrvLine32 stop_mirror;              // device copy of SrvCtl::stop
  int status;
  unsigned int launches;
  unsigned long long tasks_done;
  unsigned long long codewords;       // codewords evaluated (levels 1-3 and the level tasks)
  unsigned long long dedup_hits;
  unsigned long long finished;
  unsigned long long levels_opened;   // stage jobs pushed (two per level)
  unsigned long long wait_requeues;   // wait jobs put back behind the others
  unsigned long long host_reads;      // refreshes of the mirrors from host memory
};

struct SrvSlotHdr {
  unsigned int state;
  unsigned int id;
  int k, tmax;
  int best;    // smallest weight met (levels done and tasks counted); 64 = none
  int abort;   // a weight below the target distance was met
  int leader;
  int level;   // stage whose tasks are out
  unsigned long long claim;
  unsigned long long done;
  unsigned long long tslot;  // dedup table slot or ~0
  unsigned long long t_admit;
  int idx[24];
};

struct SrvArgs {
  SrvCtl* ctl;          // device pointer of the host-mapped control block
  const unsigned long long* pubq;
  const SrvInput* inputs;
  SrvResult* results;
  SrvDevHeader* dh;
  uint8_t* slots;
  size_t slot_bytes;
  size_t rows_off;            // the information set within a slot
  unsigned long long* jobs;   // job ring: id << 32 | stage << 24 | slot (0 = empty)
  unsigned int J;             // job ring capacity (power of two)
  unsigned long long* keys;
  unsigned long long* vals;
  unsigned long long table_cap;
  int S;
  int Q;
  int k_max;
  int lanes;                  // resident threads of the loop (task sizing)
  unsigned long long idle_ns;
  unsigned long long life_ns;
  DeviceTables tab;
};

int launch_serve_kernel(const SrvArgs& a, int grid, cudaStream_t s);

}  // namespace tg
