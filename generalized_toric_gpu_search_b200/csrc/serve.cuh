// Device-resident serving loop of max_zeros requests: shared layouts of the
// host-mapped control area and the device arena (serve_kernel.cuh, server.cu).
//
// Host-mapped (page-locked, written by one side, read by the other):
//   SrvCtl      the host's publication counter and stop flag
//   pubq        publication ring: entry i = slot | (request id i) << 32
//   SrvInput    one per slot: the request as submitted
//   SrvResult   one per slot: the answer; `seq` = id + 1 is written last
// Device arena:
//   SrvDevHeader, S slots (request state, basis, pattern table), and the
//   canonical dedup table (keys, values).
#pragma once

#include "common.cuh"

namespace tg {

constexpr int kSrvMaxK = kMaxExactK;
constexpr int kSrvTPB = 128;

enum : unsigned int { kSlotFree = 0, kSlotPrep = 1, kSlotRun = 2, kSlotWait = 3, kSlotDone = 4 };

// Dedup table value: state << 56 | max_zeros << 48 | leader id.
enum : unsigned int { kEntEmpty = 0, kEntInFlight = 1, kEntExact = 2, kEntAbort = 3 };

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

struct SrvDevHeader {
  unsigned int prep_next;             // next published request to prepare
  unsigned int lo;                    // oldest request that may still need a warp
  unsigned long long last_activity;   // globaltimer of the last useful step
  int status;
  unsigned int launches;
  unsigned long long tasks_done;
  unsigned long long codewords;
  unsigned long long dedup_hits;
  unsigned long long finished;
  unsigned int trace_n;                 // lo advances recorded so far
  unsigned int pub_mirror;              // device copy of SrvCtl::published
  unsigned long long trace[32][4];      // last lo advances: i|reason, id|state, n_tasks, claim
  unsigned int stop_mirror;             // device copy of SrvCtl::stop
  unsigned int pad1;
  unsigned long long scan_steps;        // request entries looked at by scanners
  unsigned long long host_reads;        // refreshes of the mirrors from host memory
};

struct SrvSlotHdr {
  unsigned int state;
  unsigned int id;
  int k, R, H, n_pat, tmax;
  int best;
  int abort;
  int leader;
  unsigned long long n_tasks;     // < 2^31
  unsigned long long claim;       // id << 32 | next unclaimed task (generation-tagged)
  unsigned long long done_tasks;
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
  size_t basis_off, cum_off, info_off;
  unsigned long long* ring;   // device copy of pubq, written by each request's preparer
  unsigned long long* keys;
  unsigned long long* vals;
  unsigned long long table_cap;
  int S;
  int Q;
  int k_max;
  int R;
  unsigned long long idle_ns;
  unsigned long long life_ns;
  DeviceTables tab;
};

int launch_serve_kernel(const SrvArgs& a, int grid, cudaStream_t s);

}  // namespace tg
