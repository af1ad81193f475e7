// Serving-loop kernel.  Included at the end of distance.cu, whose GF(8)
// tables and information-set device code it shares.
//
// A request is evaluated by information sets, level by level, like a code of
// a batch (infoset_kernel.cuh): its preparing warp computes its canonical
// mask and looks it up in the dedup table, then eliminates its k rows to one
// information set, walks levels 1 to 3 itself and, while the torus-orbit
// bound ceil(49 (L + 1) / k) stays below its best weight, opens level 4.
// Levels from 4 on run in two parts, as in the batch walk: the supports that
// hold the last row, after which the bound is ceil(49 w / (k - 1)), then the
// others.  Every part (stage) of every request is a job in one device ring;
// warps take 32 tasks at a time from the oldest job, so the stages of
// requests admitted at different times share the SMs (continuous batching).
// The warp that counts a stage's last task settles the request or opens its
// next stage.
//
// Every warp of the persistent grid loops:
//   1. prepare the next published request, if any;
//   2. otherwise serve the job at the head of the ring: claim 32 tasks of
//      its level, or, for a request waiting on an equivalent one still in
//      flight, resolve it once that one's answer is final (else requeue it);
//      a job with nothing left to claim is popped;
//   3. otherwise sleep briefly; leave when nothing happened for idle_ns.
// All waits are bounded: the loop exits on the host's stop flag, after
// life_ns, or after idle_ns without work; the host relaunches it while
// requests are outstanding.  No warp ever waits for another warp.
#pragma once

namespace tg {

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire_sys(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.sys.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// System-scope loads of host-mapped memory (the host writes it through the
// CPU caches; these loads never return a stale GPU-cached copy).
__device__ __forceinline__ unsigned long long ld_sys64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.sys.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_sys32(const int* p) {
  int v;
  asm volatile("ld.relaxed.sys.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_vol64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ unsigned int ld_vol32(const unsigned int* p) {
  return *reinterpret_cast<const volatile unsigned int*>(p);
}

__device__ __forceinline__ SrvSlotHdr* srv_slot(const SrvArgs& a, unsigned int slot) {
  return reinterpret_cast<SrvSlotHdr*>(a.slots + size_t(slot) * a.slot_bytes);
}

__device__ __forceinline__ V6* srv_rows(const SrvArgs& a, SrvSlotHdr* h) {
  return reinterpret_cast<V6*>(reinterpret_cast<uint8_t*>(h) + a.rows_off);
}

__device__ __forceinline__ unsigned long long ent_pack(unsigned int st, int mz, unsigned int id) {
  return (static_cast<unsigned long long>(st) << 56) |
         (static_cast<unsigned long long>(mz & 0xFF) << 48) | id;
}

// AGL2(F7) canonical mask of S (popcount >= 1), computed by one warp with the
// GL2 point table read through L1 (the anchored minimum of canonical.cu).
__device__ uint64_t canon_mask_warp(int lane, uint64_t S, const uint8_t* gl2) {
  return canon_mask_warp_min<true>(lane, S, gl2);
}

__device__ __forceinline__ int srv_stage_level(int st) { return st >> 1; }
__device__ __forceinline__ int srv_stage_part(int st) { return (st & 1) + 1; }

// Supports of stage st of a k-row request (one information set): their count
// and the rank of the first.
__device__ __forceinline__ void srv_supports(const unsigned long long (*bn)[kIsBinom], int k,
                                            int st, unsigned long long& n_sup,
                                            unsigned long long& s_off) {
  is_part_supports(kTorusBoundFlag, k, srv_stage_level(st), srv_stage_part(st), bn, n_sup, s_off);
}

// Units of stage st of a k-row request.
__device__ __forceinline__ unsigned long long srv_units(const unsigned long long (*bn)[kIsBinom],
                                                       int k, int st) {
  unsigned long long n_sup, s_off;
  srv_supports(bn, k, st, n_sup, s_off);
  return n_sup * is_units_per_support(srv_stage_level(st));
}

// Units per task of a level: the batch scan's rule for one code (about eight
// tasks per resident thread, at most 343 units, aligned with supports), grown
// by factors of 7 until the level has fewer than kSrvMaxTasks tasks (the claim
// word's task field).
__device__ __forceinline__ unsigned long long srv_task_units(unsigned long long units, int w,
                                                            int lanes) {
  const unsigned long long target = 8ull * static_cast<unsigned long long>(lanes);
  unsigned long long nb = (units + target - 1ull) / target;
  nb = max(1ull, min(nb, 343ull));
  const unsigned long long bps = is_units_per_support(w);
  if (bps > 1ull) {
    if (nb >= bps) {
      nb = (nb / bps) * bps;
    } else {
      unsigned long long p7 = 1ull;
      while (p7 * 7ull <= nb) p7 *= 7ull;
      nb = (nb * nb > 7ull * p7 * p7) ? 7ull * p7 : p7;
    }
  }
  while ((units + nb - 1ull) / nb >= kSrvMaxTasks) nb *= 7ull;
  return nb;
}

// Appends a job: stage st >= kSrvFirstStage of request gen in `slot`, or
// (st = 0) the request waiting there on an equivalent one.
__device__ void srv_push_job(const SrvArgs& a, unsigned int gen, int st, unsigned int slot) {
  const unsigned int pos = atomicAdd(&a.dh->job_tail.v, 1u);
  const unsigned long long e = (static_cast<unsigned long long>(gen) << 32) |
                               (static_cast<unsigned long long>(st) << 24) | slot;
  atomicExch(a.jobs + (pos & (a.J - 1u)), e);
}

// Writes the final answer of a request to host-mapped memory and frees the
// slot for the host.  Called by exactly one thread per request.
__device__ void srv_finish(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h, int value,
                           int flags) {
  SrvResult* r = a.results + slot;
  r->max_zeros = value;
  r->flags = flags;
  const unsigned int id = __ldcg(&h->id);
  r->id = id;
  r->t_admit_ns = __ldcg(&h->t_admit);
  r->t_done_ns = gtimer();
  atomicAdd(&a.dh->finished, 1ull);
  // The slot's last device-side write comes before the host can see the
  // answer: once `seq` is visible the host may hand the slot to a new
  // request, whose preparation must not be overwritten by this DONE.
  *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotDone;
  __threadfence_system();
  *reinterpret_cast<volatile unsigned int*>(&r->seq) = id + 1u;
}

// Settles a request with max_zeros m: records it in the dedup table (leaders
// always; other requests when the value is exact) and writes the answer.
// `witness` means m is only a witness above the threshold.
__device__ void srv_settle(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h, int m,
                           bool witness) {
  const unsigned long long ts = __ldcg(&h->tslot);
  if (ts != ~0ull && (__ldcg(&h->leader) || !witness)) {
    __threadfence();
    atomicExch(a.vals + ts, ent_pack(witness ? kEntAbort : kEntExact, m, __ldcg(&h->id)));
  }
  const int tmax = __ldcg(&h->tmax);
  srv_finish(a, slot, h, m, (witness || m > tmax) ? TG_RESULT_FAIL : TG_RESULT_PASS);
}

// Opens stage st of request gen: its done count, then its claim word (from
// here on a claim tagged (gen, st) refers to this stage), then its job.
__device__ void srv_open_level(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h,
                               unsigned int gen, int st) {
  atomicExch(&h->done, static_cast<unsigned long long>(st) << 40);
  h->level = st;
  __threadfence();
  atomicExch(&h->claim, (static_cast<unsigned long long>(gen) << 32) |
                            (static_cast<unsigned long long>(st) << 26));
  __threadfence();
  srv_push_job(a, gen, st, slot);
  atomicAdd(&a.dh->levels_opened, 1ull);
}

// After stage st of a request: settle it (a witness below the target, the
// bound met, or every level done) or open stage st + 1.  After part 1 of
// level w the unseen codewords weigh at least ceil(49 w / (k - 1)); after
// part 2, ceil(49 (w + 1) / k).  Part 2 of level k has no support.  One
// thread.
__device__ void srv_level_end(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h,
                              unsigned int gen, int st) {
  __threadfence();
  const int best = atomicAdd(&h->best, 0);
  const int k = __ldcg(&h->k);
  const int tmax = __ldcg(&h->tmax);
  if (atomicAdd(&h->abort, 0) != 0 || best < kN - tmax) {
    srv_settle(a, slot, h, kN - best, true);
    return;
  }
  const int w = srv_stage_level(st);
  const int bound = srv_stage_part(st) == 1 ? (kN * w + k - 2) / (k - 1)  // k >= w >= 4
                                            : (kN * (w + 1) + k - 1) / k;
  if (w >= k || best <= bound) {
    srv_settle(a, slot, h, kN - best, false);
    return;
  }
  srv_open_level(a, slot, h, gen, st + 1);
}

// Evaluates a request whose indices are in h->idx (warp-level): one
// information set by Gauss-Jordan elimination, levels 1 to 3 by this warp,
// then level 4 as a job unless the request is decided.
__device__ void srv_evaluate(const SrvArgs& a, int lane, unsigned int slot, SrvSlotHdr* h,
                             uint8_t* s_ord) {
  const int k = __ldcg(&h->k);
  const unsigned int gen = __ldcg(&h->id);
  const int tmax = __ldcg(&h->tmax);
  if (k == 0) {
    if (lane == 0) srv_settle(a, slot, h, 0, false);
    return;
  }
  const int my = lane < k ? __ldcg(&h->idx[lane]) : 0;
  uint64_t p0 = 0ull, p1 = 0ull, p2 = 0ull;
  if (lane < k) {
    p0 = __ldg(a.tab.Mp + my * 3);
    p1 = __ldg(a.tab.Mp + my * 3 + 1);
    p2 = __ldg(a.tab.Mp + my * 3 + 2);
  }
  is_make_order(s_ord, 0, lane);
  uint64_t used = 0ull;
  if (is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord) < k) {
    // dependent rows: a nonzero message gives the zero codeword
    if (lane == 0) srv_settle(a, slot, h, kN, false);
    return;
  }
  is_reorder_columns(used, p0, p1, p2);
  V6* rows = srv_rows(a, h);
  is_store_set(rows, lane, k, p0, p1, p2);
  __threadfence_block();
  __syncwarp();
  unsigned long long ncw = 0ull;
  const int wmin = is_levels123_sets<true>(lane, rows, 1, k, WitSrc{nullptr, nullptr, nullptr},
                                           kN - tmax, ncw);
  if (lane == 0) {
    atomicAdd(&a.dh->codewords, ncw);
    h->best = wmin;
    h->abort = 0;
    if (wmin < kN - tmax) {
      srv_settle(a, slot, h, kN - wmin, true);
    } else if (k <= 3 || wmin <= (kN * 4 + k - 1) / k) {
      srv_settle(a, slot, h, kN - wmin, false);
    } else {
      __threadfence();
      *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotRun;
      srv_open_level(a, slot, h, gen, kSrvFirstStage);
    }
  }
  __syncwarp();
}

// Answer of a request from a finished equivalent one, when conclusive.
// Returns true when the request was finished.
__device__ bool srv_from_entry(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h,
                               unsigned long long v) {
  const unsigned int st = static_cast<unsigned int>(v >> 56);
  const int mz = static_cast<int>((v >> 48) & 0xFF);
  const int tmax = __ldcg(&h->tmax);
  if (st == kEntExact) {
    atomicAdd(&a.dh->dedup_hits, 1ull);
    srv_finish(a, slot, h, mz, (mz > tmax ? TG_RESULT_FAIL : TG_RESULT_PASS) | TG_RESULT_DEDUP);
    return true;
  }
  if (st == kEntAbort && mz > tmax) {
    atomicAdd(&a.dh->dedup_hits, 1ull);
    srv_finish(a, slot, h, mz, TG_RESULT_FAIL | TG_RESULT_DEDUP);
    return true;
  }
  return false;
}

// Prepares published request `req` (warp-level).
__device__ void srv_prepare(const SrvArgs& a, int lane, unsigned int req, uint8_t* s_ord) {
  unsigned long long e = 0ull;
  if (lane == 0) {
    // pubq[req] was written before `published` moved past req; reread a
    // bounded number of times in case the store is still in flight.
    for (int tries = 0; tries < 4096; ++tries) {
      e = ld_sys64(a.pubq + (req % unsigned(a.Q)));
      if (static_cast<unsigned int>(e >> 32) == req) break;
      __nanosleep(1000);
    }
  }
  e = __shfl_sync(0xffffffffu, e, 0);
  if (static_cast<unsigned int>(e >> 32) != req) {
    if (lane == 0) atomicCAS(&a.dh->status, 0, TG_ERR_STATE);
    return;
  }
  const unsigned int slot = static_cast<unsigned int>(e);
  SrvSlotHdr* h = srv_slot(a, slot);
  const SrvInput* in = a.inputs + slot;
  if (lane == 0) {
    *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotPrep;
    __threadfence();
    *reinterpret_cast<volatile unsigned int*>(&h->id) = req;
    h->t_admit = gtimer();
  }
  __syncwarp();
  const int k = ld_sys32(&in->k);
  const int td = ld_sys32(&in->target_distance);
  const unsigned int in_id = static_cast<unsigned int>(ld_sys32(reinterpret_cast<const int*>(&in->id)));
  const int my = (lane < k && k <= kSrvMaxK) ? ld_sys32(&in->idx[lane]) : 0;
  const bool bad_k = k < 0 || k > a.k_max || in_id != req;
  const bool bad_i = __any_sync(0xffffffffu, !bad_k && lane < k && (my < 0 || my >= kN));
  if (lane == 0) {
    h->k = bad_k ? 0 : k;
    h->tmax = kN - td;
    h->tslot = ~0ull;
    h->leader = 0;
    h->level = 0;
  }
  if (lane < 24) h->idx[lane] = (!bad_k && lane < k) ? my : 0;
  __syncwarp();
  if (bad_k || bad_i) {
    if (lane == 0) srv_finish(a, slot, h, 0, TG_RESULT_BAD_INPUT);
    return;
  }
  // Exponent mask; repeated indices make popcount < k (no dedup, max_zeros 49).
  const unsigned int lo = __reduce_or_sync(0xffffffffu, lane < k && my < 32 ? 1u << my : 0u);
  const unsigned int hi =
      __reduce_or_sync(0xffffffffu, lane < k && my >= 32 ? 1u << (my - 32) : 0u);
  const uint64_t S = uint64_t(lo) | (uint64_t(hi) << 32);
  if (k >= 1 && __popcll(S) == k && a.table_cap) {
    const uint64_t key = canon_mask_warp(lane, S, a.tab.gl2);
    int outcome = 0;  // 0: no dedup (table full), 1: leader, 2: hit
    unsigned long long v = 0ull, ts = 0ull;
    if (lane == 0) {
      ts = splitmix64(key) & (a.table_cap - 1ull);
      for (int probe = 0; probe < 64; ++probe) {
        const unsigned long long old = atomicCAS(a.keys + ts, ~0ull, key);
        if (old == ~0ull) {
          atomicExch(a.vals + ts, ent_pack(kEntInFlight, 0, req));
          outcome = 1;
          break;
        }
        if (old == key) {
          v = ld_vol64(a.vals + ts);
          outcome = 2;
          break;
        }
        ts = (ts + 1ull) & (a.table_cap - 1ull);
      }
      if (outcome) h->tslot = ts;
      if (outcome == 1) h->leader = 1;
    }
    outcome = __shfl_sync(0xffffffffu, outcome, 0);
    if (outcome == 2) {
      bool done = false;
      if (lane == 0) {
        const unsigned int st = static_cast<unsigned int>(v >> 56);
        if (st == kEntEmpty || st == kEntInFlight) {
          // the equivalent request is still running: wait in the job ring
          __threadfence();
          *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotWait;
          srv_push_job(a, req, 0, slot);
          done = true;
        } else {
          done = srv_from_entry(a, slot, h, v);
        }
      }
      done = __shfl_sync(0xffffffffu, done, 0);
      if (done) return;
    }
  }
  srv_evaluate(a, lane, slot, h, s_ord);
}

// Resolves a waiting request whose equivalent has an answer (warp-level):
// from that answer when conclusive, else by its own evaluation.
__device__ void srv_resolve(const SrvArgs& a, int lane, unsigned int slot, uint8_t* s_ord) {
  SrvSlotHdr* h = srv_slot(a, slot);
  bool done = false;
  if (lane == 0) done = srv_from_entry(a, slot, h, ld_vol64(a.vals + __ldcg(&h->tslot)));
  done = __shfl_sync(0xffffffffu, done, 0);
  if (!done) srv_evaluate(a, lane, slot, h, s_ord);
}

// Runs the 32 tasks a warp claimed: `cw` is the claim word's value before
// the warp's atomicAdd (request gen, stage st, first task t0).  A claim on a
// slot that no longer serves gen, or past the stage's end, runs nothing.
// The warp that counts a stage's last task ends the stage.
__device__ void srv_run(const SrvArgs& a, int lane, unsigned int slot, unsigned long long cw,
                        const unsigned long long (*bn)[kIsBinom], uint16_t* dig, uint32_t* ez,
                        unsigned long long& n_tasks, unsigned long long& n_codewords) {
  SrvSlotHdr* h = srv_slot(a, slot);
  const unsigned int gen = static_cast<unsigned int>(cw >> 32);
  const int st = static_cast<int>((cw >> 26) & 63ull);
  const int w = srv_stage_level(st);
  const unsigned long long t0 = cw & kSrvTaskMask;
  if (ld_vol32(&h->id) != gen || st < kSrvFirstStage) return;
  __threadfence();
  const int k = __ldcg(&h->k);
  const int tmax = __ldcg(&h->tmax);
  unsigned long long n_sup, s_off;
  srv_supports(bn, k, st, n_sup, s_off);
  const unsigned long long units = n_sup * is_units_per_support(w);
  const unsigned long long nb = srv_task_units(units, w, a.lanes);
  const unsigned long long nt = (units + nb - 1ull) / nb;
  if (t0 >= nt) return;
  const int wthr = kN - tmax;
  const unsigned long long t = t0 + unsigned(lane);
  int wmin = kN + 1;
  unsigned long long ncw = 0ull;
  if (t < nt && !ld_flag(&h->abort)) {
    const unsigned long long u0 = t * nb;
    const unsigned long long u1 = min(u0 + nb, units);
    wmin = is_walk_range<kSrvTPB, false, true>(srv_rows(a, h), 1, 0, &h->abort,
                                               WitSrc{nullptr, nullptr, nullptr}, bn, dig, ez,
                                               k, w, n_sup, s_off, u0, u1, wthr,
                                               ld_flag(&h->best), ncw);
  }
  const int wl = __reduce_min_sync(0xffffffffu, wmin);
  for (int o = 16; o > 0; o >>= 1) ncw += __shfl_xor_sync(0xffffffffu, ncw, o);
  if (lane == 0) {
    n_codewords += ncw;  // this warp's statistics, flushed by the loop
    unsigned long long skipped = 0ull;
    if (wl < ld_flag(&h->best)) {
      const int best = min(atomicMin(&h->best, wl), wl);
      if (best < wthr && atomicExch(&h->abort, 1) == 0) {
        // a witness below the target: the level's unclaimed tasks are
        // skipped, and counted here
        const unsigned long long tag = cw & ~kSrvTaskMask;
        const unsigned long long old = atomicMax(&h->claim, tag | nt);
        if ((old & ~kSrvTaskMask) == tag && (old & kSrvTaskMask) < nt)
          skipped = nt - (old & kSrvTaskMask);
      }
    }
    const unsigned long long owned = min(32ull, nt - t0);
    __threadfence();
    const unsigned long long add = owned + skipped;
    const unsigned long long old = atomicAdd(&h->done, add);
    n_tasks += owned;
    if ((old >> 40) == static_cast<unsigned long long>(st) && (old & kSrvDoneMask) + add == nt)
      srv_level_end(a, slot, h, gen, st);
  }
  __syncwarp();
}

// Records activity for the idle exit: the shared word is written only when
// it is more than 50 us old, so busy warps do not queue on it.
__device__ __forceinline__ void srv_touch(const SrvArgs& a) {
  const unsigned long long now = gtimer();
  if (now > ld_vol64(&a.dh->last_activity.v) + 50000ull) atomicMax(&a.dh->last_activity.v, now);
}

__global__ void __launch_bounds__(kSrvTPB, kSrvPerSm) serve_kernel(SrvArgs a) {
  __shared__ unsigned long long s_binom[kIsBinom][kIsBinom];
  __shared__ uint16_t s_dig[kIsMaxDigits][kSrvTPB];
  __shared__ uint32_t s_ez[39][kSrvTPB];
  __shared__ uint8_t s_ord[kSrvTPB / 32][64];
  for (int i = threadIdx.x; i < kIsBinom * kIsBinom; i += kSrvTPB)
    s_binom[i / kIsBinom][i % kIsBinom] = c_binom[i / kIsBinom][i % kIsBinom];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wl = threadIdx.x >> 5;
  uint16_t* my_dig = &s_dig[0][threadIdx.x];
  uint32_t* my_ez = &s_ez[0][threadIdx.x];
  const unsigned long long t_start = gtimer();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    atomicMax(&a.dh->last_activity.v, t_start);
    atomicAdd(&a.dh->launches, 1u);
  }
  unsigned int iter = 0u;
  bool was_idle = true;
  // Host memory is read over the bus by a few doorbell warps (warp 0 of
  // every kSrvDoorbellStride-th CTA) when idle or once in 64 steps, and by
  // every other warp once in 1024 steps; all of them keep to the device
  // mirrors otherwise.
  const bool doorbell = wl == 0 && (blockIdx.x % kSrvDoorbellStride) == 0;
  unsigned long long n_tasks = 0ull, n_codewords = 0ull;  // lane 0's, flushed now and then
  for (;;) {
    int action = 0;  // -1 exit, 0 idle, 1 prepare, 2 run, 3 resolve
    unsigned int arg = 0u, slot = 0u;
    unsigned long long cw = 0ull;
    if (lane == 0) {
      ++iter;
      if (doorbell ? (was_idle || (iter & 63u) == 0u) : (iter & 1023u) == 0u) {
        const unsigned int pub = ld_acquire_sys(&a.ctl->published);
        if (pub > ld_vol32(&a.dh->pub_mirror.v)) atomicMax(&a.dh->pub_mirror.v, pub);
        if (ld_acquire_sys(&a.ctl->stop)) atomicExch(&a.dh->stop_mirror.v, 1u);
        atomicAdd(&a.dh->host_reads, 1ull);
      }
      const unsigned long long now = gtimer();
      if (ld_vol32(&a.dh->stop_mirror.v) || now - t_start > a.life_ns) {
        action = -1;
      } else {
        const unsigned int pub = ld_vol32(&a.dh->pub_mirror.v);
        unsigned int p = ld_vol32(&a.dh->prep_next.v);
        while (p < pub) {
          const unsigned int prev = atomicCAS(&a.dh->prep_next.v, p, p + 1u);
          if (prev == p) {
            action = 1;
            arg = p;
            break;
          }
          p = prev;
        }
        // The job at the head of the ring: claim from it, or pop it.  A few
        // tries per step keep the warp from looping on a busy ring.
        for (int tries = 0; action == 0 && tries < 8; ++tries) {
          const unsigned int hd = ld_vol32(&a.dh->job_head.v);
          if (hd == ld_vol32(&a.dh->job_tail.v)) break;
          unsigned long long* je = a.jobs + (hd & (a.J - 1u));
          const unsigned long long e = ld_vol64(je);
          if (e == 0ull) break;  // pushed but not yet written
          const unsigned int gen = static_cast<unsigned int>(e >> 32);
          const int st = static_cast<int>((e >> 24) & 0xFFull);
          const unsigned int sl = static_cast<unsigned int>(e & 0xFFFFFFull);
          SrvSlotHdr* h = srv_slot(a, sl);
          if (st == 0) {
            // a waiting request: take the job; resolve it once its
            // equivalent's answer is final, else put it back behind the rest
            if (atomicCAS(&a.dh->job_head.v, hd, hd + 1u) != hd) continue;
            atomicExch(je, 0ull);
            if (ld_vol32(&h->id) != gen || ld_vol32(&h->state) != kSlotWait) continue;
            const unsigned long long v = ld_vol64(a.vals + __ldcg(&h->tslot));
            if ((v >> 56) >= kEntExact &&
                atomicCAS(&h->state, kSlotWait, kSlotPrep) == kSlotWait) {
              action = 3;
              slot = sl;
            } else {
              srv_push_job(a, gen, 0, sl);
              atomicAdd(&a.dh->wait_requeues, 1ull);
            }
            continue;
          }
          const unsigned long long tag = (static_cast<unsigned long long>(gen) << 32) |
                                         (static_cast<unsigned long long>(st) << 26);
          const unsigned long long cur = ld_vol64(&h->claim);
          bool open = false;
          if ((cur & ~kSrvTaskMask) == tag) {
            const int k = __ldcg(&h->k);
            const int w = srv_stage_level(st);
            const unsigned long long units = srv_units(s_binom, k, st);
            const unsigned long long nt =
                (units + srv_task_units(units, w, a.lanes) - 1ull) /
                srv_task_units(units, w, a.lanes);
            open = (cur & kSrvTaskMask) < nt;
          }
          if (open) {
            // whatever the claim returns is this warp's to run (srv_run
            // checks the request and the level's end)
            cw = atomicAdd(&h->claim, 32ull);
            action = 2;
            slot = sl;
          } else if (atomicCAS(&a.dh->job_head.v, hd, hd + 1u) == hd) {
            atomicExch(je, 0ull);
          }
        }
        if (action == 0) {
          const unsigned long long act = max(ld_vol64(&a.dh->last_activity.v), t_start);
          if (now > act + a.idle_ns) action = -1;
        }
      }
    }
    action = __shfl_sync(0xffffffffu, action, 0);
    if (lane == 0 && (action < 0 || (iter & 63u) == 0u) && (n_tasks | n_codewords)) {
      atomicAdd(&a.dh->tasks_done, n_tasks);
      atomicAdd(&a.dh->codewords, n_codewords);
      n_tasks = n_codewords = 0ull;
    }
    if (action < 0) break;
    was_idle = action == 0;
    if (action == 0) {
      // Idle warps poll the ring every ~80 us: shorter sleeps put their
      // reads on the lines the busy warps claim from (p99 1.5 ms at 5-20 us,
      // 1.0 ms at 40-80 us on the served stream, p50 unchanged).
      __nanosleep(80000);
      continue;
    }
    arg = __shfl_sync(0xffffffffu, arg, 0);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    cw = __shfl_sync(0xffffffffu, cw, 0);
    __syncwarp();  // order every lane's loads after lane 0's acquire
    if (lane == 0) srv_touch(a);
    if (action == 1) srv_prepare(a, lane, arg, s_ord[wl]);
    else if (action == 2) srv_run(a, lane, slot, cw, s_binom, my_dig, my_ez, n_tasks, n_codewords);
    else srv_resolve(a, lane, slot, s_ord[wl]);
    if (lane == 0) srv_touch(a);
  }
}

int launch_serve_kernel(const SrvArgs& a, int grid, cudaStream_t s) {
  serve_kernel<<<grid, kSrvTPB, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "serve_kernel launch");
  return TG_OK;
}

}  // namespace tg
