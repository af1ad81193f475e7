// Serving-loop kernel.  Included at the end of distance.cu, whose GF(8)
// constant tables and prep / walk device functions it shares.
//
// Every warp of a persistent grid loops:
//   1. prepare the next published request, if any: read it from host-mapped
//      memory, compute its AGL2(F7) canonical mask, look it up in the device
//      dedup table (answer at once from an equivalent finished request when
//      that answer is conclusive for this request's threshold, wait for an
//      equivalent request in flight, else evaluate), build its basis and task
//      table and mark it runnable;
//   2. otherwise claim 32 tasks of the oldest runnable request (one per lane),
//      walk them, and finalise the request when its last task is counted;
//   3. otherwise resolve a waiting request whose equivalent has finished;
//   4. otherwise sleep briefly; leave when nothing happened for idle_ns.
// Requests published while others run are prepared and their tasks join the
// same pool, so their work overlaps on the device (continuous batching).
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

__device__ __forceinline__ unsigned long long ent_pack(unsigned int st, int mz, unsigned int id) {
  return (static_cast<unsigned long long>(st) << 56) |
         (static_cast<unsigned long long>(mz & 0xFF) << 48) | id;
}

// AGL2(F7) canonical mask of S (popcount >= 1), computed by one warp with the
// GL2 point table read through L1 (the anchored minimum of canonical.cu).
__device__ uint64_t canon_mask_warp(int lane, uint64_t S, const uint8_t* gl2) {
  return canon_mask_warp_min<true>(lane, S, gl2);
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

// Settles a request with its final value: records it in the dedup table
// (leaders always; other requests when the value is exact) and writes the
// answer.  `aborted` means the value is only a witness above the threshold.
__device__ void srv_settle(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h, int m,
                           bool aborted) {
  const unsigned long long ts = __ldcg(&h->tslot);
  if (ts != ~0ull && (__ldcg(&h->leader) || !aborted)) {
    atomicExch(a.vals + ts, ent_pack(aborted ? kEntAbort : kEntExact, m, __ldcg(&h->id)));
  }
  const int tmax = __ldcg(&h->tmax);
  srv_finish(a, slot, h, m, (aborted || m > tmax) ? TG_RESULT_FAIL : TG_RESULT_PASS);
}

// Finalises an evaluated request once all its tasks are counted.
__device__ void srv_complete(const SrvArgs& a, unsigned int slot, SrvSlotHdr* h) {
  __threadfence();
  const int m = atomicAdd(&h->best, 0);
  const bool aborted = atomicAdd(&h->abort, 0) != 0;
  srv_settle(a, slot, h, m, aborted);
}

// Builds the walk of a request whose indices are in h->idx (warp-level).
__device__ void srv_evaluate(const SrvArgs& a, int lane, unsigned int slot, SrvSlotHdr* h,
                             int* s_idx, int* s_row) {
  const int k = __ldcg(&h->k);
  s_idx[lane] = lane < k ? __ldcg(&h->idx[lane]) : -1;
  __syncwarp();
  uint8_t* base = reinterpret_cast<uint8_t*>(h);
  V6* B = reinterpret_cast<V6*>(base + a.basis_off);
  uint64_t* cum = reinterpret_cast<uint64_t*>(base + a.cum_off);
  uint32_t* info = reinterpret_cast<uint32_t*>(base + a.info_off);
  const PrepResult pr = prep_code(lane, k, s_idx, s_row, a.R, TG_ENUM_ORBIT,
                                  TG_VARIANT_HISTOGRAM, a.tab.M, B, cum, info);
  if (lane == 0) {
    if (pr.n_tasks == 0) {
      srv_settle(a, slot, h, pr.result, false);  // decided exactly without a walk
    } else {
      h->R = pr.R;
      h->H = pr.H;
      h->n_pat = pr.n_pat;
      h->best = 0;
      h->abort = 0;
      h->done_tasks = 0ull;
      h->n_tasks = pr.n_tasks;
      atomicAdd(&a.dh->codewords, static_cast<unsigned long long>(pr.n_tasks * pow8(pr.R)));
      __threadfence();
      // From here on a claim tagged with this request's id refers to the
      // tables written above, whatever the claimer believed about the slot.
      atomicExch(&h->claim, static_cast<unsigned long long>(__ldcg(&h->id)) << 32);
      __threadfence();
      *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotRun;
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
__device__ void srv_prepare(const SrvArgs& a, int lane, unsigned int req, int* s_idx,
                            int* s_row) {
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
    *reinterpret_cast<volatile unsigned long long*>(a.ring + (req % unsigned(a.Q))) = e;
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
          __threadfence();
          *reinterpret_cast<volatile unsigned int*>(&h->state) = kSlotWait;
          done = true;
        } else {
          done = srv_from_entry(a, slot, h, v);
        }
      }
      done = __shfl_sync(0xffffffffu, done, 0);
      if (done) return;
    }
  }
  srv_evaluate(a, lane, slot, h, s_idx, s_row);
}

// Resolves a waiting request (its state was moved WAIT -> PREP by lane 0).
__device__ void srv_resolve(const SrvArgs& a, int lane, unsigned int slot, int* s_idx,
                            int* s_row) {
  SrvSlotHdr* h = srv_slot(a, slot);
  bool done = false;
  if (lane == 0) done = srv_from_entry(a, slot, h, ld_vol64(a.vals + __ldcg(&h->tslot)));
  done = __shfl_sync(0xffffffffu, done, 0);
  if (!done) srv_evaluate(a, lane, slot, h, s_idx, s_row);
}

// Runs tasks c0 .. c0+31 of request `gen` in `slot`, one per lane.  The claim
// was taken on the generation-tagged counter, so `gen` is the request whose
// tables the slot holds; a claim on a generation the slot no longer serves is
// dropped (that request has finished, so no task of it was left unclaimed).
__device__ void srv_run(const SrvArgs& a, int lane, unsigned int slot, unsigned int gen,
                        unsigned long long c0) {
  SrvSlotHdr* h = srv_slot(a, slot);
  if (ld_vol32(&h->id) != gen) return;
  __threadfence();
  const unsigned long long n_tasks = __ldcg(&h->n_tasks);
  if (c0 >= n_tasks) return;
  const unsigned long long t = c0 + unsigned(lane);
  const uint8_t* base = reinterpret_cast<const uint8_t*>(h);
  const V6* B = reinterpret_cast<const V6*>(base + a.basis_off);
  const uint64_t* cum = reinterpret_cast<const uint64_t*>(base + a.cum_off);
  const uint32_t* info = reinterpret_cast<const uint32_t*>(base + a.info_off);
  bool last = false;
  if (t < n_tasks && !ld_flag(&h->abort)) {
    const int p = last_le<true>(cum, __ldcg(&h->n_pat), t);
    const uint64_t q = t - ld_u64<true>(cum + p);
    bool aborted = false;
    const int m = hist_task<true>(B, ld_u32<true>(info + p), q, __ldcg(&h->H), __ldcg(&h->k),
                                  __ldcg(&h->R), __ldcg(&h->tmax), &h->abort, aborted);
    if (m > 0) atomicMax(&h->best, m);
    if (aborted) {
      atomicExch(&h->abort, 1);
      const unsigned long long tag = static_cast<unsigned long long>(gen) << 32;
      const unsigned long long old = atomicMax(&h->claim, tag | n_tasks);
      const unsigned long long old_next = old & 0xFFFFFFFFull;
      if ((old >> 32) == gen && old_next < n_tasks) {
        __threadfence();
        const unsigned long long skipped = n_tasks - old_next;
        if (atomicAdd(&h->done_tasks, skipped) + skipped == n_tasks) last = true;
      }
    }
  }
  __syncwarp();
  const unsigned long long owned = min(32ull, n_tasks - c0);
  if (lane == 0) {
    __threadfence();
    if (atomicAdd(&h->done_tasks, owned) + owned == n_tasks) last = true;
    atomicAdd(&a.dh->tasks_done, owned);
  }
  if (last) srv_complete(a, slot, h);
}

__global__ void __launch_bounds__(kSrvTPB, 8) serve_kernel(SrvArgs a) {
  __shared__ int s_idx[kSrvTPB / 32][32];
  __shared__ int s_row[kSrvTPB / 32][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const unsigned long long t_start = gtimer();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    atomicMax(&a.dh->last_activity, t_start);
    atomicAdd(&a.dh->launches, 1u);
  }
  unsigned int iter = 0u;
  bool was_idle = true;
  for (;;) {
    int action = 0;  // -1 exit, 0 idle, 1 prepare, 2 run, 3 resolve
    unsigned int arg = 0u, slot = 0u;
    unsigned long long c0 = 0ull;
    if (lane == 0) {
      // Host memory is read over the bus: only an idle warp, or every warp
      // once in 64 steps, refreshes the device mirrors of the host's counters.
      if (was_idle || (++iter & 63u) == 0u) {
        atomicMax(&a.dh->pub_mirror, ld_acquire_sys(&a.ctl->published));
        if (ld_acquire_sys(&a.ctl->stop)) atomicExch(&a.dh->stop_mirror, 1u);
        atomicAdd(&a.dh->host_reads, 1ull);
      }
      const unsigned long long now = gtimer();
      unsigned int steps = 0u;
      if (ld_vol32(&a.dh->stop_mirror) || now - t_start > a.life_ns) {
        action = -1;
      } else {
        const unsigned int pub = ld_vol32(&a.dh->pub_mirror);
        unsigned int p = ld_vol32(&a.dh->prep_next);
        while (p < pub) {
          const unsigned int prev = atomicCAS(&a.dh->prep_next, p, p + 1u);
          if (prev == p) {
            action = 1;
            arg = p;
            break;
          }
          p = prev;
        }
        if (action == 0) {
          unsigned int lo = ld_vol32(&a.dh->lo);
          const unsigned int prepped = min(pub, ld_vol32(&a.dh->prep_next));
          for (unsigned int i = lo, n = 0; i < prepped && n < unsigned(a.S) + 1u; ++i, ++n) {
            ++steps;
            const unsigned long long e = ld_vol64(a.ring + (i % unsigned(a.Q)));
            const unsigned int eg = static_cast<unsigned int>(e >> 32);
            bool finished = false;  // nothing left to claim or resolve at i
            unsigned int why = 0u, t_hid = 0u, t_st = 0u;
            unsigned long long t_nt = 0ull, t_cw = 0ull;
            if (eg != i) {
              // A later request owns the ring entry only once request i has
              // been answered; anything else is an entry not yet visible.
              finished = eg != 0xFFFFFFFFu && eg > i && (eg - i) % unsigned(a.Q) == 0u;
              why = 1u;
              t_cw = e;
            } else {
              const unsigned int sl = static_cast<unsigned int>(e);
              SrvSlotHdr* h = srv_slot(a, sl);
              const unsigned int hid = ld_vol32(&h->id);
              t_hid = hid;
              if (hid > i) {
                finished = true;  // the slot already serves a newer request
                why = 2u;
              } else if (hid == i) {
                __threadfence();
                const unsigned int st = ld_vol32(&h->state);
                __threadfence();  // n_tasks after state: RUN publishes it
                const unsigned long long nt = __ldcg(&h->n_tasks);
                if (st == kSlotRun) {
                  const unsigned long long cw = ld_vol64(&h->claim);
                  if ((cw >> 32) == i && (cw & 0xFFFFFFFFull) < nt) {
                    const unsigned long long old = atomicAdd(&h->claim, 32ull);
                    c0 = old & 0xFFFFFFFFull;
                    arg = static_cast<unsigned int>(old >> 32);
                    if (arg != i || c0 < nt) {  // a task of generation arg, or past i's end
                      action = 2;
                      slot = sl;
                      break;
                    }
                  }
                  if ((cw >> 32) == i) finished = true;
                  why = 3u;
                  t_st = st;
                  t_nt = nt;
                  t_cw = cw;
                } else if (st == kSlotWait) {
                  const unsigned long long v = ld_vol64(a.vals + __ldcg(&h->tslot));
                  if ((v >> 56) >= kEntExact &&
                      atomicCAS(&h->state, kSlotWait, kSlotPrep) == kSlotWait) {
                    action = 3;
                    slot = sl;
                    break;
                  }
                } else if (st == kSlotDone) {
                  finished = true;
                  why = 4u;
                  t_st = st;
                }
              }
            }
            if (finished && i == lo) {
              if (atomicCAS(&a.dh->lo, lo, lo + 1u) == lo) {
                const unsigned int tn = atomicAdd(&a.dh->trace_n, 1u) & 31u;
                a.dh->trace[tn][0] = (static_cast<unsigned long long>(i) << 8) | why;
                a.dh->trace[tn][1] = (static_cast<unsigned long long>(t_hid) << 8) | t_st;
                a.dh->trace[tn][2] = t_nt;
                a.dh->trace[tn][3] = t_cw;
              }
              lo = ld_vol32(&a.dh->lo);
              if (lo > i + 1u) { i = lo - 1u; }
            }
          }
        }
        if (steps) atomicAdd(&a.dh->scan_steps, static_cast<unsigned long long>(steps));
        if (action == 0) {
          const unsigned long long act = max(ld_vol64(&a.dh->last_activity), t_start);
          if (now > act + a.idle_ns) action = -1;
        }
      }
    }
    action = __shfl_sync(0xffffffffu, action, 0);
    if (action < 0) break;
    was_idle = action == 0;
    if (action == 0) {
      __nanosleep(20000);
      continue;
    }
    arg = __shfl_sync(0xffffffffu, arg, 0);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    c0 = __shfl_sync(0xffffffffu, c0, 0);
    __syncwarp();  // order every lane's loads after lane 0's acquire
    if (lane == 0) atomicMax(&a.dh->last_activity, gtimer());
    if (action == 1) srv_prepare(a, lane, arg, s_idx[w], s_row[w]);
    else if (action == 2) srv_run(a, lane, slot, arg, c0);
    else srv_resolve(a, lane, slot, s_idx[w], s_row[w]);
    if (lane == 0) atomicMax(&a.dh->last_activity, gtimer());
  }
}

int launch_serve_kernel(const SrvArgs& a, int grid, cudaStream_t s) {
  serve_kernel<<<grid, kSrvTPB, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "serve_kernel launch");
  return TG_OK;
}

}  // namespace tg
