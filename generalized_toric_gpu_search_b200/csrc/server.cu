// Host side of the served search stream (include/toric_b200.h, tg_server_*):
// slot admission, publication of requests through page-locked mapped memory,
// relaunching of the bounded loop kernel and collection of answers.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "distance.cuh"
#include "serve.cuh"


namespace tg {

static size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

struct SrvLayout {
  int S, Q, k_max;
  unsigned int J;
  size_t slot_bytes, rows_off;
  size_t d_hdr, d_slots, d_jobs, d_keys, d_vals, d_total;
  size_t h_ctl, h_pubq, h_inputs, h_results, h_total;
  unsigned long long table_cap;
};

static int srv_defaults(const tg_server_params* p, tg_server_params& q) {
  q = *p;
  if (q.k_max < 1 || q.k_max > kSrvMaxK) {
    set_last_error("server k_max must be 1..%d", kSrvMaxK);
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (q.tail_rows != 0 && (q.tail_rows < 2 || q.tail_rows > 7)) {
    set_last_error("server tail_rows must be 0 or 2..7 (it is not used by the loop)");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (q.blocks_per_sm == 0) q.blocks_per_sm = kSrvPerSm;
  if (q.blocks_per_sm < 1 || q.blocks_per_sm > kSrvPerSm) {
    set_last_error("server blocks_per_sm must be 0..%d", kSrvPerSm);
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (q.idle_us == 0) q.idle_us = 2000;
  if (q.life_ms == 0) q.life_ms = 250;
  if (q.idle_us < 0 || q.life_ms < 0) {
    set_last_error("server idle_us and life_ms must be >= 0");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (q.table_capacity == 0) q.table_capacity = int64_t(1) << 20;
  if (q.table_capacity > 0 && (q.table_capacity < 64 || (q.table_capacity & (q.table_capacity - 1)))) {
    set_last_error("server table_capacity must be a power of two >= 64, 0 or -1");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (q.memory_fraction <= 0.0) q.memory_fraction = 0.25;
  if (q.memory_fraction > 0.9) q.memory_fraction = 0.9;
  if (q.max_slots < 0 || q.max_slots > (1 << 20)) {
    set_last_error("server max_slots must be 0..2^20");
    return TG_ERR_INVALID_ARGUMENT;
  }
  return TG_OK;
}

// Job ring capacity: a power of two above every job a full pool of requests
// can have pushed and not yet popped (each request pushes at most one job
// per stage, two per level for k - 3 <= 18 levels, plus wait jobs that
// replace one another).
static unsigned int srv_job_capacity(int S) {
  unsigned long long need = 40ull * static_cast<unsigned long long>(S) + 1024ull;
  unsigned long long J = 1024ull;
  while (J < need) J <<= 1;
  return static_cast<unsigned int>(J);
}

static SrvLayout srv_layout(const tg_server_params& q, int S) {
  SrvLayout L{};
  L.S = S;
  L.Q = 4 * S;
  L.J = srv_job_capacity(S);
  L.k_max = q.k_max;
  L.rows_off = a256(sizeof(SrvSlotHdr));
  L.slot_bytes = L.rows_off + a256(size_t(q.k_max) * kIsVecPerRow * sizeof(V6));
  L.table_cap = q.table_capacity > 0 ? static_cast<unsigned long long>(q.table_capacity) : 0ull;
  size_t off = 0;
  L.d_hdr = off;   off = a256(off + sizeof(SrvDevHeader));
  L.d_slots = off; off = a256(off + size_t(S) * L.slot_bytes);
  L.d_jobs = off;  off = a256(off + size_t(L.J) * 8);
  L.d_keys = off;  off = a256(off + L.table_cap * 8);
  L.d_vals = off;  off = a256(off + L.table_cap * 8);
  L.d_total = off;
  off = 0;
  L.h_ctl = off;     off = a256(off + sizeof(SrvCtl));
  L.h_pubq = off;    off = a256(off + size_t(L.Q) * 8);
  L.h_inputs = off;  off = a256(off + size_t(S) * sizeof(SrvInput));
  L.h_results = off; off = a256(off + size_t(S) * sizeof(SrvResult));
  L.h_total = off;
  return L;
}

// Slots from free device memory when the caller gives no count.
static int srv_slots(const tg_server_params& q, int* S) {
  if (q.max_slots > 0) {
    *S = q.max_slots;
    return TG_OK;
  }
  size_t free_b = 0, total_b = 0;
  const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
  const SrvLayout one = srv_layout(q, 1);
  const double budget = double(free_b) * q.memory_fraction -
                        double(one.table_cap) * 16.0 - 4096.0;
  // a slot and its share of the job ring
  long long s = budget > 0 ? static_cast<long long>(budget / double(one.slot_bytes + 512)) : 0;
  s = std::min<long long>(s, 1 << 16);
  if (s < 1) {
    set_last_error("not enough free device memory for one request slot");
    return TG_ERR_CAPACITY;
  }
  *S = int(s);
  return TG_OK;
}

class DeviceGuard2 {
 public:
  explicit DeviceGuard2(int dev) {
    ok_ = cudaGetDevice(&prev_) == cudaSuccess;
    err_ = cudaSetDevice(dev);
  }
  ~DeviceGuard2() {
    if (ok_) cudaSetDevice(prev_);
  }
  cudaError_t error() const { return err_; }

 private:
  int prev_ = 0;
  bool ok_ = false;
  cudaError_t err_ = cudaSuccess;
};

}  // namespace tg

using namespace tg;

struct tg_server {
  tg_context* ctx = nullptr;
  tg_server_params p{};
  SrvLayout L{};
  uint8_t* d_arena = nullptr;
  uint8_t* h_base = nullptr;
  SrvCtl* h_ctl = nullptr;
  unsigned long long* h_pubq = nullptr;
  SrvInput* h_inputs = nullptr;
  SrvResult* h_results = nullptr;
  SrvArgs args{};
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;
  std::mutex mu;
  std::vector<int> free_slots;
  std::vector<uint32_t> slot_id;
  std::vector<int> busy;           // slots with a published, unanswered request
  std::vector<uint32_t> busy_ids;  // their ids, ascending
  uint32_t next_id = 0;
  uint64_t finished = 0;
  bool launched = false;
};

extern "C" {

int tg_server_layout(tg_context* ctx, const tg_server_params* p, int32_t* h_slots,
                     size_t* h_device_bytes, size_t* h_host_bytes) {
  if (!ctx || !p) {
    set_last_error("tg_server_layout: NULL argument");
    return TG_ERR_INVALID_ARGUMENT;
  }
  tg_server_params q;
  int st = srv_defaults(p, q);
  if (st) return st;
  DeviceGuard2 g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  int S = 0;
  st = srv_slots(q, &S);
  if (st) return st;
  const SrvLayout L = srv_layout(q, S);
  if (h_slots) *h_slots = S;
  if (h_device_bytes) *h_device_bytes = L.d_total;
  if (h_host_bytes) *h_host_bytes = L.h_total;
  return TG_OK;
}

int tg_server_create(tg_context* ctx, const tg_server_params* p, void* d_arena,
                     size_t device_bytes, void* h_pinned, size_t host_bytes, tg_server** out) {
  if (!out) {
    set_last_error("tg_server_create: NULL out");
    return TG_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  if (!ctx || !p || !d_arena || !h_pinned) {
    set_last_error("tg_server_create: NULL argument");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (!ctx->is_toric) {
    set_last_error("the server needs the toric evaluation matrix");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (reinterpret_cast<uintptr_t>(d_arena) & 255u) {
    set_last_error("tg_server_create: device arena must be 256-byte aligned");
    return TG_ERR_INVALID_ARGUMENT;
  }
  tg_server_params q;
  int st = srv_defaults(p, q);
  if (st) return st;
  DeviceGuard2 g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  int S = q.max_slots;
  if (S <= 0) {
    // the caller sized the arena from tg_server_layout: recover S from it
    st = srv_slots(q, &S);
    if (st) return st;
    while (S > 1 && srv_layout(q, S).d_total > device_bytes) --S;
  }
  const SrvLayout L = srv_layout(q, S);
  if (device_bytes < L.d_total || host_bytes < L.h_total) {
    set_last_error("tg_server_create: arena %zu/%zu bytes, needs %zu/%zu", device_bytes,
                   host_bytes, L.d_total, L.h_total);
    return TG_ERR_WORKSPACE;
  }
  void* h_dev = nullptr;
  cudaError_t e = cudaHostGetDevicePointer(&h_dev, h_pinned, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaHostGetDevicePointer (host area must be pinned)");
  tg_server* srv = new tg_server();
  srv->ctx = ctx;
  srv->p = q;
  srv->L = L;
  srv->d_arena = static_cast<uint8_t*>(d_arena);
  srv->h_base = static_cast<uint8_t*>(h_pinned);
  std::memset(h_pinned, 0, L.h_total);
  srv->h_ctl = reinterpret_cast<SrvCtl*>(srv->h_base + L.h_ctl);
  srv->h_pubq = reinterpret_cast<unsigned long long*>(srv->h_base + L.h_pubq);
  srv->h_inputs = reinterpret_cast<SrvInput*>(srv->h_base + L.h_inputs);
  srv->h_results = reinterpret_cast<SrvResult*>(srv->h_base + L.h_results);
  for (int i = 0; i < L.Q; ++i) srv->h_pubq[i] = ~0ull;  // no entry published yet
  uint8_t* hd = static_cast<uint8_t*>(h_dev);
  SrvArgs& a = srv->args;
  a.ctl = reinterpret_cast<SrvCtl*>(hd + L.h_ctl);
  a.pubq = reinterpret_cast<const unsigned long long*>(hd + L.h_pubq);
  a.inputs = reinterpret_cast<const SrvInput*>(hd + L.h_inputs);
  a.results = reinterpret_cast<SrvResult*>(hd + L.h_results);
  a.dh = reinterpret_cast<SrvDevHeader*>(srv->d_arena + L.d_hdr);
  a.slots = srv->d_arena + L.d_slots;
  a.slot_bytes = L.slot_bytes;
  a.rows_off = L.rows_off;
  a.jobs = reinterpret_cast<unsigned long long*>(srv->d_arena + L.d_jobs);
  a.J = L.J;
  a.keys = reinterpret_cast<unsigned long long*>(srv->d_arena + L.d_keys);
  a.vals = reinterpret_cast<unsigned long long*>(srv->d_arena + L.d_vals);
  a.table_cap = L.table_cap;
  a.S = S;
  a.Q = L.Q;
  a.k_max = q.k_max;
  a.lanes = ctx->sm_count * q.blocks_per_sm * kSrvTPB;
  a.idle_ns = static_cast<unsigned long long>(q.idle_us) * 1000ull;
  a.life_ns = static_cast<unsigned long long>(q.life_ms) * 1000000ull;
  a.tab.M = ctx->d_M;
  a.tab.Mp = ctx->d_Mp;
  a.tab.gl2 = ctx->d_gl2;
  e = cudaStreamCreateWithFlags(&srv->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&srv->aux, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemsetAsync(srv->d_arena, 0, L.d_total, srv->aux);
  if (e == cudaSuccess && L.table_cap)
    e = cudaMemsetAsync(a.keys, 0xFF, L.table_cap * 8, srv->aux);
  if (e == cudaSuccess) e = cudaStreamSynchronize(srv->aux);
  if (e != cudaSuccess) {
    if (srv->stream) cudaStreamDestroy(srv->stream);
    if (srv->aux) cudaStreamDestroy(srv->aux);
    delete srv;
    return cuda_fail(e, "tg_server_create");
  }
  srv->free_slots.reserve(S);
  for (int i = S - 1; i >= 0; --i) srv->free_slots.push_back(i);
  srv->slot_id.assign(S, 0u);
  *out = srv;
  return TG_OK;
}

static int submit_locked(tg_server* srv, const int32_t* h_indices, int k, int target_distance,
                         uint32_t* h_id);

int tg_server_submit(tg_server* srv, const int32_t* h_indices, int32_t k, int32_t target_distance,
                     uint32_t* h_id) {
  if (!srv || (k > 0 && !h_indices)) {
    set_last_error("tg_server_submit: NULL argument");
    return TG_ERR_INVALID_ARGUMENT;
  }
  if (k < 0 || k > srv->L.k_max) {
    set_last_error("tg_server_submit: k = %d outside 0..%d", k, srv->L.k_max);
    return TG_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < k; ++i) {
    if (h_indices[i] < 0 || h_indices[i] >= kN) {
      set_last_error("tg_server_submit: index %d outside 0..48", h_indices[i]);
      return TG_ERR_INVALID_ARGUMENT;
    }
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  const int st = submit_locked(srv, h_indices, k, target_distance, h_id);
  if (st == TG_OK) __atomic_store_n(&srv->h_ctl->published, srv->next_id, __ATOMIC_RELEASE);
  return st;
}

int tg_server_submit_batch(tg_server* srv, const int32_t* h_indices, const int64_t* h_offsets,
                           int32_t n, const int32_t* h_target, uint32_t* h_ids,
                           int32_t* h_status, int32_t* h_consumed) {
  if (!srv || n < 0 || (n > 0 && (!h_offsets || !h_target || !h_ids || !h_status)) ||
      !h_consumed) {
    set_last_error("tg_server_submit_batch: NULL argument or n < 0");
    return TG_ERR_INVALID_ARGUMENT;
  }
  *h_consumed = 0;
  std::lock_guard<std::mutex> lock(srv->mu);
  int i = 0;
  for (; i < n; ++i) {
    const int64_t beg = h_offsets[i], len = h_offsets[i + 1] - beg;
    int st = TG_OK;
    if (len < 0 || len > srv->L.k_max || (len > 0 && !h_indices)) {
      st = TG_ERR_INVALID_ARGUMENT;
    } else {
      for (int64_t j = 0; j < len; ++j)
        if (h_indices[beg + j] < 0 || h_indices[beg + j] >= kN) st = TG_ERR_INVALID_ARGUMENT;
    }
    if (st == TG_OK) {
      st = submit_locked(srv, len > 0 ? h_indices + beg : nullptr, int(len), h_target[i],
                         h_ids + i);
      if (st == TG_ERR_CAPACITY) break;  // this and later requests stay with the caller
    }
    h_status[i] = st;
  }
  *h_consumed = i;
  // one publication store for the whole batch
  __atomic_store_n(&srv->h_ctl->published, srv->next_id, __ATOMIC_RELEASE);
  return TG_OK;
}

// Takes a free slot for one validated request and writes its publication
// entry (the caller holds srv->mu and publishes the new count).
static int submit_locked(tg_server* srv, const int32_t* h_indices, int k, int target_distance,
                         uint32_t* h_id) {
  if (srv->free_slots.empty()) {
    set_last_error("all %d request slots are busy", srv->L.S);
    return TG_ERR_CAPACITY;
  }
  const uint32_t id = srv->next_id;
  if (!srv->busy_ids.empty() && id - srv->busy_ids.front() >= uint32_t(srv->L.Q)) {
    set_last_error("publication ring full behind request %u", srv->busy_ids.front());
    return TG_ERR_CAPACITY;
  }
  const int slot = srv->free_slots.back();
  srv->free_slots.pop_back();
  SrvInput& in = srv->h_inputs[slot];
  in.k = k;
  in.target_distance = target_distance;
  for (int i = 0; i < 24; ++i) in.idx[i] = i < k ? h_indices[i] : 0;
  in.id = id;
  std::atomic_thread_fence(std::memory_order_release);
  srv->h_pubq[id % uint32_t(srv->L.Q)] =
      static_cast<unsigned long long>(uint32_t(slot)) | (static_cast<unsigned long long>(id) << 32);
  std::atomic_thread_fence(std::memory_order_release);
  srv->slot_id[slot] = id;
  srv->busy.push_back(slot);
  srv->busy_ids.push_back(id);
  srv->next_id = id + 1u;
  if (h_id) *h_id = id;
  return TG_OK;
}

int tg_server_debug_skip_publication(tg_server* srv) {
  if (!srv) {
    set_last_error("tg_server_debug_skip_publication: NULL server");
    return TG_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  const uint32_t id = srv->next_id;
  std::atomic_thread_fence(std::memory_order_release);
  __atomic_store_n(&srv->h_ctl->published, id + 1u, __ATOMIC_RELEASE);
  srv->next_id = id + 1u;
  return TG_OK;
}

int tg_server_pump(tg_server* srv, int32_t* h_running) {
  if (!srv) {
    set_last_error("tg_server_pump: NULL server");
    return TG_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  bool running = false;
  if (srv->launched) {
    const cudaError_t q = cudaStreamQuery(srv->stream);
    if (q == cudaErrorNotReady) {
      running = true;
    } else if (q != cudaSuccess) {
      return cuda_fail(q, "serve loop");
    } else {
      srv->launched = false;
    }
  }
  if (!running && !srv->busy.empty()) {
    DeviceGuard2 g(srv->ctx->device);
    if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
    const int grid = srv->ctx->sm_count * srv->p.blocks_per_sm;
    const int st = launch_serve_kernel(srv->args, grid, srv->stream);
    if (st) return st;
    srv->launched = true;
    running = true;
  }
  if (h_running) *h_running = running ? 1 : 0;
  return TG_OK;
}

int tg_server_poll(tg_server* srv, tg_server_result* h_out, int32_t max, int32_t* h_n) {
  if (!srv || (max > 0 && !h_out)) {
    set_last_error("tg_server_poll: NULL argument");
    return TG_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  int n = 0;
  for (size_t i = 0; i < srv->busy.size() && n < max;) {
    const int slot = srv->busy[i];
    const uint32_t id = srv->slot_id[slot];
    const SrvResult* r = &srv->h_results[slot];
    const uint32_t seq = __atomic_load_n(&r->seq, __ATOMIC_ACQUIRE);
    if (seq != id + 1u) {
      ++i;
      continue;
    }
    tg_server_result& o = h_out[n++];
    o.id = id;
    o.max_zeros = r->max_zeros;
    o.flags = r->flags;
    o.pad = 0;
    o.t_admit_ns = r->t_admit_ns;
    o.t_done_ns = r->t_done_ns;
    srv->free_slots.push_back(slot);
    srv->busy[i] = srv->busy.back();
    srv->busy.pop_back();
    auto it = std::lower_bound(srv->busy_ids.begin(), srv->busy_ids.end(), id);
    if (it != srv->busy_ids.end() && *it == id) srv->busy_ids.erase(it);
    ++srv->finished;
  }
  if (h_n) *h_n = n;
  return TG_OK;
}

int tg_server_stats(tg_server* srv, uint64_t* h_counters8) {
  if (!srv || !h_counters8) {
    set_last_error("tg_server_stats: NULL argument");
    return TG_ERR_INVALID_ARGUMENT;
  }
  SrvDevHeader dh{};
  {
    DeviceGuard2 g(srv->ctx->device);
    cudaError_t e = cudaMemcpyAsync(&dh, srv->args.dh, sizeof(dh), cudaMemcpyDeviceToHost, srv->aux);
    if (e == cudaSuccess) e = cudaStreamSynchronize(srv->aux);
    if (e != cudaSuccess) return cuda_fail(e, "tg_server_stats");
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  h_counters8[0] = srv->next_id;
  h_counters8[1] = srv->finished;
  h_counters8[2] = srv->busy.size();
  h_counters8[3] = dh.launches;
  h_counters8[4] = dh.tasks_done;
  h_counters8[5] = dh.codewords;
  h_counters8[6] = dh.dedup_hits;
  h_counters8[7] = static_cast<uint64_t>(static_cast<uint32_t>(dh.status));
  return TG_OK;
}

int tg_server_destroy(tg_server* srv) {
  if (!srv) return TG_OK;
  __atomic_store_n(&srv->h_ctl->stop, 1u, __ATOMIC_RELEASE);
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::seconds(20);
  for (;;) {
    const cudaError_t q = cudaStreamQuery(srv->stream);
    if (q != cudaErrorNotReady) break;
    if (std::chrono::steady_clock::now() > deadline) {
      set_last_error("serve loop did not stop within 20 s; server left allocated");
      return TG_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::milliseconds(1));
  }
  cudaStreamDestroy(srv->stream);
  cudaStreamDestroy(srv->aux);
  delete srv;
  return TG_OK;
}

}  // extern "C"
