// AGL2(F7) canonical forms of exponent sets and a device hash set for
// canonical dedup.
//
// Canonical form (the reference's canonical_forms kernel, kernel_canon.py:44-129,
// and canonical_forms_batch, champion_search_canonical.py:115-140): the
// minimum over A in GL2(F7) and anchor s in S of sort(A.S - A.s), packed 6 bits
// per index with the largest index most significant.  For sets of equal size
// that order is the order of 49-bit masks (bit i = exponent index i), so the
// key is the smallest mask among the AGL2 images of S that contain the origin.
// This file computes that mask for any popcount 1..49 and derives the
// reference's packed 128-bit key from it for k <= 16.
//
// Kernel: one warp per set, persistent CTAs; the 2016 x 49 point permutation
// table of GL2(F7) (98,784 bytes) sits in shared memory.  Lane l handles the
// matrices l, l + 32, ...: it maps the mask point by point, then for every
// point q of the image translates the image by -q on the torus Z_7^2
// (a per-row 7-bit rotation followed by a 49-bit rotation by 7 rows) and keeps
// the smallest mask, skipping the translations whose top row already exceeds
// the best (canon_mask_warp_min in common.cuh).  A 64-bit warp min-reduction
// finishes the set.
#include "common.cuh"
#include "canonical.cuh"

namespace tg {

constexpr int kCanonTPB = 512;                     // 2 CTAs per SM: 32 warps
constexpr int kGl2Row = 52;                        // padded row in shared memory
constexpr int kGl2SharedBytes = kGl2Order * kGl2Row;  // 104,832

struct CanonArgs {
  const int32_t* sets;    // (n, k) rows, or NULL
  const uint64_t* masks;  // n masks when sets == NULL (parents when expand)
  int expand;             // set s = parent s / 49 plus point s % 49 (0 if present)
  int n;
  int k;
  uint64_t* out_mask;
  uint64_t* out_lo;
  uint64_t* out_hi;
  int32_t* status;
  const uint8_t* gl2;
};

__global__ void __launch_bounds__(kCanonTPB, 2) canon_kernel(CanonArgs a) {
  extern __shared__ __align__(16) uint8_t s_perm[];
  // the GL2 table, rows padded from 49 to kGl2Row bytes
  for (int i = threadIdx.x; i < kGl2Order * kN; i += blockDim.x) {
    const int m = i / kN;
    s_perm[m * kGl2Row + (i - m * kN)] = __ldg(a.gl2 + i);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps_per_block = blockDim.x >> 5;
  const int n_warps = gridDim.x * warps_per_block;
  for (int s = blockIdx.x * warps_per_block + (threadIdx.x >> 5); s < a.n; s += n_warps) {
    uint64_t S = 0ull;
    bool bad = false;
    if (a.sets) {
      const int k = a.k;
      const int32_t* row = a.sets + size_t(s) * size_t(k);
      const int i_a = lane < k ? row[lane] : 0;
      const int i_b = lane + 32 < k ? row[lane + 32] : 0;
      const bool bad_a = lane < k && (i_a < 0 || i_a >= kN);
      const bool bad_b = lane + 32 < k && (i_b < 0 || i_b >= kN);
      uint64_t mine = 0ull;
      if (lane < k && !bad_a) mine |= 1ull << i_a;
      if (lane + 32 < k && !bad_b) mine |= 1ull << i_b;
      const uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(mine));
      const uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(mine >> 32));
      S = uint64_t(lo) | (uint64_t(hi) << 32);
      bad = __any_sync(0xffffffffu, bad_a || bad_b) || __popcll(S) != k;
    } else if (a.expand) {
      const uint64_t parent = a.masks[s / kN] & kMask49;
      const int p = s % kN;
      S = (parent >> p & 1ull) ? 0ull : (parent | (1ull << p));
    } else {
      S = a.masks[s] & kMask49;
    }
    if (bad || S == 0ull) {
      if (lane == 0) {
        a.out_mask[s] = 0ull;
        if (a.out_lo) a.out_lo[s] = ~0ull;
        if (a.out_hi) a.out_hi[s] = ~0ull;
        if (bad && a.status) atomicCAS(a.status, 0, TG_ERR_BAD_INPUT);
      }
      continue;
    }
    const uint64_t best = canon_mask_warp_min<false, kGl2Row>(lane, S, s_perm);
    if (lane == 0) {
      a.out_mask[s] = best;
      uint64_t lo, hi;
      key_from_mask(best, lo, hi);
      if (a.out_lo) a.out_lo[s] = lo;
      if (a.out_hi) a.out_hi[s] = hi;
    }
  }
}

static bool g_canon_attr[64] = {false};

int run_canonical(int device, int sm_count, const uint8_t* d_gl2, const int32_t* d_sets,
                  const uint64_t* d_masks, int n, int k, uint64_t* d_out_mask,
                  uint64_t* d_lo, uint64_t* d_hi, int32_t* d_status, cudaStream_t s,
                  int expand) {
  if (n <= 0) return TG_OK;
  if (!g_canon_attr[device]) {
    cudaError_t e = cudaFuncSetAttribute(canon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kGl2SharedBytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(canon_kernel)");
    g_canon_attr[device] = true;
  }
  CanonArgs a{d_sets, d_masks, expand, n, k, d_out_mask, d_lo, d_hi, d_status, d_gl2};
  const int warps_needed = n;
  int grid = sm_count * 2;
  const int max_grid = (warps_needed + (kCanonTPB / 32) - 1) / (kCanonTPB / 32);
  if (grid > max_grid) grid = max_grid;
  canon_kernel<<<grid, kCanonTPB, kGl2SharedBytes, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "canon_kernel launch");
  return TG_OK;
}

// ---------------------------------------------------------------------------
// Device hash set: open addressing, linear probing, 64-bit keys.
// Layout: [256-byte header][keys: cap x u64][tags: cap x u64].
// A tag is (call_id << 32 | index of first insertion in that call); the
// smallest tag wins, so old keys stay old and within a call the first index
// is the representative, whatever the thread order.
// ---------------------------------------------------------------------------

constexpr uint64_t kEmpty = ~0ull;

struct HashHeader {
  unsigned long long count;  // occupied slots
};

__device__ __forceinline__ uint64_t hash_slot(uint64_t key, uint64_t cap) {
  return splitmix64(key) & (cap - 1ull);
}

__global__ void hash_clear_kernel(uint64_t* keys, uint64_t* tags, uint64_t cap, HashHeader* h) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < cap; i += stride) {
    keys[i] = kEmpty;
    tags[i] = kEmpty;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) h->count = 0ull;
}

__global__ void hash_insert_kernel(uint64_t* keys, uint64_t* tags, uint64_t cap, HashHeader* h,
                                   const uint64_t* in, int n, uint32_t call_id, int32_t* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t key = in[i];
  if (key == kEmpty || key == 0ull) return;  // not a key: never new
  const unsigned long long tag = (static_cast<unsigned long long>(call_id) << 32) | uint32_t(i);
  uint64_t slot = hash_slot(key, cap);
  for (uint64_t probe = 0; probe < cap; ++probe) {
    const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(keys + slot),
                                             static_cast<unsigned long long>(kEmpty),
                                             static_cast<unsigned long long>(key));
    if (old == kEmpty || old == key) {
      if (old == kEmpty) {
        const unsigned long long cnt = atomicAdd(&h->count, 1ull) + 1ull;
        if (cnt > cap / 2 && status) atomicCAS(status, 0, TG_ERR_CAPACITY);
      }
      atomicMin(reinterpret_cast<unsigned long long*>(tags + slot), tag);
      return;
    }
    slot = (slot + 1ull) & (cap - 1ull);
  }
  if (status) atomicCAS(status, 0, TG_ERR_CAPACITY);
}

__global__ void hash_mark_kernel(const uint64_t* keys, const uint64_t* tags, uint64_t cap,
                                 const uint64_t* in, int n, uint32_t call_id, uint8_t* is_new,
                                 int32_t* n_new) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool fresh = false;
  if (i < n) {
    const uint64_t key = in[i];
    if (key != kEmpty && key != 0ull) {
      const unsigned long long tag = (static_cast<unsigned long long>(call_id) << 32) | uint32_t(i);
      uint64_t slot = hash_slot(key, cap);
      for (uint64_t probe = 0; probe < cap; ++probe) {
        const uint64_t k = keys[slot];
        if (k == key) {
          fresh = tags[slot] == tag;
          break;
        }
        if (k == kEmpty) break;
        slot = (slot + 1ull) & (cap - 1ull);
      }
    }
    if (is_new) is_new[i] = fresh ? 1 : 0;
  }
  if (n_new) {
    const unsigned b = __ballot_sync(0xffffffffu, fresh);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(n_new, __popc(b));
  }
}

size_t hashset_bytes(int64_t cap) { return 256 + size_t(cap) * 16; }

// ---------------------------------------------------------------------------
// Order-preserving compaction of flagged masks into sorted index rows.
// ---------------------------------------------------------------------------

constexpr int kCompactTPB = 256;

__global__ void compact_count_kernel(const uint8_t* flags, int n, int* block_counts) {
  __shared__ int s_cnt;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool f = i < n && flags[i];
  const unsigned b = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(&s_cnt, __popc(b));
  __syncthreads();
  if (threadIdx.x == 0) block_counts[blockIdx.x] = s_cnt;
}

__global__ void compact_scan_kernel(int* block_counts, int nb, int* total) {
  // one thread: the number of blocks is n / 256 (a few tens of thousands)
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int run = 0;
    for (int b = 0; b < nb; ++b) {
      const int c = block_counts[b];
      block_counts[b] = run;
      run += c;
    }
    *total = run;
  }
}

__global__ void compact_write_kernel(const uint64_t* masks, const uint8_t* flags, int n, int k,
                                     const int* block_offsets, uint64_t* out_masks,
                                     int32_t* out_sets, int64_t* out_offsets) {
  __shared__ int s_warp[kCompactTPB / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool f = i < n && flags[i];
  const unsigned b = __ballot_sync(0xffffffffu, f);
  if (lane == 0) s_warp[w] = __popc(b);
  __syncthreads();
  int before = block_offsets[blockIdx.x];
  for (int j = 0; j < w; ++j) before += s_warp[j];
  before += __popc(b & ((1u << lane) - 1u));
  if (f) {
    const uint64_t m = masks[i];
    if (out_masks) out_masks[before] = m;
    if (out_sets) {
      int32_t* row = out_sets + size_t(before) * size_t(k);
      uint64_t x = m;
      for (int j = 0; j < k; ++j) {
        const int idx = x ? __ffsll(static_cast<long long>(x)) - 1 : 0;
        x &= x - 1ull;
        row[j] = idx;
      }
    }
    if (out_offsets) {
      out_offsets[before] = int64_t(before) * k;
      out_offsets[before + 1] = int64_t(before + 1) * k;
    }
  }
}

size_t compact_scratch_bytes(int n) {
  return size_t((n + kCompactTPB - 1) / kCompactTPB + 1) * sizeof(int);
}

int run_compact(const uint64_t* d_masks, const uint8_t* d_flags, int n, int k, void* d_scratch,
                uint64_t* d_out_masks, int32_t* d_out_sets, int64_t* d_out_offsets,
                int32_t* d_count, cudaStream_t s) {
  if (n <= 0) {
    cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(count)");
    if (d_out_offsets) {
      e = cudaMemsetAsync(d_out_offsets, 0, sizeof(int64_t), s);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(offsets)");
    }
    return TG_OK;
  }
  const int nb = (n + kCompactTPB - 1) / kCompactTPB;
  int* counts = static_cast<int*>(d_scratch);
  compact_count_kernel<<<nb, kCompactTPB, 0, s>>>(d_flags, n, counts);
  compact_scan_kernel<<<1, 32, 0, s>>>(counts, nb, d_count);
  if (d_out_offsets) {
    cudaError_t e = cudaMemsetAsync(d_out_offsets, 0, sizeof(int64_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(offsets)");
  }
  compact_write_kernel<<<nb, kCompactTPB, 0, s>>>(d_masks, d_flags, n, k, counts, d_out_masks,
                                                   d_out_sets, d_out_offsets);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "compact kernels launch");
  return TG_OK;
}

int run_hash_clear(void* table, int64_t cap, cudaStream_t s) {
  uint8_t* base = static_cast<uint8_t*>(table);
  uint64_t* keys = reinterpret_cast<uint64_t*>(base + 256);
  uint64_t* tags = keys + cap;
  HashHeader* h = reinterpret_cast<HashHeader*>(base);
  int grid = int((cap + 255) / 256);
  if (grid > 4096) grid = 4096;
  hash_clear_kernel<<<grid, 256, 0, s>>>(keys, tags, uint64_t(cap), h);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "hash_clear_kernel launch");
  return TG_OK;
}

int run_hash_insert(void* table, int64_t cap, const uint64_t* d_keys, int n, uint32_t call_id,
                    uint8_t* d_is_new, int32_t* d_n_new, int32_t* d_status, cudaStream_t s) {
  if (n <= 0) {
    if (d_n_new) {
      cudaError_t e = cudaMemsetAsync(d_n_new, 0, sizeof(int32_t), s);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(n_new)");
    }
    return TG_OK;
  }
  uint8_t* base = static_cast<uint8_t*>(table);
  uint64_t* keys = reinterpret_cast<uint64_t*>(base + 256);
  uint64_t* tags = keys + cap;
  HashHeader* h = reinterpret_cast<HashHeader*>(base);
  if (d_n_new) {
    cudaError_t e = cudaMemsetAsync(d_n_new, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(n_new)");
  }
  const int grid = (n + 255) / 256;
  hash_insert_kernel<<<grid, 256, 0, s>>>(keys, tags, uint64_t(cap), h, d_keys, n, call_id, d_status);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "hash_insert_kernel launch");
  hash_mark_kernel<<<grid, 256, 0, s>>>(keys, tags, uint64_t(cap), d_keys, n, call_id, d_is_new,
                                        d_n_new);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "hash_mark_kernel launch");
  return TG_OK;
}

}  // namespace tg
