// Information-set enumeration of max_zeros (Brouwer-Zimmermann).  Included by
// distance.cu, whose GF(8) tables, descriptors and helpers it shares.
//
// max_zeros = 49 - d, d the minimum weight of a nonzero codeword.  For a code
// of k rows, a warp finds information sets I_1..I_s: pairwise disjoint sets of
// columns, the first m of them of rank k ("full") and possibly a last one of
// rank r = k - delta ("partial").  Gauss-Jordan elimination on I_j gives a
// generator G_j of the same code that is the identity on I_j's pivot columns,
// and rows r..k-1 of a partial set's G_j vanish on all of its columns.  A
// codeword c = u G_j then has wt(c restricted to I_j) >= wt(u) - delta_j.
// Level w enumerates, for every set, the projective messages u of weight
// exactly w, so once levels 1..L are complete every codeword not yet seen
// has weight >= m (L + 1) + max(0, L + 1 - delta) (the columns of different
// sets are disjoint).  A code is finished when
//   * its best weight is <= that bound (the best weight is then d), or
//   * all k levels are complete (every message has been seen), or
//   * a weight below the target distance appears (the decision of the early
//     exit: max_zeros > 49 - target_distance).
//
// Sets are found by greedy elimination over a column order; the identity
// order first, then up to kIsTries - 1 pseudo-random orders (a fixed
// sequence), keeping the order with the most full sets and then the largest
// partial rank.  One lane holds one row, bit-sliced over the 49 columns, so a
// pivot step is a ballot, a row swap and one broadcast.
//
// Tasks: (level w, code, set j, support T of w rows, block of outer
// coefficients).  The first row of T has coefficient 1; the next
// w - 1 - inner rows ("outer") take the block's base-7 digits as powers
// alpha^e; the last inner = min(w - 1, 5) rows walk a reflected base-7 Gray
// code over alpha^0..alpha^6, one XOR of a precomputed delta
// (alpha^v + alpha^(v+1)) g per codeword.  The global queue is level-major
// over the batch, so a code's level w + 1 starts after its level w has been
// handed out, and a finished code's remaining range is skipped by moving the
// counter past it.
#pragma once

namespace tg {

constexpr int kIsInner = 5;       // Gray-walked coefficients per task (7^5 codewords)
constexpr int kIsTries = 32;      // column orders tried per code
constexpr int kIsBinom = 22;      // binomial table side (n, r <= 21)

// ---------------------------------------------------------------------------
// Preparation: one warp per code, lane r holds row r bit-sliced (3 x 49 bits).
// ---------------------------------------------------------------------------

constexpr int kIsPrepWarps = 4;

// x <- c x for a GF(8) constant c, on bit-sliced planes.
__device__ __forceinline__ void gf8_scale64(uint32_t c, uint64_t& x0, uint64_t& x1,
                                            uint64_t& x2) {
  uint64_t r0 = 0ull, r1 = 0ull, r2 = 0ull;
  uint64_t a0 = x0, a1 = x1, a2 = x2;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const uint64_t m = 0ull - uint64_t((c >> b) & 1u);
    r0 ^= a0 & m;
    r1 ^= a1 & m;
    r2 ^= a2 & m;
    const uint64_t t = a2;  // a <- alpha a: (a0, a1, a2) -> (a2, a0 ^ a2, a1)
    a2 = a1;
    a1 = a0 ^ t;
    a0 = t;
  }
  x0 = r0;
  x1 = r1;
  x2 = r2;
}

__device__ __forceinline__ V6 v6_of_planes(uint64_t p0, uint64_t p1, uint64_t p2) {
  V6 v;
  v.l0 = uint32_t(p0);
  v.l1 = uint32_t(p1);
  v.l2 = uint32_t(p2);
  v.h0 = uint32_t(p0 >> 32) & kHiMask;
  v.h1 = uint32_t(p1 >> 32) & kHiMask;
  v.h2 = uint32_t(p2 >> 32) & kHiMask;
  v.pad0 = v.pad1 = 0u;
  return v;
}

// Column order of try t: identity for t = 0, else a Fisher-Yates shuffle
// driven by splitmix64.
__device__ void is_make_order(uint8_t* ord, int t, int lane) {
  if (lane == 0) {
    for (int i = 0; i < kN; ++i) ord[i] = uint8_t(i);
    if (t > 0) {
      uint64_t s = 0x6A09E667F3BCC909ull + uint64_t(t);
      for (int i = kN - 1; i > 0; --i) {
        s = splitmix64(s);
        const int j = int(s % uint64_t(i + 1));
        const uint8_t x = ord[i];
        ord[i] = ord[j];
        ord[j] = x;
      }
    }
  }
  __syncwarp();
}

// Gauss-Jordan elimination over the unused columns in `ord` order until k
// pivots are found; returns the rank reached.  Pivot columns are added to
// `used`.  All values are warp-uniform except the rows.
__device__ int is_gauss_jordan(int lane, int k, uint64_t& p0, uint64_t& p1, uint64_t& p2,
                               uint64_t& used, const uint8_t* ord) {
  int rank = 0;
  for (int ci = 0; ci < kN && rank < k; ++ci) {
    const int col = ord[ci];
    if ((used >> col) & 1ull) continue;
    const uint32_t coef = uint32_t((p0 >> col) & 1ull) | (uint32_t((p1 >> col) & 1ull) << 1) |
                          (uint32_t((p2 >> col) & 1ull) << 2);
    const unsigned cand = __ballot_sync(0xffffffffu, lane >= rank && lane < k && coef != 0u);
    if (cand == 0u) continue;
    const int pr = __ffs(cand) - 1;
    const int src = lane == rank ? pr : (lane == pr ? rank : lane);
    p0 = __shfl_sync(0xffffffffu, p0, src);
    p1 = __shfl_sync(0xffffffffu, p1, src);
    p2 = __shfl_sync(0xffffffffu, p2, src);
    const uint32_t cf = __shfl_sync(0xffffffffu, coef, src);
    const uint32_t inv = c_inv[__shfl_sync(0xffffffffu, cf, rank)];
    uint64_t q0 = __shfl_sync(0xffffffffu, p0, rank);
    uint64_t q1 = __shfl_sync(0xffffffffu, p1, rank);
    uint64_t q2 = __shfl_sync(0xffffffffu, p2, rank);
    gf8_scale64(inv, q0, q1, q2);
    if (lane == rank) {
      p0 = q0;
      p1 = q1;
      p2 = q2;
    } else {
      gf8_scale64(cf, q0, q1, q2);
      p0 ^= q0;
      p1 ^= q1;
      p2 ^= q2;
    }
    used |= 1ull << col;
    ++rank;
  }
  return rank;
}

// Writes the rows of one set: g and the six Gray-step deltas per row.
__device__ __forceinline__ void is_store_set(V6* dst, int lane, int k, uint64_t p0, uint64_t p1,
                                             uint64_t p2) {
  if (lane >= k) return;
  V6* R = dst + size_t(lane) * kIsVecPerRow;
  v6_stg(R, v6_of_planes(p0, p1, p2));
  // (1 + alpha) g, then multiplied by alpha for each next delta
  uint64_t d0 = p0 ^ p2, d1 = p1 ^ p0 ^ p2, d2 = p2 ^ p1;
  for (int v = 0; v < 6; ++v) {
    v6_stg(R + 1 + v, v6_of_planes(d0, d1, d2));
    const uint64_t t = d2;
    d2 = d1;
    d1 = d0 ^ t;
    d0 = t;
  }
}

// Shape of the level-w tasks of one set, n_supports = C(k, w).  Every task
// covers about 7^kIsInner codewords: below level kIsInner + 1 a task walks
// `group` consecutive supports completely; from there on a task is one
// support and one block of the outer coefficients (group = 1).
struct IsTaskShape {
  int inner;                     // Gray-walked coefficients per support
  int outer;                     // coefficients fixed by the task's block
  unsigned long long group;      // supports per task
  unsigned long long per_set;    // tasks per set
};

__device__ __forceinline__ IsTaskShape is_task_shape(unsigned long long n_supports, int w) {
  IsTaskShape s;
  s.inner = min(w - 1, kIsInner);
  s.outer = w - 1 - s.inner;
  if (s.outer > 0) {
    s.group = 1ull;
    s.per_set = n_supports * c_pow7[s.outer];
  } else {
    s.group = c_pow7[kIsInner - s.inner];
    s.per_set = (n_supports + s.group - 1ull) / s.group;
  }
  return s;
}

__device__ __forceinline__ unsigned long long is_tasks_per_set(int k, int w) {
  return is_task_shape(c_binom[k][w], w).per_set;
}

__global__ void __launch_bounds__(kIsPrepWarps * 32) prep_infoset_kernel(DistArgs a) {
  __shared__ uint8_t s_ord[kIsPrepWarps][64];
  const int wl = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kIsPrepWarps + wl;
  if (c >= a.n) return;  // warp-uniform
  const int64_t beg = a.off[c];
  const int64_t klong = a.off[c + 1] - beg;
  // Codes below the threshold, and invalid ones, belong to the other path
  // (which reports bad input).
  int k = (klong >= a.is_min_k && klong <= a.k_max) ? int(klong) : 0;
  const int my = lane < k ? a.idx[beg + lane] : 0;
  if (__any_sync(0xffffffffu, lane < k && (my < 0 || my >= kN))) k = 0;
  if (k == 0) {
    for (int w = lane; w < a.k_max; w += 32) {
      a.is_cnt[size_t(w) * a.n + c] = 0ull;
      a.is_done[size_t(w) * a.n + c] = 0ull;
    }
    return;
  }
  uint64_t o0 = 0ull, o1 = 0ull, o2 = 0ull;
  if (lane < k) {
    for (int j = 0; j < kN; ++j) {
      const uint64_t v = a.tab.M[my * kN + j];
      o0 |= (v & 1ull) << j;
      o1 |= ((v >> 1) & 1ull) << j;
      o2 |= ((v >> 2) & 1ull) << j;
    }
  }
  const int cap_sets = min(kIsMaxSets, kIsMaxRows / k);
  const int full_max = min(cap_sets, kN / k);
  const bool partial_ok = full_max < cap_sets && kN - full_max * k > 0;
  const int ideal = full_max * 64 + (partial_ok ? min(k, kN - full_max * k) : 0);
  int best_score = -1, best_t = 0;
  bool deficient = false;
  for (int t = 0; t < kIsTries; ++t) {
    is_make_order(s_ord[wl], t, lane);
    uint64_t p0 = o0, p1 = o1, p2 = o2, used = 0ull;
    int m = 0, rp = 0;
    while (m < full_max) {
      const int r = is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord[wl]);
      if (r < k) {
        rp = r;
        break;
      }
      ++m;
    }
    if (t == 0 && m == 0) {
      deficient = true;  // dependent rows: some nonzero message gives the zero codeword
      break;
    }
    if (m == full_max && partial_ok) rp = is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord[wl]);
    const int score = m * 64 + rp;
    if (score > best_score) {
      best_score = score;
      best_t = t;
    }
    if (best_score >= ideal) break;
  }
  int n_sets = 0, m_full = 0, delta = 0;
  if (!deficient) {
    is_make_order(s_ord[wl], best_t, lane);
    uint64_t p0 = o0, p1 = o1, p2 = o2, used = 0ull;
    V6* base = a.is_rows + size_t(c) * a.is_stride;
    while (n_sets < cap_sets) {
      const int r = is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord[wl]);
      if (r < k && (r == 0 || k - r > kIsMaxDelta)) break;
      is_store_set(base + size_t(n_sets) * k * kIsVecPerRow, lane, k, p0, p1, p2);
      ++n_sets;
      if (r < k) {
        delta = k - r;
        break;
      }
      ++m_full;
    }
  }
  for (int w = 1 + lane; w <= a.k_max; w += 32) {
    unsigned long long cnt = 0ull;
    if (!deficient && w <= k) cnt = static_cast<unsigned long long>(n_sets) * is_tasks_per_set(k, w);
    a.is_cnt[size_t(w - 1) * a.n + c] = cnt;
    a.is_done[size_t(w - 1) * a.n + c] = 0ull;
  }
  if (lane == 0) {
    CodeDesc d{};
    d.k = k;
    d.R = m_full;
    d.H = n_sets;
    d.n_pat = delta;
    d.tmax = kN - (a.target ? a.target[c] : a.td_default);
    d.flags = kIsCodeFlag | (deficient ? kDecidedFlag : 0);
    d.set_id = c;
    d.n_tasks = 0ull;
    a.desc[c] = d;
    a.out[c] = deficient ? kN : 0;
    a.abort[c] = deficient ? 1 : 0;
    a.is_best[c] = deficient ? 0 : 64;
    a.is_bits[c] = 0u;
    atomicAdd(&a.hdr->ref_messages, double(pow8(k)) - 1.0);
  }
}

// Exclusive scan of the level-major task counts (one CTA of 1024 threads).
__global__ void __launch_bounds__(kScanThreads) scan_levels_kernel(DistArgs a) {
  __shared__ unsigned long long s_part[kScanThreads / 32];
  __shared__ int s_over;
  const int t = threadIdx.x;
  const long long N = static_cast<long long>(a.n) * a.k_max;
  if (t == 0) s_over = 0;
  __syncthreads();
  const long long chunk = (N + kScanThreads - 1) / kScanThreads;
  const long long beg = min(N, t * chunk);
  const long long end = min(N, beg + chunk);
  unsigned long long sum = 0ull;
  bool over = false;
  for (long long i = beg; i < end; ++i) {
    const unsigned long long x = a.is_cnt[i];
    if (sum + x < sum) over = true;
    sum += x;
  }
  const int lane = t & 31, wid = t >> 5;
  unsigned long long incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) {
      if (incl + y < incl) over = true;
      incl += y;
    }
  }
  if (lane == 31) s_part[wid] = incl;
  if (over) s_over = 1;
  __syncthreads();
  if (wid == 0) {
    unsigned long long v = s_part[lane];
    bool ov = false;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) {
        if (v + y < v) ov = true;
        v += y;
      }
    }
    if (ov) s_over = 1;
    s_part[lane] = v;
  }
  __syncthreads();
  unsigned long long run = incl - sum + (wid > 0 ? s_part[wid - 1] : 0ull);
  for (long long i = beg; i < end; ++i) {
    a.is_off[i] = run;
    run += a.is_cnt[i];
  }
  if (t == kScanThreads - 1) {
    a.is_off[N] = s_part[31];
    a.is_hdr->total_tasks = s_part[31];
    a.is_hdr->counter = 0ull;
  }
  __syncthreads();
  if (t == 0 && s_over) {
    // Work beyond 2^64 tasks: nothing runs.
    for (long long i = 0; i <= N; ++i) a.is_off[i] = 0ull;
    a.is_hdr->total_tasks = 0ull;
    report_status(a.hdr, TG_ERR_INVALID_ARGUMENT);
  }
}

// ---------------------------------------------------------------------------
// Walk.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void is_weight(const V6& p, int& wmin) {
  const int lo = __popc(lop3<0xFE>(p.l0, p.l1, p.l2));
  const int hi = __popc(lop3<0xFE>(p.h0, p.h1, p.h2));
  wmin = __viaddmin_s32(lo, hi, wmin);
}

// p <- alpha p on the bit-sliced planes.
__device__ __forceinline__ void v6_alpha(V6& p) {
  uint32_t t = p.l2;
  p.l2 = p.l1;
  p.l1 = p.l0 ^ t;
  p.l0 = t;
  t = p.h2;
  p.h2 = p.h1;
  p.h1 = p.h0 ^ t;
  p.h0 = t;
}

// Delta of the move between 49-codeword blocks b - 1 and b (b >= 1): digit
// 2 + tz moves, tz = trailing base-7 zeros of b.  It runs up when the digits
// above it sum to an even number, between alpha^v and alpha^(v+1).
__device__ __forceinline__ const V6* is_block_move(const V6* rows, unsigned b, uint32_t r2,
                                                  uint32_t r3, uint32_t r4) {
  unsigned q = b;
  int tz = 0;
  while (q % 7u == 0u) {
    q /= 7u;
    ++tz;
  }
  const unsigned ot = q % 7u;
  const int v = ((q / 7u) & 1u) ? int(6u - ot) : int(ot - 1u);
  const uint32_t R = tz == 0 ? r2 : (tz == 1 ? r3 : r4);
  return rows + R + 1 + v;
}

#define TG_IS_STEP(D) \
  v6_xor(cw, D);      \
  is_weight(cw, wmin)
#define TG_IS_SWEEP_UP \
  TG_IS_STEP(d0); TG_IS_STEP(d1); TG_IS_STEP(d2); TG_IS_STEP(d3); TG_IS_STEP(d4); TG_IS_STEP(d5)
#define TG_IS_SWEEP_DOWN \
  TG_IS_STEP(d5); TG_IS_STEP(d4); TG_IS_STEP(d3); TG_IS_STEP(d2); TG_IS_STEP(d1); TG_IS_STEP(d0)

// Walks the 7^inner codewords of one support from cw (every walked
// coefficient alpha^0).  Digit 0 (row r0) and digit 1 (row r1) keep their six
// deltas in registers, so the walk is straight-line code over blocks of 49
// codewords; the one move between blocks (digits 2..4, rows r2..r4) is loaded
// a block ahead.  Rows are vector offsets from `rows`.  Returns the codewords
// evaluated.
__device__ __forceinline__ unsigned long long is_walk_support(V6 cw, int inner, const V6* rows,
                                                              uint32_t r0, uint32_t r1,
                                                              uint32_t r2, uint32_t r3,
                                                              uint32_t r4, int wthr,
                                                              const int32_t* stop, int& wmin) {
  is_weight(cw, wmin);
  if (inner == 0) return 1ull;
  const V6* R0 = rows + r0;
  const V6 d0 = v6_ldg(R0 + 1), d1 = v6_ldg(R0 + 2), d2 = v6_ldg(R0 + 3);
  const V6 d3 = v6_ldg(R0 + 4), d4 = v6_ldg(R0 + 5), d5 = v6_ldg(R0 + 6);
  if (inner == 1) {
    TG_IS_SWEEP_UP;
    return 7ull;
  }
  const V6* R1 = rows + r1;
  const V6 e0 = v6_ldg(R1 + 1), e1 = v6_ldg(R1 + 2), e2 = v6_ldg(R1 + 3);
  const V6 e3 = v6_ldg(R1 + 4), e4 = v6_ldg(R1 + 5), e5 = v6_ldg(R1 + 6);
  const unsigned blocks = static_cast<unsigned>(c_pow7[inner - 2]);
  V6 nx;
  v6_zero(nx);
  if (blocks > 1u) nx = v6_ldg(is_block_move(rows, 1u, r2, r3, r4));
  unsigned b = 0;
  for (; b < blocks; ++b) {
    if (b) {
      TG_IS_STEP(nx);
      if (b + 1u < blocks) nx = v6_ldg(is_block_move(rows, b + 1u, r2, r3, r4));
    }
    // Digit 0 runs up in sweep s of block b when b + s is even; digit 1 runs
    // up through the block when b is even.
    if ((b & 1u) == 0u) {
      TG_IS_SWEEP_UP;   TG_IS_STEP(e0);
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e1);
      TG_IS_SWEEP_UP;   TG_IS_STEP(e2);
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e3);
      TG_IS_SWEEP_UP;   TG_IS_STEP(e4);
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e5);
      TG_IS_SWEEP_UP;
    } else {
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e5);
      TG_IS_SWEEP_UP;   TG_IS_STEP(e4);
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e3);
      TG_IS_SWEEP_UP;   TG_IS_STEP(e2);
      TG_IS_SWEEP_DOWN; TG_IS_STEP(e1);
      TG_IS_SWEEP_UP;   TG_IS_STEP(e0);
      TG_IS_SWEEP_DOWN;
    }
    if (wmin < wthr) break;
    if ((b & 15u) == 15u && ld_flag(stop)) break;
  }
  return 49ull * (min(b, blocks - 1u) + 1u);
}

#undef TG_IS_SWEEP_DOWN
#undef TG_IS_SWEEP_UP
#undef TG_IS_STEP

// One task: its supports walked completely; the smallest weight met, and the
// codewords evaluated in ncw.
__device__ __forceinline__ int is_task(const DistArgs& a,
                                       const unsigned long long (*bn)[kIsBinom], int c, int k,
                                       int w, unsigned long long local, int wthr,
                                       unsigned long long& ncw) {
  const unsigned long long n_sup = bn[k][w];
  const IsTaskShape sh = is_task_shape(n_sup, w);
  const int j = int(local / sh.per_set);
  const unsigned long long rr = local - static_cast<unsigned long long>(j) * sh.per_set;
  const unsigned long long B = c_pow7[sh.outer];
  // supports [s_beg, s_end) of C(k, w) <= C(21, 10) fit 32 bits
  uint32_t s_beg, s_end;
  unsigned long long blk0;
  if (sh.outer > 0) {
    s_beg = uint32_t(rr / B);
    s_end = s_beg + 1u;
    blk0 = rr - static_cast<unsigned long long>(s_beg) * B;
  } else {
    s_beg = uint32_t(rr * sh.group);
    s_end = uint32_t(min(rr * sh.group + sh.group, n_sup));
    blk0 = 0ull;
  }
  const V6* rows = a.is_rows + size_t(c) * a.is_stride + size_t(j) * k * kIsVecPerRow;
  const int32_t* stop = a.abort + c;
  int wmin = 64;
  ncw = 0ull;
  for (uint32_t s = s_beg; s < s_end; ++s) {
    // Support rows from the largest down (combinadic unranking).  The q-th
    // row found is inner digit q while q < inner, then the outer rows from the
    // top block digit down, and last the row with coefficient 1.
    V6 cw;
    v6_zero(cw);
    uint32_t r0 = 0u, r1 = 0u, r2 = 0u, r3 = 0u, r4 = 0u;
    unsigned long long srank = s, blk = blk0;
    unsigned long long P = sh.outer > 0 ? c_pow7[sh.outer - 1] : 1ull;
    int rem = w, q = 0;
    for (int pos = k - 1; pos >= 0 && rem > 0; --pos) {
      const unsigned long long b = bn[pos][rem];
      if (srank < b) continue;
      srank -= b;
      --rem;
      const uint32_t R = uint32_t(pos * kIsVecPerRow);
      V6 g = v6_ldg(rows + R);
      if (q < sh.inner) {
        if (q == 0) r0 = R;
        else if (q == 1) r1 = R;
        else if (q == 2) r2 = R;
        else if (q == 3) r3 = R;
        else r4 = R;
      } else if (rem > 0) {
        const unsigned long long e = blk / P;
        blk -= e * P;
        P /= 7ull;
        for (unsigned long long i = 0; i < e; ++i) v6_alpha(g);
      }
      v6_xor(cw, g);
      ++q;
    }
    ncw += is_walk_support(cw, sh.inner, rows, r0, r1, r2, r3, r4, wthr, stop, wmin);
    if (wmin < wthr) break;
  }
  return wmin;
}

// Marks code c finished and moves the counter past its current level range.
__device__ __forceinline__ void is_finish(const DistArgs& a, int c, unsigned long long range_end) {
  atomicExch(a.abort + c, 1);
  atomicMax(&a.is_hdr->counter, range_end);
}

template <int kTPB, int kMinBlocks>
__global__ void __launch_bounds__(kTPB, kMinBlocks) walk_infoset_kernel(DistArgs a) {
  __shared__ unsigned long long s_binom[kIsBinom][kIsBinom];
  for (int i = threadIdx.x; i < kIsBinom * kIsBinom; i += kTPB)
    s_binom[i / kIsBinom][i % kIsBinom] = c_binom[i / kIsBinom][i % kIsBinom];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned long long total = a.is_hdr->total_tasks;
  const int NW = a.n * a.k_max;
  unsigned long long evaluated = 0ull;
  for (;;) {
    unsigned long long base = 0ull;
    if (lane == 0) base = atomicAdd(&a.is_hdr->counter, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    int f0 = 0;
    if (lane == 0) f0 = last_le(a.is_off, NW + 1, base);
    f0 = __shfl_sync(0xffffffffu, f0, 0);
    const unsigned long long t = base + lane;
    if (t >= total) continue;
    const int f = t < __ldg(a.is_off + f0 + 1) ? f0 : last_le(a.is_off, NW + 1, t);
    const int w = f / a.n + 1;
    const int c = f - (w - 1) * a.n;
    const unsigned long long r_beg = __ldg(a.is_off + f), r_end = __ldg(a.is_off + f + 1);
    if (ld_flag(a.abort + c)) {
      atomicMax(&a.is_hdr->counter, r_end);
      continue;
    }
    const int wthr = kN - a.desc[c].tmax;
    unsigned long long ncw = 0ull;
    const int wmin = is_task(a, s_binom, c, a.desc[c].k, w, t - r_beg, wthr, ncw);
    evaluated += ncw;
    const int best = min(atomicMin(a.is_best + c, wmin), wmin);
    if (best < wthr) {
      is_finish(a, c, r_end);  // a witness below the target distance
      continue;
    }
    __threadfence();
    if (atomicAdd(a.is_done + f, 1ull) + 1ull == __ldg(a.is_cnt + f)) {
      // The last task of level w: check the bound of the complete levels.
      const unsigned bit = 1u << (w - 1);
      const unsigned bits = atomicOr(a.is_bits + c, bit) | bit;
      const int L = __ffs(~bits) - 1;
      const int now = atomicAdd(a.is_best + c, 0);
      const CodeDesc d = a.desc[c];
      const int bound = d.R * (L + 1) + (d.n_pat > 0 ? max(0, L + 1 - d.n_pat) : 0);
      if (L >= d.k || now <= bound) is_finish(a, c, r_end);
    }
  }
  // codewords evaluated, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
  if (lane == 0 && evaluated) atomicAdd(&a.is_hdr->codewords, evaluated);
}

__global__ void finalize_infoset_kernel(DistArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  const CodeDesc d = a.desc[c];
  if ((d.flags & kIsCodeFlag) == 0 || (d.flags & kDecidedFlag) != 0) return;
  a.out[c] = kN - a.is_best[c];
}

}  // namespace tg
