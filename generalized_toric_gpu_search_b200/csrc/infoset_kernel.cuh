// Information-set enumeration of max_zeros (Brouwer-Zimmermann).  Included by
// distance.cu, whose GF(8) tables, descriptors and helpers it shares.
//
// max_zeros = 49 - d, d the minimum weight of a nonzero codeword.  Gauss-Jordan
// elimination on an information set I (k columns of rank k) gives a generator
// of the code that is the identity on I, so a codeword c = u G equals the
// message u on I.  Level w enumerates the projective messages of weight
// exactly w.  After levels 1..L every codeword not yet seen weighs at least
//   * ceil(49 (L + 1) / k) for a toric code, from one set: the torus
//     translations permute the 49 columns regularly and map the code onto
//     itself, so every translate of I is an information set too, and each
//     column lies in exactly k of the 49 translates;
//   * m (L + 1) + max(0, L + 1 - delta) for any other matrix, from pairwise
//     disjoint sets I_1..I_s found by greedy elimination over column orders
//     (m full sets, and possibly a last one of rank k - delta).
// A code is finished when its best weight is <= that bound (the best weight
// is then d), when all k levels are complete, or when a weight below the
// target distance appears (the early-exit decision).  One lane holds one row,
// bit-sliced over the 49 columns, so a pivot step is a ballot, a row swap and
// one broadcast; each set's columns are reordered with the pivots last (in
// the high word).
//
// Levels 1 to 3 run as one launch (levels123_kernel, one CTA per set).  From
// level 4 on, each level runs in two parts (supports with the set's last row,
// then the rest), each a launch triple: plan_level_kernel finishes the codes
// whose bound is met and sizes the part for the others, scan_level_kernel
// picks the task size and the offsets, and walk_level_kernel hands the tasks
// to a persistent grid.  No code starts a part before the previous one is
// complete, so no work is spent on parts a code turns out not to need.
//
// Walk.  A support of w rows has its last row at coefficient 1.  A block is 49
// codewords: digit 0 swept through its 7 multiples, digit 1 stepping
// alpha^0..alpha^6 between the sweeps; digits 2.. follow a reflected base-7
// Gray code over the blocks, whose start state has a closed form, so a task
// (a range of blocks) may start anywhere.  The zeros of a sweep's 7 codewords
// on the 32 low columns are one-LOP3 selections in the domain W = P / g; a
// threshold test on them (single counts, or pairs of codewords at high
// thresholds) sends the rare sweep that may hold a lighter codeword to an
// exact count.
#pragma once

namespace tg {

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

// Move masks of a bit compress (gather the bits of x selected by m to the low
// end, in order): six rounds, round i shifting some bits right by 2^i (the
// parallel-suffix method of Hacker's Delight, 7-4).  They depend on m only.
struct IsCompress {
  uint64_t m;
  uint64_t mv[6];
};

__device__ __forceinline__ IsCompress is_compress_masks(uint64_t m) {
  IsCompress c;
  c.m = m;
  uint64_t mk = ~m << 1;  // the zeros of m to the right of each bit
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    uint64_t mp = mk ^ (mk << 1);  // parity of those zeros, by a prefix XOR
    mp ^= mp << 2;
    mp ^= mp << 4;
    mp ^= mp << 8;
    mp ^= mp << 16;
    mp ^= mp << 32;
    const uint64_t mv = mp & m;  // bits that move by 2^i this round
    c.mv[i] = mv;
    m = (m ^ mv) | (mv >> (1 << i));
    mk &= ~mp;
  }
  return c;
}

__device__ __forceinline__ uint64_t is_compress(uint64_t x, const IsCompress& c) {
  x &= c.m;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const uint64_t t = x & c.mv[i];
    x = (x ^ t) | (t >> (1 << i));
  }
  return x;
}

// Reorders the 49 columns of a bit-sliced row: the columns outside `piv`
// first (increasing), then those in `piv`.  Weights do not depend on the
// column order, and a set's codewords are sparse on its own pivot columns;
// with those last, the low 32 columns look like random columns, so the walk's
// low-half weight bound is tight.
__device__ __forceinline__ void is_reorder_columns(uint64_t piv, uint64_t& p0, uint64_t& p1,
                                                   uint64_t& p2) {
  // The non-pivot columns in increasing order, then the pivot columns.
  const uint64_t rest = ~piv & kMask49;
  const IsCompress cr = is_compress_masks(rest);
  const IsCompress cp = is_compress_masks(piv & kMask49);
  const int nr = __popcll(rest);
  p0 = is_compress(p0, cr) | (is_compress(p0, cp) << nr);
  p1 = is_compress(p1, cr) | (is_compress(p1, cp) << nr);
  p2 = is_compress(p2, cr) | (is_compress(p2, cp) << nr);
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
  if (k == 0) return;
  uint64_t o0 = 0ull, o1 = 0ull, o2 = 0ull;
  if (lane < k) {
    o0 = __ldg(a.tab.Mp + my * 3);
    o1 = __ldg(a.tab.Mp + my * 3 + 1);
    o2 = __ldg(a.tab.Mp + my * 3 + 2);
  }
  V6* base = a.is_rows + size_t(c) * a.is_stride;
  bool deficient = false;
  int n_sets = 0, m_full = 0, delta = 0;
  int32_t flags = kIsCodeFlag;
  if (a.is_toric) {
    // One information set, the first k independent columns: the torus
    // translations act regularly on the columns and map the code onto
    // itself, so E's 49 translates are information sets whose light
    // codewords are shifted copies of E's (with the same weights).  After
    // levels 1..L on E alone, a codeword not seen has weight >= L + 1 on every
    // translate, and each column lies in k of them: k wt >= 49 (L + 1).
    is_make_order(s_ord[wl], 0, lane);
    uint64_t p0 = o0, p1 = o1, p2 = o2, used = 0ull;
    if (is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord[wl]) < k) {
      deficient = true;  // dependent rows: some nonzero message gives the zero codeword
    } else {
      is_reorder_columns(used, p0, p1, p2);
      is_store_set(base, lane, k, p0, p1, p2);
      if (a.is_piv && lane == 0) a.is_piv[size_t(c) * kIsMaxSets] = used;
      n_sets = 1;
      m_full = 1;
      flags |= kTorusBoundFlag;
    }
  } else {
    // Disjoint information sets, greedily along a column order: the identity
    // and up to kIsTries - 1 shuffles, keeping the most full sets and then the
    // largest partial rank.
    const int cap_sets = min(kIsMaxSets, kIsMaxRows / k);
    const int full_max = min(cap_sets, kN / k);
    const bool partial_ok = full_max < cap_sets && kN - full_max * k > 0;
    const int ideal = full_max * 64 + (partial_ok ? min(k, kN - full_max * k) : 0);
    int best_score = -1, best_t = 0;
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
    if (!deficient) {
      is_make_order(s_ord[wl], best_t, lane);
      uint64_t p0 = o0, p1 = o1, p2 = o2, used = 0ull;
      while (n_sets < cap_sets) {
        const uint64_t used_before = used;
        const int r = is_gauss_jordan(lane, k, p0, p1, p2, used, s_ord[wl]);
        if (r < k && (r == 0 || k - r > kIsMaxDelta)) break;
        uint64_t q0 = p0, q1 = p1, q2 = p2;
        is_reorder_columns(used & ~used_before, q0, q1, q2);
        is_store_set(base + size_t(n_sets) * k * kIsVecPerRow, lane, k, q0, q1, q2);
        if (a.is_piv && lane == 0) a.is_piv[size_t(c) * kIsMaxSets + n_sets] = used & ~used_before;
        ++n_sets;
        if (r < k) {
          delta = k - r;
          break;
        }
        ++m_full;
      }
    }
  }
  if (lane == 0) {
    CodeDesc d{};
    d.k = k;
    d.R = m_full;
    d.H = n_sets;
    d.n_pat = delta;
    d.tmax = kN - (a.target ? a.target[c] : a.td_default);
    d.flags = flags | (deficient ? kDecidedFlag : 0);
    d.set_id = c;
    d.n_tasks = 0ull;
    a.desc[c] = d;
    a.out[c] = deficient ? kN : 0;
    a.abort[c] = deficient ? 1 : 0;
    a.is_best[c] = deficient ? 0 : 64;
    atomicAdd(&a.hdr->ref_messages, double(pow8(k)) - 1.0);
  }
}

// ---------------------------------------------------------------------------
// One level at a time: plan (which codes go on, how many units each), scan
// (task size and offsets), walk.  Units are 49-codeword Gray blocks of one
// support (whole supports of 1 or 7 codewords at levels 1 and 2).
// ---------------------------------------------------------------------------

// Units of one support at level w.
__device__ __forceinline__ unsigned long long is_units_per_support(int w) {
  return w >= 3 ? c_pow7[w - 3] : 1ull;
}

// Most units a task takes at level w (about 16807 codewords).
__device__ __forceinline__ unsigned long long is_max_task_units(int w) {
  return w >= 3 ? 343ull : (w == 2 ? 2401ull : 16807ull);
}

// Orders the codes by k for the level walks (is_perm: position -> code).
// Tasks are numbered over positions, so where a warp's 32 tasks span two
// codes those have the same k, the same loop lengths and, mostly, the same
// threshold mode (in batch order, a batch of 10,000 sets with k from 6 to 14
// ran 3 % slower).  One CTA;
// the order within a k is that of the atomics (it changes no result).
__global__ void __launch_bounds__(kScanThreads) order_codes_kernel(DistArgs a) {
  __shared__ int s_cnt[kIsBinom + 1];
  const int t = threadIdx.x;
  for (int i = t; i <= kIsBinom; i += kScanThreads) s_cnt[i] = 0;
  __syncthreads();
  for (int c = t; c < a.n; c += kScanThreads)
    atomicAdd(&s_cnt[max(0, min(a.desc[c].k, kIsBinom))], 1);
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int i = 0; i <= kIsBinom; ++i) {
      const int x = s_cnt[i];
      s_cnt[i] = run;
      run += x;
    }
  }
  __syncthreads();
  for (int c = t; c < a.n; c += kScanThreads)
    a.is_perm[atomicAdd(&s_cnt[max(0, min(a.desc[c].k, kIsBinom))], 1)] = c;
}

// Level w of a toric code runs in two parts.  Part 1 takes the supports that
// hold the last row (index k - 1): C(k-1, w-1) of them, support ranks
// C(k-1, w) .. C(k, w) - 1.  Part 2 takes the others: C(k-1, w), ranks
// 0 .. C(k-1, w) - 1.  Let e be the pivot column of row k - 1.  A codeword c
// not met by levels 1..w-1 and part 1 weighs at least w on every translate
// E + t of the information set, and w + 1 on each translate whose
// restriction of c holds e + t (had it weighed w there, its shift by t
// would be a part-1 message).  Those are the wt(c) translates with e + t in
// the support of c, so k wt >= 49 w + wt, i.e.
//   wt >= ceil(49 w / (k - 1))   after part 1,
// against ceil(49 w / k) before it and ceil(49 (w + 1) / k) after part 2.
// Any other code walks its whole level in part 1 and nothing in part 2.
__device__ __forceinline__ bool is_split_level(int32_t flags) {
  return (flags & kTorusBoundFlag) != 0;
}

// Supports of part `part` of level w of a k-row code: their count and the
// rank of the first.
__device__ __forceinline__ void is_part_supports(int32_t flags, int k, int w, int part,
                                                 const unsigned long long (*bn)[kIsBinom],
                                                 unsigned long long& n_sup,
                                                 unsigned long long& s_off) {
  if (!is_split_level(flags)) {
    n_sup = part == 1 ? bn[k][w] : 0ull;
    s_off = 0ull;
  } else if (part == 1) {
    n_sup = bn[k - 1][w - 1];
    s_off = bn[k - 1][w];
  } else {
    n_sup = bn[k - 1][w];
    s_off = 0ull;
  }
}

// Decides, with everything before part `part` (1 or 2) of level w complete,
// whether each code is finished, and the units of that part for the others.
__global__ void plan_level_kernel(DistArgs a, int w, int part) {
  // One thread per code position (is_perm order): the units are written by
  // position, so the scan and the walk read them in their own order.
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = p < a.n ? __ldg(a.is_perm + p) : 0;
  unsigned long long units = 0ull;
  const CodeDesc d = p < a.n ? a.desc[c] : CodeDesc{};
  if (p < a.n && (d.flags & kIsCodeFlag) != 0 && (d.flags & kDecidedFlag) == 0 &&
      a.abort[c] == 0 && (part == 1 || is_split_level(d.flags))) {
    const int best = a.is_best[c];
    bool done = w > d.k || best < kN - d.tmax;  // every message seen, or a witness
    if (!done) {
      int bound;
      if (!is_split_level(d.flags)) {
        const int L = w - 1;
        bound = d.R * (L + 1) + (d.n_pat > 0 ? max(0, L + 1 - d.n_pat) : 0);
      } else if (part == 1) {
        bound = (kN * w + d.k - 1) / d.k;
      } else {
        bound = (kN * w + d.k - 2) / (d.k - 1);  // w <= k, so k >= 4 here
      }
      done = best <= bound;
    }
    if (done) {
      a.abort[c] = 1;  // exact (bound met or every message seen), or a witness
    } else {
      unsigned long long n_sup, s_off;
      is_part_supports(d.flags, d.k, w, part, c_binom, n_sup, s_off);
      units = static_cast<unsigned long long>(d.H) * n_sup * is_units_per_support(w);
    }
  }
  if (p < a.n) a.is_units[p] = units;
  // Lets scan_level_kernel and walk_level_kernel skip a part no set needs.
  if (__any_sync(0xffffffffu, units != 0ull) && (threadIdx.x & 31) == 0) a.is_hdr->work = 1;
}

// Task size of level w (units per task, sized so the level has about eight
// tasks per resident thread) and the task offsets of the code positions (the
// codes in is_perm order).  One CTA.
__global__ void __launch_bounds__(kScanThreads) scan_level_kernel(DistArgs a, int w) {
  __shared__ unsigned long long s_part[kScanThreads / 32];
  __shared__ unsigned long long s_nb;
  __shared__ int s_over;
  const int t = threadIdx.x;
  const int lane = t & 31, wid = t >> 5;
  const int n = a.n;
  if (a.is_hdr->work == 0) {  // written by plan_level_kernel; the same for every thread
    if (t == 0) {
      a.is_hdr->counter = 0ull;
      a.is_hdr->total = 0ull;
      a.is_hdr->units = 1ull;
      a.is_hdr->level = w;
    }
    return;
  }
  if (t == 0) s_over = 0;
  __syncthreads();
  const int chunk = (n + kScanThreads - 1) / kScanThreads;
  const int beg = min(n, t * chunk);
  const int end = min(n, beg + chunk);
  // pass 1: total units
  unsigned long long sum = 0ull;
  bool over = false;
  for (int i = beg; i < end; ++i) {
    const unsigned long long x = a.is_units[i];
    if (sum + x < sum) over = true;
    sum += x;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, sum, o);
    if (sum + y < sum) over = true;
    sum += y;
  }
  if (lane == 0) s_part[wid] = sum;
  if (over) s_over = 1;
  __syncthreads();
  if (t == 0) {
    unsigned long long tot = 0ull;
    for (int i = 0; i < kScanThreads / 32; ++i) {
      if (tot + s_part[i] < tot) s_over = 1;
      tot += s_part[i];
    }
    const unsigned long long target = static_cast<unsigned long long>(a.is_tasks_per_thread) *
                                      static_cast<unsigned long long>(a.is_lanes);
    unsigned long long nb = (tot + target - 1ull) / target;
    // the largest task: the tunable limit from level 3 on (49 by default)
    nb = max(1ull, min(nb, w >= 3 ? static_cast<unsigned long long>(a.is_max_task_units)
                                  : is_max_task_units(w)));
    // Align tasks with supports (units per support is a power of 7): whole
    // supports, or the power of 7 dividing one that is nearest on a log
    // scale, so the lanes of a warp walk equal block counts.
    const unsigned long long bps = is_units_per_support(w);
    if (bps > 1ull) {
      if (nb >= bps) {
        nb = (nb / bps) * bps;
      } else {
        unsigned long long p7 = 1ull;
        while (p7 * 7ull <= nb) p7 *= 7ull;
        // 7 p7 when nb > sqrt(7) p7 (nb^2 > 7 p7^2); 7 p7 <= bps here
        nb = (nb * nb > 7ull * p7 * p7) ? 7ull * p7 : p7;
      }
    }
    s_nb = nb;
  }
  __syncthreads();
  const unsigned long long nb = s_nb;
  // pass 2: tasks per code, exclusive scan
  unsigned long long tsum = 0ull;
  for (int i = beg; i < end; ++i) tsum += (a.is_units[i] + nb - 1ull) / nb;
  unsigned long long incl = tsum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();
  if (lane == 31) s_part[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    unsigned long long v = s_part[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    s_part[lane] = v;
  }
  __syncthreads();
  unsigned long long run = incl - tsum + (wid > 0 ? s_part[wid - 1] : 0ull);
  for (int i = beg; i < end; ++i) {
    a.is_off[i] = run;
    run += (a.is_units[i] + nb - 1ull) / nb;
  }
  __syncthreads();
  if (t == 0) {
    unsigned long long total = s_part[31];
    if (s_over) {
      // Work beyond 2^64 units: nothing runs.
      for (int i = 0; i <= n; ++i) a.is_off[i] = 0ull;
      total = 0ull;
      report_status(a.hdr, TG_ERR_INVALID_ARGUMENT);
    }
    a.is_off[n] = total;
    a.is_hdr->counter = 0ull;
    a.is_hdr->total = total;
    a.is_hdr->units = nb;
    a.is_hdr->level = w;
    a.is_hdr->tasks_all += total;
    a.is_hdr->work = 0;  // every thread read it before the first barrier
  }
}

// p <- alpha^e p on the bit-sliced planes, e in 0..6.
__device__ __forceinline__ void v6_alpha_pow(V6& p, int e) {
  for (int i = 0; i < e; ++i) {
    uint32_t t = p.l2;
    p.l2 = p.l1;
    p.l1 = p.l0 ^ t;
    p.l0 = t;
    t = p.h2;
    p.h2 = p.h1;
    p.h1 = p.h0 ^ t;
    p.h0 = t;
  }
}

// Gray value of digit 2 + i at the start of block b: the base-7 digit o_i of
// b, reflected (6 - o_i) when the digits above it sum to an odd number.
__device__ __forceinline__ int is_block_digit(unsigned long long& rest) {
  int o;
  if ((rest >> 32) == 0ull) {  // 32-bit arithmetic whenever it fits (w <= 14)
    const uint32_t r = uint32_t(rest);
    o = int(r % 7u);
    rest = r / 7u;
  } else {
    o = int(rest % 7ull);
    rest /= 7ull;
  }
  return (rest & 1ull) ? 6 - o : o;
}

// Delta of the move from block b - 1 to block b (b >= 1): digit 2 + tz moves,
// tz = trailing base-7 zeros of b, up when the digits above it sum to an even
// number, between alpha^v and alpha^(v+1).  dig[i * kStride] is the row of
// digit 2 + i.
template <int kStride>
__device__ __forceinline__ const V6* is_block_move(const V6* rows, const uint16_t* dig,
                                                  unsigned long long b) {
  int tz = 0;
  while (b % 7ull == 0ull) {
    b /= 7ull;
    ++tz;
  }
  const int ot = int(b % 7ull);
  const int v = ((b / 7ull) & 1ull) ? 6 - ot : ot - 1;
  return rows + dig[tz * kStride] + 1 + v;
}

// Where the witness pass records a codeword of one code: the pivot columns of
// the information set it was found on, the code's 49-symbol output row and
// its claim word (first writer wins).
struct WitOut {
  const uint64_t* piv;
  uint8_t* dst;
  int32_t* lock;
};

// Records a codeword, given in its information set's column order (positions
// 0..31 in the lo words, 32..48 in bits 0..16 of the hi words), as the code's
// witness in the original column order: the set's non-pivot columns first
// (increasing), then its pivots, as prep_infoset_kernel ordered them.  Only
// the first caller per code writes, so the row is never torn; its claim word
// takes the codeword's weight + 1, the value the pass reports (lanes of other
// warps may meet lighter codewords in the same round).
__device__ __noinline__ void is_put_witness(WitOut wo, uint32_t l0, uint32_t l1, uint32_t l2,
                                            uint32_t h0, uint32_t h1, uint32_t h2) {
  const int wt = __popc(l0 | l1 | l2) + __popc((h0 | h1 | h2) & kHiMask);
  if (atomicCAS(wo.lock, 0, wt + 1) != 0) return;
  const uint64_t piv = *wo.piv & kMask49;
  const uint64_t q0 = uint64_t(l0) | (uint64_t(h0 & kHiMask) << 32);
  const uint64_t q1 = uint64_t(l1) | (uint64_t(h1 & kHiMask) << 32);
  const uint64_t q2 = uint64_t(l2) | (uint64_t(h2 & kHiMask) << 32);
  uint64_t rest = ~piv & kMask49, tail = piv;
  for (int d = 0; d < kN; ++d) {
    const bool front = rest != 0ull;
    const uint64_t pick = front ? rest : tail;
    const int col = __ffsll(static_cast<long long>(pick)) - 1;
    if (front) rest &= rest - 1ull;
    else tail &= tail - 1ull;
    wo.dst[col] = uint8_t(((q0 >> d) & 1ull) | (((q1 >> d) & 1ull) << 1) |
                          (((q2 >> d) & 1ull) << 2));
  }
}

// is_sweep_exact of the witness pass: also records the first codeword
// lighter than wthr.
__device__ __noinline__ int is_sweep_exact_w(V6 P, const V6* g_row, int wmin, WitOut wo,
                                             int wthr) {
  V6 g = v6_ldg(g_row);
  for (int v = 0; v < 7; ++v) {
    const uint32_t x0 = P.l0 ^ g.l0, x1 = P.l1 ^ g.l1, x2 = P.l2 ^ g.l2;
    const uint32_t y0 = P.h0 ^ g.h0, y1 = P.h1 ^ g.h1, y2 = P.h2 ^ g.h2;
    const int wt = __popc(lop3<0xFE>(x0, x1, x2)) + __popc(lop3<0xFE>(y0, y1, y2));
    if (wt < wthr) is_put_witness(wo, x0, x1, x2, y0, y1, y2);
    wmin = min(wmin, wt);
    v6_alpha_pow(g, 1);
  }
  return wmin;
}

// Exact weights of the seven codewords P + alpha^v g, v = 0..6, min'd into
// wmin (kCG: g_row may have been written during the kernel, so it is read
// through L2 only).
template <bool kCG>
__device__ __noinline__ int is_sweep_exact(V6 P, const V6* g_row, int wmin) {
  V6 g = v6_load<kCG>(g_row);
  for (int v = 0; v < 7; ++v) {
    const int lo = __popc(lop3<0xFE>(P.l0 ^ g.l0, P.l1 ^ g.l1, P.l2 ^ g.l2));
    const int hi = __popc(lop3<0xFE>(P.h0 ^ g.h0, P.h1 ^ g.h1, P.h2 ^ g.h2));
    wmin = min(wmin, lo + hi);
    v6_alpha_pow(g, 1);
  }
  return wmin;
}

// Three bit planes of 32 columns of GF(8) values.
struct Pl3 {
  uint32_t x0, x1, x2;
};

// Column-wise product modulo x^3 + x + 1.
__device__ __forceinline__ Pl3 pl3_mul(const Pl3& a, const Pl3& b) {
  const uint32_t t0 = a.x0 & b.x0;
  const uint32_t t1 = lop3<0x6A>(a.x0, b.x1, a.x1 & b.x0);  // (a & b) ^ c
  const uint32_t t2 = lop3<0x6A>(a.x0, b.x2, lop3<0x6A>(a.x1, b.x1, a.x2 & b.x0));
  const uint32_t t3 = lop3<0x6A>(a.x1, b.x2, a.x2 & b.x1);
  const uint32_t t4 = a.x2 & b.x2;
  return Pl3{t0 ^ t3, lop3<0x96>(t1, t3, t4), t2 ^ t4};
}

// Column-wise inverse x^6 = x^2 x^4 (0 stays 0); squaring is linear.
__device__ __forceinline__ Pl3 pl3_inv(const Pl3& a) {
  const Pl3 s2{a.x0, a.x2, a.x1 ^ a.x2};
  const Pl3 s4{s2.x0, s2.x2, s2.x1 ^ s2.x2};
  return pl3_mul(s2, s4);
}

__device__ __forceinline__ Pl3 pl3_lo(const V6& v) { return Pl3{v.l0, v.l1, v.l2}; }

__device__ __forceinline__ Pl3 pl3_and(const Pl3& a, uint32_t m) {
  return Pl3{a.x0 & m, a.x1 & m, a.x2 & m};
}

__device__ __forceinline__ void pl3_xor(Pl3& a, const Pl3& b) {
  a.x0 ^= b.x0;
  a.x1 ^= b.x1;
  a.x2 ^= b.x2;
}

// c x for a constant c of GF(8), on three bit planes (x0, x1, x2) of 32
// columns; folds to a few XORs when c is known at compile time.
__device__ __forceinline__ void gf8_scale32(uint32_t c, uint32_t& x0, uint32_t& x1, uint32_t& x2) {
  uint32_t r0 = 0u, r1 = 0u, r2 = 0u;
  uint32_t a0 = x0, a1 = x1, a2 = x2;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if ((c >> b) & 1u) {
      r0 ^= a0;
      r1 ^= a1;
      r2 ^= a2;
    }
    const uint32_t t = a2;  // a <- alpha a
    a2 = a1;
    a1 = a0 ^ t;
    a0 = t;
  }
  x0 = r0;
  x1 = r1;
  x2 = r2;
}

// The rare path of a sweep whose lower bound reaches below wmin: exact
// weights of its seven codewords P + alpha^v g.  The low half comes from the
// sweep's zero counts z[v] (plus zz, the zeros on g's zero columns); the high
// half is rebuilt from Ph, P's high word without digit 1's term, plus kC r1
// (kC = digit 1's coefficient in this sweep).
// Witness pass: rebuilds the codeword P + alpha^v g of a sweep from its W
// domain state and records it.  The low columns of P are W g where g is
// nonzero and Pz where g is zero; its high word is ph (digit 1's term
// included); gh is the high word of alpha^v g.
__device__ __noinline__ void is_sweep_witness(Pl3 W, Pl3 Pz, const V6* g_row, int v,
                                              uint32_t ph0, uint32_t ph1, uint32_t ph2,
                                              uint32_t gh0, uint32_t gh1, uint32_t gh2,
                                              WitOut wo) {
  Pl3 gl = pl3_lo(v6_ldg(g_row));
  Pl3 P = pl3_mul(W, gl);
  P.x0 |= Pz.x0;
  P.x1 |= Pz.x1;
  P.x2 |= Pz.x2;
  for (int i = 0; i < v; ++i) gl = Pl3{gl.x2, gl.x0 ^ gl.x2, gl.x1};  // alpha gl
  is_put_witness(wo, P.x0 ^ gl.x0, P.x1 ^ gl.x1, P.x2 ^ gl.x2, ph0 ^ gh0, ph1 ^ gh1, ph2 ^ gh2);
}

template <bool kW, bool kCG>
__device__ __forceinline__ int is_sweep_fix(uint32_t kC, const int (&z)[7], int zz, uint32_t ph0,
                                            uint32_t ph1, uint32_t ph2, const V6* g_row,
                                            const V6* r1_row, int wmin, const Pl3& W,
                                            const Pl3& Pz, WitOut wo, int wthr) {
  uint32_t d0 = ld_u32<kCG>(&r1_row->h0), d1 = ld_u32<kCG>(&r1_row->h1),
           d2 = ld_u32<kCG>(&r1_row->h2);
  gf8_scale32(kC, d0, d1, d2);
  ph0 ^= d0;
  ph1 ^= d1;
  ph2 ^= d2;
  uint32_t g0 = ld_u32<kCG>(&g_row->h0), g1 = ld_u32<kCG>(&g_row->h1),
           g2 = ld_u32<kCG>(&g_row->h2);
  const int lo_base = 32 - zz;
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    const int hi = __popc(lop3<0xFE>(ph0 ^ g0, ph1 ^ g1, ph2 ^ g2));
    const int wt = lo_base - z[v] + hi;
    if (kW && wt < wthr) is_sweep_witness(W, Pz, g_row, v, ph0, ph1, ph2, g0, g1, g2, wo);
    wmin = min(wmin, wt);
    const uint32_t t = g2;  // g <- alpha g
    g2 = g1;
    g1 = g0 ^ t;
    g0 = t;
  }
  return wmin;
}

// One sweep of digit 0, on the low 32 columns in the domain W = P / g
// (column-wise; g the digit-0 row): P + alpha^v g vanishes at column j
// exactly when W_j = alpha^v (g_j != 0) or P_j = 0 (g_j = 0).  So the zeros
// of all seven codewords are seven one-LOP3 selections plus the zero columns
// of g (tracked as Pz = P & gz: ngz less its nonzero columns).  The high
// columns weigh at least hb, so only a sweep with more than thr = 32 + hb -
// wmin low zeros can hold a codeword lighter than wmin; that sweep is counted
// exactly (kC: digit 1's coefficient in this sweep).  thz = thr - ngz is the
// test on the selection count less Pz's nonzero columns.
#define TG_IS_ZCOUNTS(z_)                                                                        \
  int z_[7];                                                                                     \
  z_[0] = __popc(lop3<sel_lut(1)>(W.x0, W.x1, W.x2));                                            \
  z_[1] = __popc(lop3<sel_lut(2)>(W.x0, W.x1, W.x2));                                            \
  z_[2] = __popc(lop3<sel_lut(4)>(W.x0, W.x1, W.x2));                                            \
  z_[3] = __popc(lop3<sel_lut(3)>(W.x0, W.x1, W.x2));                                            \
  z_[4] = __popc(lop3<sel_lut(6)>(W.x0, W.x1, W.x2));                                            \
  z_[5] = __popc(lop3<sel_lut(7)>(W.x0, W.x1, W.x2));                                            \
  z_[6] = __popc(lop3<sel_lut(5)>(W.x0, W.x1, W.x2));
// Sweep S of a block (digit 1 at alpha^S, alpha^0..6 = 1, 2, 4, 3, 6, 7, 5 =
// kC): a sweep that may hold a codeword lighter than wmin is counted exactly
// on the spot.  This form serves low thresholds, where that happens often.
#define TG_IS_SWEEP1(S, kC)                                                                      \
  {                                                                                              \
    TG_IS_ZCOUNTS(z_)                                                                            \
    const int pz_ = __popc(lop3<0xFE>(Pz.x0, Pz.x1, Pz.x2));                                    \
    const int zm_ = __vimax3_s32(__vimax3_s32(z_[0], z_[1], z_[2]),                              \
                                 __vimax3_s32(z_[3], z_[4], z_[5]), z_[6]) - pz_;                \
    if (__builtin_expect(zm_ > thz, 0)) {                                                        \
      wmin = is_sweep_fix<kW, kCG>(kC, z_, ngz - pz_, qh0, qh1, qh2, rows + r0, rows + r1, wmin, \
                                   W, Pz, wo, wthr);                                             \
      thz = thz_base - wmin;                                                                     \
    }                                                                                            \
  }
// The same single-count test with the flagged sweeps counted after the
// block (bit S of fl), so the block is one stretch of straight-line code.
#define TG_IS_SWEEP1F(S)                                                                         \
  {                                                                                              \
    TG_IS_ZCOUNTS(z_)                                                                            \
    const int pz_ = __popc(lop3<0xFE>(Pz.x0, Pz.x1, Pz.x2));                                    \
    const int zm_ = __vimax3_s32(__vimax3_s32(z_[0], z_[1], z_[2]),                              \
                                 __vimax3_s32(z_[3], z_[4], z_[5]), z_[6]) - pz_;                \
    fl |= zm_ > thz ? (1u << (S)) : 0u;                                                          \
  }
// The same test on pairs of codewords: the selections of alpha^0|alpha^1,
// alpha^2|alpha^3 and alpha^4|alpha^5 are disjoint, so each pair's count
// bounds both of its codewords' zeros; four counts instead of seven.  Used at
// high thresholds, where flags are rare: bit S of fl marks the sweep, and the
// block's flagged sweeps are counted after it, so the seven sweeps are one
// stretch of straight-line code.
#define TG_IS_SWEEP2(S)                                                                          \
  {                                                                                              \
    const int y0_ = __popc(lop3<sel_lut(1) | sel_lut(2)>(W.x0, W.x1, W.x2));                     \
    const int y1_ = __popc(lop3<sel_lut(4) | sel_lut(3)>(W.x0, W.x1, W.x2));                     \
    const int y2_ = __popc(lop3<sel_lut(6) | sel_lut(7)>(W.x0, W.x1, W.x2));                     \
    const int y3_ = __popc(lop3<sel_lut(5)>(W.x0, W.x1, W.x2));                                  \
    const int pz_ = __popc(lop3<0xFE>(Pz.x0, Pz.x1, Pz.x2));                                    \
    const int ym_ = __vimax3_s32(y0_, y1_, max(y2_, y3_)) - pz_;                                 \
    fl |= ym_ > thz ? (1u << (S)) : 0u;                                                          \
  }
#define TG_IS_MOVE(I)                                                        \
  {                                                                          \
    W.x0 ^= ez[(6 * (I) + 0) * kStride];                                     \
    W.x1 ^= ez[(6 * (I) + 1) * kStride];                                     \
    W.x2 ^= ez[(6 * (I) + 2) * kStride];                                     \
    Pz.x0 ^= ez[(6 * (I) + 3) * kStride];                                    \
    Pz.x1 ^= ez[(6 * (I) + 4) * kStride];                                    \
    Pz.x2 ^= ez[(6 * (I) + 5) * kStride];                                    \
  }

// The rare path of a block: the sweeps flagged in fl are counted exactly.
// W and Pz are the state of sweep 6; stepping back through digit 1's moves
// (ez, stride kStride) gives each earlier sweep's.  Sweep s has digit 1 at
// alpha^s (alpha^0..6 = 1, 2, 4, 3, 6, 7, 5, packed in nibbles).
template <int kStride, bool kW, bool kCG>
__device__ __forceinline__ int is_block_fix(unsigned fl, Pl3 W, Pl3 Pz, const uint32_t* ez, int ngz,
                                         uint32_t qh0, uint32_t qh1, uint32_t qh2,
                                         const V6* g_row, const V6* r1_row, int wmin, WitOut wo,
                                         int wthr) {
  for (int s = 6; s >= 0 && fl != 0u; --s) {
    if ((fl >> s) & 1u) {
      TG_IS_ZCOUNTS(z_)
      const int pz_ = __popc(lop3<0xFE>(Pz.x0, Pz.x1, Pz.x2));
      wmin = is_sweep_fix<kW, kCG>((0x05763421u >> (4 * s)) & 0xFu, z_, ngz - pz_, qh0, qh1, qh2,
                              g_row, r1_row, wmin, W, Pz, wo, wthr);
      fl &= ~(1u << s);
    }
    if (s > 0) {
      W.x0 ^= ez[(6 * (s - 1) + 0) * kStride];
      W.x1 ^= ez[(6 * (s - 1) + 1) * kStride];
      W.x2 ^= ez[(6 * (s - 1) + 2) * kStride];
      Pz.x0 ^= ez[(6 * (s - 1) + 3) * kStride];
      Pz.x1 ^= ez[(6 * (s - 1) + 4) * kStride];
      Pz.x2 ^= ez[(6 * (s - 1) + 5) * kStride];
    }
  }
  return wmin;
}

// Smallest thr at which a block is tested on pairs of codewords (with seven
// selections of about 7/64 of the 32 low columns each, a pair's count tops 15
// in about 0.3 % of the sweeps and 16 in about 0.08 %, against 1.3e-5 for the
// largest single count over 14).  At thr = 15 about half of a warp's blocks
// hold a flagged sweep, and counting it leaves the other lanes idle: single
// counts there made a batch of 10,000 sets with k from 6 to 14 0.9 % faster.
constexpr int kIsPairThr = 16;
// Smallest thr at which single counts are flagged and counted after the block
// rather than on the spot.  A single count tops 10 in about 0.1 % of the
// codewords, so few blocks hold a flag; below that, stepping back through
// digit 1's moves to a flagged sweep costs more than a branch per sweep.  The
// straight-line blocks made a batch of 10,000 sets with k from 6 to 14 0.3 %
// faster, 1,000 sets of 14 rows (level 4 at thr 14 and 15) 4.5 % faster and
// 1,000 sets of 12 rows (thr 11 to 13) 1.2 % slower; starting them at thr 13
// or 14 instead was slower on all three batches.
constexpr int kIsDeferThr = 10;

// Walks blocks [b0, b0 + nblk) of one support; P is the sum of its rows other
// than digit 0 at the start of block b0.  Each block is 7 sweeps of digit 0
// (row r0) with digit 1 (row r1) stepping alpha^0 .. alpha^6 between them:
// 49 codewords of straight-line code, the same in every block, so the lanes
// of a warp never split on the block's parity.  Digit 1's six steps, in the
// W domain and on g's zero columns, are kept in this thread's shared-memory
// slots ez (stride kStride), and its return alpha^6 -> alpha^0 in slots
// 36..38; the move between blocks (digits 2.., rows dig[]) is loaded a block
// ahead.
// P's high word without digit 1's term (qh, which only the block moves
// change) is kept for the exact count of a rare sweep.  Returns the codewords
// evaluated.
template <int kStride, bool kW, bool kCG>
__device__ __forceinline__ unsigned long long is_walk_blocks(
    const V6& P, const V6* rows, uint32_t r0, uint32_t r1, const uint16_t* dig, uint32_t* ez,
    unsigned long long b0, unsigned long long nblk, int hb, int wthr, const int32_t* stop,
    int& wmin, WitOut wo) {
  const Pl3 g = pl3_lo(v6_load<kCG>(rows + r0));
  const Pl3 h = pl3_inv(g);
  const uint32_t gz = ~(g.x0 | g.x1 | g.x2);  // low columns where g is 0
  const int ngz = __popc(gz);
  // Digit 1's step i is (alpha^i + alpha^(i+1)) r1 = alpha^i (1 + alpha) r1:
  // one product with h for the first, then a multiplication by alpha (one
  // XOR) for each next, in both domains.
  const Pl3 d0 = pl3_lo(v6_load<kCG>(rows + r1 + 1));
  Pl3 e = pl3_mul(d0, h);
  Pl3 zq = pl3_and(d0, gz);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    ez[(6 * i + 0) * kStride] = e.x0;
    ez[(6 * i + 1) * kStride] = e.x1;
    ez[(6 * i + 2) * kStride] = e.x2;
    ez[(6 * i + 3) * kStride] = zq.x0;
    ez[(6 * i + 4) * kStride] = zq.x1;
    ez[(6 * i + 5) * kStride] = zq.x2;
    e = Pl3{e.x2, e.x0 ^ e.x2, e.x1};  // alpha e
    zq = Pl3{zq.x2, zq.x0 ^ zq.x2, zq.x1};
  }
  {
    // (alpha^6 + alpha^0) r1 = alpha^2 r1
    const Pl3 r = pl3_lo(v6_load<kCG>(rows + r1));
    ez[36 * kStride] = r.x1;
    ez[37 * kStride] = r.x1 ^ r.x2;
    ez[38 * kStride] = r.x0 ^ r.x2;
  }
  Pl3 W = pl3_mul(pl3_lo(P), h);
  Pl3 Pz = pl3_and(pl3_lo(P), gz);
  // digit 1 starts at alpha^0
  uint32_t qh0 = P.h0 ^ ld_u32<kCG>(&rows[r1].h0);
  uint32_t qh1 = P.h1 ^ ld_u32<kCG>(&rows[r1].h1);
  uint32_t qh2 = P.h2 ^ ld_u32<kCG>(&rows[r1].h2);
  const int thz_base = 32 + hb - ngz;
  int thz = thz_base - wmin;
  // The move into block m = b0 + i + 1 changes digit 2 when m % 7 != 0 (six
  // blocks in seven): up from alpha^(m7 - 1) when m / 7 is even, else down
  // from alpha^(7 - m7); the rest take the general form.
  // A task's blocks in one support: at most 343 in the batch walk; the served
  // loop's largest stages (k >= 15) take 343 x 7^j so their task count fits
  // the claim word.
  const int n = int(nblk);
  int m7 = int((b0 + 1ull) % 7ull);
  int par = int(((b0 + 1ull) / 7ull) & 1ull);
  V6 nx;
  v6_zero(nx);
  if (n > 1) nx = v6_load<kCG>(is_block_move<kStride>(rows, dig, b0 + 1ull));
  int i = 0;
  for (; i < n; ++i) {
    if (i) {
      // digits 2.. move to block b, digit 1 returns to alpha^0
      Pl3 d = pl3_lo(nx);
      d.x0 ^= ez[36 * kStride];
      d.x1 ^= ez[37 * kStride];
      d.x2 ^= ez[38 * kStride];
      pl3_xor(W, pl3_mul(d, h));
      pl3_xor(Pz, pl3_and(d, gz));
      qh0 ^= nx.h0;
      qh1 ^= nx.h1;
      qh2 ^= nx.h2;
      if (++m7 == 7) {
        m7 = 0;
        par ^= 1;
      }
      if (i + 1 < n) {
        const V6* mv = m7 != 0 ? rows + dig[0] + 1 + (par ? 6 - m7 : m7 - 1)
                               : is_block_move<kStride>(rows, dig, b0 + unsigned(i) + 1ull);
        nx = v6_load<kCG>(mv);
      }
    }
    // Sweep s at digit-1 coefficient alpha^s; the flagged ones are counted
    // exactly after the block.
    // The pair test pays once thr >= kIsPairThr: below it a pair's count
    // passes thr so often that the exact path costs more than it saves.
    unsigned fl = 0u;
    if (thz + ngz >= kIsPairThr) {
      TG_IS_SWEEP2(0); TG_IS_MOVE(0); TG_IS_SWEEP2(1); TG_IS_MOVE(1); TG_IS_SWEEP2(2);
      TG_IS_MOVE(2); TG_IS_SWEEP2(3); TG_IS_MOVE(3); TG_IS_SWEEP2(4); TG_IS_MOVE(4);
      TG_IS_SWEEP2(5); TG_IS_MOVE(5); TG_IS_SWEEP2(6);
    } else if (thz + ngz >= kIsDeferThr) {
      TG_IS_SWEEP1F(0); TG_IS_MOVE(0); TG_IS_SWEEP1F(1); TG_IS_MOVE(1); TG_IS_SWEEP1F(2);
      TG_IS_MOVE(2); TG_IS_SWEEP1F(3); TG_IS_MOVE(3); TG_IS_SWEEP1F(4); TG_IS_MOVE(4);
      TG_IS_SWEEP1F(5); TG_IS_MOVE(5); TG_IS_SWEEP1F(6);
    } else {
      TG_IS_SWEEP1(0, 1u); TG_IS_MOVE(0); TG_IS_SWEEP1(1, 2u); TG_IS_MOVE(1); TG_IS_SWEEP1(2, 4u);
      TG_IS_MOVE(2); TG_IS_SWEEP1(3, 3u); TG_IS_MOVE(3); TG_IS_SWEEP1(4, 6u); TG_IS_MOVE(4);
      TG_IS_SWEEP1(5, 7u); TG_IS_MOVE(5); TG_IS_SWEEP1(6, 5u);
    }
    if (__builtin_expect(fl != 0u, 0)) {
      wmin = is_block_fix<kStride, kW, kCG>(fl, W, Pz, ez, ngz, qh0, qh1, qh2, rows + r0, rows + r1,
                                       wmin, wo, wthr);
      thz = thz_base - wmin;
    }
    if (wmin < wthr) break;
    // Another task's witness (a weight below wthr) stops the code; with
    // wthr <= 1 there is none, and the flag is not polled.
    if (wthr > 1 && (i & 15) == 15 && ld_flag(stop)) break;
  }
  return 49ull * static_cast<unsigned long long>(min(i, n - 1) + 1);
}

#undef TG_IS_MOVE
#undef TG_IS_SWEEP2
#undef TG_IS_SWEEP1F
#undef TG_IS_SWEEP1
#undef TG_IS_ZCOUNTS

// Units [u0, u1) of code c at level w (flat over set, support, block); the
// smallest weight met (or wmin when none is smaller), and the codewords
// evaluated in ncw.  dig and ez (stride kStride) are this thread's shared
// scratch: the rows of digits 2..w-2 and digit 1's moves.
// Where the witness pass of one code records its witness (pivot words of
// its sets, output row, claim word); all NULL outside the witness pass.
struct WitSrc {
  const uint64_t* piv;
  uint8_t* dst;
  int32_t* lock;
};

// Units [u0, u1) of one part of level w of one code whose information sets
// start at `base` (n_sets sets of k rows, the last with rank deficit delta):
// per set, the n_sup supports of ranks s_off .. s_off + n_sup - 1.  `stop`
// is the code's abort flag.  The smallest weight met (or wmin when none is
// smaller), and the codewords evaluated in ncw.  dig and ez (stride kStride)
// are this thread's shared scratch: the rows of digits 2..w-2 and digit 1's
// moves.  Serves the batch walk and the served loop alike.
template <int kStride, bool kW, bool kCG>
__device__ __forceinline__ int is_walk_range(const V6* base, int n_sets, int delta,
                                             const int32_t* stop, WitSrc wsrc,
                                             const unsigned long long (*bn)[kIsBinom],
                                             uint16_t* dig, uint32_t* ez, int k, int w,
                                             unsigned long long n_sup, unsigned long long s_off,
                                             unsigned long long u0, unsigned long long u1,
                                             int wthr, int wmin, unsigned long long& ncw) {
  const unsigned long long bps = is_units_per_support(w);
  const unsigned long long per_set = n_sup * bps;
  ncw = 0ull;
  unsigned long long u = u0;
  while (u < u1) {
    unsigned long long j, s, b;
    if (((u | per_set) >> 32) == 0ull) {  // 32-bit divisions whenever they fit
      const uint32_t u32 = uint32_t(u), ps = uint32_t(per_set), bp = uint32_t(bps);
      const uint32_t j32 = u32 / ps, r32 = u32 - j32 * ps, s32 = r32 / bp;
      j = j32;
      s = s32;
      b = r32 - s32 * bp;
    } else {
      j = u / per_set;
      const unsigned long long r = u - j * per_set;
      s = r / bps;
      b = r - s * bps;
    }
    const unsigned long long nblk = min(bps - b, u1 - u);
    const V6* rows = base + size_t(j) * k * kIsVecPerRow;
    // Support rows from the largest down (combinadic unranking).  The q-th
    // row found is Gray digit q (q < w - 1); the last one has coefficient 1.
    // Digit 0 is swept through all seven values and stays out of P; digit 1
    // starts every block at alpha^0; digit 2 + i starts at the Gray value of
    // base-7 digit i of b.  The positions are found first, by a loop whose
    // body is a few predicated instructions (every lane runs all k steps, so
    // the warp stays converged whatever its lanes' supports), and the rows
    // are loaded after it, by a loop over the w digits.
    uint32_t r0 = 0u, r1 = 0u, rl = 0u;
    {
      unsigned long long srank = s + s_off;
      int rem = w, q = 0;
      for (int pos = k - 1; pos >= 0; --pos) {
        const unsigned long long bb = bn[pos][rem];
        if (rem > 0 && srank >= bb) {
          const uint32_t R = uint32_t(pos * kIsVecPerRow);
          if (rem == 1) rl = R;
          else if (q == 0) r0 = R;
          else if (q == 1) r1 = R;
          else dig[(q - 2) * kStride] = uint16_t(R);
          srank -= bb;
          --rem;
          ++q;
        }
      }
    }
    V6 P = v6_load<kCG>(rows + rl);
    if (w >= 3) v6_xor(P, v6_load<kCG>(rows + r1));
    {
      unsigned long long rest = b;
      for (int i = 0; i < w - 3; ++i) {
        V6 g = v6_load<kCG>(rows + dig[i * kStride]);
        v6_alpha_pow(g, is_block_digit(rest));
        v6_xor(P, g);
      }
    }
    if (w == 1) {
      const int wt = __popc(lop3<0xFE>(P.l0, P.l1, P.l2)) + __popc(lop3<0xFE>(P.h0, P.h1, P.h2));
      wmin = min(wmin, wt);
      ncw += 1ull;
    } else if (w == 2) {
      wmin = is_sweep_exact<kCG>(P, rows + r0, wmin);
      ncw += 7ull;
    } else {
      // Weight on the set's pivot columns: the message restricted to the rows
      // with pivots (w, less the deficit of a partial set), less the pivots
      // that do not fit in the 17 high columns (k > 17).
      const int dj = int(j) == n_sets - 1 ? delta : 0;
      const int hb = max(0, w - dj - max(0, (k - dj) - 17));
      const WitOut wo = kW ? WitOut{wsrc.piv + j, wsrc.dst, wsrc.lock}
                           : WitOut{nullptr, nullptr, nullptr};
      ncw += is_walk_blocks<kStride, kW, kCG>(P, rows, r0, r1, dig, ez, b, nblk, hb, wthr, stop, wmin,
                                         wo);
    }
    u += nblk;
    if (wmin < wthr) break;
  }
  return wmin;
}

// is_walk_range for part `part` of level w of code c of a batch.
template <int kStride, bool kW>
__device__ __forceinline__ int is_walk_units(const DistArgs& a,
                                             const unsigned long long (*bn)[kIsBinom],
                                             uint16_t* dig, uint32_t* ez, int c, int k, int w,
                                             int part, unsigned long long u0,
                                             unsigned long long u1, int wthr, int wmin,
                                             unsigned long long& ncw) {
  const WitSrc wsrc = kW ? WitSrc{a.is_piv + size_t(c) * kIsMaxSets, a.witness + size_t(c) * kN,
                                  a.wit_lock + c}
                         : WitSrc{nullptr, nullptr, nullptr};
  const CodeDesc& d = a.desc[c];
  unsigned long long n_sup, s_off;
  is_part_supports(d.flags, k, w, part, bn, n_sup, s_off);
  return is_walk_range<kStride, kW, false>(a.is_rows + size_t(c) * a.is_stride, d.H, d.n_pat,
                                           a.abort + c, wsrc, bn, dig, ez, k, w, n_sup, s_off,
                                           u0, u1, wthr, wmin, ncw);
}

constexpr int kIsMaxDigits = kMaxExactK - 3;  // digits 2..w-2, w <= 21

// kW: the witness pass (per-code targets 50 - max_zeros; the first codeword
// below a target is recorded as that code's witness).
template <int kTPB, int kMinBlocks, bool kW>
__global__ void __launch_bounds__(kTPB, kMinBlocks) walk_level_kernel(DistArgs a, int w,
                                                                       int part) {
  __shared__ unsigned long long s_binom[kIsBinom][kIsBinom];
  __shared__ uint16_t s_dig[kIsMaxDigits][kTPB];
  __shared__ uint32_t s_ez[39][kTPB];
  if (a.is_hdr->total == 0ull) return;  // no set needs this level (uniform per block)
  for (int i = threadIdx.x; i < kIsBinom * kIsBinom; i += kTPB)
    s_binom[i / kIsBinom][i % kIsBinom] = c_binom[i / kIsBinom][i % kIsBinom];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned long long total = a.is_hdr->total;
  const unsigned long long nb = a.is_hdr->units;
  unsigned long long evaluated = 0ull;
  uint16_t* my_dig = &s_dig[0][threadIdx.x];  // this thread's digit rows, stride kTPB
  uint32_t* my_ez = &s_ez[0][threadIdx.x];     // this thread's digit-1 moves, stride kTPB
  // Tasks are numbered over code positions (codes ordered by k, is_perm);
  // p0 is the position of the warp's first task, claimed in increasing order.
  int p0 = 0;
  for (;;) {
    unsigned long long base = 0ull;
    if (lane == 0) base = atomicAdd(&a.is_hdr->counter, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    if (lane == 0) p0 = last_le_from(a.is_off, p0, a.n + 1, base);
    p0 = __shfl_sync(0xffffffffu, p0, 0);
    // The code's abort flag and best weight sit in a few cache lines that
    // every lane would poll, so lane 0 reads them for the warp's first code.
    const int c0 = __ldg(a.is_perm + p0);
    int abort0 = 0, best0 = 0;
    if (lane == 0) {
      abort0 = ld_flag(a.abort + c0);
      best0 = ld_flag(a.is_best + c0);
    }
    abort0 = __shfl_sync(0xffffffffu, abort0, 0);
    best0 = __shfl_sync(0xffffffffu, best0, 0);
    const unsigned long long t = base + lane;
    int c = -1, p = -1, wmin = kN + 1;
    if (t < total) {
      p = t < __ldg(a.is_off + p0 + 1) ? p0 : last_le_from(a.is_off, p0, a.n + 1, t);
      c = p == p0 ? c0 : __ldg(a.is_perm + p);
      if (p != p0) {
        abort0 = ld_flag(a.abort + c);
        best0 = ld_flag(a.is_best + c);
      }
      if (abort0) {
        atomicMax(&a.is_hdr->counter, __ldg(a.is_off + p + 1));
        c = -1;
      } else {
        const unsigned long long u0 = (t - __ldg(a.is_off + p)) * nb;
        const unsigned long long u1 =
            min(u0 + nb, static_cast<unsigned long long>(a.is_units[p]));
        unsigned long long ncw = 0ull;
        // Codewords no lighter than the code's best so far cannot change it,
        // so the walk starts from that best.
        wmin = is_walk_units<kTPB, kW>(a, s_binom, my_dig, my_ez, c, a.desc[c].k, w, part, u0,
                                       u1, kN - a.desc[c].tmax, best0, ncw);
        evaluated += ncw;
      }
    }
    // One atomic per code and warp, and only when the warp's lightest
    // codeword improves the code's best: the lanes of a warp mostly share a
    // code, and most tasks find nothing lighter.
    for (unsigned pend = __ballot_sync(0xffffffffu, c >= 0); pend != 0u;) {
      const int leader = __ffs(pend) - 1;
      const int cl = __shfl_sync(0xffffffffu, c, leader);
      const int pl = __shfl_sync(0xffffffffu, p, leader);
      const bool mine = c == cl;
      const int wl = __reduce_min_sync(0xffffffffu, mine ? wmin : kN + 1);
      pend &= ~__ballot_sync(0xffffffffu, mine);
      if (lane == leader && wl < ld_flag(a.is_best + cl)) {
        const int best = min(atomicMin(a.is_best + cl, wl), wl);
        if (best < kN - a.desc[cl].tmax) {
          // a witness below the target distance: the code is decided
          atomicExch(a.abort + cl, 1);
          atomicMax(&a.is_hdr->counter, __ldg(a.is_off + pl + 1));
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
  if (lane == 0 && evaluated) {
    atomicAdd(&a.is_hdr->codewords, evaluated);
    atomicAdd(&a.is_hdr->stage_codewords[2 * w + part - 1], evaluated);
  }
}

// Levels 1 to 3 of n_sets information sets of k rows (at base), by nthr
// threads (this one is tid): the rows themselves (weight-1 messages); for
// each pair of rows q < p the sweep alpha^v row_p + row_q; for each triple
// q < p < t the seven sweeps alpha^v row_t + alpha^s row_p + row_q
// (messages up to scalars).  Returns this thread's smallest weight; ncw =
// codewords evaluated by all nthr threads.  With wsrc.dst set (the witness
// pass) the first codeword lighter than wthr is recorded.  kCG: the rows may
// have been written during the launch.
template <bool kCG>
__device__ int is_levels123_part(int tid, int nthr, const V6* base, int n_sets, int k,
                                 WitSrc wsrc, int wthr, unsigned long long& ncw) {
  const int n1 = k, n2 = k * (k - 1) / 2, n3 = k * (k - 1) * (k - 2) / 6;
  const int per_set = n1 + n2 + n3;
  const int total = n_sets * per_set;
  const bool wit = wsrc.dst != nullptr;
  int wmin = kN + 1;
  // Units from the last down: the 49-codeword triples first, the rows and
  // pairs (1 and 7 codewords) last, where they even out the threads' loads.
  for (int uu = tid; uu < total; uu += nthr) {
    const int u = total - 1 - uu;
    const int j = u / per_set;
    int r = u - j * per_set;
    const V6* rows = base + size_t(j) * k * kIsVecPerRow;
    const WitOut wo{wsrc.piv + j, wsrc.dst, wsrc.lock};
    if (r < n1) {
      const V6 P = v6_load<kCG>(rows + r * kIsVecPerRow);
      const int wt = __popc(lop3<0xFE>(P.l0, P.l1, P.l2)) + __popc(lop3<0xFE>(P.h0, P.h1, P.h2));
      if (wit && wt < wthr) is_put_witness(wo, P.l0, P.l1, P.l2, P.h0, P.h1, P.h2);
      wmin = min(wmin, wt);
      continue;
    }
    r -= n1;
    int t = -1;  // the third row of a triple: C(t, 3) <= r < C(t + 1, 3)
    if (r >= n2) {
      r -= n2;
      t = 2;
      while ((t + 1) * t * (t - 1) / 6 <= r) ++t;
      r -= t * (t - 1) * (t - 2) / 6;
    }
    int p = 1;  // pair q < p: C(p, 2) <= r < C(p + 1, 2)
    while ((p + 1) * p / 2 <= r) ++p;
    const int q = r - p * (p - 1) / 2;
    const V6 Q = v6_load<kCG>(rows + q * kIsVecPerRow);
    if (t < 0) {
      wmin = wit ? is_sweep_exact_w(Q, rows + p * kIsVecPerRow, wmin, wo, wthr)
                 : is_sweep_exact<kCG>(Q, rows + p * kIsVecPerRow, wmin);
    } else {
      V6 X = v6_load<kCG>(rows + p * kIsVecPerRow);  // alpha^s row_p, s = 0..6
      for (int s7 = 0; s7 < 7; ++s7) {
        V6 P = Q;
        v6_xor(P, X);
        wmin = wit ? is_sweep_exact_w(P, rows + t * kIsVecPerRow, wmin, wo, wthr)
                   : is_sweep_exact<kCG>(P, rows + t * kIsVecPerRow, wmin);
        v6_alpha_pow(X, 1);
      }
    }
  }
  ncw = static_cast<unsigned long long>(n_sets) *
        static_cast<unsigned long long>(n1 + 7 * n2 + 49 * n3);
  return wmin;
}

// is_levels123_part by one warp, the smallest weight reduced over it.
template <bool kCG>
__device__ int is_levels123_sets(int lane, const V6* base, int n_sets, int k, WitSrc wsrc,
                                 int wthr, unsigned long long& ncw) {
  int wmin = is_levels123_part<kCG>(lane, 32, base, n_sets, k, wsrc, wthr, ncw);
  for (int o = 16; o > 0; o >>= 1) wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
  return wmin;
}

// Levels 1 to 3 of every set of a batch in one launch, one CTA of
// kL123Threads per set (a 14-row set has 469 row, pair and triple units, so
// the larger sets no longer hold one warp each for the whole launch).  These
// levels are too small to fill the GPU one launch each, and running them
// without the bound check between them only adds codewords (the best weight
// stays that of a codeword); level 4 onwards then follows the plan / scan /
// walk triples.
constexpr int kL123Threads = 128;

__global__ void __launch_bounds__(kL123Threads) levels123_kernel(DistArgs a) {
  __shared__ int s_min[kL123Threads / 32];
  const int c = blockIdx.x;
  const int tid = threadIdx.x;
  const CodeDesc d = a.desc[c];
  if ((d.flags & kIsCodeFlag) == 0 || (d.flags & kDecidedFlag) != 0 || ld_flag(a.abort + c) != 0)
    return;  // uniform over the CTA
  // The witness pass records the first codeword lighter than the target.
  const WitSrc wsrc = a.witness ? WitSrc{a.is_piv + size_t(c) * kIsMaxSets,
                                         a.witness + size_t(c) * kN, a.wit_lock + c}
                                : WitSrc{nullptr, nullptr, nullptr};
  unsigned long long ncw = 0ull;
  int wmin = is_levels123_part<false>(tid, kL123Threads, a.is_rows + size_t(c) * a.is_stride, d.H,
                                      d.k, wsrc, kN - d.tmax, ncw);
  for (int o = 16; o > 0; o >>= 1) wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
  if ((tid & 31) == 0) s_min[tid >> 5] = wmin;
  __syncthreads();
  if (tid == 0) {
    for (int i = 1; i < kL123Threads / 32; ++i) wmin = min(wmin, s_min[i]);
    atomicAdd(&a.is_hdr->codewords, ncw);
    if (wmin < a.is_best[c]) a.is_best[c] = wmin;
    if (a.is_best[c] < kN - d.tmax) a.abort[c] = 1;  // a witness below the target distance
  }
}

__global__ void finalize_infoset_kernel(DistArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  const CodeDesc d = a.desc[c];
  if ((d.flags & kIsCodeFlag) == 0 || (d.flags & kDecidedFlag) != 0) return;
  a.out[c] = kN - a.is_best[c];
}

// Targets of the witness pass: 50 - out, so that the pass stops at the first
// codeword with at least out zeros (1 for an empty set).
__global__ void witness_targets_kernel(const int32_t* out, const int64_t* off, int32_t* td, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int m = min(max(out[c], 0), kN);
  td[c] = off[c + 1] > off[c] ? kN + 1 - m : 1;
}

// After the witness pass: the zeros of each recorded witness (its claim word
// holds weight + 1) become the results, the pass's values elsewhere (codes
// decided without a walk); a code evaluated by the walk without a witness
// raises TG_ERR_STATE, and any status of the pass is copied into the first
// pass's header hdr1 (the one tg_distance_status reads).
__global__ void witness_finish_kernel(DistArgs a2, int32_t* out, WsHeader* hdr1) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a2.n) return;
  const CodeDesc d = a2.desc[c];
  const int lock = a2.wit_lock[c];
  if ((d.flags & kIsCodeFlag) != 0 && (d.flags & kDecidedFlag) == 0 && lock == 0)
    report_status(hdr1, TG_ERR_STATE);
  if (c == 0 && a2.hdr->status != TG_OK) report_status(hdr1, a2.hdr->status);
  out[c] = lock != 0 ? kN - (lock - 1) : a2.out[c];
}

}  // namespace tg
