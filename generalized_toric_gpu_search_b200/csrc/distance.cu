// max_zeros of GF(8) generalized toric codes: exact enumeration and the
// reference's sampled screening mode, for batches of codes of mixed size in
// one persistent launch.
//
// What is computed (the reference's eval_min_distance_batch_bp,
// kernel_cuda_bp.py:146-238, and its OpenCL twin kernel.py:97-203): for each
// exponent set S (k rows of the evaluation matrix M) the largest number of
// zero coordinates of c . M[S] over nonzero messages c in GF(8)^k, with the
// early exit "stop once zeros > tmax = 49 - target_distance".
//
// How (B200 design, not the reference's per-message loop):
//  * Enumeration.  Scalar multiples of a codeword have the same zeros, so only
//    projective messages (first nonzero coefficient 1) are needed.  When M is
//    the toric matrix the torus (x, y) -> (l x, m y) also permutes
//    coordinates and multiplies coefficient i by alpha^(e1 a_i + e2 b_i), so
//    the first two nonzero coefficients -- and the third when its exponent
//    point is not collinear with the first two -- can be normalised to 1 as
//    well ("orbit" enumeration, ~49x fewer codewords).  The row order is
//    chosen so the leading rows are in general position.
//  * Tasks.  The last R rows ("tail") of a code are walked completely inside
//    one task; the leading H = k - R rows ("head") carry the normalised
//    message patterns.  Every task covers 8^R codewords, so tasks of codes
//    of any size cost the same and a global atomic counter hands them out to
//    a persistent grid (equal-cost slices).
//  * Walk.  Inside a task the codeword moves along a binary-reflected Gray
//    code over the GF(2) coordinates of the tail coefficients: one XOR of a
//    bit-sliced basis vector per step.
//  * Histogram variant (toric M, every entry of a row nonzero).  The eight
//    codewords P + c g (c in GF(8), g the last row) have zero sets that
//    partition the 49 coordinates by w_j = P_j / g_j, so their zero counts are
//    the 8-bin histogram of w.  The walk runs on w directly (the basis is
//    divided coordinate-wise by g) and every state yields 8 codewords for
//    14 LOP3 + 14 POPC.
//  * Direct variant (any M).  One OR of the three planes and two POPC per
//    codeword.
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "distance.cuh"
#include "serve.cuh"

namespace tg {

__constant__ uint8_t c_mul[64];
__constant__ uint8_t c_inv[8];
// Binomials C(n, r), n, r <= 21 (0 for r > n), and powers of 7 for the
// weight-ordered enumeration of free head coefficients (task_start) and the
// information-set levels.
__constant__ unsigned long long c_binom[22][22];
__constant__ unsigned long long c_pow7[22];

static bool g_tables_ready[64] = {false};

int upload_field_tables(int device) {
  if (device < 0 || device >= 64) return TG_ERR_NO_DEVICE;
  if (g_tables_ready[device]) return TG_OK;
  uint8_t mul[64], inv[8];
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) mul[a * 8 + b] = gf8_mul_c(uint8_t(a), uint8_t(b));
  inv[0] = 0;
  for (int a = 1; a < 8; ++a)
    for (int b = 1; b < 8; ++b)
      if (mul[a * 8 + b] == 1) inv[a] = uint8_t(b);
  cudaError_t e = cudaMemcpyToSymbol(c_mul, mul, sizeof(mul));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(c_mul)");
  e = cudaMemcpyToSymbol(c_inv, inv, sizeof(inv));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(c_inv)");
  unsigned long long binom[22][22] = {}, pow7[22];
  for (int n = 0; n <= 21; ++n) {
    binom[n][0] = 1;
    for (int r = 1; r <= n; ++r) binom[n][r] = binom[n - 1][r - 1] + (r <= n - 1 ? binom[n - 1][r] : 0);
  }
  pow7[0] = 1;
  for (int i = 1; i <= 21; ++i) pow7[i] = pow7[i - 1] * 7ull;
  e = cudaMemcpyToSymbol(c_binom, binom, sizeof(binom));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_pow7, pow7, sizeof(pow7));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(c_binom)");
  g_tables_ready[device] = true;
  return TG_OK;
}

// ---------------------------------------------------------------------------
// Workspace layout
// ---------------------------------------------------------------------------

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
size_t align_ws(size_t x) { return align256(x); }

int max_patterns(int H) {
  if (H <= 0) return 1;
  return 1 + H + H * (H - 1) / 2 + H * (H - 1) * (H - 2) / 6;
}

int default_tail_rows(const tg_distance_params& p) {
  return p.tail_rows > 0 ? p.tail_rows : 4;
}

// Smallest k evaluated by information sets (kNever: none).
constexpr int kNever = 1 << 20;
int infoset_min_k(const tg_distance_params& p) {
  if (p.sample_count > 0) return kNever;
  if (p.enumeration == TG_ENUM_INFOSET) return 2;
  if (p.enumeration == kEnumInfosetAll) return 1;
  if (p.enumeration == TG_ENUM_AUTO) return TG_INFOSET_AUTO_MIN_K;
  return kNever;
}

// Rows (sets x k) an information-set code of k_lo <= k <= k_hi may store.
static int infoset_rows(int k_lo, int k_hi) {
  int rows = 0;
  for (int k = k_lo; k <= k_hi; ++k) rows = std::max(rows, infoset_max_sets(k) * k);
  return rows;
}

WsLayout ws_layout(const tg_distance_params& p) {
  WsLayout L{};
  const size_t n = size_t(p.n_sets > 0 ? p.n_sets : 0);
  const bool sampled = p.sample_count > 0;
  const int kmax = p.k_max > 0 ? p.k_max : 1;
  const int R = default_tail_rows(p);
  const int Hmax = kmax > R ? kmax - R : 0;
  L.basis_stride = sampled ? 0 : kmax * 3;
  L.pat_stride = sampled ? 0 : max_patterns(Hmax);
  L.bitpat_stride = sampled ? kmax * 8 : 0;
  size_t off = 0;
  L.hdr = off;      off = align256(off + sizeof(WsHeader));
  L.desc = off;     off = align256(off + n * sizeof(CodeDesc));
  L.task_off = off; off = align256(off + (n + 1) * sizeof(uint64_t));
  L.abort = off;    off = align256(off + n * sizeof(int32_t));
  L.basis = off;    off = align256(off + n * size_t(L.basis_stride) * sizeof(V6));
  L.pat_cum = off;  off = align256(off + n * size_t(L.pat_stride) * sizeof(uint64_t));
  L.pat_info = off; off = align256(off + n * size_t(L.pat_stride) * sizeof(uint32_t));
  L.bitpat = off;   off = align256(off + n * size_t(L.bitpat_stride) * sizeof(V6));
  L.is_min_k = infoset_min_k(p);
  const bool infoset = L.is_min_k <= kmax;
  const size_t n_is = infoset ? n : 0;
  L.is_stride = infoset ? infoset_rows(L.is_min_k, kmax) * kIsVecPerRow : 0;
  L.is_hdr = off;   off = align256(off + (infoset ? sizeof(IsHeader) : 0));
  L.is_rows = off;  off = align256(off + n * size_t(L.is_stride) * sizeof(V6));
  L.is_units = off; off = align256(off + n_is * sizeof(uint64_t));
  L.is_off = off;   off = align256(off + (infoset ? n + 1 : 0) * sizeof(uint64_t));
  L.is_best = off;  off = align256(off + n_is * sizeof(int32_t));
  L.is_perm = off;  off = align256(off + n_is * sizeof(int32_t));
  L.total = off;
  return L;
}

// ---------------------------------------------------------------------------
// Per-code preparation: validation, row order, bit-sliced basis, patterns.
// One warp per code.
// ---------------------------------------------------------------------------

constexpr int kPrepWarps = 4;

__device__ __forceinline__ void report_status(WsHeader* h, int code) {
  atomicCAS(&h->status, 0, code);
}

__device__ __forceinline__ int pt_a(int idx) { return idx / 7; }
__device__ __forceinline__ int pt_b(int idx) { return idx % 7; }

// Exponent points p, q, r of Z_7^2 on one affine line.
__device__ __forceinline__ bool collinear3(int p, int q, int r) {
  const int ua = pt_a(q) - pt_a(p), ub = pt_b(q) - pt_b(p);
  const int va = pt_a(r) - pt_a(p), vb = pt_b(r) - pt_b(p);
  int det = (ua * vb - ub * va) % 7;
  if (det < 0) det += 7;
  return det == 0;
}

// Pattern descriptor bits: i0 [0,5) i1 [5,10) i2 [10,15) nfix [15,17)
// mult7 [17] free_from [18,23).
__device__ __forceinline__ uint32_t pat_pack(int i0, int i1, int i2, int nfix,
                                             int mult7, int free_from) {
  return uint32_t(i0) | (uint32_t(i1) << 5) | (uint32_t(i2) << 10) |
         (uint32_t(nfix) << 15) | (uint32_t(mult7) << 17) |
         (uint32_t(free_from) << 18);
}

__device__ __forceinline__ uint64_t pow8(int e) { return e <= 0 ? 1ull : (1ull << (3 * e)); }

// Bit-sliced planes of v_j for j = lane and 32 + lane, gathered by ballot.
__device__ __forceinline__ V6 ballot_planes(int lane, uint32_t v_lo, uint32_t v_hi) {
  V6 r;
  r.l0 = __ballot_sync(0xffffffffu, v_lo & 1u);
  r.l1 = __ballot_sync(0xffffffffu, (v_lo >> 1) & 1u);
  r.l2 = __ballot_sync(0xffffffffu, (v_lo >> 2) & 1u);
  r.h0 = __ballot_sync(0xffffffffu, v_hi & 1u) & kHiMask;
  r.h1 = __ballot_sync(0xffffffffu, (v_hi >> 1) & 1u) & kHiMask;
  r.h2 = __ballot_sync(0xffffffffu, (v_hi >> 2) & 1u) & kHiMask;
  r.pad0 = r.pad1 = 0u;
  (void)lane;
  return r;
}

struct PrepResult {
  int result;        // max_zeros when decided without enumeration
  uint64_t n_tasks;  // tasks of the walk (0 when decided)
  int n_pat;
  int R;
  int H;
};

// Warp-level preparation of one code whose k (< 32) valid exponent indices
// are in s_idx[0..k): repeated rows and k <= 1 are decided directly; else
// the rows are ordered (leading head rows in general position for the orbit
// enumeration), the bit-sliced basis B[r*3 + t] = alpha^t row_r (divided
// coordinate-wise by the last row for the histogram variant) and the pattern
// table (cum, info) are written.  s_row is per-warp scratch of 32 ints.
__device__ PrepResult prep_code(int lane, int k, const int* s_idx, int* s_row, int R_param,
                                int enumeration, int variant, const uint8_t* M, V6* B,
                                uint64_t* cum, uint32_t* info) {
  PrepResult out{0, 0ull, 0, 0, 0};
  const int my = lane < k ? s_idx[lane] : -1 - lane;
  bool dup = false;
  if (k > 1) {
    const unsigned act = __ballot_sync(0xffffffffu, lane < k);
    const unsigned m = __match_any_sync(0xffffffffu, my);
    dup = __any_sync(0xffffffffu, (act >> lane & 1u) && __popc(m) > 1);
  }
  if (k == 0) return out;
  if (dup) {
    // Two equal rows: c_i = c_j = 1 is a nonzero message with the zero
    // codeword, so max_zeros = 49.
    out.result = kN;
    return out;
  }
  if (k == 1) {
    // All nonzero multiples of one row have the row's zero set.
    const int row = s_idx[0];
    const int z0 = (lane < kN && M[row * kN + lane] == 0) ? 1 : 0;
    const int z1 = (lane + 32 < kN && M[row * kN + lane + 32] == 0) ? 1 : 0;
    out.result = __popc(__ballot_sync(0xffffffffu, z0)) + __popc(__ballot_sync(0xffffffffu, z1));
    return out;
  }
  const int R = min(R_param, k);
  const int H = k - R;
  out.R = R;
  out.H = H;
  // Row order: leading head rows in general position (orbit mode).
  if (lane == 0) {
    int used = 0;  // bitmask over set positions
    int nsel = 0;
    if (enumeration == TG_ENUM_ORBIT) {
      for (int pos = 0; pos < H; ++pos) {
        int best = -1, best_cost = 1 << 30;
        for (int cand = 0; cand < k; ++cand) {
          if (used >> cand & 1) continue;
          int cost = 0;
          for (int x = 0; x < nsel; ++x)
            for (int y = x + 1; y < nsel; ++y)
              cost += collinear3(s_idx[s_row[x]], s_idx[s_row[y]], s_idx[cand]) ? 1 : 0;
          if (cost < best_cost) { best_cost = cost; best = cand; }
        }
        s_row[nsel++] = best;
        used |= 1 << best;
      }
    }
    for (int cand = 0; cand < k; ++cand)
      if (!(used >> cand & 1)) s_row[nsel++] = cand;
  }
  __syncwarp();

  // Bit-sliced basis, coordinates j = lane and 32 + lane.
  const int last = s_idx[s_row[k - 1]];
  const bool hist = variant == TG_VARIANT_HISTOGRAM;
  uint32_t inv_lo = 1, inv_hi = 1;
  if (hist) {
    inv_lo = c_inv[M[last * kN + lane]];
    inv_hi = lane + 32 < kN ? c_inv[M[last * kN + lane + 32]] : 0u;
  }
  for (int r = 0; r < k; ++r) {
    const int row = s_idx[s_row[r]];
    const uint32_t g_lo = M[row * kN + lane];
    const uint32_t g_hi = lane + 32 < kN ? M[row * kN + lane + 32] : 0u;
    uint32_t e = 1;  // alpha^t
    for (int t = 0; t < 3; ++t) {
      uint32_t v_lo = c_mul[e * 8 + g_lo];
      uint32_t v_hi = c_mul[e * 8 + g_hi];
      if (hist) {
        v_lo = c_mul[v_lo * 8 + inv_lo];
        v_hi = lane + 32 < kN ? c_mul[v_hi * 8 + inv_hi] : 0u;
      }
      const V6 v = ballot_planes(lane, v_lo, v_hi);
      if (lane == 0) v6_stg(B + r * 3 + t, v);
      e = c_mul[e * 8 + 2];
    }
  }

  // Message patterns over the head rows.
  uint64_t n_tasks = 0;
  int np = 0;
  if (lane == 0) {
    uint64_t acc = 0;
    cum[np] = acc; info[np] = pat_pack(0, 0, 0, 0, 0, H); ++np; acc += 1;
    if (enumeration == TG_ENUM_ORBIT) {
      for (int i0 = 0; i0 < H; ++i0) {
        cum[np] = acc; info[np] = pat_pack(i0, 0, 0, 1, 0, H); ++np; acc += 1;
      }
      for (int i0 = 0; i0 < H; ++i0)
        for (int i1 = i0 + 1; i1 < H; ++i1) {
          cum[np] = acc; info[np] = pat_pack(i0, i1, 0, 2, 0, H); ++np; acc += 1;
        }
      for (int i0 = 0; i0 < H; ++i0)
        for (int i1 = i0 + 1; i1 < H; ++i1)
          for (int i2 = i1 + 1; i2 < H; ++i2) {
            const bool col = collinear3(s_idx[s_row[i0]], s_idx[s_row[i1]], s_idx[s_row[i2]]);
            cum[np] = acc;
            info[np] = pat_pack(i0, i1, i2, 3, col ? 1 : 0, i2 + 1);
            ++np;
            acc += (col ? 7ull : 1ull) * pow8(H - 1 - i2);
          }
    } else {
      for (int i0 = 0; i0 < H; ++i0) {
        cum[np] = acc; info[np] = pat_pack(i0, 0, 0, 1, 0, i0 + 1); ++np;
        acc += pow8(H - 1 - i0);
      }
    }
    n_tasks = acc;
  }
  out.n_tasks = __shfl_sync(0xffffffffu, n_tasks, 0);
  out.n_pat = __shfl_sync(0xffffffffu, np, 0);
  return out;
}

__global__ void __launch_bounds__(kPrepWarps * 32)
prep_exact_kernel(DistArgs a) {
  __shared__ int s_idx[kPrepWarps][32];
  __shared__ int s_row[kPrepWarps][32];
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kPrepWarps + w;
  if (c >= a.n) return;  // warp-uniform

  const int64_t beg = a.off[c];
  const int64_t end = a.off[c + 1];
  const int64_t klong = end - beg;
  CodeDesc d{};
  d.set_id = c;
  d.tmax = kN - (a.target ? a.target[c] : a.td_default);
  d.flags = 0;
  bool ok = true;
  if (klong < 0 || klong > a.k_max) {
    ok = false;
    if (lane == 0) report_status(a.hdr, TG_ERR_BAD_INPUT);
  }
  const int k = ok ? int(klong) : 0;
  int my = -1;
  if (ok && lane < k) my = a.idx[beg + lane];
  const bool bad = __any_sync(0xffffffffu, lane < k && (my < 0 || my >= kN));
  if (bad) {
    ok = false;
    if (lane == 0) report_status(a.hdr, TG_ERR_BAD_INPUT);
  }
  if (lane < 32) s_idx[w][lane] = my;
  __syncwarp();
  if (ok && k >= a.is_min_k) {
    // Evaluated by information sets (prep_infoset_kernel fills the rest).
    if (lane == 0) {
      d.k = k;
      d.flags = kIsCodeFlag;
      d.n_tasks = 0ull;
      a.desc[c] = d;
    }
    return;
  }
  PrepResult pr{0, 0ull, 0, 0, 0};
  if (ok) {
    V6* B = a.basis + size_t(c) * a.basis_stride;
    uint64_t* cum = a.pat_cum + size_t(c) * a.pat_stride;
    uint32_t* info = a.pat_info + size_t(c) * a.pat_stride;
    pr = prep_code(lane, k, s_idx[w], s_row[w], a.R, a.enumeration, a.variant, a.tab.M, B, cum,
                   info);
  }
  if (lane == 0) {
    d.k = k;
    d.R = pr.R;
    d.H = pr.H;
    d.n_pat = pr.n_pat;
    d.n_tasks = pr.n_tasks;
    a.desc[c] = d;
    a.out[c] = pr.result;
    a.abort[c] = 0;
    if (pr.n_tasks) {
      atomicAdd(&a.hdr->codewords, (unsigned long long)(pr.n_tasks * pow8(pr.R)));
      a.hdr->has_tasks = 1;
    }
    if (ok && k > 0) atomicAdd(&a.hdr->ref_messages, double(pow8(k)) - 1.0);
  }
}

// ---------------------------------------------------------------------------
// Exclusive scan of per-code task counts (one CTA of 1024 threads).
// ---------------------------------------------------------------------------

constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) scan_tasks_kernel(DistArgs a) {
  __shared__ unsigned long long s_part[kScanThreads / 32];
  __shared__ int s_over;
  const int t = threadIdx.x;
  const int n = a.n;
  if (a.hdr->has_tasks == 0) {
    // No code has walk tasks (every set takes the information-set path, or
    // none needs enumerating): the walks read no offset when the total is 0.
    if (t == 0) {
      a.task_off[n] = 0ull;
      a.hdr->total_tasks = 0ull;
      a.hdr->counter = 0ull;
    }
    return;
  }
  if (t == 0) s_over = 0;
  const int chunk = (n + kScanThreads - 1) / kScanThreads;
  const int beg = min(n, t * chunk);
  const int end = min(n, beg + chunk);
  unsigned long long sum = 0;
  bool over = false;
  for (int i = beg; i < end; ++i) {
    const unsigned long long x = a.desc[i].n_tasks;
    if (sum + x < sum) over = true;
    sum += x;
  }
  // warp inclusive scan
  const int lane = t & 31, wid = t >> 5;
  unsigned long long incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_part[wid] = incl;
  __syncthreads();
  if (over) s_over = 1;
  if (wid == 0) {
    unsigned long long v = s_part[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    s_part[lane] = v;  // inclusive over warps
  }
  __syncthreads();
  unsigned long long run = incl - sum + (wid > 0 ? s_part[wid - 1] : 0ull);
  for (int i = beg; i < end; ++i) {
    a.task_off[i] = run;
    run += a.desc[i].n_tasks;
  }
  if (t == kScanThreads - 1) {
    const unsigned long long total = s_part[31];
    a.task_off[n] = total;
    a.hdr->total_tasks = total;
    a.hdr->counter = 0ull;
  }
  __syncthreads();
  if (t == 0 && s_over) {
    // Work larger than 2^64 tasks: nothing runs.
    a.task_off[n] = 0ull;
    a.hdr->total_tasks = 0ull;
    for (int i = 0; i <= n; ++i) a.task_off[i] = 0ull;
    report_status(a.hdr, TG_ERR_INVALID_ARGUMENT);
  }
}

// ---------------------------------------------------------------------------
// Persistent walk kernels.
// ---------------------------------------------------------------------------

// Start vector of local task q of a pattern: the head coefficients in the
// domain of the basis.
template <bool kCG = false>
__device__ __forceinline__ V6 task_start(const V6* B, uint32_t info, uint64_t q, int H) {
  const int i0 = int(info & 31u), i1 = int((info >> 5) & 31u), i2 = int((info >> 10) & 31u);
  const int nfix = int((info >> 15) & 3u);
  const int mult7 = int((info >> 17) & 1u);
  const int ff = int((info >> 18) & 31u);
  V6 s;
  v6_zero(s);
  int c2 = 1;
  if (mult7) {
    c2 = int(q % 7ull) + 1;
    q /= 7ull;
  }
  if (nfix >= 1) v6_xor(s, v6_load<kCG>(B + i0 * 3));
  if (nfix >= 2) v6_xor(s, v6_load<kCG>(B + i1 * 3));
  if (nfix >= 3) {
    for (int t = 0; t < 3; ++t)
      if (c2 >> t & 1) v6_xor(s, v6_load<kCG>(B + i2 * 3 + t));
  }
  // Free rows ff..H-1 take every vector of GF(8)^F exactly once, ordered by
  // the number of nonzero coefficients: light messages come first, so an
  // early exit meets its witness sooner; the full set is unchanged.
  const int F = H - ff;
  int w = 0;
  unsigned long long size = 1ull;  // C(F, 0) * 7^0
  while (q >= size && w < F) {
    q -= size;
    ++w;
    size = c_binom[F][w] * c_pow7[w];
  }
  unsigned long long comb = q / c_pow7[w];
  unsigned long long dig = q - comb * c_pow7[w];
  int rem = w;
  for (int pos = F - 1; pos >= 0 && rem > 0; --pos) {
    const unsigned long long b = c_binom[pos][rem];
    if (comb >= b) {
      comb -= b;
      --rem;
      const int dgt = int(dig % 7ull) + 1;
      dig /= 7ull;
      const int r = ff + pos;
      for (int t = 0; t < 3; ++t)
        if (dgt >> t & 1) v6_xor(s, v6_load<kCG>(B + r * 3 + t));
    }
  }
  return s;
}

// Histogram of the eight codewords P + c g: running max of the bins.
// bin 0 (c = 0, the codeword P itself) is skipped when !bin0.
__device__ __forceinline__ void hist8(const V6& w, int& m, bool bin0) {
  int s = 0;
#define TG_BIN(V)                                                          \
  {                                                                        \
    const int lo = __popc(lop3<sel_lut(V)>(w.l0, w.l1, w.l2));             \
    const int hi = __popc(lop3<sel_lut(V)>(w.h0, w.h1, w.h2));             \
    m = __viaddmax_s32(lo, hi, m);                                         \
    s += lo + hi;                                                          \
  }
  TG_BIN(1) TG_BIN(2) TG_BIN(3) TG_BIN(4) TG_BIN(5) TG_BIN(6) TG_BIN(7)
#undef TG_BIN
  const int c0 = bin0 ? (kN - s) : 0;
  m = max(m, c0);
}

// Weight of a bit-sliced codeword folded into a running minimum.
__device__ __forceinline__ void weight_min(const V6& p, int& wmin) {
  const int lo = __popc(lop3<0xFE>(p.l0, p.l1, p.l2));
  const int hi = __popc(lop3<0xFE>(p.h0, p.h1, p.h2));
  wmin = __viaddmin_s32(lo, hi, wmin);
}

struct WalkState {
  uint64_t total;
  int c;
};

// Claims 32 consecutive tasks per warp; returns false when the queue is empty.
__device__ __forceinline__ bool claim_task(const DistArgs& a, uint64_t total, int lane,
                                           uint64_t& t, int& c, bool& active) {
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(&a.hdr->counter, 32ull);
  base = __shfl_sync(0xffffffffu, base, 0);
  if (base >= total) return false;
  int c0 = 0;
  if (lane == 0) c0 = last_le(a.task_off, a.n + 1, base);
  c0 = __shfl_sync(0xffffffffu, c0, 0);
  t = base + lane;
  active = t < total;
  c = c0;
  if (active)
    while (__ldg(a.task_off + c + 1) <= t) ++c;
  return true;
}

// One task of the histogram walk: the Gray walk of the tail rows H..k-2 from
// the pattern's start vector, 8 codewords per state.  Returns the largest
// zero count seen; sets `aborted` when it exceeds tmax.  Polls *abort_flag
// every 512 codewords and stops when another task aborted the code.
template <bool kCG = false>
__device__ __forceinline__ int hist_task(const V6* B, uint32_t info, uint64_t q, int H, int k,
                                         int R, int tmax, const int32_t* abort_flag,
                                         bool& aborted) {
  V6 w = task_start<kCG>(B, info, q, H);
  const bool zero_head = ((info >> 15) & 3u) == 0u;
  const V6 g0 = v6_load<kCG>(B + (k - 2) * 3 + 0);
  const V6 g1 = v6_load<kCG>(B + (k - 2) * 3 + 1);
  const V6 g2 = v6_load<kCG>(B + (k - 2) * 3 + 2);
  const uint32_t n_mid = 1u << (3 * (R - 2));
  int m = 0;
  aborted = false;
  for (uint32_t mi = 0; mi < n_mid; ++mi) {
    if (mi) {
      const int f = __ffs(int(mi)) - 1;
      const int row = k - 3 - f / 3;
      v6_xor(w, v6_load<kCG>(B + row * 3 + f % 3));
    }
    hist8(w, m, mi != 0u || !zero_head);
    v6_xor(w, g0); hist8(w, m, true);
    v6_xor(w, g1); hist8(w, m, true);
    v6_xor(w, g0); hist8(w, m, true);
    v6_xor(w, g2); hist8(w, m, true);
    v6_xor(w, g0); hist8(w, m, true);
    v6_xor(w, g1); hist8(w, m, true);
    v6_xor(w, g0); hist8(w, m, true);
    if (m > tmax) {
      aborted = true;
      break;
    }
    if ((mi & 7u) == 7u && ld_flag(abort_flag)) break;
  }
  return m;
}

// Moves the task counter past the remaining tasks of an aborted code: every
// task in [counter, task_off[c + 1]) belongs to code c once a lane of c has
// been claimed, so the jump loses no other code's work.
__device__ __forceinline__ void skip_code(const DistArgs& a, int c) {
  atomicMax(&a.hdr->counter, static_cast<unsigned long long>(__ldg(a.task_off + c + 1)));
}

template <int kTPB, int kMinBlocks>
__global__ void __launch_bounds__(kTPB, kMinBlocks) walk_hist_kernel(DistArgs a) {
  const int lane = threadIdx.x & 31;
  const uint64_t total = a.hdr->total_tasks;
  for (;;) {
    uint64_t t;
    int c;
    bool active;
    if (!claim_task(a, total, lane, t, c, active)) break;
    if (!active) continue;
    if (ld_flag(a.abort + c)) {
      skip_code(a, c);
      continue;
    }
    const CodeDesc d = a.desc[c];
    const uint64_t local = t - __ldg(a.task_off + c);
    const uint64_t* cum = a.pat_cum + size_t(c) * a.pat_stride;
    const int p = last_le(cum, d.n_pat, local);
    const uint64_t q = local - __ldg(cum + p);
    const uint32_t info = __ldg(a.pat_info + size_t(c) * a.pat_stride + p);
    const V6* B = a.basis + size_t(c) * a.basis_stride;
    bool aborted = false;
    const int m = hist_task(B, info, q, d.H, d.k, d.R, d.tmax, a.abort + c, aborted);
    if (m > 0) atomicMax(a.out + c, m);
    if (aborted) {
      atomicExch(a.abort + c, 1);
      skip_code(a, c);
    }
  }
}

template <int kTPB, int kMinBlocks>
__global__ void __launch_bounds__(kTPB, kMinBlocks) walk_direct_kernel(DistArgs a) {
  const int lane = threadIdx.x & 31;
  const uint64_t total = a.hdr->total_tasks;
  for (;;) {
    uint64_t t;
    int c;
    bool active;
    if (!claim_task(a, total, lane, t, c, active)) break;
    if (!active) continue;
    if (ld_flag(a.abort + c)) {
      skip_code(a, c);
      continue;
    }
    const CodeDesc d = a.desc[c];
    const uint64_t local = t - __ldg(a.task_off + c);
    const uint64_t* cum = a.pat_cum + size_t(c) * a.pat_stride;
    const int p = last_le(cum, d.n_pat, local);
    const uint64_t q = local - __ldg(cum + p);
    const uint32_t info = __ldg(a.pat_info + size_t(c) * a.pat_stride + p);
    const V6* B = a.basis + size_t(c) * a.basis_stride;
    V6 w = task_start(B, info, q, d.H);
    const bool zero_head = ((info >> 15) & 3u) == 0u;
    const int k = d.k;
    // Inner 64 states: rows k-1 (bits 0..2) and k-2 (bits 3..5).
    const V6 e0 = v6_ldg(B + (k - 1) * 3 + 0);
    const V6 e1 = v6_ldg(B + (k - 1) * 3 + 1);
    const V6 e2 = v6_ldg(B + (k - 1) * 3 + 2);
    const V6 e3 = v6_ldg(B + (k - 2) * 3 + 0);
    const V6 e4 = v6_ldg(B + (k - 2) * 3 + 1);
    const V6 e5 = v6_ldg(B + (k - 2) * 3 + 2);
    const uint32_t n_mid = 1u << (3 * (d.R - 2));
    const int wthr = kN - d.tmax;  // abort when a weight < wthr appears
    int wmin = 64;
    bool aborted = false;
    for (uint32_t mi = 0; mi < n_mid; ++mi) {
      if (mi) {
        const int f = __ffs(int(mi)) - 1;
        const int row = k - 3 - f / 3;
        v6_xor(w, v6_ldg(B + row * 3 + f % 3));
      }
      {
        int w0 = 64;
        weight_min(w, w0);
        if (mi != 0u || !zero_head) wmin = min(wmin, w0);
      }
#pragma unroll
      for (int s = 1; s < 64; ++s) {
        const int f = __ffs(s) - 1;
        if (f == 0) v6_xor(w, e0);
        else if (f == 1) v6_xor(w, e1);
        else if (f == 2) v6_xor(w, e2);
        else if (f == 3) v6_xor(w, e3);
        else if (f == 4) v6_xor(w, e4);
        else v6_xor(w, e5);
        weight_min(w, wmin);
      }
      if (wmin < wthr) {
        aborted = true;
        break;
      }
      if ((mi & 7u) == 7u && ld_flag(a.abort + c)) break;
    }
    const int m = kN - wmin;
    if (m > 0) atomicMax(a.out + c, m);
    if (aborted) {
      atomicExch(a.abort + c, 1);
      skip_code(a, c);
    }
  }
}

// ---------------------------------------------------------------------------
// Sampled screening (kernel_cuda_bp.py:167-236): work_id = 1..sample_count,
// poly_id or per-coefficient splitmix64 hashing, bit-exact to the reference.
// ---------------------------------------------------------------------------

constexpr uint64_t kSampleChunk = 64;  // work ids per task

__global__ void __launch_bounds__(kPrepWarps * 32) prep_sampled_kernel(DistArgs a) {
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kPrepWarps + w;
  if (c >= a.n) return;
  const int64_t beg = a.off[c];
  const int64_t klong = a.off[c + 1] - beg;
  CodeDesc d{};
  d.set_id = a.set_ids ? a.set_ids[c] : c;
  d.tmax = kN - (a.target ? a.target[c] : a.td_default);
  bool ok = klong >= 0 && klong <= a.k_max;
  const int k = ok ? int(klong) : 0;
  // Each lane loads up to two indices (k <= 49 < 64).
  const int i_a = (ok && lane < k) ? a.idx[beg + lane] : 0;
  const int i_b = (ok && lane + 32 < k) ? a.idx[beg + lane + 32] : 0;
  const bool bad = __any_sync(0xffffffffu, (ok && lane < k && (i_a < 0 || i_a >= kN)) ||
                                               (ok && lane + 32 < k && (i_b < 0 || i_b >= kN)));
  if (!ok || bad) {
    ok = false;
    if (lane == 0) report_status(a.hdr, TG_ERR_BAD_INPUT);
  }
  uint64_t n_tasks = 0;
  int result = 0;
  if (ok && k == 0) {
    // The reference evaluates the empty message sum, the zero codeword.
    result = a.sample_count > 0 ? kN : 0;
  } else if (ok) {
    V6* T = a.bitpat + size_t(c) * a.bitpat_stride;
    for (int i = 0; i < k; ++i) {
      const int row = __shfl_sync(0xffffffffu, i < 32 ? i_a : i_b, i & 31);
      const uint32_t g_lo = a.tab.M[row * kN + lane];
      const uint32_t g_hi = lane + 32 < kN ? a.tab.M[row * kN + lane + 32] : 0u;
      for (int v = 0; v < 8; ++v) {
        const V6 p = ballot_planes(lane, c_mul[v * 8 + g_lo], c_mul[v * 8 + g_hi]);
        if (lane == 0) v6_stg(T + i * 8 + v, p);
      }
    }
    n_tasks = (uint64_t(a.sample_count) + kSampleChunk - 1) / kSampleChunk;
  }
  if (lane == 0) {
    d.k = k;
    d.n_tasks = n_tasks;
    a.desc[c] = d;
    a.out[c] = result;
    a.abort[c] = 0;
    if (n_tasks) {
      atomicAdd(&a.hdr->codewords, (unsigned long long)a.sample_count);
      a.hdr->has_tasks = 1;
    }
  }
}

template <int kTPB>
__global__ void __launch_bounds__(kTPB) walk_sampled_kernel(DistArgs a) {
  const int lane = threadIdx.x & 31;
  const uint64_t total = a.hdr->total_tasks;
  const uint64_t seed = a.seed;
  const uint64_t count = uint64_t(a.sample_count);
  for (;;) {
    uint64_t t;
    int c;
    bool active;
    if (!claim_task(a, total, lane, t, c, active)) break;
    if (!active) continue;
    if (ld_flag(a.abort + c)) {
      skip_code(a, c);
      continue;
    }
    const CodeDesc d = a.desc[c];
    const uint64_t j = t - __ldg(a.task_off + c);
    const V6* T = a.bitpat + size_t(c) * a.bitpat_stride;
    const int k = d.k;
    const uint64_t sid = uint64_t(int64_t(d.set_id));
    const bool poly_mode = 3 * k <= 63;
    const uint64_t w_beg = j * kSampleChunk + 1;
    const uint64_t w_end = min(count, (j + 1) * kSampleChunk);
    int m = 0;
    bool aborted = false;
    for (uint64_t wid = w_beg; wid <= w_end; ++wid) {
      V6 v;
      v6_zero(v);
      if (poly_mode) {
        const uint64_t x = seed ^ (sid * 0x9E3779B97F4A7C15ull) ^ (wid * 0xBF58476D1CE4E5B9ull);
        uint64_t pid = mod_mersenne(splitmix64(x), 3 * k) + 1ull;
        for (int i = 0; i < k; ++i) {
          v6_xor(v, v6_ldg(T + i * 8 + int(pid & 7ull)));
          pid >>= 3;
        }
      } else {
        const uint64_t xf = seed ^ (sid * 0xD6E8FEB86659FD93ull) ^ (wid * 0xA5A3564E27F8861Full);
        const int forced = int(splitmix64(xf) % uint64_t(k));
        const uint64_t base = seed ^ (sid * 0x9E3779B97F4A7C15ull) ^ (wid * 0xBF58476D1CE4E5B9ull);
        for (int i = 0; i < k; ++i) {
          int cf = int(splitmix64(base ^ (uint64_t(i + 1) * 0x94D049BB133111EBull)) & 7ull);
          if (i == forced && cf == 0) cf = 1;
          v6_xor(v, v6_ldg(T + i * 8 + cf));
        }
      }
      const int wt = __popc(lop3<0xFE>(v.l0, v.l1, v.l2)) + __popc(lop3<0xFE>(v.h0, v.h1, v.h2));
      const int zeros = kN - wt;
      if (zeros > d.tmax) {
        m = max(m, zeros);
        aborted = true;
        break;
      }
      m = max(m, zeros);
      if ((wid & 15ull) == 0ull && ld_flag(a.abort + c)) break;
    }
    if (m > 0) atomicMax(a.out + c, m);
    if (aborted) {
      atomicExch(a.abort + c, 1);
      skip_code(a, c);
    }
  }
}

}  // namespace tg

#include "infoset_kernel.cuh"

namespace tg {

// ---------------------------------------------------------------------------
// Host launcher
// ---------------------------------------------------------------------------

constexpr int kIsWalkThreads = 128;

// Two register budgets per CTA shape: 1024 resident threads per SM (64
// registers per thread) or 512 (128 registers).
template <int kTPB>
static cudaError_t launch_walk(int variant, bool sampled, int grid, int blocks_per_sm,
                               const DistArgs& args, cudaStream_t s) {
  constexpr int kFull = 1024 / kTPB;
  constexpr int kHalf = 512 / kTPB;
  const bool full = blocks_per_sm * kTPB >= 1024;
  if (sampled) {
    walk_sampled_kernel<kTPB><<<grid, kTPB, 0, s>>>(args);
  } else if (variant == TG_VARIANT_HISTOGRAM) {
    if (full) walk_hist_kernel<kTPB, kFull><<<grid, kTPB, 0, s>>>(args);
    else walk_hist_kernel<kTPB, kHalf><<<grid, kTPB, 0, s>>>(args);
  } else {
    if (full) walk_direct_kernel<kTPB, kFull><<<grid, kTPB, 0, s>>>(args);
    else walk_direct_kernel<kTPB, kHalf><<<grid, kTPB, 0, s>>>(args);
  }
  return cudaGetLastError();
}

// Last level the information-set walk can need for a batch whose sets have
// at most k_max rows.  With the toric matrix, after levels 1..L every unseen
// codeword of a k-row code weighs at least ceil(49 (L + 1) / k); the Griesmer
// bound n >= sum_{i < k} ceil(d / 8^i) caps the distance d of any [49, k]
// code over GF(8) at some G(k).  Once ceil(49 (L + 1) / k) > G(k) a
// minimum-weight codeword has been met and plan_level_kernel stops the code,
// so no level after that L is needed by any k <= k_max.  Other matrices use
// the disjoint-set bound: every level up to k_max.
int infoset_last_level(int k_max, int is_toric) {
  if (!is_toric) return k_max;
  int last = 0;
  for (int k = 1; k <= k_max; ++k) {
    int G = 0;
    for (int d = 1; d <= kN; ++d) {
      long long sum = 0, q = 1;
      for (int i = 0; i < k && sum <= kN; ++i) {
        sum += (d + q - 1) / q;
        if (q < (1ll << 40)) q *= 8;
      }
      if (sum <= kN) G = d;
    }
    int L = 0;
    while ((kN * (L + 1) + k - 1) / k < G + 1) ++L;
    last = std::max(last, std::min(L, k));
  }
  return last;
}

int run_prepare(const DistArgs& args, cudaStream_t s) {
  if (args.n <= 0) return TG_OK;
  const bool sampled = args.sample_count > 0;
  cudaError_t e = cudaMemsetAsync(args.hdr, 0, sizeof(WsHeader), s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(header)");
  const int prep_grid = (args.n + kPrepWarps - 1) / kPrepWarps;
  if (sampled) prep_sampled_kernel<<<prep_grid, kPrepWarps * 32, 0, s>>>(args);
  else prep_exact_kernel<<<prep_grid, kPrepWarps * 32, 0, s>>>(args);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "prep kernel launch");
  if (args.is_min_k <= args.k_max) {
    e = cudaMemsetAsync(args.is_hdr, 0, sizeof(IsHeader), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(information-set header)");
    prep_infoset_kernel<<<(args.n + kIsPrepWarps - 1) / kIsPrepWarps, kIsPrepWarps * 32, 0, s>>>(
        args);
    order_codes_kernel<<<1, kScanThreads, 0, s>>>(args);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "information-set prep launch");
  }
  scan_tasks_kernel<<<1, kScanThreads, 0, s>>>(args);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "scan kernel launch");
  return TG_OK;
}

int run_walk(const DistArgs& args, int sm_count, int blocks_per_sm, int tpb, cudaStream_t s,
             int parts) {
  if (args.n <= 0) return TG_OK;
  const bool sampled = args.sample_count > 0;
  const int grid = sm_count * blocks_per_sm;
  cudaError_t e = cudaSuccess;
  if (parts & kWalkEnumeration) {
    switch (tpb) {
      case 64: e = launch_walk<64>(args.variant, sampled, grid, blocks_per_sm, args, s); break;
      case 256: e = launch_walk<256>(args.variant, sampled, grid, blocks_per_sm, args, s); break;
      default: e = launch_walk<128>(args.variant, sampled, grid, blocks_per_sm, args, s); break;
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "walk kernel launch");
  if ((parts & kWalkInfoset) && args.is_min_k <= args.k_max) {
    // Information-set walk: levels 1 to 3 in one launch, then a plan / scan /
    // walk triple per part of each level; 5 CTAs of 128 threads per SM for
    // the walk (96 registers, no spills, 28 KB of shared memory each; 6 CTAs
    // at 80 registers spill and ran 1 % slower).  Parts no code needs return
    // before any setup.
    constexpr int kPerSm = 5;  // register budget of the walk (96 per thread)
    DistArgs la = args;
    const int per_sm = args.is_blocks_per_sm > 0 ? min(args.is_blocks_per_sm, kPerSm) : kPerSm;
    la.is_lanes = sm_count * per_sm * kIsWalkThreads;
    const int plan_grid = (args.n + 255) / 256;
    levels123_kernel<<<args.n, kL123Threads, 0, s>>>(la);
    const int w_last = infoset_last_level(args.k_max, args.is_toric);
    // Each level in two parts (a toric code's supports with and without its
    // last row; other codes walk the whole level in part 1).
    for (int w = 4; w <= w_last; ++w) {
      for (int part = 1; part <= 2; ++part) {
        plan_level_kernel<<<plan_grid, 256, 0, s>>>(la, w, part);
        scan_level_kernel<<<1, kScanThreads, 0, s>>>(la, w);
        if (la.witness)
          walk_level_kernel<kIsWalkThreads, kPerSm, true>
              <<<sm_count * per_sm, kIsWalkThreads, 0, s>>>(la, w, part);
        else
          walk_level_kernel<kIsWalkThreads, kPerSm, false>
              <<<sm_count * per_sm, kIsWalkThreads, 0, s>>>(la, w, part);
      }
    }
    finalize_infoset_kernel<<<plan_grid, 256, 0, s>>>(la);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "information-set walk launch");
  }
  return TG_OK;
}

int run_witness_targets(const int32_t* out, const int64_t* off, int32_t* td, int n,
                        cudaStream_t s) {
  if (n <= 0) return TG_OK;
  witness_targets_kernel<<<(n + 255) / 256, 256, 0, s>>>(out, off, td, n);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TG_OK : cuda_fail(e, "witness target launch");
}

int run_witness_finish(const DistArgs& a2, int32_t* out, WsHeader* hdr1, cudaStream_t s) {
  if (a2.n <= 0) return TG_OK;
  witness_finish_kernel<<<(a2.n + 255) / 256, 256, 0, s>>>(a2, out, hdr1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TG_OK : cuda_fail(e, "witness finish launch");
}

}  // namespace tg

#include "serve_kernel.cuh"
