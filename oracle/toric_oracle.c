/*
 * ORACLE — test infrastructure only.  CPU restatement of the reference's
 * algorithms for the GF(8) toric-code hot path, used by tests/, by
 * __graft_entry__.smoke() to check the device results and by bench.py's
 * CPU-baseline leg.
 * The product (generalized_toric_gpu_search_b200) never links or calls it.
 *
 * Restated from (paths inside the reference project):
 *   gf8.py:9-21                 GF(8) = GF(2)[x]/(x^3+x+1) multiplication
 *   precompute.py:17-43         evaluation matrix M (built by the caller)
 *   kernel.py:35-60             bitpat[b][i][v] construction
 *   kernel.py:97-203            batched max_zeros: messages 1..8^k-1 in base-8
 *                               digit order (coefficient i = digit i), zeros =
 *                               popcount(~v0 & ~v1 & ~v2 & mask49), stop once
 *                               zeros > tmax; sampled mode with splitmix64
 *                               (same as kernel_cuda_bp.py:47-66, 167-236)
 *   kernel_canon.py:44-129      canonical key: min over GL2(F7) x anchors of
 *                               sort(rel(anchor, perm)) packed 6 bits per
 *                               index, 128-bit unsigned compare
 *   champion_search_canonical.py:61-108   GL2 permutations, rel_table
 *
 * Early exit: the reference's value after an abort depends on GPU thread
 * timing.  This restatement walks messages in increasing id order per chunk
 * and reports the largest zero count it saw; only "value > tmax" is
 * comparable for failing sets.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define NP 49
#define MASK49 ((1ULL << 49) - 1ULL)

static uint8_t MUL[64];
static int mul_ready = 0;

static uint8_t gf8_mul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  for (int i = 0; i < 3; ++i) {
    if (b & 1) r ^= a;
    a = (uint8_t)(a << 1);
    if (a & 8) a ^= 0xB;
    b >>= 1;
  }
  return r;
}

static void init_mul(void) {
  if (mul_ready) return;
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) MUL[a * 8 + b] = gf8_mul((uint8_t)a, (uint8_t)b);
  mul_ready = 1;
}

void or_mul_table(int32_t* out64) {
  init_mul();
  for (int i = 0; i < 64; ++i) out64[i] = MUL[i];
}

/* bitpat[(b*k + i)*8 + v], kernel.py:35-60 */
static void build_bitpat(const int32_t* M, const int32_t* S, int k, uint64_t* bp) {
  for (int b = 0; b < 3; ++b)
    for (int i = 0; i < k; ++i)
      for (int v = 0; v < 8; ++v) {
        uint64_t m = 0;
        for (int j = 0; j < NP; ++j)
          if ((MUL[v * 8 + M[S[i] * NP + j]] >> b) & 1) m |= 1ULL << j;
        bp[(b * k + i) * 8 + v] = m;
      }
}

static inline int zeros_of(uint64_t v0, uint64_t v1, uint64_t v2) {
  return __builtin_popcountll(~v0 & ~v1 & ~v2 & MASK49);
}

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

/* Evaluates messages of one set.  Exact: ids [lo, hi].  Sampled: work ids
 * [lo, hi].  Stops at the first zeros > tmax when *abort_flag is set or
 * becomes set by another thread. */
static int eval_range(const uint64_t* bp, int k, int tmax, uint64_t lo, uint64_t hi,
                      int64_t sample_count, uint64_t seed, uint64_t set_id,
                      volatile int* abort_flag) {
  const uint64_t total = (3 * k <= 63) ? ((1ULL << (3 * k)) - 1ULL) : ~0ULL;
  const int poly_mode = sample_count > 0 && 3 * k <= 63;
  int best = 0;
  for (uint64_t w = lo; w <= hi; ++w) {
    if (abort_flag && *abort_flag) break;
    uint64_t pid = w;
    if (poly_mode) {
      uint64_t x = seed ^ (set_id * 0x9E3779B97F4A7C15ULL) ^ (w * 0xBF58476D1CE4E5B9ULL);
      pid = (splitmix64(x) % total) + 1ULL;
    }
    int forced = 0;
    if (sample_count > 0 && !poly_mode) {
      uint64_t x = seed ^ (set_id * 0xD6E8FEB86659FD93ULL) ^ (w * 0xA5A3564E27F8861FULL);
      forced = (int)(splitmix64(x) % (uint64_t)k);
    }
    uint64_t v0 = 0, v1 = 0, v2 = 0, tmp = pid;
    for (int i = 0; i < k; ++i) {
      int c;
      if (sample_count > 0 && !poly_mode) {
        uint64_t x = seed ^ (set_id * 0x9E3779B97F4A7C15ULL) ^ (w * 0xBF58476D1CE4E5B9ULL) ^
                     ((uint64_t)(i + 1) * 0x94D049BB133111EBULL);
        c = (int)(splitmix64(x) & 7ULL);
        if (i == forced && c == 0) c = 1;
      } else {
        c = (int)(tmp & 7ULL);
        tmp >>= 3;
      }
      v0 ^= bp[(0 * k + i) * 8 + c];
      v1 ^= bp[(1 * k + i) * 8 + c];
      v2 ^= bp[(2 * k + i) * 8 + c];
    }
    const int z = zeros_of(v0, v1, v2);
    if (z > best) best = z;
    if (z > tmax) {
      if (abort_flag) *abort_flag = 1;
      break;
    }
  }
  return best;
}

/*
 * max_zeros of n sets (flat indices + n+1 offsets), target distance per set
 * (td == NULL -> td_default), sampled when sample_count > 0 with
 * set_id = set_ids[s] (NULL -> s).  Work is cut into chunks of 2^18 messages
 * spread over `threads` OpenMP threads.
 */
int or_max_zeros_batch(const int32_t* M, const int32_t* flat, const int64_t* offsets, int n,
                       const int32_t* td, int td_default, int64_t sample_count, uint64_t seed,
                       const int32_t* set_ids, int32_t* out, int threads) {
  init_mul();
  if (n <= 0) return 0;
  const uint64_t CH = 1ULL << 18;
  uint64_t* first_chunk = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n + 1));
  uint64_t** bps = (uint64_t**)calloc((size_t)n, sizeof(uint64_t*));
  int* abort_flags = (int*)calloc((size_t)n, sizeof(int));
  if (!first_chunk || !bps || !abort_flags) return -1;
  uint64_t total_chunks = 0;
  for (int s = 0; s < n; ++s) {
    const int k = (int)(offsets[s + 1] - offsets[s]);
    first_chunk[s] = total_chunks;
    out[s] = 0;
    uint64_t items;
    if (sample_count > 0) items = (uint64_t)sample_count;
    else items = (k == 0) ? 0 : ((1ULL << (3 * k)) - 1ULL);
    if (k == 0) items = sample_count > 0 ? (uint64_t)sample_count : 0;
    total_chunks += (items + CH - 1) / CH;
    bps[s] = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(3 * (k > 0 ? k : 1) * 8));
    if (k > 0) build_bitpat(M, flat + offsets[s], k, bps[s]);
  }
  first_chunk[n] = total_chunks;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t ch = 0; ch < (int64_t)total_chunks; ++ch) {
    int lo = 0, hi = n - 1;
    while (lo < hi) { /* last set with first_chunk <= ch */
      int mid = (lo + hi + 1) / 2;
      if (first_chunk[mid] <= (uint64_t)ch) lo = mid; else hi = mid - 1;
    }
    const int s = lo;
    if (abort_flags[s]) continue;
    const int k = (int)(offsets[s + 1] - offsets[s]);
    const int tmax = NP - (td ? td[s] : td_default);
    uint64_t items = sample_count > 0 ? (uint64_t)sample_count : ((1ULL << (3 * k)) - 1ULL);
    const uint64_t c0 = (uint64_t)ch - first_chunk[s];
    const uint64_t a = c0 * CH + 1ULL;
    uint64_t b = a + CH - 1ULL;
    if (b > items) b = items;
    int z;
    if (k == 0) {
      z = NP; /* sampled k = 0: the empty sum, the zero codeword */
      if (z > tmax) abort_flags[s] = 1;
    } else {
      z = eval_range(bps[s], k, tmax, a, b, sample_count, seed,
                     (uint64_t)(int64_t)(set_ids ? set_ids[s] : s), &abort_flags[s]);
    }
#pragma omp critical
    {
      if (z > out[s]) out[s] = z;
    }
  }
  for (int s = 0; s < n; ++s) free(bps[s]);
  free(bps);
  free(first_chunk);
  free(abort_flags);
  return 0;
}

/* Evaluates `count` consecutive exact messages of one set starting at id
 * `first` with no early exit (the reference's per-message work); returns the
 * largest zero count.  Used to time the CPU baseline. */
int or_eval_messages(const int32_t* M, const int32_t* S, int k, uint64_t first, uint64_t count) {
  init_mul();
  uint64_t bp[3 * 21 * 8];
  if (k < 1 || k > 21) return -1;
  build_bitpat(M, S, k, bp);
  return eval_range(bp, k, NP, first, first + count - 1ULL, 0, 0, 0, NULL);
}

/* Evaluates messages 1..min(count, 8^k - 1) of every set with no early exit,
 * spread over `threads` OpenMP threads in chunks of 2^16 messages; returns
 * the number of messages evaluated.  This is the CPU baseline's timed work:
 * the reference's per-message loop (kernel.py:147-180) on a bounded prefix. */
int64_t or_eval_prefix_batch(const int32_t* M, const int32_t* flat, const int64_t* offsets, int n,
                             uint64_t count, int threads, int32_t* out) {
  init_mul();
  const uint64_t CH = 1ULL << 16;
  uint64_t* first = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n + 1));
  uint64_t* items = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n + 1));
  uint64_t** bps = (uint64_t**)calloc((size_t)(n > 0 ? n : 1), sizeof(uint64_t*));
  if (!first || !items || !bps) return -1;
  uint64_t tot = 0, msgs = 0;
  for (int s = 0; s < n; ++s) {
    const int k = (int)(offsets[s + 1] - offsets[s]);
    const uint64_t full = (k >= 1 && k <= 21) ? ((1ULL << (3 * k)) - 1ULL) : 0ULL;
    items[s] = full < count ? full : count;
    first[s] = tot;
    tot += (items[s] + CH - 1) / CH;
    msgs += items[s];
    out[s] = 0;
    bps[s] = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(3 * (k > 0 ? k : 1) * 8));
    if (k > 0) build_bitpat(M, flat + offsets[s], k, bps[s]);
  }
  first[n] = tot;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t ch = 0; ch < (int64_t)tot; ++ch) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) / 2;
      if (first[mid] <= (uint64_t)ch) lo = mid; else hi = mid - 1;
    }
    const int s = lo;
    const int k = (int)(offsets[s + 1] - offsets[s]);
    const uint64_t a = ((uint64_t)ch - first[s]) * CH + 1ULL;
    uint64_t b = a + CH - 1ULL;
    if (b > items[s]) b = items[s];
    const int z = eval_range(bps[s], k, NP, a, b, 0, 0, 0, NULL);
#pragma omp critical
    {
      if (z > out[s]) out[s] = z;
    }
  }
  for (int s = 0; s < n; ++s) free(bps[s]);
  free(bps);
  free(first);
  free(items);
  return (int64_t)msgs;
}

/* ---- canonical forms -------------------------------------------------- */

static int32_t GL2[2016 * NP];
static uint8_t REL[NP * NP];
static int canon_ready = 0;

static void init_canon(void) {
  if (canon_ready) return;
  int m = 0;
  for (int a = 0; a < 7; ++a)
    for (int b = 0; b < 7; ++b)
      for (int c = 0; c < 7; ++c)
        for (int d = 0; d < 7; ++d) {
          if ((((a * d - b * c) % 7) + 7) % 7 == 0) continue;
          for (int p = 0; p < NP; ++p) {
            const int x = p / 7, y = p % 7;
            GL2[m * NP + p] = ((a * x + b * y) % 7) * 7 + (c * x + d * y) % 7;
          }
          ++m;
        }
  for (int p = 0; p < NP; ++p)
    for (int q = 0; q < NP; ++q)
      REL[p * NP + q] = (uint8_t)(((q / 7 - p / 7 + 7) % 7) * 7 + (q % 7 - p % 7 + 7) % 7);
  canon_ready = 1;
}

void or_gl2_perms(int32_t* out) {
  init_canon();
  memcpy(out, GL2, sizeof(GL2));
}

void or_rel_table(uint8_t* out) {
  init_canon();
  memcpy(out, REL, sizeof(REL));
}

/* The reference's packed key for rows of k <= 16 (kernel_canon.py:44-129). */
void or_canonical_keys(const int32_t* sets, int n, int k, uint64_t* out_lo, uint64_t* out_hi,
                       int threads) {
  init_canon();
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (int s = 0; s < n; ++s) {
    uint64_t best_lo = ~0ULL, best_hi = ~0ULL;
    const int32_t* S = sets + (size_t)s * (size_t)k;
    for (int pi = 0; pi < 2016; ++pi) {
      int perm[16];
      for (int i = 0; i < k; ++i) perm[i] = GL2[pi * NP + S[i]];
      for (int anc = 0; anc < k; ++anc) {
        int t[16];
        for (int i = 0; i < k; ++i) t[i] = REL[perm[anc] * NP + perm[i]];
        for (int i = 1; i < k; ++i) {
          int v = t[i], j = i;
          while (j > 0 && t[j - 1] > v) { t[j] = t[j - 1]; --j; }
          t[j] = v;
        }
        uint64_t lo = 0, hi = 0;
        const int pf = k <= 10 ? 0 : 1;
        for (int i = pf; i < k; ++i) {
          const int off = 6 * (i - pf);
          const uint64_t v = (uint64_t)t[i];
          if (off + 6 <= 64) lo |= v << off;
          else if (off < 64) { lo |= v << off; hi |= v >> (64 - off); }
          else hi |= v << (off - 64);
        }
        if (hi < best_hi || (hi == best_hi && lo < best_lo)) { best_lo = lo; best_hi = hi; }
      }
    }
    out_lo[s] = best_lo;
    out_hi[s] = best_hi;
  }
}

/* Anchored-min canonical mask for any popcount: min over A in GL2(F7) and
 * anchor s of the mask of A(S - s). */
void or_canonical_masks(const uint64_t* masks, int n, uint64_t* out, int threads) {
  init_canon();
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (int s = 0; s < n; ++s) {
    const uint64_t S = masks[s] & MASK49;
    int pts[NP], k = 0;
    for (int p = 0; p < NP; ++p)
      if (S >> p & 1ULL) pts[k++] = p;
    uint64_t best = ~0ULL;
    if (k == 0) best = 0;
    for (int pi = 0; pi < 2016 && k > 0; ++pi) {
      for (int anc = 0; anc < k; ++anc) {
        const int a = GL2[pi * NP + pts[anc]];
        uint64_t m = 0;
        for (int i = 0; i < k; ++i) m |= 1ULL << REL[a * NP + GL2[pi * NP + pts[i]]];
        if (m < best) best = m;
      }
    }
    out[s] = best;
  }
}

/* ---- witness check (a test helper with no reference counterpart) ---------
 * Solves m A = c over GF(8) for A = M[S] (k x 49 rows of the code) by
 * Gauss-Jordan elimination of the 49 x (k + 1) system A^T m^T = c^T.  When c
 * is a codeword it writes a message m with m A = c (nonzero whenever one
 * exists: for c = 0 a null-space vector of a rank-deficient A), recomputes
 * m A with the reference's evaluation (kernel.py:97-203: the sum over i of
 * coefficient m_i times row S[i]) and returns the zero count of c.  Returns
 * -1 when c is not in the row space or the recomputed codeword differs, -2
 * when c = 0 and A has full rank (no nonzero message gives it), -3 for k out
 * of 1..49. */
int or_codeword_message(const int32_t* M, const int32_t* S, int k, const uint8_t* cw,
                        int32_t* msg) {
  init_mul();
  if (k < 1 || k > NP) return -3;
  uint8_t inv[8] = {0};
  for (int a = 1; a < 8; ++a)
    for (int b = 1; b < 8; ++b)
      if (MUL[a * 8 + b] == 1) inv[a] = (uint8_t)b;
  uint8_t E[NP][NP + 1];
  for (int j = 0; j < NP; ++j) {
    for (int i = 0; i < k; ++i) E[j][i] = (uint8_t)M[S[i] * NP + j];
    E[j][k] = cw[j];
  }
  int pivrow_col[NP];
  int is_pivot[NP];
  for (int i = 0; i < k; ++i) is_pivot[i] = 0;
  int r = 0;
  for (int i = 0; i < k && r < NP; ++i) {
    int p = -1;
    for (int j = r; j < NP; ++j)
      if (E[j][i]) { p = j; break; }
    if (p < 0) continue;
    if (p != r)
      for (int t = 0; t <= k; ++t) { uint8_t x = E[p][t]; E[p][t] = E[r][t]; E[r][t] = x; }
    const uint8_t s = inv[E[r][i]];
    for (int t = 0; t <= k; ++t) E[r][t] = MUL[s * 8 + E[r][t]];
    for (int j = 0; j < NP; ++j) {
      if (j == r || !E[j][i]) continue;
      const uint8_t f = E[j][i];
      for (int t = 0; t <= k; ++t) E[j][t] ^= MUL[f * 8 + E[r][t]];
    }
    pivrow_col[r] = i;
    is_pivot[i] = 1;
    ++r;
  }
  for (int j = r; j < NP; ++j)
    if (E[j][k]) return -1;  /* inconsistent: c is not a codeword */
  int all_zero = 1;
  for (int j = 0; j < NP; ++j)
    if (cw[j]) all_zero = 0;
  for (int i = 0; i < k; ++i) msg[i] = 0;
  if (all_zero) {
    int f = -1;
    for (int i = 0; i < k && f < 0; ++i)
      if (!is_pivot[i]) f = i;
    if (f < 0) return -2;
    msg[f] = 1;
  }
  for (int rr = 0; rr < r; ++rr) {
    uint8_t v = E[rr][k];
    for (int i = 0; i < k; ++i)
      if (!is_pivot[i] && msg[i]) v ^= MUL[E[rr][i] * 8 + msg[i]];
    msg[pivrow_col[rr]] = v;
  }
  int zeros = 0;
  for (int j = 0; j < NP; ++j) {
    uint8_t v = 0;
    for (int i = 0; i < k; ++i) v ^= MUL[msg[i] * 8 + M[S[i] * NP + j]];
    if (v != cw[j]) return -1;
    if (v == 0) ++zeros;
  }
  return zeros;
}
