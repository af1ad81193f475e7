// Shared definitions of libtoric_b200: GF(8) arithmetic, bit-sliced codeword
// vectors, status words and small device helpers.
//
// Field: GF(8) = GF(2)[x]/(x^3 + x + 1), elements 0..7 as polynomial bit
// patterns, the modulus of gf8.py:9 (POLY = 0b1011).  A codeword of length 49
// is stored bit-sliced: plane p holds bit p of the 49 GF(8) coordinates, the
// coordinates 0..31 in a `lo` word and 32..48 in bits 0..16 of a `hi` word.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/toric_b200.h"

namespace tg {

constexpr int kN = 49;                       // code length = torus points
constexpr int kMaxExactK = 21;               // exact enumeration limit (kernel_cuda_bp.py:270)
constexpr int kMaxSampledK = 49;             // sampled limit (kernel_cuda_bp.py:301)
constexpr uint32_t kHiMask = (1u << 17) - 1; // coordinates 32..48
constexpr uint64_t kMask49 = (1ull << 49) - 1;
constexpr int kGl2Order = 2016;              // |GL2(F7)|

// Carry-less product modulo x^3 + x + 1 (gf8.py:11-21).
constexpr uint8_t gf8_mul_c(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  for (int i = 0; i < 3; ++i) {
    if (b & 1) r ^= a;
    a = static_cast<uint8_t>(a << 1);
    if (a & 8) a ^= 0xB;
    b >>= 1;
  }
  return r;
}

// Bit-sliced codeword: three planes x (lo, hi).  32 bytes with padding so a
// vector loads as two 16-byte words.
struct alignas(16) V6 {
  uint32_t l0, l1, l2, h0, h1, h2, pad0, pad1;
};

__host__ __device__ __forceinline__ void v6_zero(V6& v) {
  v.l0 = v.l1 = v.l2 = v.h0 = v.h1 = v.h2 = 0u;
  v.pad0 = v.pad1 = 0u;
}

__device__ __forceinline__ void v6_xor(V6& a, const V6& b) {
  a.l0 ^= b.l0; a.l1 ^= b.l1; a.l2 ^= b.l2;
  a.h0 ^= b.h0; a.h1 ^= b.h1; a.h2 ^= b.h2;
}

// Loads a bit-sliced vector through the read-only path (two 16-byte loads).
__device__ __forceinline__ V6 v6_ldg(const V6* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 a = __ldg(q);
  const uint4 b = __ldg(q + 1);
  V6 v;
  v.l0 = a.x; v.l1 = a.y; v.l2 = a.z; v.h0 = a.w;
  v.h1 = b.x; v.h2 = b.y; v.pad0 = 0u; v.pad1 = 0u;
  return v;
}

__device__ __forceinline__ void v6_stg(V6* p, const V6& v) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(v.l0, v.l1, v.l2, v.h0);
  q[1] = make_uint4(v.h1, v.h2, 0u, 0u);
}

// 3-input logic op with an immediate truth table (one LOP3).
template <int kLut>
__device__ __forceinline__ uint32_t lop3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(kLut));
  return d;
}

// Truth table of "(a, b, c) == (bit0, bit1, bit2) of v" for lop3 inputs
// a = 0xF0, b = 0xCC, c = 0xAA.
constexpr int sel_lut(int v) {
  return ((v & 1) ? 0xF0 : 0x0F) & ((v & 2) ? 0xCC : 0x33) & ((v & 4) ? 0xAA : 0x55);
}

// Relaxed device-scope load of a flag written by other CTAs.
__device__ __forceinline__ int ld_flag(const int32_t* p) {
  return *reinterpret_cast<const volatile int32_t*>(p);
}

// Loads of data that no thread writes during the kernel (kCG = false, the
// non-coherent read-only path) or that other SMs may rewrite while the kernel
// runs (kCG = true: cached in L2 only, so never a stale L1 line).
template <bool kCG>
__device__ __forceinline__ uint64_t ld_u64(const uint64_t* p) {
  if (kCG) return __ldcg(reinterpret_cast<const unsigned long long*>(p));
  return __ldg(reinterpret_cast<const unsigned long long*>(p));
}

template <bool kCG>
__device__ __forceinline__ uint32_t ld_u32(const uint32_t* p) {
  return kCG ? __ldcg(p) : __ldg(p);
}

template <bool kCG>
__device__ __forceinline__ V6 v6_load(const V6* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 a = kCG ? __ldcg(q) : __ldg(q);
  const uint4 b = kCG ? __ldcg(q + 1) : __ldg(q + 1);
  V6 v;
  v.l0 = a.x; v.l1 = a.y; v.l2 = a.z; v.h0 = a.w;
  v.h1 = b.x; v.h2 = b.y; v.pad0 = 0u; v.pad1 = 0u;
  return v;
}

// Index of the last element of sorted a[0..n) that is <= x (a[0] <= x).
template <bool kCG = false>
__device__ __forceinline__ int last_le(const uint64_t* a, int n, uint64_t x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ld_u64<kCG>(a + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The same search starting from a known lo (a[lo] <= x), galloping forward:
// O(log distance) loads when x lies close after a[lo].
template <bool kCG = false>
__device__ __forceinline__ int last_le_from(const uint64_t* a, int lo, int n, uint64_t x) {
  int hi = n - 1;
  for (int step = 1; lo + step < n; step <<= 1) {
    if (ld_u64<kCG>(a + lo + step) > x) {
      hi = lo + step - 1;
      break;
    }
    lo += step;
  }
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ld_u64<kCG>(a + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// splitmix64 finaliser (kernel_cuda_bp.py:47-52, kernel.py:10-15).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// x mod (2^m - 1) for 1 <= m <= 63, by folding m-bit digits (2^m == 1).
__host__ __device__ __forceinline__ uint64_t mod_mersenne(uint64_t x, int m) {
  const uint64_t M = (1ull << m) - 1ull;
  while (x > M) x = (x & M) + (x >> m);
  return x == M ? 0ull : x;
}

constexpr uint64_t kRep7 = 0x0000040810204081ull;  // bits 0, 7, ..., 42

// Translation of a 49-bit torus mask by -(qa, qb): columns rotate right by qb
// inside each row of 7, rows rotate down by qa.
__device__ __forceinline__ uint64_t torus_shift(uint64_t m, int qa, int qb) {
  const uint64_t low = ((1ull << (7 - qb)) - 1ull) * kRep7;
  const uint64_t cr = ((m >> qb) & low) | ((m << (7 - qb)) & (kMask49 & ~low));
  const int r = 7 * qa;
  return ((cr >> r) | (cr << (kN - r))) & kMask49;
}

// Top row of a nonempty 49-bit mask (the highest row of Z_7^2 it occupies)
// and that row's 7 bits.
__device__ __forceinline__ void mask_top_row(uint64_t m, int& t, uint32_t& bits) {
  t = ((63 - __clzll(static_cast<long long>(m))) * 37) >> 8;  // (highest bit) / 7
  bits = uint32_t(m >> (7 * t)) & 0x7Fu;
}

// Smallest top row of the translates of an image with row occupancy R,
// anchored at its points: the translation by -q moves row qa to row 0, and
// the candidate's top row is the highest occupied row after that shift.
__device__ __forceinline__ int min_top_row(uint32_t R) {
  int tmin = 9;
  for (uint32_t rows = R; rows != 0u; rows &= rows - 1u) {
    const int qa = __ffs(rows) - 1;
    const uint32_t rr = ((R >> qa) | (R << (7 - qa))) & 0x7Fu;
    tmin = min(tmin, 31 - __clz(rr));
  }
  return tmin;
}

// AGL2(F7) canonical mask of S != 0 (the smallest mask among the images of S
// that contain the origin), by one warp.  A candidate's order is decided
// first by its top row, then by that row's bits.
//
// Stage 1.  The image of point (x, y) under A = (a b; c d) lies in row
// a x + b y: the row occupancy of A S, and so the smallest top row its
// translates can reach, depend on A's first row only.  The table holds the
// 2016 matrices in lexicographic order of (a, b, c, d), so each of the 48
// first rows heads 42 consecutive matrices; the lanes take the 48 first rows
// and find the smallest top row t* over all.
//
// Stage 2.  Only the matrices whose first row reaches t* can give the
// minimum.  The lanes map S by those (lane l takes l, l + 32, ... of them,
// from the table `perm`, read through the read-only path when kLdg), then
// translate each image by -q for every point q of its rows that reach t*;
// candidates above the best so far are skipped on their top-row bits without
// the full translation.  The lanes share their best every 8 matrices.
// Returns the mask in every lane.
// kRow: bytes between the table's rows (49 in global memory; the shared copy
// pads rows to 52 bytes, a 13-word stride that keeps the lanes' loads on
// distinct banks).
template <bool kLdg, int kRow = kN>
__device__ __forceinline__ uint64_t canon_mask_warp_min(int lane, uint64_t S,
                                                         const uint8_t* perm) {
  constexpr int kGroups = kGl2Order / 42;  // first rows (a, b) != (0, 0)
  int tg[2] = {9, 9};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int g = lane + 32 * h;
    if (g < kGroups) {
      const uint8_t* P = perm + g * 42 * kRow;
      uint32_t R = 0u;
      for (uint64_t x = S; x != 0ull; x &= x - 1ull) {
        const int p = __ffsll(static_cast<long long>(x)) - 1;
        const int idx = kLdg ? __ldg(P + p) : P[p];
        R |= 1u << ((idx * 37) >> 8);  // row idx / 7
      }
      tg[h] = min_top_row(R);
    }
  }
  int tstar = min(tg[0], tg[1]);
  for (int o = 16; o > 0; o >>= 1) tstar = min(tstar, __shfl_xor_sync(0xffffffffu, tstar, o));
  const unsigned cand0 = __ballot_sync(0xffffffffu, tg[0] == tstar);
  const unsigned cand1 = __ballot_sync(0xffffffffu, tg[1] == tstar) & 0xFFFFu;  // groups 32..47
  const int n0 = __popc(cand0);
  const int n_mat = 42 * (n0 + __popc(cand1));

  uint64_t best = ~0ull;
  int tb = tstar;       // no candidate can have a lower top row
  uint32_t pb = 0x7Fu;  // best's top-row bits (none yet)
  for (int j = lane, it = 0; j - lane < n_mat; j += 32, ++it) {
    if (j < n_mat) {
      // the (j / 42)-th candidate first row, matrix j % 42 of its group
      const int q = j / 42;
      const int g = q < n0 ? __fns(cand0, 0, q + 1) : 32 + __fns(cand1, 0, q - n0 + 1);
      const uint8_t* P = perm + (g * 42 + (j - 42 * q)) * kRow;
      uint64_t img = 0ull;
      uint32_t R = 0u;
      for (uint64_t x = S; x != 0ull; x &= x - 1ull) {
        const int p = __ffsll(static_cast<long long>(x)) - 1;
        const int idx = kLdg ? __ldg(P + p) : P[p];
        img |= 1ull << idx;
        R |= 1u << ((idx * 37) >> 8);  // row idx / 7
      }
      // Anchors q = (qa, qb) row by row: the rows after the shift, and so the
      // top row t and the image row ra that lands on it, depend on qa only.
      for (uint32_t rows = R; rows != 0u; rows &= rows - 1u) {
        const int qa = __ffs(rows) - 1;
        const uint32_t rr = ((R >> qa) | (R << (7 - qa))) & 0x7Fu;  // rows after the shift
        const int t = 31 - __clz(rr);
        if (t > tb) continue;
        int ra = qa + t;
        ra = ra >= 7 ? ra - 7 : ra;
        const uint32_t rb = uint32_t(img >> (7 * ra)) & 0x7Fu;
        for (uint32_t cols = uint32_t(img >> (7 * qa)) & 0x7Fu; cols != 0u; cols &= cols - 1u) {
          const int qb = __ffs(cols) - 1;
          // t == tb here (tb is already the smallest possible top row)
          if ((((rb >> qb) | (rb << (7 - qb))) & 0x7Fu) > pb) continue;
          const uint64_t cand = torus_shift(img, qa, qb);
          if (cand < best) {
            best = cand;
            mask_top_row(best, tb, pb);
          }
        }
      }
    }
    if ((it & 7) == 7 || j + 32 - lane >= n_mat) {
      uint64_t m = best;
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xffffffffu, m, o);
        m = other < m ? other : m;
      }
      if (m < best) {
        best = m;
        mask_top_row(best, tb, pb);
      }
    }
  }
  return best;
}

__device__ __forceinline__ void key_from_mask(uint64_t m, uint64_t& lo, uint64_t& hi) {
  const int k = __popcll(m);
  if (k < 1 || k > 16) {
    lo = ~0ull;
    hi = ~0ull;
    return;
  }
  const int pf = k <= 10 ? 0 : 1;
  lo = 0ull;
  hi = 0ull;
  int i = 0;
  while (m) {
    const int idx = __ffsll(static_cast<long long>(m)) - 1;
    m &= m - 1ull;
    if (i >= pf) {
      const int off = 6 * (i - pf);
      const uint64_t v = uint64_t(idx);
      if (off < 64) {
        lo |= v << off;
        if (off + 6 > 64) hi |= v >> (64 - off);
      } else {
        hi |= v << (off - 64);
      }
    }
    ++i;
  }
}

// Context tables shared by the kernels (device memory of one context).
struct DeviceTables {
  const uint8_t* M;       // 49 x 49 matrix entries (row-major)
  const uint64_t* Mp;     // 49 rows x 3 bit planes of M (bit j of plane b = bit b of M[row][j])
  const uint8_t* gl2;     // 2016 x 49 point permutations of GL2(F7)
};

}  // namespace tg

// Host-side helpers implemented in abi.cu.
namespace tg {
void set_last_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
}  // namespace tg
