// ORACLE — test infrastructure only.  Launch wrappers for the reference's own
// CUDA kernels, whose source strings build_ref.py extracts from the reference
// modules (kernel_cuda_bp.py:41-239 `_CUDA_BP_SRC`, kernel_canon.py:26-130
// `_CUDA_CANON_SRC`) into _ref/ and compiles together with this file.
// The launch geometry is the one of the reference Python wrappers:
//   eval_min_distance_batch_bp: grid = num_sets, block 256,
//       smem = align8(4k) + 192k + 8            (kernel_cuda_bp.py:262-264, 311-321)
//   eval_min_distance_single_bp: grid = ceil((8^k-1)/256), block 256,
//       smem = 192k                            (kernel_cuda_bp.py:260-261, 276-286)
//   canonical_forms: grid = ceil(32n/256), block 256, out_lo preset to
//       all ones and out_hi to zero             (kernel_canon.py:163-173)
// The tests use these kernels as the bit-exact GPU reference on the B200.
#include <cuda_runtime.h>

#include "_ref/ref_bp_src.cu"
#include "_ref/ref_canon_src.cu"

extern "C" int ref_bp_batch(const int* d_M, const int* d_sets, int k, int tmax, int n,
                            long long sample_count, unsigned long long seed, int* d_out,
                            void* stream) {
  if (n <= 0) return 0;
  const int s_bytes = ((k * 4 + 7) / 8) * 8;
  const int smem = s_bytes + 3 * k * 8 * 8 + 8;
  eval_min_distance_batch_bp<<<n, 256, smem, static_cast<cudaStream_t>(stream)>>>(
      d_M, d_sets, k, tmax, n, sample_count, seed, d_out);
  return static_cast<int>(cudaGetLastError());
}

// d_out must hold 0 before the call (cp.zeros in the reference).
extern "C" int ref_bp_single(const int* d_M, const int* d_s, int k, int tmax, int* d_out,
                             void* stream) {
  if (k <= 0 || k > 12) return -1;  // grid.x overflows 2^31-1 for k >= 13 in the reference
  const long long total = (1LL << (3 * k)) - 1;
  const long long grid = (total + 255) / 256;
  eval_min_distance_single_bp<<<static_cast<unsigned>(grid), 256, 3 * k * 8 * 8,
                                static_cast<cudaStream_t>(stream)>>>(d_M, d_s, k, tmax, total,
                                                                     d_out);
  return static_cast<int>(cudaGetLastError());
}

// out_lo must hold all ones and out_hi zero before the call.
extern "C" int ref_canon(const int* d_sets, const int* d_perms, const unsigned char* d_rel,
                         unsigned long long* d_lo, unsigned long long* d_hi, int n, int k,
                         void* stream) {
  if (n <= 0) return 0;
  const int threads = 256;
  const int grid = (n * 32 + threads - 1) / threads;
  canonical_forms<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      d_sets, d_perms, d_rel, d_lo, d_hi, n, k);
  return static_cast<int>(cudaGetLastError());
}
