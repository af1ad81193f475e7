// Integer pipe throughput of the SM, the denominators of the distance
// kernel's roofline.  Each variant runs 8 independent dependency chains per
// thread, 1024 threads per CTA and one CTA per SM, and reports operations per
// SM per clock from clock64() around the timed loop.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "canonical.cuh"

namespace tg {

enum PipeOp { kOpLop3 = 0, kOpPopc = 1, kOpIadd = 2, kOpAddMax = 3, kOpLop3Popc = 4 };

constexpr int kChains = 8;
constexpr int kUnroll = 16;
constexpr int kPipeThreads = 1024;

template <int kOp>
__global__ void __launch_bounds__(kPipeThreads, 1)
pipe_kernel(uint32_t* sink, long long* cycles, int iters) {
  uint32_t x[kChains], y[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) {
    x[i] = threadIdx.x * 0x9E3779B9u + uint32_t(i) * 0x85EBCA6Bu + blockIdx.x;
    y[i] = x[i] ^ 0x5BD1E995u;
  }
  const uint32_t b = threadIdx.x ^ 0x27D4EB2Du;
  const uint32_t c = blockIdx.x * 0x165667B1u + 7u;
  __syncthreads();
  const long long t0 = clock64();
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int i = 0; i < kChains; ++i) {
        if (kOp == kOpLop3) {
          asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[i]) : "r"(b), "r"(c));
        } else if (kOp == kOpPopc) {
          asm volatile("popc.b32 %0, %0;" : "+r"(x[i]));
        } else if (kOp == kOpIadd) {
          asm volatile("add.u32 %0, %0, %1;" : "+r"(x[i]) : "r"(b));
        } else if (kOp == kOpAddMax) {
          x[i] = uint32_t(__viaddmax_s32(int(x[i]), int(b), int(c ^ x[i])));
        } else {
          asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[i]) : "r"(b), "r"(c));
          asm volatile("popc.b32 %0, %0;" : "+r"(y[i]));
        }
      }
    }
  }
  __syncthreads();
  const long long t1 = clock64();
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) acc ^= x[i] ^ y[i];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

template <int kOp>
static int run_pipe(int sm_count, uint32_t* sink, long long* cyc, int iters, double ops_per_iter,
                    double* rate, double* mhz) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  pipe_kernel<kOp><<<sm_count, kPipeThreads>>>(sink, cyc, 2);  // warm-up
  cudaEventRecord(e0);
  pipe_kernel<kOp><<<sm_count, kPipeThreads>>>(sink, cyc, iters);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "pipe_kernel");
  std::vector<long long> h(sm_count);
  e = cudaMemcpy(h.data(), cyc, sizeof(long long) * sm_count, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(cycles)");
  std::sort(h.begin(), h.end());
  const double med = double(h[sm_count / 2]);
  const double ops = double(kPipeThreads) * iters * kUnroll * kChains * ops_per_iter;
  *rate = ops / med;
  if (mhz) *mhz = med / (double(ms) * 1e3);
  return TG_OK;
}

int measure_int_pipes(int sm_count, void* d_scratch, double* out6) {
  uint32_t* sink = static_cast<uint32_t*>(d_scratch);
  long long* cyc = reinterpret_cast<long long*>(static_cast<uint8_t*>(d_scratch) + (768 << 10));
  if (size_t(sm_count) * kPipeThreads * 4 > (768u << 10)) return TG_ERR_INVALID_ARGUMENT;
  const int iters = 4096;
  int st;
  double mhz = 0.0;
  if ((st = run_pipe<kOpLop3>(sm_count, sink, cyc, iters, 1.0, &out6[0], &mhz))) return st;
  if ((st = run_pipe<kOpPopc>(sm_count, sink, cyc, iters, 1.0, &out6[1], nullptr))) return st;
  if ((st = run_pipe<kOpIadd>(sm_count, sink, cyc, iters, 1.0, &out6[2], nullptr))) return st;
  if ((st = run_pipe<kOpAddMax>(sm_count, sink, cyc, iters, 1.0, &out6[3], nullptr))) return st;
  if ((st = run_pipe<kOpLop3Popc>(sm_count, sink, cyc, iters, 2.0, &out6[4], nullptr))) return st;
  out6[5] = mhz;
  return TG_OK;
}

}  // namespace tg
