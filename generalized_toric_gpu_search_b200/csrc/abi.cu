// extern "C" boundary of libtoric_b200.so (declared in include/toric_b200.h):
// argument checks, device selection, context tables and launch dispatch.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "canonical.cuh"
#include "distance.cuh"


namespace tg {

static thread_local char g_err[512] = "";

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what) {
  set_last_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return TG_ERR_CUDA;
}

static int invalid(const char* msg) {
  set_last_error("%s", msg);
  return TG_ERR_INVALID_ARGUMENT;
}

// Restores the calling thread's current device on scope exit.
class DeviceGuard {
 public:
  explicit DeviceGuard(int dev) {
    ok_ = cudaGetDevice(&prev_) == cudaSuccess;
    err_ = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (ok_) cudaSetDevice(prev_);
  }
  cudaError_t error() const { return err_; }

 private:
  int prev_ = 0;
  bool ok_ = false;
  cudaError_t err_ = cudaSuccess;
};

// The toric evaluation matrix of precompute.py:32-43: row a*7+b is x^a y^b,
// column j is the torus point (x, y) = (1 + j/7, 1 + j%7).
static void toric_matrix(uint8_t out[kN * kN]) {
  auto pw = [](uint8_t base, int e) {
    uint8_t r = 1;
    for (int i = 0; i < e; ++i) r = gf8_mul_c(r, base);
    return r;
  };
  for (int i = 0; i < kN; ++i)
    for (int j = 0; j < kN; ++j)
      out[i * kN + j] = gf8_mul_c(pw(uint8_t(1 + j / 7), i / 7), pw(uint8_t(1 + j % 7), i % 7));
}

// GL2(F7) as permutations of the 49 points, matrices (a b; c d) in the
// lexicographic order of (a, b, c, d) with nonzero determinant; point (x, y)
// maps to (a x + b y, c x + d y) (champion_search_canonical.py:61-74).
static void gl2_table(uint8_t out[kGl2Order * kN]) {
  int m = 0;
  for (int a = 0; a < 7; ++a)
    for (int b = 0; b < 7; ++b)
      for (int c = 0; c < 7; ++c)
        for (int d = 0; d < 7; ++d) {
          if (((a * d - b * c) % 7 + 7) % 7 == 0) continue;
          for (int p = 0; p < kN; ++p) {
            const int x = p / 7, y = p % 7;
            out[m * kN + p] = uint8_t(((a * x + b * y) % 7) * 7 + (c * x + d * y) % 7);
          }
          ++m;
        }
}

}  // namespace tg

using namespace tg;

extern "C" {

const char* tg_status_string(int status) {
  switch (status) {
    case TG_OK: return "TG_OK";
    case TG_ERR_INVALID_ARGUMENT: return "TG_ERR_INVALID_ARGUMENT";
    case TG_ERR_CUDA: return "TG_ERR_CUDA";
    case TG_ERR_WORKSPACE: return "TG_ERR_WORKSPACE";
    case TG_ERR_NO_DEVICE: return "TG_ERR_NO_DEVICE";
    case TG_ERR_CAPACITY: return "TG_ERR_CAPACITY";
    case TG_ERR_TIMEOUT: return "TG_ERR_TIMEOUT";
    case TG_ERR_BAD_INPUT: return "TG_ERR_BAD_INPUT";
    case TG_ERR_STATE: return "TG_ERR_STATE";
    default: return "TG_ERR_UNKNOWN";
  }
}

const char* tg_last_error(void) { return g_err; }

int tg_abi_version(void) { return TG_ABI_VERSION; }

int tg_device_count(int32_t* h_count) {
  if (!h_count) return invalid("tg_device_count: NULL output");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *h_count = 0;
    cudaGetLastError();
    set_last_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? TG_OK : TG_ERR_CUDA;
  }
  *h_count = n;
  return TG_OK;
}

int tg_device_info(int device, int32_t* h_sm_count, int32_t* h_cc_major, int32_t* h_cc_minor,
                   char* h_name, int32_t name_len) {
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    set_last_error("cudaGetDeviceProperties(%d): %s", device, cudaGetErrorString(e));
    return TG_ERR_NO_DEVICE;
  }
  if (h_sm_count) *h_sm_count = prop.multiProcessorCount;
  if (h_cc_major) *h_cc_major = prop.major;
  if (h_cc_minor) *h_cc_minor = prop.minor;
  if (h_name && name_len > 0) {
    std::strncpy(h_name, prop.name, size_t(name_len) - 1);
    h_name[name_len - 1] = '\0';
  }
  return TG_OK;
}

int tg_context_create(int device, const int32_t* h_M, tg_context** out_ctx) {
  if (!out_ctx) return invalid("tg_context_create: NULL out_ctx");
  *out_ctx = nullptr;
  if (!h_M) return invalid("tg_context_create: NULL matrix");
  uint8_t M[kN * kN];
  for (int i = 0; i < kN * kN; ++i) {
    if (h_M[i] < 0 || h_M[i] > 7) return invalid("tg_context_create: matrix entries must be 0..7");
    M[i] = uint8_t(h_M[i]);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_last_error("No CUDA GPU found.");
    return TG_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_last_error("device %d out of range (%d devices)", device, ndev);
    return TG_ERR_NO_DEVICE;
  }
  DeviceGuard g(device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  int st = upload_field_tables(device);
  if (st) return st;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
  uint8_t T[kN * kN];
  toric_matrix(T);
  std::vector<uint8_t> gl2(size_t(kGl2Order) * kN);
  gl2_table(gl2.data());
  tg_context* ctx = new tg_context();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  ctx->is_toric = std::memcmp(T, M, sizeof(M)) == 0 ? 1 : 0;
  // The rows of M bit-sliced (one 49-bit word per GF(8) bit), as the
  // information-set preparation loads them.
  uint64_t planes[kN * 3] = {};
  for (int r = 0; r < kN; ++r)
    for (int j = 0; j < kN; ++j)
      for (int b = 0; b < 3; ++b)
        planes[r * 3 + b] |= uint64_t((M[r * kN + j] >> b) & 1u) << j;
  e = cudaMalloc(&ctx->d_M, sizeof(M));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_Mp, sizeof(planes));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_gl2, gl2.size());
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_M, M, sizeof(M), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_Mp, planes, sizeof(planes), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_gl2, gl2.data(), gl2.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (ctx->d_M) cudaFree(ctx->d_M);
    if (ctx->d_Mp) cudaFree(ctx->d_Mp);
    if (ctx->d_gl2) cudaFree(ctx->d_gl2);
    delete ctx;
    return cuda_fail(e, "context tables");
  }
  *out_ctx = ctx;
  return TG_OK;
}

int tg_context_destroy(tg_context* ctx) {
  if (!ctx) return TG_OK;
  DeviceGuard g(ctx->device);
  if (ctx->d_M) cudaFree(ctx->d_M);
  if (ctx->d_Mp) cudaFree(ctx->d_Mp);
  if (ctx->d_gl2) cudaFree(ctx->d_gl2);
  delete ctx;
  return TG_OK;
}

int tg_context_is_toric(const tg_context* ctx, int32_t* h_is_toric) {
  if (!ctx || !h_is_toric) return invalid("tg_context_is_toric: NULL argument");
  *h_is_toric = ctx->is_toric;
  return TG_OK;
}

static int check_distance_params(const tg_distance_params* p) {
  if (!p) return invalid("NULL tg_distance_params");
  if (p->n_sets < 0) return invalid("n_sets must be >= 0");
  if (p->sample_count < 0) return invalid("sample_count must be >= 0");
  if (p->sample_count > 0) {
    if (p->k_max < 0 || p->k_max > kMaxSampledK)
      return invalid("CUDA-BP bit-parallel kernel supports k <= 49");
  } else if (p->k_max < 0 || p->k_max > kMaxExactK) {
    return invalid("Exact CUDA-BP batch evaluation supports k <= 21");
  }
  if (p->tail_rows != 0 && (p->tail_rows < 2 || p->tail_rows > 7))
    return invalid("tail_rows must be 0 or 2..7");
  if (p->enumeration < TG_ENUM_AUTO || p->enumeration > TG_ENUM_INFOSET)
    return invalid("unknown enumeration");
  if (p->variant < TG_VARIANT_AUTO || p->variant > TG_VARIANT_DIRECT)
    return invalid("unknown variant");
  if (p->blocks_per_sm < 0 || p->blocks_per_sm > 16) return invalid("blocks_per_sm must be 0..16");
  if (p->threads_per_block != 0 && p->threads_per_block != 64 && p->threads_per_block != 128 &&
      p->threads_per_block != 256)
    return invalid("threads_per_block must be 0, 64, 128 or 256");
  if (p->is_blocks_per_sm < 0 || p->is_blocks_per_sm > 5)
    return invalid("is_blocks_per_sm must be 0..5");
  if (p->is_tasks_per_thread < 0 || p->is_tasks_per_thread > 64)
    return invalid("is_tasks_per_thread must be 0..64");
  if (p->is_max_task_units < 0 || p->is_max_task_units > 2401)
    return invalid("is_max_task_units must be 0..2401");
  return TG_OK;
}

int tg_distance_workspace_size(const tg_distance_params* p, size_t* h_bytes) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!h_bytes) return invalid("NULL h_bytes");
  *h_bytes = ws_layout(*p).total;
  return TG_OK;
}

static void bind_workspace(DistArgs& a, const WsLayout& L, void* ws) {
  uint8_t* b = static_cast<uint8_t*>(ws);
  a.hdr = reinterpret_cast<WsHeader*>(b + L.hdr);
  a.desc = reinterpret_cast<CodeDesc*>(b + L.desc);
  a.task_off = reinterpret_cast<uint64_t*>(b + L.task_off);
  a.abort = reinterpret_cast<int32_t*>(b + L.abort);
  a.basis = reinterpret_cast<V6*>(b + L.basis);
  a.pat_cum = reinterpret_cast<uint64_t*>(b + L.pat_cum);
  a.pat_info = reinterpret_cast<uint32_t*>(b + L.pat_info);
  a.bitpat = reinterpret_cast<V6*>(b + L.bitpat);
  a.basis_stride = L.basis_stride;
  a.pat_stride = L.pat_stride;
  a.bitpat_stride = L.bitpat_stride;
  a.is_min_k = L.is_min_k;
  a.is_stride = L.is_stride;
  a.is_hdr = reinterpret_cast<IsHeader*>(b + L.is_hdr);
  a.is_rows = reinterpret_cast<V6*>(b + L.is_rows);
  a.is_units = reinterpret_cast<uint64_t*>(b + L.is_units);
  a.is_off = reinterpret_cast<uint64_t*>(b + L.is_off);
  a.is_best = reinterpret_cast<int32_t*>(b + L.is_best);
  a.is_perm = reinterpret_cast<int32_t*>(b + L.is_perm);
}

// Validates a max_zeros call and fills the kernel arguments.
static int bind_distance(tg_context* ctx, const tg_distance_params* p, const int32_t* d_indices,
                         const int64_t* d_offsets, const int32_t* d_target,
                         const int32_t* d_set_ids, int32_t* d_out, void* d_workspace,
                         size_t workspace_bytes, bool need_inputs, DistArgs& a) {
  if (!ctx) return invalid("tg_max_zeros: NULL context");
  int st = check_distance_params(p);
  if (st) return st;
  if (p->n_sets == 0) return TG_OK;
  if ((need_inputs && (!d_indices || !d_offsets)) || !d_out)
    return invalid("tg_max_zeros: NULL device pointer");
  if (!d_workspace || (reinterpret_cast<uintptr_t>(d_workspace) & 255u))
    return invalid("tg_max_zeros: workspace must be non-NULL and 256-byte aligned");
  const WsLayout L = ws_layout(*p);
  if (workspace_bytes < L.total) {
    set_last_error("tg_max_zeros: workspace has %zu bytes, needs %zu", workspace_bytes, L.total);
    return TG_ERR_WORKSPACE;
  }
  // Enumeration of the codes below the information-set threshold.
  int enumeration = p->enumeration;
  if (enumeration == TG_ENUM_AUTO) enumeration = ctx->is_toric ? TG_ENUM_ORBIT : TG_ENUM_PROJECTIVE;
  if (enumeration == TG_ENUM_INFOSET) enumeration = TG_ENUM_PROJECTIVE;
  if (enumeration == TG_ENUM_ORBIT && !ctx->is_toric)
    return invalid("orbit enumeration needs the toric evaluation matrix");
  int variant = p->variant;
  if (variant == TG_VARIANT_AUTO) variant = ctx->is_toric ? TG_VARIANT_HISTOGRAM : TG_VARIANT_DIRECT;
  if (variant == TG_VARIANT_HISTOGRAM && !ctx->is_toric)
    return invalid("histogram variant needs the toric evaluation matrix");
  a = DistArgs{};
  a.idx = d_indices;
  a.off = d_offsets;
  a.target = d_target;
  a.set_ids = d_set_ids;
  a.out = d_out;
  a.n = p->n_sets;
  a.k_max = p->k_max;
  a.R = default_tail_rows(*p);
  a.enumeration = enumeration;
  a.variant = variant;
  a.td_default = p->target_distance;
  a.sample_count = p->sample_count;
  a.seed = p->sample_seed;
  a.tab.M = ctx->d_M;
  a.tab.Mp = ctx->d_Mp;
  a.tab.gl2 = ctx->d_gl2;
  a.is_toric = ctx->is_toric;
  a.is_blocks_per_sm = p->is_blocks_per_sm > 0 ? p->is_blocks_per_sm : 5;
  // defaults: the shape the tuner picks for k = 14, the largest codes of a
  // batch of 10,000 sets with k from 6 to 14
  a.is_tasks_per_thread = p->is_tasks_per_thread > 0 ? p->is_tasks_per_thread : 4;
  a.is_max_task_units = p->is_max_task_units > 0 ? p->is_max_task_units : 49;
  bind_workspace(a, L, d_workspace);
  return TG_OK;
}

static int launch_shape(const tg_distance_params* p, int* bps, int* tpb) {
  *bps = p->blocks_per_sm > 0 ? p->blocks_per_sm : 8;
  *tpb = p->threads_per_block > 0 ? p->threads_per_block : 128;
  return TG_OK;
}

int tg_max_zeros_prepare(tg_context* ctx, const tg_distance_params* p, const int32_t* d_indices,
                         const int64_t* d_offsets, const int32_t* d_target,
                         const int32_t* d_set_ids, int32_t* d_out, void* d_workspace,
                         size_t workspace_bytes, void* stream) {
  DistArgs a;
  int st = bind_distance(ctx, p, d_indices, d_offsets, d_target, d_set_ids, d_out, d_workspace,
                         workspace_bytes, true, a);
  if (st || p->n_sets == 0) return st;
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  return run_prepare(a, static_cast<cudaStream_t>(stream));
}

int tg_max_zeros_walk_part(tg_context* ctx, const tg_distance_params* p, int32_t parts,
                           int32_t* d_out, void* d_workspace, size_t workspace_bytes,
                           void* stream) {
  if (parts < 1 || parts > (TG_WALK_ENUMERATION | TG_WALK_INFOSET))
    return invalid("tg_max_zeros_walk_part: parts must be a nonempty mask of TG_WALK_*");
  DistArgs a;
  int st = bind_distance(ctx, p, nullptr, nullptr, nullptr, nullptr, d_out, d_workspace,
                         workspace_bytes, false, a);
  if (st || p->n_sets == 0) return st;
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  int bps, tpb;
  launch_shape(p, &bps, &tpb);
  return run_walk(a, ctx->sm_count, bps, tpb, static_cast<cudaStream_t>(stream),
                  (parts & TG_WALK_ENUMERATION ? kWalkEnumeration : 0) |
                      (parts & TG_WALK_INFOSET ? kWalkInfoset : 0));
}

int tg_max_zeros_walk(tg_context* ctx, const tg_distance_params* p, int32_t* d_out,
                      void* d_workspace, size_t workspace_bytes, void* stream) {
  return tg_max_zeros_walk_part(ctx, p, TG_WALK_ENUMERATION | TG_WALK_INFOSET, d_out,
                                d_workspace, workspace_bytes, stream);
}

int tg_max_zeros(tg_context* ctx, const tg_distance_params* p, const int32_t* d_indices,
                 const int64_t* d_offsets, const int32_t* d_target, const int32_t* d_set_ids,
                 int32_t* d_out, void* d_workspace, size_t workspace_bytes, void* stream) {
  DistArgs a;
  int st = bind_distance(ctx, p, d_indices, d_offsets, d_target, d_set_ids, d_out, d_workspace,
                         workspace_bytes, true, a);
  if (st || p->n_sets == 0) return st;
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = run_prepare(a, s);
  if (st) return st;
  int bps, tpb;
  launch_shape(p, &bps, &tpb);
  return run_walk(a, ctx->sm_count, bps, tpb, s);
}

}  // extern "C"

namespace tg {

// Workspace of tg_max_zeros_witness: the first pass (the caller's
// parameters), the witness pass (information sets for every k >= 1), and the
// pass's values, targets, claim words and pivot columns.
struct WitLayout {
  WsLayout p1, p2;
  size_t off2, out2, td2, lock, piv, total;
};

static tg_distance_params witness_pass_params(const tg_distance_params& p) {
  tg_distance_params q = p;
  q.enumeration = kEnumInfosetAll;
  q.target_distance = 1;
  q.sample_count = 0;
  return q;
}

static WitLayout witness_layout(const tg_distance_params& p) {
  WitLayout L{};
  const size_t n = size_t(p.n_sets > 0 ? p.n_sets : 0);
  L.p1 = ws_layout(p);
  L.p2 = ws_layout(witness_pass_params(p));
  size_t off = align_ws(L.p1.total);
  L.off2 = off;  off = align_ws(off + L.p2.total);
  L.out2 = off;  off = align_ws(off + n * sizeof(int32_t));
  L.td2 = off;   off = align_ws(off + n * sizeof(int32_t));
  L.lock = off;  off = align_ws(off + n * sizeof(int32_t));
  L.piv = off;   off = align_ws(off + n * kIsMaxSets * sizeof(uint64_t));
  L.total = off;
  return L;
}

}  // namespace tg

extern "C" {

int tg_infoset_last_level(int32_t k_max, int32_t is_toric, int32_t* h_level) {
  if (!h_level) return invalid("tg_infoset_last_level: NULL output");
  if (k_max < 0 || k_max > kMaxExactK) return invalid("k_max must be 0..21");
  *h_level = infoset_last_level(k_max, is_toric ? 1 : 0);
  return TG_OK;
}

int tg_witness_workspace_size(const tg_distance_params* p, size_t* h_bytes) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!h_bytes) return invalid("NULL h_bytes");
  if (p->sample_count > 0) return invalid("witnesses are defined for exact max_zeros only");
  *h_bytes = witness_layout(*p).total;
  return TG_OK;
}

int tg_max_zeros_witness(tg_context* ctx, const tg_distance_params* p, const int32_t* d_indices,
                         const int64_t* d_offsets, const int32_t* d_target,
                         const int32_t* d_set_ids, int32_t* d_out, uint8_t* d_witness,
                         void* d_workspace, size_t workspace_bytes, void* stream) {
  if (!ctx) return invalid("tg_max_zeros_witness: NULL context");
  int st = check_distance_params(p);
  if (st) return st;
  if (p->sample_count > 0) return invalid("witnesses are defined for exact max_zeros only");
  if (p->n_sets == 0) return TG_OK;
  if (!d_witness) return invalid("tg_max_zeros_witness: NULL witness buffer");
  const WitLayout W = witness_layout(*p);
  if (workspace_bytes < W.total) {
    set_last_error("tg_max_zeros_witness: workspace has %zu bytes, needs %zu", workspace_bytes,
                   W.total);
    return TG_ERR_WORKSPACE;
  }
  DistArgs a1;
  st = bind_distance(ctx, p, d_indices, d_offsets, d_target, d_set_ids, d_out, d_workspace,
                     workspace_bytes, true, a1);
  if (st) return st;
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int bps, tpb;
  launch_shape(p, &bps, &tpb);
  // Pass 1: max_zeros as tg_max_zeros computes it.
  st = run_prepare(a1, s);
  if (!st) st = run_walk(a1, ctx->sm_count, bps, tpb, s);
  if (st) return st;
  // Pass 2: information sets with per-set targets 50 - out, recording the
  // first codeword below each target.
  uint8_t* b = static_cast<uint8_t*>(d_workspace);
  DistArgs a2 = a1;
  bind_workspace(a2, W.p2, b + W.off2);
  a2.sample_count = 0;
  a2.td_default = 1;
  a2.target = reinterpret_cast<int32_t*>(b + W.td2);
  a2.out = reinterpret_cast<int32_t*>(b + W.out2);
  a2.is_piv = reinterpret_cast<uint64_t*>(b + W.piv);
  a2.witness = d_witness;
  a2.wit_lock = reinterpret_cast<int32_t*>(b + W.lock);
  cudaError_t e = cudaMemsetAsync(d_witness, 0, size_t(p->n_sets) * kN, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(a2.wit_lock, 0, size_t(p->n_sets) * sizeof(int32_t), s);
  if (e != cudaSuccess) return cuda_fail(e, "tg_max_zeros_witness: clear witness buffers");
  st = run_witness_targets(d_out, d_offsets, reinterpret_cast<int32_t*>(b + W.td2), p->n_sets, s);
  if (!st) st = run_prepare(a2, s);
  if (!st) st = run_walk(a2, ctx->sm_count, bps, tpb, s);
  if (!st) st = run_witness_finish(a2, d_out, a1.hdr, s);
  return st;
}

int tg_distance_status(const tg_distance_params* p, const void* d_workspace, void* stream,
                       int32_t* h_status) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!d_workspace || !h_status) return invalid("tg_distance_status: NULL argument");
  const WsLayout L = ws_layout(*p);
  WsHeader h{};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(&h, static_cast<const uint8_t*>(d_workspace) + L.hdr, sizeof(h),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "tg_distance_status");
  *h_status = h.status;
  return TG_OK;
}

int tg_distance_counters(const tg_distance_params* p, const void* d_workspace, void* stream,
                         uint64_t* h_tasks, uint64_t* h_codewords, double* h_reference_messages) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!d_workspace) return invalid("tg_distance_counters: NULL workspace");
  const WsLayout L = ws_layout(*p);
  WsHeader h{};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(&h, static_cast<const uint8_t*>(d_workspace) + L.hdr, sizeof(h),
                                  cudaMemcpyDeviceToHost, s);
  IsHeader hi{};
  if (e == cudaSuccess && L.is_min_k <= p->k_max && p->n_sets > 0)
    e = cudaMemcpyAsync(&hi, static_cast<const uint8_t*>(d_workspace) + L.is_hdr, sizeof(hi),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "tg_distance_counters");
  if (h_tasks) *h_tasks = h.total_tasks + hi.tasks_all;
  if (h_codewords) *h_codewords = h.codewords + hi.codewords;
  if (h_reference_messages) *h_reference_messages = h.ref_messages;
  return TG_OK;
}

int tg_distance_path_counters(const tg_distance_params* p, const void* d_workspace, void* stream,
                              uint64_t* h_counts) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!d_workspace || !h_counts) return invalid("tg_distance_path_counters: NULL argument");
  const WsLayout L = ws_layout(*p);
  WsHeader h{};
  IsHeader hi{};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint8_t* b = static_cast<const uint8_t*>(d_workspace);
  cudaError_t e = cudaMemcpyAsync(&h, b + L.hdr, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && L.is_min_k <= p->k_max && p->n_sets > 0)
    e = cudaMemcpyAsync(&hi, b + L.is_hdr, sizeof(hi), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "tg_distance_path_counters");
  h_counts[0] = h.total_tasks;
  h_counts[1] = h.codewords;
  h_counts[2] = hi.tasks_all;
  h_counts[3] = hi.codewords;
  return TG_OK;
}

static_assert(kIsStages == TG_INFOSET_STAGES, "stage count of the header");

int tg_distance_stage_counters(const tg_distance_params* p, const void* d_workspace, void* stream,
                               uint64_t* h_counts, int32_t n) {
  int st = check_distance_params(p);
  if (st) return st;
  if (!d_workspace || !h_counts) return invalid("tg_distance_stage_counters: NULL argument");
  if (n < 0) return invalid("tg_distance_stage_counters: n must be >= 0");
  const WsLayout L = ws_layout(*p);
  IsHeader hi{};
  if (L.is_min_k <= p->k_max && p->n_sets > 0) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&hi, static_cast<const uint8_t*>(d_workspace) + L.is_hdr,
                                    sizeof(hi), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "tg_distance_stage_counters");
  }
  // Levels 1 to 3 add to the total only (one CTA per set; no second atomic).
  unsigned long long later = 0ull;
  for (int i = 1; i < kIsStages; ++i) later += hi.stage_codewords[i];
  hi.stage_codewords[0] = hi.codewords - later;
  for (int i = 0; i < n && i < kIsStages; ++i) h_counts[i] = hi.stage_codewords[i];
  return TG_OK;
}

int tg_canonical_sets(tg_context* ctx, const int32_t* d_sets, int32_t n, int32_t k,
                      uint64_t* d_out_mask, uint64_t* d_out_key_lo, uint64_t* d_out_key_hi,
                      int32_t* d_status, void* stream) {
  if (!ctx) return invalid("tg_canonical_sets: NULL context");
  if (n < 0) return invalid("tg_canonical_sets: n must be >= 0");
  if (k < 0 || k > kN) return invalid("tg_canonical_sets: k must be 0..49");
  if (n == 0) return TG_OK;
  if ((k > 0 && !d_sets) || !d_out_mask) return invalid("tg_canonical_sets: NULL device pointer");
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  static const int32_t kDummy = 0;
  return run_canonical(ctx->device, ctx->sm_count, ctx->d_gl2, k > 0 ? d_sets : &kDummy, nullptr,
                       n, k, d_out_mask, d_out_key_lo, d_out_key_hi, d_status,
                       static_cast<cudaStream_t>(stream));
}

int tg_canonical_masks(tg_context* ctx, const uint64_t* d_masks, int32_t n, uint64_t* d_out_mask,
                       uint64_t* d_out_key_lo, uint64_t* d_out_key_hi, void* stream) {
  if (!ctx) return invalid("tg_canonical_masks: NULL context");
  if (n < 0) return invalid("tg_canonical_masks: n must be >= 0");
  if (n == 0) return TG_OK;
  if (!d_masks || !d_out_mask) return invalid("tg_canonical_masks: NULL device pointer");
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  return run_canonical(ctx->device, ctx->sm_count, ctx->d_gl2, nullptr, d_masks, n, 0, d_out_mask,
                       d_out_key_lo, d_out_key_hi, nullptr, static_cast<cudaStream_t>(stream));
}

int tg_expand_canonical(tg_context* ctx, const uint64_t* d_parents, int32_t n, uint64_t* d_out,
                        void* stream) {
  if (!ctx) return invalid("tg_expand_canonical: NULL context");
  if (n < 0 || int64_t(n) * kN > int64_t(0x7fffffff))
    return invalid("tg_expand_canonical: n must be >= 0 and n * 49 < 2^31");
  if (n == 0) return TG_OK;
  if (!d_parents || !d_out) return invalid("tg_expand_canonical: NULL device pointer");
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  return run_canonical(ctx->device, ctx->sm_count, ctx->d_gl2, nullptr, d_parents, n * kN, 0,
                       d_out, nullptr, nullptr, nullptr, static_cast<cudaStream_t>(stream), 1);
}

int tg_compact_scratch_bytes(int32_t n, size_t* h_bytes) {
  if (!h_bytes || n < 0) return invalid("tg_compact_scratch_bytes: bad argument");
  *h_bytes = compact_scratch_bytes(n);
  return TG_OK;
}

int tg_compact_sets(const uint64_t* d_masks, const uint8_t* d_flags, int32_t n, int32_t k,
                    void* d_scratch, uint64_t* d_out_masks, int32_t* d_out_sets,
                    int64_t* d_out_offsets, int32_t* d_count, void* stream) {
  if (n < 0 || k < 0 || k > kN) return invalid("tg_compact_sets: bad n or k");
  if (!d_count || (n > 0 && (!d_masks || !d_flags || !d_scratch)))
    return invalid("tg_compact_sets: NULL device pointer");
  return run_compact(d_masks, d_flags, n, k, d_scratch, d_out_masks, d_out_sets, d_out_offsets,
                     d_count, static_cast<cudaStream_t>(stream));
}

int tg_hashset_bytes(int64_t capacity, size_t* h_bytes) {
  if (!h_bytes) return invalid("tg_hashset_bytes: NULL output");
  if (capacity < 64 || (capacity & (capacity - 1)))
    return invalid("hash set capacity must be a power of two >= 64");
  *h_bytes = hashset_bytes(capacity);
  return TG_OK;
}

int tg_hashset_clear(void* d_table, int64_t capacity, void* stream) {
  if (!d_table) return invalid("tg_hashset_clear: NULL table");
  if (capacity < 64 || (capacity & (capacity - 1)))
    return invalid("hash set capacity must be a power of two >= 64");
  return run_hash_clear(d_table, capacity, static_cast<cudaStream_t>(stream));
}

int tg_hashset_insert(void* d_table, int64_t capacity, const uint64_t* d_keys, int32_t n,
                      uint32_t call_id, uint8_t* d_is_new, int32_t* d_n_new, int32_t* d_status,
                      void* stream) {
  if (!d_table) return invalid("tg_hashset_insert: NULL table");
  if (capacity < 64 || (capacity & (capacity - 1)))
    return invalid("hash set capacity must be a power of two >= 64");
  if (n < 0) return invalid("tg_hashset_insert: n must be >= 0");
  if (n > 0 && !d_keys) return invalid("tg_hashset_insert: NULL keys");
  if (call_id == 0) return invalid("tg_hashset_insert: call_id must be >= 1");
  return run_hash_insert(d_table, capacity, d_keys, n, call_id, d_is_new, d_n_new, d_status,
                         static_cast<cudaStream_t>(stream));
}

int tg_measure_int_pipes(int device, void* d_scratch, double* h_out6) {
  if (!d_scratch || !h_out6) return invalid("tg_measure_int_pipes: NULL argument");
  int32_t sm = 0;
  int st = tg_device_info(device, &sm, nullptr, nullptr, nullptr, 0);
  if (st) return st;
  DeviceGuard g(device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  return measure_int_pipes(sm, d_scratch, h_out6);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Zero-allocation max_zeros: the workspace is a scratch array compiled into
// the library instead of caller memory.
// ---------------------------------------------------------------------------

namespace tg {

constexpr size_t kStaticWorkspaceBytes = size_t(TG_STATIC_WORKSPACE_BYTES);

// One copy per device that loads the library, alive until the process exits.
static __device__ __align__(256) uint8_t g_static_workspace[kStaticWorkspaceBytes];

// Device address of g_static_workspace per device ordinal.  In host code the
// symbol itself is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and cached here.
static void* g_static_workspace_addr[64] = {nullptr};
static std::mutex g_static_workspace_mu;

static int static_workspace_address(int device, void** out) {
  if (device < 0 || device >= 64) {
    set_last_error("device %d has no static workspace slot", device);
    return TG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_static_workspace_mu);
  if (!g_static_workspace_addr[device]) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_workspace);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_workspace)");
    g_static_workspace_addr[device] = addr;
  }
  *out = g_static_workspace_addr[device];
  return TG_OK;
}

}  // namespace tg

extern "C" int tg_max_zeros_noalloc(tg_context* ctx, const tg_distance_params* p,
                                    const int32_t* d_indices, const int64_t* d_offsets,
                                    const int32_t* d_target, const int32_t* d_set_ids,
                                    int32_t* d_out, void* stream) {
  if (!ctx) return invalid("tg_max_zeros_noalloc: NULL context");
  int st = check_distance_params(p);
  if (st) return st;
  if (p->n_sets == 0) return TG_OK;
  const size_t need = ws_layout(*p).total;
  if (need > kStaticWorkspaceBytes) {
    set_last_error("tg_max_zeros_noalloc: this batch needs %zu bytes of workspace but the "
                   "static workspace holds %zu; split the batch or use tg_max_zeros",
                   need, kStaticWorkspaceBytes);
    return TG_ERR_WORKSPACE;
  }
  DeviceGuard g(ctx->device);
  if (g.error() != cudaSuccess) return cuda_fail(g.error(), "cudaSetDevice");
  void* ws = nullptr;
  st = static_workspace_address(ctx->device, &ws);
  if (st) return st;
  DistArgs a;
  st = bind_distance(ctx, p, d_indices, d_offsets, d_target, d_set_ids, d_out, ws,
                     kStaticWorkspaceBytes, true, a);
  if (st) return st;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = run_prepare(a, s);
  if (st) return st;
  int bps, tpb;
  launch_shape(p, &bps, &tpb);
  return run_walk(a, ctx->sm_count, bps, tpb, s);
}
