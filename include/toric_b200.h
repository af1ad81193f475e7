/*
 * toric_b200.h — C ABI of libtoric_b200.so, the sm_100a implementation of the
 * GF(8) generalized-toric-code hot path:
 *
 *   - max_zeros: for a code spanned by the rows M[S] of the 49x49 evaluation
 *     matrix, the largest number of zero coordinates of a nonzero codeword
 *     (minimum distance d = 49 - max_zeros), with the reference's early-exit
 *     threshold and its splitmix64 sampled screening mode;
 *   - the AGL2(F7) canonical form of an exponent set (anchored minimum, with
 *     the reference's packed 6-bit key for k <= 16 and a 49-bit mask for any k);
 *   - a device hash set that deduplicates canonical keys;
 *   - a device-resident serving loop (continuous batching of max_zeros
 *     requests with per-request thresholds and canonical dedup).
 *
 * Conventions
 *   - Every entry point returns a status code (TG_OK == 0); no exception ever
 *     crosses the boundary.  tg_status_string() names a code and
 *     tg_last_error() gives the message of the calling thread's last failure.
 *   - Pointers named d_* are device pointers on the context's device; h_*
 *     are host pointers.  `stream` is a cudaStream_t passed as void*
 *     (NULL = legacy default stream).  Work is enqueued on `stream` and the
 *     call returns without synchronising unless stated otherwise.
 *   - The library owns only its small per-context constant tables.  All
 *     per-call scratch lives in caller-provided workspaces, so the calls are
 *     re-entrant per stream and can be captured into CUDA graphs.
 *   - Exponent index i in 0..48 is the point (a, b) = (i / 7, i % 7) of Z_7^2;
 *     row i of M is the monomial x^a y^b evaluated at the 49 torus points.
 */
#ifndef TORIC_B200_H
#define TORIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TG_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
enum {
  TG_OK = 0,
  TG_ERR_INVALID_ARGUMENT = 1, /* bad size, k out of range, NULL pointer   */
  TG_ERR_CUDA = 2,             /* a CUDA runtime call failed               */
  TG_ERR_WORKSPACE = 3,        /* workspace smaller than required          */
  TG_ERR_NO_DEVICE = 4,        /* no CUDA device / bad device ordinal      */
  TG_ERR_CAPACITY = 5,         /* hash table or serving ring full          */
  TG_ERR_TIMEOUT = 6,          /* a bounded device wait gave up            */
  TG_ERR_BAD_INPUT = 7,        /* index outside 0..48 found on the device  */
  TG_ERR_STATE = 8             /* call not valid in the object's state     */
};

typedef struct tg_context tg_context;

/* Name of a status code (static string). */
const char* tg_status_string(int status);
/* Message of the calling thread's most recent failed call (static per thread). */
const char* tg_last_error(void);
/* TG_ABI_VERSION of the loaded library. */
int tg_abi_version(void);

/* ---- device and context ------------------------------------------------ */

/* Number of visible CUDA devices (0 when none). */
int tg_device_count(int32_t* h_count);

/* SM count, compute capability and name of a device. */
int tg_device_info(int device, int32_t* h_sm_count, int32_t* h_cc_major,
                   int32_t* h_cc_minor, char* h_name, int32_t name_len);

/* Creates a context on `device` from the 49x49 evaluation matrix M (host,
 * row-major int32, entries 0..7).  Replaces DistanceOracleCUDABP.__init__
 * (kernel_cuda_bp.py:251-258) and CanonicalOracle.__init__
 * (kernel_canon.py:137-148): uploads the matrix tables and the GL2(F7) point
 * permutations once.  When M equals the toric matrix of precompute.py:32-43
 * the context enables the torus-orbit enumeration (see tg_distance_params). */
int tg_context_create(int device, const int32_t* h_M, tg_context** out_ctx);
int tg_context_destroy(tg_context* ctx);
/* 1 when the context's M is the toric evaluation matrix, else 0. */
int tg_context_is_toric(const tg_context* ctx, int32_t* h_is_toric);

/* ---- max_zeros (exact and sampled) -------------------------------------- */

/* Exact enumeration strategies.  All give the same max_zeros (and the same
 * pass/fail decision under an early exit); they differ in how many codewords
 * they evaluate.
 *   AUTO        sets with k >= TG_INFOSET_AUTO_MIN_K (2) by information
 *               sets, the others (k = 1) by orbit (toric context) or
 *               projective enumeration
 *   PROJECTIVE  every message whose first nonzero coefficient is 1
 *   ORBIT       projective + torus-orbit normalisation (toric context only)
 *   INFOSET     information sets (Brouwer-Zimmermann) for every set, k >= 2:
 *               messages of weight 1, 2, ... on disjoint information sets,
 *               stopping when the weight bound of the unseen codewords
 *               reaches the best weight found; any evaluation matrix */
enum {
  TG_ENUM_AUTO = 0,
  TG_ENUM_PROJECTIVE = 1,
  TG_ENUM_ORBIT = 2,
  TG_ENUM_INFOSET = 3
};
#define TG_INFOSET_AUTO_MIN_K 2
enum {
  TG_VARIANT_AUTO = 0,      /* histogram when the context is toric            */
  TG_VARIANT_HISTOGRAM = 1, /* last row via an 8-bin zero histogram           */
  TG_VARIANT_DIRECT = 2     /* one popcount pair per codeword                 */
};

typedef struct tg_distance_params {
  int32_t n_sets;          /* number of codes in the batch (>= 0)            */
  int32_t k_max;           /* largest k in the batch (exact: <= 21, sampled: <= 49) */
  int32_t tail_rows;       /* R: rows walked inside one task; 0 = default    */
  int32_t enumeration;     /* TG_ENUM_*                                      */
  int32_t variant;         /* TG_VARIANT_*                                   */
  int32_t blocks_per_sm;   /* persistent CTAs per SM; 0 = default            */
  int32_t threads_per_block; /* 0 = default (128)                            */
  int32_t target_distance; /* used for every set when d_target is NULL       */
  int64_t sample_count;    /* 0 = exact; > 0 = reference sampled screening   */
  uint64_t sample_seed;    /* splitmix64 seed of the sampled mode            */
  /* Launch shape of the information-set walk (ABI version 2): */
  int32_t is_blocks_per_sm;    /* CTAs of 128 threads per SM, 1..5; 0 = 5        */
  int32_t is_tasks_per_thread; /* a level is cut into about this many tasks per
                                  resident thread, 1..64; 0 = 4                  */
  int32_t is_max_task_units;   /* largest task, in 49-codeword blocks, 1..2401;
                                  0 = 49                                         */
  int32_t is_pad;
} tg_distance_params;

/* Bytes of workspace tg_max_zeros needs for these parameters. */
int tg_distance_workspace_size(const tg_distance_params* p, size_t* h_bytes);

/* max_zeros of every set of a batch of mixed sizes, in one persistent launch.
 * Replaces DistanceOracleCUDABP.max_zeros_batch (kernel_cuda_bp.py:290-323,
 * kernel eval_min_distance_batch_bp :146-238) and DistanceOracle.max_zeros_batch
 * (kernel.py:276-323); a one-set batch replaces max_zeros
 * (kernel_cuda_bp.py:266-288, kernel.py:241-274).
 *   d_indices  flat exponent indices of all sets (int32, 0..48)
 *   d_offsets  n_sets+1 int64 offsets into d_indices (set s = [off[s], off[s+1]))
 *   d_target   per-set target_distance (int32) or NULL (p->target_distance)
 *   d_set_ids  per-set sampling id (the reference's blockIdx.x) or NULL (= s)
 *   d_out      per-set max_zeros (int32).  A set passes iff out <= 49 - td, and
 *              then out is exact; a failing set returns a witness > 49 - td.
 * The workspace must be 256-byte aligned and hold tg_distance_workspace_size
 * bytes.  Indices outside 0..48 make the call report TG_ERR_BAD_INPUT through
 * tg_distance_status() after the stream reaches it. */
int tg_max_zeros(tg_context* ctx, const tg_distance_params* p,
                 const int32_t* d_indices, const int64_t* d_offsets,
                 const int32_t* d_target, const int32_t* d_set_ids,
                 int32_t* d_out, void* d_workspace, size_t workspace_bytes,
                 void* stream);

/* The two halves of tg_max_zeros, for callers that time or capture them
 * separately: _prepare validates the sets, orders rows, builds the bit-sliced
 * bases, the information sets and the task tables (prep + scan kernels);
 * _walk runs the persistent enumeration kernels over the prepared tasks and
 * writes d_out.  Same arguments and workspace as tg_max_zeros; d_out of
 * _prepare receives the values of sets decided without enumeration (k <= 1,
 * dependent rows). */
int tg_max_zeros_prepare(tg_context* ctx, const tg_distance_params* p,
                         const int32_t* d_indices, const int64_t* d_offsets,
                         const int32_t* d_target, const int32_t* d_set_ids,
                         int32_t* d_out, void* d_workspace,
                         size_t workspace_bytes, void* stream);
int tg_max_zeros_walk(tg_context* ctx, const tg_distance_params* p,
                      int32_t* d_out, void* d_workspace, size_t workspace_bytes,
                      void* stream);

/* One part of tg_max_zeros_walk, for callers that time the two walks apart:
 * TG_WALK_ENUMERATION runs the orbit / projective / sampled walk (sets below
 * the information-set threshold), TG_WALK_INFOSET the information-set walk
 * and the step that writes its results.  tg_max_zeros_walk is both, in that
 * order; the parts touch disjoint sets, so either order gives the same d_out. */
enum { TG_WALK_ENUMERATION = 1, TG_WALK_INFOSET = 2 };
int tg_max_zeros_walk_part(tg_context* ctx, const tg_distance_params* p,
                           int32_t parts, int32_t* d_out, void* d_workspace,
                           size_t workspace_bytes, void* stream);

/* Last information-set level a batch with sets of at most k_max rows can
 * need (levels 1..3 always run; levels 4..*h_level are launched).  For the
 * toric matrix: the smallest L with ceil(49 (L + 1) / k) above the Griesmer
 * cap of a [49, k] code over GF(8), maximised over k <= k_max (9 for
 * k_max = 14); for other matrices k_max.  No
 * counterpart in the reference, which walks every message.  Needs no GPU. */
int tg_infoset_last_level(int32_t k_max, int32_t is_toric, int32_t* h_level);

/* Bytes of workspace tg_max_zeros_witness needs (exact parameters only). */
int tg_witness_workspace_size(const tg_distance_params* p, size_t* h_bytes);

/* tg_max_zeros plus, for every set, a witness codeword: 49 GF(8) symbols
 * (uint8, values 0..7, in M's column order) at d_witness + 49 * s, with
 * exactly d_out[s] zero coordinates.  For a passing set it is a codeword of
 * minimum weight; for a failing set one of weight below the target
 * distance, whose zero count d_out[s] then reports (still > 49 - td).  A set
 * with dependent rows gets the zero codeword (d_out = 49); an empty set
 * gets zeros.  The reference returns only the count
 * (DistanceOracleCUDABP.max_zeros_batch, kernel_cuda_bp.py:290-323; its
 * message poly_id stays inside eval_min_distance_batch_bp :146-238); the
 * witness lets a caller check a result on the host by solving m M[S] = c.
 * Runs a second information-set pass whose per-set targets are 50 - d_out,
 * recording the first codeword that reaches them; a set evaluated by the walk
 * without a witness raises TG_ERR_STATE through tg_distance_status (same
 * workspace).  Exact parameters only (sample_count == 0). */
int tg_max_zeros_witness(tg_context* ctx, const tg_distance_params* p,
                         const int32_t* d_indices, const int64_t* d_offsets,
                         const int32_t* d_target, const int32_t* d_set_ids,
                         int32_t* d_out, uint8_t* d_witness, void* d_workspace,
                         size_t workspace_bytes, void* stream);

/* Size of the library-owned scratch area tg_max_zeros_noalloc works in. */
#define TG_STATIC_WORKSPACE_BYTES (16u << 20)

/* tg_max_zeros for callers that must not allocate device memory.
 * No counterpart in the reference (its oracles allocate per call through
 * CuPy).  Meant for hosts where device memory is carved out up front or owned
 * by another allocator -- an application that hands this library a fixed
 * pool, a plugin whose host forbids cudaMalloc after start-up, a latency-bound
 * loop that cannot afford an allocation's implicit synchronisation.  It takes
 * the same inputs and writes the same d_out as tg_max_zeros but runs in a
 * TG_STATIC_WORKSPACE_BYTES scratch array compiled into the library (held on
 * every device that loads it) and allocates nothing.  The first call on a
 * device looks the array's device address up (cudaGetSymbolAddress), so make
 * that first call before any stream capture on that device.  Batches whose
 * tg_distance_workspace_size exceeds the array are refused with
 * TG_ERR_WORKSPACE.  All calls share the one array: calls that may overlap on
 * the GPU (different streams, or different host threads) race and must be
 * serialised by the caller.  Sets with indices outside 0..48 come back as 0;
 * there is no status query for this path. */
int tg_max_zeros_noalloc(tg_context* ctx, const tg_distance_params* p,
                         const int32_t* d_indices, const int64_t* d_offsets,
                         const int32_t* d_target, const int32_t* d_set_ids,
                         int32_t* d_out, void* stream);

/* Device status word of the last tg_max_zeros run on this workspace
 * (synchronises `stream`): TG_OK or TG_ERR_BAD_INPUT. */
int tg_distance_status(const tg_distance_params* p, const void* d_workspace,
                       void* stream, int32_t* h_status);

/* Work accounting of the last run on this workspace (synchronises `stream`):
 * tasks queued, codewords evaluated (orbit / projective: the codewords the
 * queued tasks cover; information sets: the codewords the walk evaluated) and
 * the reference-equivalent message count sum(8^k - 1) over exact sets. */
int tg_distance_counters(const tg_distance_params* p, const void* d_workspace,
                         void* stream, uint64_t* h_tasks,
                         uint64_t* h_codewords, double* h_reference_messages);

/* The same accounting per walk (synchronises `stream`): h_counts[0..3] =
 * enumeration walk tasks and codewords, information-set tasks queued (levels
 * 4 and up; levels 1-3 run as one warp per set, without tasks) and codewords
 * the information-set walk evaluated (all levels). */
int tg_distance_path_counters(const tg_distance_params* p, const void* d_workspace,
                              void* stream, uint64_t* h_counts);

/* Codewords the information-set walk evaluated per stage (synchronises
 * `stream`): h_counts[0] = levels 1 to 3, h_counts[2 w + part - 1] = part
 * `part` (1 or 2) of level w >= 4.  Part 1 of a level takes the supports
 * holding the set's last row, part 2 the others (a non-toric matrix walks
 * whole levels in part 1).  Writes min(n, TG_INFOSET_STAGES) entries.  No
 * counterpart in the reference (profiling aid). */
#define TG_INFOSET_STAGES 44
int tg_distance_stage_counters(const tg_distance_params* p, const void* d_workspace,
                               void* stream, uint64_t* h_counts, int32_t n);

/* ---- canonical forms ---------------------------------------------------- */

/* Canonical form of n exponent sets given as rows of a (n, k) int32 matrix.
 * Replaces CanonicalOracle.compute (kernel_canon.py:151-176; kernel
 * canonical_forms :44-129) and canonical_forms_batch
 * (champion_search_canonical.py:115-140).
 *   d_out_mask  canonical 49-bit mask (bit i = exponent index i): the
 *               smallest mask of an AGL2(F7) image of the set that contains
 *               the origin.  Defined for every k in 1..49.
 *   d_out_key_lo/hi  the reference's packed key (6 bits per sorted index,
 *               index 0 skipped for k >= 11) for k <= 16, else all ones.
 * Rows with repeated or out-of-range indices get mask 0 and key all ones and
 * raise TG_ERR_BAD_INPUT in *d_status (int32, may be NULL). */
int tg_canonical_sets(tg_context* ctx, const int32_t* d_sets, int32_t n,
                      int32_t k, uint64_t* d_out_mask, uint64_t* d_out_key_lo,
                      uint64_t* d_out_key_hi, int32_t* d_status, void* stream);

/* Same for sets given as 49-bit masks (popcount 1..49; 0 -> mask 0). */
int tg_canonical_masks(tg_context* ctx, const uint64_t* d_masks, int32_t n,
                       uint64_t* d_out_mask, uint64_t* d_out_key_lo,
                       uint64_t* d_out_key_hi, void* stream);

/* Canonical masks of all one-point extensions of n parent masks (49-bit):
 * d_out[49 * i + p] = canonical mask of parent_i with point p added, or 0 when
 * p is already in parent_i.  The expansion of the canonical BFS
 * (champion_search_canonical.py:496-506) fused with its canonicalisation
 * (kernel_canon.py:151-176), on the device.  n * 49 must fit in int32. */
int tg_expand_canonical(tg_context* ctx, const uint64_t* d_parents, int32_t n,
                        uint64_t* d_out, void* stream);

/* Scratch bytes of tg_compact_sets for n entries. */
int tg_compact_scratch_bytes(int32_t n, size_t* h_bytes);
/* Order-preserving compaction of the entries i with d_flags[i] != 0: their
 * masks (d_out_masks, may be NULL), their sorted exponent indices as rows of
 * k int32 (d_out_sets, may be NULL; each mask must hold k points) and
 * count+1 row offsets (d_out_offsets, may be NULL); *d_count = count.  Feeds
 * a level of new canonical sets straight into tg_max_zeros. */
int tg_compact_sets(const uint64_t* d_masks, const uint8_t* d_flags, int32_t n,
                    int32_t k, void* d_scratch, uint64_t* d_out_masks,
                    int32_t* d_out_sets, int64_t* d_out_offsets, int32_t* d_count,
                    void* stream);

/* ---- device hash set (canonical dedup) ----------------------------------- */

/* Bytes of a hash set with `capacity` slots (power of two >= 64). */
int tg_hashset_bytes(int64_t capacity, size_t* h_bytes);
/* Empties a hash set. */
int tg_hashset_clear(void* d_table, int64_t capacity, void* stream);
/* Inserts n 64-bit keys; 0 and all ones are not keys (never new, not stored).
 * d_is_new[i] = 1 iff key i
 * was absent before this call and i is its first index in this call — the
 * semantics of the reference's `seen` set walk in
 * champion_search_canonical.py:337-345.  `call_id` must grow from call to
 * call on one table (1, 2, ...).  d_n_new (may be NULL) receives the count.
 * A table fuller than half its capacity sets TG_ERR_CAPACITY in *d_status. */
int tg_hashset_insert(void* d_table, int64_t capacity, const uint64_t* d_keys,
                      int32_t n, uint32_t call_id, uint8_t* d_is_new,
                      int32_t* d_n_new, int32_t* d_status, void* stream);

/* ---- served search stream (device-resident request loop) ---------------- */

/* A server evaluates max_zeros requests as they arrive: requests are admitted
 * into a fixed pool of device slots (sized from free device memory), each is
 * deduplicated by its AGL2(F7) canonical form in a device hash table, carries
 * its own early-exit threshold, and is evaluated by information sets level
 * by level; every open level of every request is a job of one device ring,
 * whose tasks the warps of one persistent loop kernel claim in arrival order,
 * so the work of requests admitted at different times overlaps on the GPU.
 * This is the
 * B200 form of the reference's host pipeline _pipelined_eval + _dispatch
 * (champion_search_canonical.py:281-378, 237-271) and evolve_search's
 * evaluate_sets (evolve_search.py:266-282), request by request. */

typedef struct tg_server tg_server;

typedef struct tg_server_params {
  int32_t max_slots;       /* request slots; 0 = from free device memory     */
  int32_t k_max;           /* largest request size, <= 21                    */
  int32_t tail_rows;       /* unused by the information-set loop; 0 or 2..7  */
  int32_t blocks_per_sm;   /* loop CTAs (128 threads) per SM, 1..5; 0 = 5    */
  int32_t idle_us;         /* the loop exits after this long without work; 0 = 2000 */
  int32_t life_ms;         /* one loop launch ends after this long; 0 = 250  */
  int64_t table_capacity;  /* dedup table slots, power of two; 0 = 2^20; -1 = no dedup */
  double memory_fraction;  /* share of free device memory for slots (max_slots == 0); 0 = 0.25 */
} tg_server_params;

#define TG_RESULT_PASS 1      /* max_zeros <= 49 - td; the value is exact          */
#define TG_RESULT_FAIL 2      /* a codeword beyond the threshold; value is a witness */
#define TG_RESULT_DEDUP 4     /* answered from an earlier request of the same canonical form */
#define TG_RESULT_BAD_INPUT 8 /* k or an index out of range                         */

typedef struct tg_server_result {
  uint32_t id;          /* the id tg_server_submit returned                  */
  int32_t max_zeros;
  int32_t flags;        /* TG_RESULT_* bits                                  */
  int32_t pad;
  uint64_t t_admit_ns;  /* device globaltimer when the loop took the request */
  uint64_t t_done_ns;   /* device globaltimer when the answer was written    */
} tg_server_result;

/* Slots, device bytes and page-locked host bytes a server needs. */
int tg_server_layout(tg_context* ctx, const tg_server_params* p, int32_t* h_slots,
                     size_t* h_device_bytes, size_t* h_host_bytes);
/* Creates a server in caller memory: d_arena (device, 256-byte aligned) and
 * h_pinned (page-locked host memory the device can map, e.g. cudaHostAlloc). */
int tg_server_create(tg_context* ctx, const tg_server_params* p, void* d_arena,
                     size_t device_bytes, void* h_pinned, size_t host_bytes,
                     tg_server** out);
/* Queues one request; TG_ERR_CAPACITY when every slot is busy. */
int tg_server_submit(tg_server* srv, const int32_t* h_indices, int32_t k,
                     int32_t target_distance, uint32_t* h_id);
/* Queues requests 0..n-1 in order (request i: h_indices[h_offsets[i] ..
 * h_offsets[i+1]), threshold h_target[i]) under one lock and one publication
 * store, until the slots run out.  *h_consumed = how many were taken from the
 * front: h_status[i] is TG_OK (h_ids[i] = its id) or TG_ERR_INVALID_ARGUMENT
 * (k or an index out of range; no id) for each of them; the rest stay with
 * the caller.  Returns TG_OK, or TG_ERR_INVALID_ARGUMENT for bad pointers.
 * No counterpart in the reference (its drivers evaluate batches). */
int tg_server_submit_batch(tg_server* srv, const int32_t* h_indices, const int64_t* h_offsets,
                           int32_t n, const int32_t* h_target, uint32_t* h_ids,
                           int32_t* h_status, int32_t* h_consumed);
/* (Re)launches the loop kernel when requests are outstanding and it has
 * exited; *h_running = 1 while a loop launch is executing. */
int tg_server_pump(tg_server* srv, int32_t* h_running);
/* Collects up to max finished results (in completion order) and frees slots. */
int tg_server_poll(tg_server* srv, tg_server_result* h_out, int32_t max, int32_t* h_n);
/* Counters: [0] published, [1] finished, [2] outstanding, [3] loop launches,
 * [4] level tasks run, [5] codewords evaluated, [6] dedup answers, [7] device
 * status. */
int tg_server_stats(tg_server* srv, uint64_t* h_counters8);
/* Fault injection for failure tests: moves the publication counter past one
 * request id without publishing that request.  The loop's bounded wait for
 * the missing publication entry runs out (a few milliseconds) and sets
 * TG_ERR_STATE in the device status (tg_server_stats counter 7); the loop and
 * the requests published after it go on.  No counterpart in the reference. */
int tg_server_debug_skip_publication(tg_server* srv);
/* Stops the loop (bounded wait) and frees the server object. */
int tg_server_destroy(tg_server* srv);

/* ---- integer pipe throughput (roofline denominators) --------------------- */

/* Measures per-SM issue rates (operations per SM per clock) of the integer
 * instructions the distance kernel uses: out[0] LOP3, out[1] POPC, out[2]
 * IADD3, out[3] fused add+max, out[4] LOP3+POPC interleaved 1:1 (ops of both
 * kinds), out[5] the SM clock in MHz seen during the run.  Needs
 * d_scratch of 1 MiB.  Synchronises. */
int tg_measure_int_pipes(int device, void* d_scratch, double* h_out6);

#ifdef __cplusplus
}
#endif

#endif /* TORIC_B200_H */
