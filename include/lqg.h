/* liteqg_b200 — C ABI of the B200 quantized-graph query path.
 *
 * A drop-in for the query path of LiteQG's symphonyqg.Index (a SymphonyQG
 * fork): the same index file, the same search semantics, bit-exact ids, on one
 * NVIDIA B200 (sm_100a). Plain pointers and sizes only; every call returns an
 * lqg_status and never throws. Host buffers belong to the caller, device
 * buffers to the library. One lqg_index may be used from one host thread at a
 * time; distinct indexes may be used concurrently on distinct streams.
 *
 * Reference interfaces replaced (paths inside the LiteQG project):
 *   python/bindings.cpp:38-61   Index(index_type, metric, num_elements, dimension, degree_bound)
 *   python/bindings.cpp:63,65   Index.load / Index.save
 *   python/bindings.cpp:67      Index.set_ef
 *   python/bindings.cpp:69-90   Index.build_index
 *   python/bindings.cpp:92-98   Index.search(query, k)
 *   symqglib/qg/qg.hpp:206-243  QuantizedGraph::save_index/load_index/set_ef/search
 *   symqglib/qg/qg.hpp:298-344  QuantizedGraph::search_qg_with_heap
 */
#ifndef LQG_H
#define LQG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define LQG_API __attribute__((visibility("default")))
#else
#define LQG_API
#endif

typedef struct lqg_index lqg_index;

typedef enum {
    LQG_OK = 0,
    LQG_ERR_ARG = 1,      /* bad argument (shape, metric, degree, k, ef ...) */
    LQG_ERR_IO = 2,       /* file missing, short, or of the wrong size */
    LQG_ERR_CUDA = 3,     /* a CUDA runtime call failed */
    LQG_ERR_NOMEM = 4,    /* device or host allocation failed */
    LQG_ERR_STATE = 5,    /* call made in the wrong state (no data, ef unset) */
    LQG_ERR_CAPACITY = 6, /* a per-query work area overflowed; see lqg_last_error */
    LQG_ERR_CORRUPT = 7   /* index content invalid (neighbour id out of range) */
} lqg_status;

#define LQG_NO_ID 0xFFFFFFFFu /* output slot the reference leaves unwritten */

/* Text of the last error on this host thread ("" if none). */
LQG_API const char* lqg_last_error(void);

/* Index(index_type, metric, num_elements, dimension, degree_bound):
 * python/bindings.cpp:38-61. index_type must be "QG", metric "L2",
 * degree_bound a positive multiple of 32 (up to 128 on the GPU), and
 * dimension in [33, 2048] (the reference's rotator aborts outside it,
 * symqglib/utils/rotator.hpp:55-76). device: CUDA ordinal. */
LQG_API lqg_status lqg_create(const char* index_type, const char* metric,
                      uint64_t num_elements, uint32_t dimension,
                      uint32_t degree_bound, int device, lqg_index** out);

/* Frees everything the index owns. NULL is accepted. */
LQG_API void lqg_free(lqg_index* ix);

/* Index.load: symqglib/qg/qg.hpp:217-224. The file must be exactly
 * 4 + 4*N*(D+deg) + N*D + 8*D bytes, optionally followed by a FastScan
 * section (see lqg_fs_build); every neighbour id must be < N.
 * Uploads the neighbour lists, codes and SQ8 parameters to the device. */
LQG_API lqg_status lqg_load(lqg_index* ix, const char* path);

/* Index.save: symqglib/qg/qg.hpp:206-215 (same bytes). */
LQG_API lqg_status lqg_save(const lqg_index* ix, const char* path);

/* Sets the index content from host arrays (the file's fields):
 * vectors[N][D] f32 (stored, not searched), nbrs[N][deg] u32,
 * codes[N][D] u8, params[D][2] f32 (min, scale). Validates and uploads. */
LQG_API lqg_status lqg_set_arrays(lqg_index* ix, uint32_t entry, const float* vectors,
                          const uint32_t* nbrs, const uint8_t* codes,
                          const float* params);

/* Copies the index content out (any pointer may be NULL). */
LQG_API lqg_status lqg_get_arrays(const lqg_index* ix, uint32_t* entry, float* vectors,
                          uint32_t* nbrs, uint8_t* codes, float* params);

/* Index.build_index(data, EF, num_iter): python/bindings.cpp:69-90 ->
 * QGBuilder (symqglib/qg/qg_builder.hpp:48-91), built on the GPU.
 * data: HOST [N][D] f32. EF in [1, 512], num_iter >= 2. Deterministic for a
 * given seed (the reference seeds from std::random_device). random_edges
 * (< degree_bound) slots of every list are seeded random long-range links
 * (the reference's builder keeps leftover random links in slots its pruning
 * leaves empty, qg.hpp:475-487); they keep well-separated clusters reachable
 * from the single entry point. Produces the same file layout; the graph is
 * the GPU builder's, not bit-identical to the reference builder's. */
LQG_API lqg_status lqg_build(lqg_index* ix, const float* data, uint32_t ef_build,
                             uint32_t num_iter, uint64_t seed, uint32_t random_edges);

/* lqg_build with search-path long links (no reference counterpart; the
 * reference's heuristic_prune, qg_builder.hpp:155-200, is alpha = 1,
 * path_take = far_budget = 0, which lqg_build uses):
 *   alpha >= 1   a kept neighbour j removes a later candidate i only when
 *                alpha * |j - i| < |node - i|; alpha > 1 keeps longer, more
 *                diverse links (the Vamana rule);
 *   path_take    the first path_take nodes popped by each node's build search
 *                (from the entry point toward the node) join its candidates,
 *                up to 32 of them beyond the nearest ones;
 *   far_budget   slots of each list that only candidates farther than twice
 *                the nearest candidate's distance may take.
 * With reverse edges these become routes from the entry region into every
 * cluster of clustered data.
 *   pair_kernel  candidate-to-candidate distances of the prune: 0 FP32 on the
 *                CUDA cores; 1 Gram matrices on the tensor cores (tcgen05,
 *                each value split into BF16 hi + lo, FP32 accumulation in
 *                tensor memory) with every prune decision near its threshold
 *                re-checked in FP32, which gives the same graph as 0.
 *   report       optional: prune kernel time and FP32 re-checks of the build. */
typedef struct {
    double prune_ms;    /* all prune launches (CUDA events) */
    double build_ms;    /* the whole build on the device */
    uint64_t rechecks;  /* pair_kernel 1: decisions re-checked in FP32 */
} lqg_build_report;
LQG_API lqg_status lqg_build_ex(lqg_index* ix, const float* data, uint32_t ef_build,
                                uint32_t num_iter, uint64_t seed, uint32_t random_edges,
                                float alpha, uint32_t path_take, uint32_t far_budget,
                                uint32_t pair_kernel, lqg_build_report* report);

/* Index.set_ef: symqglib/qg/qg.hpp:226-230. ef in [1, 512]. */
LQG_API lqg_status lqg_set_ef(lqg_index* ix, uint32_t ef);

/* Index.search(query, k): python/bindings.cpp:92-98 -> qg.hpp:235-243.
 * One query, host buffers, synchronous; the plain one-query-per-launch form.
 * results[k] receives exactly the ids the reference writes (its worst-k of
 * the ef pool in ascending distance, qg.hpp:340-343); slots it would leave
 * unwritten (pool smaller than k) are LQG_NO_ID. */
LQG_API lqg_status lqg_search(lqg_index* ix, const float* query, uint32_t k,
                      uint32_t* results);

/* Batched search (no reference counterpart; M > 1 form of Index.search).
 * All pointers are DEVICE pointers; the call is asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default stream).
 *   queries  [m][D] f32
 *   k, ef    per-query arrays [m] (u32) or NULL, then k0/ef0 apply to all
 *            (ef0 == 0 means the value given to lqg_set_ef). With a per-query
 *            ef array, ef0 must be an upper bound of its values (it sizes the
 *            kernel's pool): a per-query ef above ef0 runs at ef0, and 0 runs
 *            at 1; per-query k values above kstride are clamped.
 *   ids      [m][kstride] u32, compat output as lqg_search writes it
 *   pool_ids [m][pstride] u32, pool_d [m][pstride] f32: the full final pool
 *            in ascending distance (NULL to skip); unused slots LQG_NO_ID/inf
 *   stats    [m][4] u32 (NULL to skip): pops, distance computations,
 *            kernel that finished the query (0 fast, 1 heap, 2 global exact;
 *            the global exact kernel counts exactly the reference's
 *            evaluations, the others also count re-evaluations), pool size
 * Queries whose pool meets two equal distances are re-run by the exact
 * kernel (libstdc++ heap order) inside the same call, so ids always equal the
 * reference's. */
LQG_API lqg_status lqg_search_batch_device(lqg_index* ix, const float* queries,
                                   int64_t m, const uint32_t* k, uint32_t k0,
                                   const uint32_t* ef, uint32_t ef0,
                                   uint32_t* ids, uint32_t kstride,
                                   uint32_t* pool_ids, float* pool_d,
                                   uint32_t pstride, uint32_t* stats,
                                   void* stream);

/* Waits for `stream` and reports what the device-side search recorded since
 * the last batch started on this index: LQG_OK, or LQG_ERR_CAPACITY when a
 * query overflowed the exact kernel's work area (its ids are LQG_NO_ID). */
LQG_API lqg_status lqg_stream_status(lqg_index* ix, void* stream);

/* The same with HOST buffers: copies in, searches, copies out, synchronizes.
 * Pinned host memory gives the fastest copies. */
LQG_API lqg_status lqg_search_batch(lqg_index* ix, const float* queries, int64_t m,
                            const uint32_t* k, uint32_t k0, const uint32_t* ef,
                            uint32_t ef0, uint32_t* ids, uint32_t kstride,
                            uint32_t* pool_ids, float* pool_d,
                            uint32_t pstride, uint32_t* stats, void* stream);

/* Runs every query of the batch through the exact (heap-emulating) kernel
 * only; same arguments and outputs as lqg_search_batch_device. Used to check
 * the fast kernel and to count the reference's distance evaluations. */
LQG_API lqg_status lqg_search_exact_device(lqg_index* ix, const float* queries,
                                   int64_t m, const uint32_t* k, uint32_t k0,
                                   const uint32_t* ef, uint32_t ef0,
                                   uint32_t* ids, uint32_t kstride,
                                   uint32_t* pool_ids, float* pool_d,
                                   uint32_t pstride, uint32_t* stats,
                                   void* stream);

/* The exact kernel with NO allocation: this entry point has no counterpart in
 * the reference. It is for callers that cannot let a library allocate GPU
 * memory — applications whose device memory is already reserved by another
 * allocator (a framework's caching pool), and latency-sensitive loops where a
 * cudaMalloc/cudaFree could synchronize the device and stall other streams.
 * Same arguments and outputs as lqg_search_exact_device (DEVICE pointers), but
 * the work areas live in a fixed array inside the library (about 1.1 MB per
 * GPU, held until the process exits). ef (or the per-query ef bound ef0) above
 * 512 is rejected at the call with LQG_ERR_ARG, as in every search entry
 * point; a query that needs more than 8192 visited nodes or 8192 search-heap
 * entries makes the call return LQG_ERR_CAPACITY, with that query's ids set to
 * LQG_NO_ID and every other query of the batch answered normally. The call
 * waits for `stream` before returning. The first call on a device looks up
 * the array's device address and keeps it; make that first call before any
 * stream capture, and do not reset the device (cudaDeviceReset) after it. All
 * calls share the array, so calls that overlap on the GPU (other threads or
 * streams) race: serialize them. */
LQG_API lqg_status lqg_search_exact_noalloc(lqg_index* ix, const float* queries,
                                           int64_t m, const uint32_t* k, uint32_t k0,
                                           const uint32_t* ef, uint32_t ef0,
                                           uint32_t* ids, uint32_t kstride,
                                           uint32_t* pool_ids, float* pool_d,
                                           uint32_t pstride, uint32_t* stats,
                                           void* stream);

/* Launch shape and policy. 0 fields keep the current value. A new index
 * starts with mode 6, lanes_per_cand 2, visited_bits 10, warps_per_block 8,
 * heap_warps 4, heap_scap 256.
 *   lanes_per_cand  {1,2,4,8,16}: lanes sharing one distance (both kernels)
 *   visited_bits    [8, 13]: slots of the per-query visited cache (2^bits)
 *   warps_per_block {1..16} and blocks_per_sm {1..32}: fast kernel shape
 *                   (blocks_per_sm 0 = as many as fit)
 *   mode            1: fast kernel for every query, heap kernel for the
 *                   queries whose distances tie; 2: heap kernel for every
 *                   query; 3: replay kernel for every query (sorted-pool
 *                   search warps, heap replay lanes; exact under ties);
 *                   4: split kernel for every query (exact search heap per
 *                   warp, result heap replayed afterwards from a log);
 *                   5: batch kernel for every query (as 4, with each
 *                   expansion's candidates decided at once against a
 *                   sorted pool in shared memory); 6: batch kernel with
 *                   the search heap built only when a pop meets equal
 *                   smallest distances (until then the heap's top is the
 *                   sorted pool's first unpopped entry)
 *   heap_warps      {1..8}: warps per block of the heap kernel, {1..5} of
 *                   the split and batch kernels (modes 4-6)
 *   heap_scap       [256, 16384]: search-pool slots per query in shared
 *                   memory (heap and replay kernels; larger pools spill to
 *                   global memory, then to the global-memory kernel)
 *   replay_warps    {1..15}: search warps per block of the replay kernel
 *                   (plus one replay warp)
 *   replay_all      modes 4-6: 1 sends every query through the checked result
 *                   replay pass (0, the default: only queries whose output
 *                   the heap layout decides); set on every call, not kept
 *                   when 0 is passed
 *   small_batch     modes 5-6: a batch of at most this many queries runs one
 *                   query per block of 4 warps (each expansion's distances
 *                   split over the warps: lower latency per query, fewer
 *                   queries resident); LQG_SMALL_BATCH_AUTO (the default):
 *                   as many queries as such blocks fit on the GPU at once;
 *                   LQG_SMALL_BATCH_OFF: never. The same ids either way. */
typedef struct {
    uint32_t lanes_per_cand;
    uint32_t visited_bits;
    uint32_t warps_per_block;
    uint32_t blocks_per_sm;
    uint32_t mode;
    uint32_t heap_warps;
    uint32_t heap_scap;
    uint32_t replay_warps;
    uint32_t replay_all;
    uint32_t small_batch;
} lqg_tuning;

#define LQG_SMALL_BATCH_AUTO 0xFFFFFFFEu
#define LQG_SMALL_BATCH_OFF 0xFFFFFFFFu
LQG_API lqg_status lqg_set_tuning(lqg_index* ix, const lqg_tuning* t);
LQG_API lqg_status lqg_get_tuning(const lqg_index* ix, lqg_tuning* t);

/* ---- Serving loop (no reference counterpart) ----------------------------
 * Continuous batching of single-query requests over one resident index: a
 * dispatcher launches whatever is pending as one batch as soon as one of
 * `streams` contexts is free, so requests that arrive while other batches
 * are on the GPU are admitted as contexts free up and overlap with them.
 * Admission is by each request's own device state (query, k, ef, ids, and
 * the per-query candidate logs, sized by its ef): requests fall in ef classes
 * (<= 64, 128, 256, 512); a batch takes the oldest pending request and every
 * pending request of the same or a smaller class, in arrival order, up to
 * the count of that class whose state fits the context's share
 * (state_budget / streams, default budget 4 GiB); `max_batch`, if set,
 * caps every class. Start runs one full-size batch of every class on every
 * context (in the index's current tuning mode) so that the contexts' work
 * areas are at their largest before the first request: growing them later
 * would allocate device memory, which waits for the whole device. Set the
 * tuning before starting. A batch's state is released when its batch ends.
 * Results are exactly those of a search of the query alone. While a server
 * runs, use the index only through it. */
typedef struct lqg_server lqg_server;
typedef struct {
    uint32_t streams;      /* contexts (batches in flight), default 4 */
    uint32_t max_batch;    /* cap on requests per batch (0: from state_budget per class) */
    uint64_t state_budget; /* device bytes for admitted requests, default 4 GiB */
    uint32_t max_k;        /* largest k of a request, default 100 */
    uint32_t max_ef;       /* largest ef of a request, default 512 */
} lqg_server_config;
typedef struct {
    uint64_t completed;    /* requests finished since start / reset */
    uint64_t batches;
    double mean_batch;
    double p50_us, p99_us; /* latency arrival -> result */
    double qps;            /* completed / elapsed */
    uint32_t max_batch, streams;  /* max_batch: the largest class's count */
} lqg_server_metrics;

LQG_API lqg_status lqg_server_start(lqg_index* ix, const lqg_server_config* cfg,
                                    lqg_server** out);
/* Copies `query` (D floats, host) and queues it; ef 0 = the index's set_ef. */
LQG_API lqg_status lqg_server_submit(lqg_server* s, const float* query, uint32_t k,
                                     uint32_t ef, uint64_t* ticket);
/* Waits for a ticket (timeout_us < 0: forever), copies its k ids, releases it. */
LQG_API lqg_status lqg_server_wait(lqg_server* s, uint64_t ticket, uint32_t* ids,
                                   int64_t timeout_us, double* latency_us);
/* Open-loop driver: submits query i at arrival_us[i] (from the call's start;
 * NULL = as fast as possible) from a client thread (all requests already due
 * in one step), waits for all; ids [m][kstride], latency_us [m] (may be
 * NULL), measured from each request's scheduled arrival. */
LQG_API lqg_status lqg_server_replay(lqg_server* s, const float* queries, int64_t m,
                                     const uint32_t* k, const uint32_t* ef,
                                     const double* arrival_us, uint32_t* ids,
                                     uint32_t kstride, double* latency_us);
LQG_API lqg_status lqg_server_stats(lqg_server* s, lqg_server_metrics* out);
LQG_API lqg_status lqg_server_reset_stats(lqg_server* s);
/* Finishes queued requests, stops the threads, frees the contexts. */
LQG_API lqg_status lqg_server_stop(lqg_server* s);

/* Profiling hook: when both are non-NULL cudaEvent_t handles, every later
 * batch records `start` just before its first search kernel and `stop` just
 * after its last, on the batch's stream (NULL, NULL turns it off). The events
 * stay owned by the caller. */
LQG_API lqg_status lqg_set_kernel_events(lqg_index* ix, void* start, void* stop);

/* Basic properties. */
LQG_API lqg_status lqg_info(const lqg_index* ix, uint64_t* num_elements,
                    uint32_t* dimension, uint32_t* degree_bound,
                    uint32_t* entry, uint32_t* ef);

/* Device pointers of the resident index (for callers that fuse their own
 * work): nbrs [N][deg] u32, codes [N][cstride] u8, params [D][2] f32. */
LQG_API lqg_status lqg_device_arrays(const lqg_index* ix, const uint32_t** nbrs,
                             const uint8_t** codes, const float** params,
                             uint32_t* code_stride);

/* ---- FastScan / RaBitQ search (upstream SymphonyQG) ----------------------
 * The query path this fork still carries but no longer calls:
 * QuantizedGraph::search_qg (symqglib/qg/qg.hpp:252-287, the call commented
 * out at qg.hpp:241) with scan_neighbors (:348-393), the sorted SearchBuffer
 * and ResultBuffer (utils/buffer.hpp:10-119) and update_results (:395-418).
 * It needs per-node RaBitQ codes and factors of the node's neighbours
 * (quantization/rabitq.hpp:23-108), which the fork's builder never writes
 * (update_qg, qg.hpp:475-502, was truncated): lqg_fs_build writes them.
 * P = 2^ceil(log2 D). In the index file they follow the reference's bytes as
 * a section ("LQGFS1", P, degree_bound, D, the rotation's diagonal[P], then
 * per node deg*P/8 code bytes in upstream's FastScan block layout and
 * triple_x/factor_dq/factor_vq[deg]); lqg_load reads it when present and
 * lqg_save writes it. The reference's loader reads its own bytes and stops
 * there, so such a file still loads in the reference. */

/* Encodes the current graph: a seeded +-1/sqrt(P) rotation diagonal (the
 * reference's FHTRotator seeds from std::random_device and does not save it,
 * utils/rotator.hpp:31-47), the FHT of every vector, and for every node and
 * neighbour the sign bits of the rotated residual and its three factors
 * (norms and inner products reduced in FP64). A neighbour equal to its node
 * gets zero factors (the reference would divide 0 by 0). No reference
 * counterpart runs: upstream's QuantizedGraph::update_qg. */
LQG_API lqg_status lqg_fs_build(lqg_index* ix, uint64_t seed);

/* The section's arrays (host buffers): diag[P]; packed[N][deg*P/8] in
 * upstream's FastScan block layout (quantization/fastscan_impl.hpp:63-123);
 * factors[N][3][deg]. set replaces them (for codes made elsewhere, e.g. by
 * the reference's own rabitq_codes); get copies them out (any pointer may be
 * NULL; padded_dim receives P). */
LQG_API lqg_status lqg_fs_set_arrays(lqg_index* ix, const float* diag, const uint8_t* packed,
                                     const float* factors);
LQG_API lqg_status lqg_fs_get_arrays(const lqg_index* ix, uint32_t* padded_dim, float* diag,
                                     uint8_t* packed, float* factors);

/* search_qg for m queries. DEVICE pointers, asynchronous on `stream`.
 * k/ef per query or k0/ef0 for all (ef0 == 0: the set_ef value; with a
 * per-query ef array ef0 bounds it); ef in [1, 512], kstride <= 1024.
 * ids[m][kstride]: the k ids the reference copies out, ascending exact
 * distance; slots its zero-initialised result buffer never fills hold 0, as
 * in the reference. stats[m][4] (NULL to skip): search-buffer pops, exact
 * distances of popped nodes, exact distances in update_results, results. */
LQG_API lqg_status lqg_fs_search_batch_device(lqg_index* ix, const float* queries, int64_t m,
                                              const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                              uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                              uint32_t* stats, void* stream);
/* Waits for `stream`; LQG_OK, or the first device-side failure of the last
 * FastScan batch (a non-finite distance: that query's ids are LQG_NO_ID). */
LQG_API lqg_status lqg_fs_stream_status(lqg_index* ix, void* stream);
/* The same with HOST buffers (copies in, searches, copies out, synchronizes). */
LQG_API lqg_status lqg_fs_search_batch(lqg_index* ix, const float* queries, int64_t m,
                                       const uint32_t* k, uint32_t k0, const uint32_t* ef,
                                       uint32_t ef0, uint32_t* ids, uint32_t kstride,
                                       uint32_t* stats, void* stream);
/* One query, host buffers (upstream's Index.search: qg.hpp:235-243 with
 * search_qg); results[k]. */
LQG_API lqg_status lqg_fs_search(lqg_index* ix, const float* query, uint32_t k,
                                 uint32_t* results);

/* Self-test of the kernels' failure path (no reference counterpart): every
 * wait in this library's kernels (mbarrier completions of bulk copies and
 * tensor-core work, waits between warps) is bounded, and on running out the
 * kernel records an error the host reads and returns; it never traps or
 * hangs. This launches one warp that waits `tries` times (1..2^20) on an
 * mbarrier nothing arrives on; *timed_out receives 1 when the wait ran out
 * (the expected outcome) and the context stays usable. */
LQG_API lqg_status lqg_selftest_bounded_wait(int device, uint32_t tries, uint32_t* timed_out);

#ifdef __cplusplus
}
#endif
#endif
