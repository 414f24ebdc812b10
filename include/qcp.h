/*
 * qcp.h -- C ABI of the B200 spatial-index range-search library.
 *
 * The library builds a bulk-loaded R-tree over points or rectangles on one
 * GPU (Hilbert keys -> device radix sort -> bottom-up packing) and answers
 * batches of axis-aligned box queries with the exact hit set of every query
 * as a sorted list of int32 object ids (0-based input positions).
 *
 * Each entry point replaces a piece of the reference's tree interface
 * (paths inside JinwoongKim/Query-Co-processing-on-Heterogeneous-Architectures):
 *
 *   qcp_index_build    tree::Tree::Build            src/tree/tree.h:24
 *                      (MPHR::Build src/tree/mphr.cpp:35-136 and the
 *                      ChunkManager::Init/CopyNode residency of
 *                      src/manager/chunk_manager.cpp:16-40)
 *   qcp_query_batch    tree::Tree::Search           src/tree/tree.h:47-48
 *                      (MPHR::Search src/tree/mphr.cpp:196-272), returning
 *                      per-query id lists instead of a logged hit total
 *   qcp_query_counts   the per-block hit counters of MPHR::Search
 *                      (src/tree/mphr.cpp:219-252)
 *   qcp_index_save     tree::Tree::DumpToFile       src/tree/tree.h:28
 *   qcp_index_load     tree::Tree::DumpFromFile     src/tree/tree.h:26
 *   qcp_index_free     the destructors src/tree/mphr.cpp:21-28 (the reference
 *                      never frees device memory)
 *   qcp_result_release (no counterpart: the reference returns no lists)
 *   qcp_last_error     stands in for cudaErrCheck -> exit (src/common/macro.h:100-108)
 *
 * Conventions: every call returns a qcp_status and never exits the process;
 * the caller owns the input buffers; the library owns the index and each
 * result's buffers until qcp_index_free / qcp_result_release.  Queries on
 * one index may run concurrently from several host threads; building, saving
 * or freeing an index must not overlap queries on it.
 */
#ifndef QCP_H_
#define QCP_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qcp_status {
  QCP_OK = 0,
  QCP_ERR_BAD_ARG = 1,         /* invalid argument (message in qcp_last_error) */
  QCP_ERR_OOM = 2,             /* device or pinned host allocation failed */
  QCP_ERR_OUTPUT_OVERFLOW = 3, /* a result exceeds the configured output cap */
  QCP_ERR_TIMEOUT = 4,         /* a bounded device wait ran out */
  QCP_ERR_CUDA = 5,            /* any other CUDA error */
  QCP_ERR_NO_DEVICE = 6,       /* no usable CUDA device */
  QCP_ERR_IO = 7               /* index file could not be read or written */
} qcp_status;

/* Where a buffer lives. */
typedef enum qcp_mem { QCP_MEM_HOST = 0, QCP_MEM_DEVICE = 1 } qcp_mem;

/* Hilbert key quantisation. */
typedef enum qcp_key_mode {
  /* floor(clamp(p,0,1) * 2^bits) with bits = 32 (2-D), 21 (3-D) or
   * floor(64/D) otherwise; the default. */
  QCP_KEY_NORM = 0,
  /* The reference's key: (long long)(1e6f * p) with 20 bits per dimension
   * for D > 2 and 31 for D == 2 (src/tree/tree.cpp:597,
   * src/mapper/hilbert_mapper.cpp:21-23).  Defined for D*bits <= 64. */
  QCP_KEY_REF = 1,
  /* k-means-clustered keys (the reference's CLUSTER_TYPE_KMEANSHILBERT,
   * src/mapper/kmeans_mapper.cpp:204-259), cluster-major: the objects are
   * clustered by k-means (kmeans_clusters centres, at most kmeans_iters
   * assignments), the clusters are ranked by the QCP_KEY_NORM key of their
   * centres, and an object's 64-bit key is its cluster's rank in the top
   * ceil(log2 K) bits followed by its own QCP_KEY_NORM key.  Deterministic:
   * centres start at the objects floor(k*n/K), sums are exact fixed point. */
  QCP_KEY_KMEANS = 2
} qcp_key_mode;

typedef struct qcp_build_opts {
  uint32_t fanout;    /* entries per node, a multiple of 32 in [32, 256]; 0 = 128 */
  uint32_t key_mode;  /* qcp_key_mode */
  uint32_t key_bits;  /* bits per dimension; 0 = the mode's default */
  uint32_t input_mem; /* qcp_mem of objs */
  void* stream;       /* cudaStream_t for the build; NULL = legacy default stream */
  uint32_t kmeans_clusters; /* QCP_KEY_KMEANS: centres; 0 = min(1024, n) (the reference uses 20000) */
  uint32_t kmeans_iters;    /* QCP_KEY_KMEANS: most assignments; 0 = 30 (the reference: 1000) */
} qcp_build_opts;

typedef struct qcp_index qcp_index; /* opaque, device resident */

typedef struct qcp_index_info {
  uint64_t n;               /* objects indexed */
  uint32_t dims;
  uint32_t is_rect;
  uint32_t fanout;
  uint32_t levels;          /* tree height; level 0 = leaves */
  uint64_t level_nodes[16]; /* nodes per level, leaves first */
  uint64_t device_bytes;    /* bytes of the resident index */
  uint32_t key_mode;
  uint32_t key_bits;
} qcp_index_info;

/* Traversal algorithm. */
typedef enum qcp_algo {
  /* All queries of the batch in one work-queue pipeline: level-synchronous
   * expansion of (query, node) items, then one persistent pass per output
   * phase with dynamically fetched items; the default. */
  QCP_ALGO_BATCHED = 0,
  /* One query per CUDA block, restart-scanning + parent-check traversal
   * (the reference's MPRS, src/tree/mphr.cpp:303-438), emitting ids. */
  QCP_ALGO_PLAIN = 1,
  /* CPU + GPU co-processing (the reference's Hybrid tree,
   * src/tree/hybrid.cpp:451-760): host threads walk the internal levels of
   * every query down to opts->handoff_level and hand the (query, node) items
   * of that level to the GPU, which expands the rest and scans the leaves,
   * writes and sorts as QCP_ALGO_BATCHED does. */
  QCP_ALGO_HYBRID = 2
} qcp_algo;

typedef struct qcp_query_opts {
  uint32_t algo;       /* qcp_algo */
  uint32_t boxes_mem;  /* qcp_mem of the query boxes */
  uint32_t result_mem; /* qcp_mem where offsets/ids (or counts) are delivered */
  uint32_t unsorted;   /* 1 = skip the per-query id sort (hit SET still exact) */
  void* stream;        /* cudaStream_t; NULL = legacy default stream */
  uint32_t flags;      /* QCP_QUERY_* bits */
  /* Tuning knobs (0 = default; qcp_autotune picks them): CUDA blocks per SM
   * of the batched traversal kernels (default 8, at most 32), and log2 of
   * the id window of the per-query sort (default 17, largest 18, smallest
   * 12; raised where the id range would need more than 8192 windows). */
  uint32_t blocks_per_sm;
  uint32_t win_bits;
  /* QCP_ALGO_HYBRID: host threads of the upper-tree walk (0 = all cores) and
   * the tree level whose items go to the GPU (0 or 1 = the leaves' parents;
   * the root's level = everything on the GPU). */
  uint32_t cpu_threads;
  uint32_t handoff_level;
  /* Leaf prefetch of the batched traversal (0 = default): partially covered
   * leaves are copied into a per-warp shared-memory ring by bulk copies
   * (cp.async.bulk on the TMA unit) this many leaves ahead of the one being
   * tested; 0 = 2 buffers, 1 = no ring (every lane loads its coordinates
   * itself), 2..4 = that many buffers (fewer where shared memory is short).
   * qcp_autotune picks it. */
  uint32_t leaf_prefetch;
  /* Queries per warp of the batched traversal's level expansion: lanes
   * that share one (query, node) item, 32 (default, 0), 16 or 8 (two or
   * four items per warp at once).  qcp_autotune picks it. */
  uint32_t lanes_per_item;
  /* Hit cache between the two leaf passes of a call that writes ids: the
   * count pass records which leaves overlap and which objects of partially
   * covered leaves hit, and the write pass replays that instead of testing
   * again.  0 = on (default), 1 = off (the count pass runs leaner, the write
   * pass tests again).  qcp_autotune picks it. */
  uint32_t hit_cache;
} qcp_query_opts;

/* flags: record CUDA events around every phase of the call; the times are
 * reported by qcp_query_stats_last. */
#define QCP_QUERY_TIMING 1u

/* Work and time of the last query call made on the calling host thread. */
typedef struct qcp_query_stats {
  uint32_t algo;
  uint32_t num_queries;
  uint64_t frontier_items[16]; /* (query, node) items per level, leaves first */
  uint64_t leaf_items;         /* (query, leaf-parent) items scanned */
  uint64_t leaves_covered;     /* overlapping leaves whose MBR lies inside the query */
  uint64_t leaves_partial;     /* overlapping leaves whose objects were tested */
  uint64_t objects_covered;    /* objects of covered leaves (hits without a test) */
  uint64_t hits;
  uint32_t sort_small_jobs;    /* per-query slices sorted directly */
  uint32_t sort_msd_jobs;      /* slices split by MSD rounds (all rounds) */
  /* device milliseconds per phase (only with QCP_QUERY_TIMING) */
  float ms_expand, ms_count, ms_scan, ms_write, ms_sort, ms_total;
  /* parts of ms_sort: small slices, window partition, window sort */
  float ms_sort_small, ms_sort_partition, ms_sort_windows;
  uint64_t sort_window_ids;    /* ids of the slices sorted through windows (with QCP_QUERY_TIMING) */
  /* the window sort's two kernels: the bitmap sort of the windows of more
   * than 512 ids (its milliseconds and ids) and the one-warp sort of the
   * rest (ms_sort_windows minus ms_sort_windows_bitmap) */
  float ms_sort_windows_bitmap;
  uint64_t sort_window_bitmap_ids;
} qcp_query_stats;

qcp_status qcp_query_stats_last(qcp_query_stats* out);

/* Result of one batch in CSR form: the ids of query i are
 * ids[offsets[i] .. offsets[i+1]), ascending unless opts.unsorted. */
typedef struct qcp_result {
  uint32_t num_queries;
  uint32_t mem;           /* qcp_mem of offsets and ids */
  uint64_t total_hits;
  const uint64_t* offsets; /* num_queries + 1 entries */
  const int32_t* ids;      /* total_hits entries */
  void* owner_;            /* library-owned arena; release with qcp_result_release */
} qcp_result;

/* Build the index.  objs: n rows of dims floats (points, is_rect = 0) or of
 * 2*dims floats [lo0..lo(D-1), hi0..hi(D-1)] (rectangles, is_rect = 1).
 * Coordinates must be finite; 1 <= dims <= 8; 1 <= n < 2^31. */
qcp_status qcp_index_build(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                           const qcp_build_opts* opts, qcp_index** out);

qcp_status qcp_index_free(qcp_index* index);

qcp_status qcp_index_get_info(const qcp_index* index, qcp_index_info* info);

/* Run q box queries.  boxes: q rows of 2*dims floats [lo.., hi..]; an object
 * is a hit iff for every dim d: !(q.lo[d] > e.hi[d] || q.hi[d] < e.lo[d])
 * (src/node/node_soa.cpp:94-113).  opts may be NULL (batched, host memory,
 * sorted, default stream).  The call returns after the result is complete. */
qcp_status qcp_query_batch(qcp_index* index, const float* boxes, uint32_t q,
                           const qcp_query_opts* opts, qcp_result* out);

/* Hit count of each of q queries into counts[q] (host or device memory per
 * opts->result_mem). */
qcp_status qcp_query_counts(qcp_index* index, const float* boxes, uint32_t q,
                            const qcp_query_opts* opts, uint64_t* counts);

qcp_status qcp_result_release(qcp_result* result);

/* Write the index to a versioned binary file / read it back onto the current
 * device. */
qcp_status qcp_index_save(const qcp_index* index, const char* path);
qcp_status qcp_index_load(const char* path, void* stream, qcp_index** out);

/* Copy the sorted Hilbert keys, the permutation (sorted position -> input id)
 * and the node MBRs of one level back to host buffers (for tests).  keys
 * and ids take n entries; mbr takes 2*dims*level_nodes[level] floats laid out
 * node-major [lo.., hi..].  Any pointer may be NULL. */
qcp_status qcp_index_export(const qcp_index* index, uint64_t* keys, int32_t* ids,
                            uint32_t level, float* mbr);

/* Captured build: the device bulk load of n objects of one shape (dims,
 * is_rect, fan-out, key mode and bits from opts; QCP_KEY_NORM or
 * QCP_KEY_REF) recorded once into a CUDA graph -- Hilbert keys, the 64-bit
 * radix sort, packing into the SoA leaf layout and the bottom-up MBR levels
 * -- over buffers the plan owns, and replayed by qcp_build_plan_run with no
 * allocation and no host round trip between the steps.  The plan owns the
 * index it builds: qcp_build_plan_run sets *index to it (valid until the
 * next run or qcp_build_plan_free; queries on it work as on any index, and a
 * run must not overlap queries on it).  objs: n rows as for qcp_index_build
 * in host or device memory (objs_mem), copied into the plan's input buffer,
 * or NULL when the caller has written them into qcp_build_plan_input(plan)
 * itself.  Non-finite coordinates fail the run with QCP_ERR_BAD_ARG.
 * Replaces the reference's host build and its copy of the tree to the device
 * (Tree::Bottom_Up, src/tree/tree.cpp:410-495; MPHR::Build,
 * src/tree/mphr.cpp:60-133). */
typedef struct qcp_build_plan qcp_build_plan;

qcp_status qcp_build_plan_create(uint64_t n, uint32_t dims, uint32_t is_rect, const qcp_build_opts* opts,
                                 qcp_build_plan** plan);
float* qcp_build_plan_input(qcp_build_plan* plan);
qcp_status qcp_build_plan_run(qcp_build_plan* plan, const float* objs, uint32_t objs_mem, void* stream,
                              qcp_index** index);
qcp_status qcp_build_plan_free(qcp_build_plan* plan);

/* Hit count of each of q (<= 262144) queries, computed by the batched
 * traversal, without allocating any memory -- for callers that must not call
 * cudaMalloc while they query (device memory owned by another allocator,
 * serving loops that cannot take cudaMalloc's implicit synchronisation,
 * allocation only at start-up by policy).  d_boxes (q rows of 2*dims floats)
 * and d_counts (q entries) are device memory the caller owns, on the
 * index's device (or managed memory); device memory of another GPU is
 * refused with QCP_ERR_BAD_ARG.  The traversal's scratch is one fixed array
 * of about 20 MiB in the library's device image, held by every GPU that
 * loads the library until exit and shared by all calls: calls that overlap
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the array's device address and keeps it for the life of
 * the process; make it before any stream capture.  A cudaDeviceReset after
 * that first call is not supported (it invalidates every index as well).  A
 * batch whose traversal frontier exceeds the scratch's 2^20 (query, node)
 * items returns QCP_ERR_OUTPUT_OVERFLOW (split the batch); d_counts is then
 * undefined.  No counterpart in the reference. */
qcp_status qcp_query_counts_noalloc(qcp_index* index, const float* d_boxes, uint32_t q,
                                    uint64_t* d_counts, void* stream);

/* Autotuner: picks the build fan-out and the query knobs (blocks_per_sm,
 * win_bits, leaf_prefetch, lanes_per_item) for a data set and a sample of
 * its queries by timing trials on the current device: every fan-out in {64,
 * 128, 256} is built and queried with the default knobs, then blocks_per_sm
 * in {4, 8, 16}, win_bits in {16, 17, 18}, leaf_prefetch in {1, 2, 3},
 * lanes_per_item in {8, 16, 32} and hit_cache on/off are tried one after
 * the other at the best fan-out (coordinate descent); each trial is the median of `repeats` timed batches of the
 * sample (sorted output) after one untimed batch.  objs and boxes are host
 * memory as for qcp_index_build / qcp_query_batch; `base` supplies the key
 * mode, key bits and stream (its fanout is ignored).  The reference fixes
 * its fan-out at compile time (NODE_SIZE, src/common/config.h) and has no
 * tuner. */
#define QCP_TUNE_MAX_TRIALS 16
typedef struct qcp_tune_result {
  uint32_t fanout;            /* best build fan-out */
  uint32_t blocks_per_sm;     /* best qcp_query_opts.blocks_per_sm */
  uint32_t win_bits;          /* best qcp_query_opts.win_bits */
  uint32_t trials;            /* entries used in the arrays below */
  float best_ms;              /* batch time of the best trial */
  float build_ms;             /* build time at the best fan-out */
  uint32_t trial_fanout[QCP_TUNE_MAX_TRIALS];
  uint32_t trial_blocks_per_sm[QCP_TUNE_MAX_TRIALS];
  uint32_t trial_win_bits[QCP_TUNE_MAX_TRIALS];
  float trial_ms[QCP_TUNE_MAX_TRIALS];
  uint32_t leaf_prefetch;     /* best qcp_query_opts.leaf_prefetch */
  uint32_t trial_leaf_prefetch[QCP_TUNE_MAX_TRIALS];
  uint32_t lanes_per_item;    /* best qcp_query_opts.lanes_per_item */
  uint32_t trial_lanes_per_item[QCP_TUNE_MAX_TRIALS];
  uint32_t hit_cache;         /* best qcp_query_opts.hit_cache */
  uint32_t trial_hit_cache[QCP_TUNE_MAX_TRIALS];
} qcp_tune_result;

qcp_status qcp_autotune(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect, const float* boxes,
                        uint32_t q, const qcp_build_opts* base, uint32_t repeats, qcp_tune_result* out);

/* Query plans: the batched pipeline (sorted ids unless opts->unsorted) for at
 * most max_queries boxes and max_hits ids per batch, captured once into a
 * CUDA graph and replayed per batch.  qcp_query_batch sizes its buffers and
 * launches from host readbacks between its phases; a plan fixes them at
 * creation (device memory for max_queries boxes, the frontier, max_hits ids
 * twice, the sort's tables) so every phase runs from device-resident counts,
 * and one graph launch replaces its ~20 kernel launches and 3 host round
 * trips.  opts: blocks_per_sm, win_bits, leaf_prefetch, lanes_per_item and
 * unsorted are used (algo must be
 * batched; NULL = defaults).  qcp_plan_create runs the pipeline once on an
 * empty batch before capturing it.
 *
 * qcp_plan_run: boxes (q <= max_queries rows, host or device memory per
 * boxes_mem) are copied in and the batch is padded with empty boxes; on
 * return *total_hits is set and *d_offsets (q + 1 entries) / *d_ids point to
 * the plan's device result, valid until the next run or qcp_plan_free.  A
 * batch whose hits exceed max_hits, or whose traversal frontier exceeds the
 * plan's item capacity (64 per query + 1 per 1024 hits + 65536), returns
 * QCP_ERR_OUTPUT_OVERFLOW (run it through qcp_query_batch or a larger plan).
 * A plan runs one batch at a time; plans of one index may run concurrently
 * on different streams.  The reference launches one kernel per 128 queries
 * with host synchronisation in between (MPHR::Search,
 * src/tree/mphr.cpp:231-258). */
typedef struct qcp_plan qcp_plan;

qcp_status qcp_plan_create(qcp_index* index, uint32_t max_queries, uint64_t max_hits,
                           const qcp_query_opts* opts, qcp_plan** out);
qcp_status qcp_plan_run(qcp_plan* plan, const float* boxes, uint32_t q, uint32_t boxes_mem, void* stream,
                        uint64_t* total_hits, const uint64_t** d_offsets, const int32_t** d_ids);
qcp_status qcp_plan_free(qcp_plan* plan);

/* Serving: replays an open-loop arrival trace through continuous batching
 * over the resident index.  Request i (box i, q rows of 2*dims floats in
 * host memory) arrives arrival_s[i] seconds after the call starts
 * (non-decreasing).  `streams` worker threads, each with its own CUDA stream
 * and two captured query plans (qcp_plan, up to 256 and up to 4096 queries),
 * take every request that has arrived (up to max_batch) and run it as plan
 * replays; batches of different workers overlap on the device.  Admission by
 * output memory: each worker's plans reserve result buffers for
 * output_cap_bytes / streams bytes of results, so the results held at once
 * stay under the cap; a batch whose results do not fit is split, and a
 * single request larger than that runs alone through qcp_query_batch once
 * its counted result bytes (4 per id + 8 per query) fit the cap next to what
 * the other workers hold.  Plans and buffers are set up before the clock
 * starts.  deliver (optional) receives every request's ascending ids, from
 * the worker threads, once each.  latency_ms (optional, q entries) gets
 * arrival -> results-on-host time per request; trace (optional) gets one
 * qcp_serve_batch per run, in completion order (stats->batches runs in all).
 * No counterpart in the reference (its Evaluator replays fixed query files
 * through Tree::Search, src/evaluator/evaluator.cpp:171-280). */
typedef void (*qcp_deliver_fn)(void* user, uint32_t request, const int32_t* ids, uint64_t n);

/* One plan replay (or one alone run) of a serving replay, recorded when
 * qcp_serve_opts.trace is set.  Times are seconds since the replay started. */
typedef struct qcp_serve_batch {
  uint32_t worker;     /* worker thread (stream) index */
  uint32_t requests;   /* requests in this run */
  uint32_t path;       /* 0: small plan, 1: large plan, 2: alone through qcp_query_batch */
  uint32_t split;      /* 1: part of a batch split after an overflow */
  uint64_t hits;
  double t_taken;      /* the batch was taken from the queue */
  double t_start;      /* this run started */
  double t_run;        /* this run's hit total was on the host */
  double t_admitted;   /* its result bytes were admitted under the cap */
  double t_done;       /* its results were on the host and delivered */
} qcp_serve_batch;

typedef struct qcp_serve_opts {
  uint32_t streams;          /* batches in flight; 0 = 4 */
  uint32_t max_batch;        /* queries per batch at most; 0 = 16384 */
  uint64_t output_cap_bytes; /* result bytes held at once; 0 = 2 GiB */
  qcp_deliver_fn deliver;    /* NULL: results are dropped after the copy */
  void* user;                /* passed to deliver */
  qcp_serve_batch* trace;    /* NULL, or room for trace_cap records (the first ones are kept) */
  uint64_t trace_cap;
} qcp_serve_opts;

typedef struct qcp_serve_stats {
  uint64_t requests;
  uint64_t hits;
  uint64_t batches;
  double mean_batch;         /* requests per batch */
  double seconds;            /* first arrival -> last completion */
  double qps;                /* requests / seconds */
  double p50_ms, p99_ms, max_ms, mean_ms;  /* with latency_ms only */
  uint32_t max_inflight;     /* most batches on the device at once */
  uint32_t reserved_;
  uint64_t max_output_bytes; /* most result bytes held at once */
} qcp_serve_stats;

qcp_status qcp_serve_replay(qcp_index* index, const float* boxes, const double* arrival_s, uint32_t q,
                            const qcp_serve_opts* opts, float* latency_ms, qcp_serve_stats* stats);

/* Message of the last error on the calling host thread ("" if none). */
const char* qcp_last_error(void);

/* Kernels this library launched on the calling host thread since the last
 * reset (reset = 1 clears the counter after reading). */
uint64_t qcp_launch_count(int reset);

/* Library version string. */
const char* qcp_version(void);

#ifdef __cplusplus
}
#endif
#endif /* QCP_H_ */
