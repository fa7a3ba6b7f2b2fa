/*
 * apspie.h -- C ABI of apspie_b200, a B200-native (sm_100a) implementation of
 * apspie's SpMSpV / hash-SpGEMM hot path.
 *
 * Conventions
 *   - Every entry point returns an int status (APSPIE_OK == 0) and never
 *     exits the process.  apspie_last_error() gives a message for the last
 *     failure on a context.
 *   - Pointers named d_* are device pointers on the context's device; h_*
 *     are host pointers.  Graphs are CSR with int32 row offsets and int32
 *     column indices (the reference's layout, src/matrix.hpp:6-37).  For
 *     traversal the CSR row of u lists u's out-neighbours, which is the
 *     "CSC" the reference drivers pass to mXv (test/bfs/main.cu:140).
 *   - Work is stream-ordered on the context's stream.  Calls that return a
 *     value to the host (counts, statistics) synchronise that stream.
 *   - A context must not be used from two host threads at once.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * the apspie source tree).
 */
#ifndef APSPIE_H
#define APSPIE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  APSPIE_OK = 0,
  APSPIE_ERR_INVALID = 1,     /* bad argument (size, vertex id, null pointer) */
  APSPIE_ERR_OOM = 2,         /* device or host allocation failed */
  APSPIE_ERR_CUDA = 3,        /* CUDA runtime error */
  APSPIE_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  APSPIE_ERR_OVERFLOW = 5,    /* a result does not fit the int32 layout */
  APSPIE_ERR_UNSUPPORTED = 6, /* feature not available on this device */
  APSPIE_ERR_BUSY = 7,        /* serving queue full / admission refused */
  APSPIE_ERR_TOO_LARGE = 8    /* input exceeds a fixed buffer's stated maximum */
} apspie_status;

typedef struct apspie_context *apspie_ctx;

/* ------------------------------------------------------------ context ---
 * Replaces mgpu::CreateCudaDevice (test/bfs/main.cu:27) plus the scratch
 * workspace of allocScratch (src/util.cuh:646-672, src/scratch.hpp:5-31):
 * the context owns a grow-only device workspace reused across calls, so no
 * call allocates once the workspace has grown to the graph's size.
 * stream may be NULL (the legacy default stream). */
int apspie_ctx_create(int device, void *stream, apspie_ctx *out);
int apspie_ctx_destroy(apspie_ctx ctx);
int apspie_ctx_set_stream(apspie_ctx ctx, void *stream);
/* Caps the blocks of this context's persistent launches (BFS, SSSP, MIS,
 * batch); 0 = as many as fit (the default).  Two contexts whose caps add up
 * to at most apspie_ctx_resident_blocks can run persistent kernels at the
 * same time on different streams. */
int apspie_ctx_set_max_grid(apspie_ctx ctx, int blocks);
/* A cap that every persistent kernel of the library fits (2 per SM). */
int apspie_ctx_resident_blocks(apspie_ctx ctx, int *blocks);
int apspie_ctx_sync(apspie_ctx ctx);
/* Number of kernels this context has launched since creation. */
int apspie_ctx_launch_count(apspie_ctx ctx, uint64_t *out);
/* Bytes of device workspace currently held by the context (its
 * sub-contexts' included). */
int apspie_ctx_workspace_bytes(apspie_ctx ctx, size_t *out);
const char *apspie_last_error(apspie_ctx ctx);
const char *apspie_status_string(int status);

/* ---------------------------------------------------------------- BFS ---
 * Replaces bfs<T>() (src/bfs.cuh:33-125, mXv + addResult per level) and the
 * keys-only spmspvBfs() (src/spmspvBfs.cuh:96-243).
 * d_depth[v] = level of v (source 0, unreached -1), bit-exact with the
 * reference's CPU BFS (src/testBfs.cpp:7-72).  max_levels > 0 stops after
 * levels 1..max_levels-1 have been assigned, as the reference's fixed
 * iteration count does (src/bfs.cuh:87); max_levels <= 0 runs to convergence.
 * Direction-optimising: push over the frontier queue (out-adjacency d_ptr /
 * d_ind) while it is small, pull over the unvisited vertices while it is
 * large.  Pull reads the in-adjacency d_tptr / d_tind (CSR of the transpose);
 * pass d_ptr / d_ind again for an undirected graph, or NULL to push only. */
int apspie_bfs(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
               const int *d_ind, const int *d_tptr, const int *d_tind,
               int32_t *d_depth, int max_levels);

typedef struct {
  int32_t levels;            /* deepest level + 1 (the reference's "search depth") */
  int32_t pull_levels;       /* levels run in the pull direction */
  int64_t vertices_reached;  /* |R| */
  int64_t edges_traversed;   /* E_R = sum of out-degrees of reached vertices */
} apspie_bfs_stats;

/* Statistics of the last apspie_bfs on this context (synchronises). Also
 * reports a device-side timeout of that run as APSPIE_ERR_TIMEOUT. */
int apspie_bfs_get_stats(apspie_ctx ctx, apspie_bfs_stats *out);

/* Transpose of an m x n CSR (the CSC of the matrix; csr2csc,
 * src/util.cuh:474, extract_csr2csc, src/matrix.cpp:230): d_tptr n + 1
 * offsets, d_tind nnz row ids ascending within each column, d_tval nnz values
 * (may be NULL; d_val NULL = ones).  Caller-allocated outputs; a stable radix
 * sort of the edges on the device. */
int apspie_csr_transpose(apspie_ctx ctx, int m, int n, int64_t nnz,
                         const int *d_ptr, const int *d_ind, const float *d_val,
                         int *d_tptr, int *d_tind, float *d_tval);

/* Builds the in-adjacency that apspie_bfs pulls over (d_tptr: m + 1
 * offsets, d_tind: nnz indices, caller-allocated) from the out-adjacency,
 * each row ordered by the neighbours' out-degree, highest first (ties by
 * id).  A vertex still unvisited at level L has no neighbour above depth L,
 * and its best-connected neighbours are the likeliest to be in the level's
 * frontier, so a pull probe hits sooner.  Depths do not depend on the order.
 * A one-time graph build step (a radix sort of the edges), like building
 * the transpose; pass the result as d_tptr / d_tind (also for an undirected
 * graph, instead of repeating d_ptr / d_ind). */
int apspie_bfs_prepare(apspie_ctx ctx, int m, int64_t nnz, const int *d_ptr,
                       const int *d_ind, int *d_tptr, int *d_tind);

/* Per-level trace of the last apspie_bfs (synchronises): for each level
 * i < max_levels (at most 64) the direction (1 push, 2 pull), frontier size,
 * frontier out-edges, device time in ns, and two self-checks: vertices
 * queued from an implicit (pull-produced) frontier before a push level, and
 * edges the push expansion walked (== frontier out-edges); and the ns from
 * the level's start until the first and the last block finished its share of
 * the level (the remainder of h_ns is the grid barrier).  *n_out = levels
 * written.  The array outputs may be NULL. */
int apspie_bfs_get_trace(apspie_ctx ctx, int max_levels, int *n_out,
                         int32_t *h_mode, int64_t *h_frontier,
                         int64_t *h_frontier_edges, int64_t *h_ns,
                         int64_t *h_queued, int64_t *h_expanded,
                         int64_t *h_work_first_ns, int64_t *h_work_last_ns);

/* BFS that allocates no memory: apspie_bfs's traversal (same arguments and
 * result, push/pull chosen automatically, or push only when d_tptr is NULL)
 * for callers that cannot call cudaMalloc -- code running while a stream is
 * captured into a CUDA graph, hosts whose device memory is fixed up front,
 * plugins inside a process whose allocator they do not own.  No context is
 * needed: work goes on `stream` (NULL = legacy default stream) of the current
 * device.  Its scratch is one fixed array in device memory, held by every GPU
 * that loads the library until the process exits, sized for at most 2^20
 * vertices and 2^24 edges; larger inputs return APSPIE_ERR_TOO_LARGE without
 * launching anything.  The first call on a device looks up that array's
 * device address (and may load the library's device code); make that first
 * call before any stream capture.  All calls share the one array, so calls
 * that overlap on the GPU (other streams, other host threads) race; run them
 * one after another.  The array's address is cached per CUDA context (a
 * driver-API context of the caller's, or the device's primary context, which
 * cudaDeviceReset replaces).  Statistics are not reported; the run's status
 * is read with apspie_bfs_noalloc_status.  No counterpart in the reference. */
int apspie_bfs_noalloc(void *stream, int src, int64_t nnz, int m,
                       const int *d_ptr, const int *d_ind, const int *d_tptr,
                       const int *d_tind, int32_t *d_depth, int max_levels);
/* Status of the last apspie_bfs_noalloc on the current device: enqueues on
 * `stream` a copy of its status word into d_status (one int of device
 * memory), stream-ordered and without a host synchronisation -- 0, or
 * APSPIE_ERR_TIMEOUT when a bounded grid-barrier wait gave up (the depths are
 * then incomplete).  Enqueue it on the traversal's stream, after the
 * traversal and before the next apspie_bfs_noalloc on the device: every call
 * shares the one status word.  Allocates nothing. */
int apspie_bfs_noalloc_status(void *stream, int32_t *d_status);

/* Direction-switch thresholds (Beamer's alpha, beta; defaults 14 and 24):
 * push -> pull when frontier edges * alpha > unexplored edges, pull -> push
 * when frontier vertices * beta < m (alpha 0 never pulls).  mode: 0 = switch
 * automatically, 1 = push only, 2 = pull only. */
int apspie_bfs_set_params(apspie_ctx ctx, int alpha, int beta, int mode);

/* --------------------------------------------------------------- SSSP ---
 * Replaces sssp<V>() (src/sssp.cuh:28-115) with its per-iteration min-plus
 * spmspvSssp<V>() (src/spmspvSssp.cuh:92-291).  Frontier-driven
 * Bellman-Ford: each round expands the vertices whose distance dropped in the
 * previous round, relaxing with atomicMin.  Unreached vertices get
 * UINT32_MAX (u32) or +inf (f32); the reference uses -1 on the CPU and
 * 1.70141e38 on the GPU.  u32 sums saturate at UINT32_MAX - 1.  The f32
 * result is bit-identical to the reference's CPU SSSP (src/testSssp.cpp:33-
 * 115): every relaxation is one round-to-nearest single add and both reach
 * the same fixpoint.  max_rounds > 0 bounds the number of rounds (the
 * reference's `depth` argument; its unit-weight rounds after the first,
 * src/sssp.cuh:83,91, are not reproduced); <= 0 runs to convergence. */
int apspie_sssp_u32(apspie_ctx ctx, int src, int64_t nnz, int m,
                    const int *d_ptr, const int *d_ind, const uint32_t *d_w,
                    uint32_t *d_dist, int max_rounds);
int apspie_sssp_f32(apspie_ctx ctx, int src, int64_t nnz, int m,
                    const int *d_ptr, const int *d_ind, const float *d_w,
                    float *d_dist, int max_rounds);
/* The same, direction-optimising: given the in-adjacency with its weights
 * (d_tptr / d_tind / d_tw, e.g. from apspie_csr_transpose with the weights
 * as the values), a round whose frontier's out-edges times alpha exceed nnz
 * (apspie_sssp_set_pull; default 0 = never: with the staged push rounds,
 * push-only measured 3.1 ms per source on R-MAT 22 symmetrised against 3.7
 * at alpha 2, and 6.2 against 7.3 ms on R-MAT 23) scans every in-edge
 * instead: each vertex takes the least d[u] + w(u,v) over its in-neighbours
 * in the frontier and writes its own distance, without atomics.  Same
 * results as apspie_sssp_u32 / _f32 (the same min-plus fixpoint); pull
 * rounds are only taken with the near-far step at 0.  With the switch at 0
 * the in-adjacency is not read and the call runs as apspie_sssp_u32 / _f32
 * (the same kernel).  Replaces the same
 * reference calls (src/sssp.cuh:28-115), whose every iteration scans all
 * finite vertices' edges. */
int apspie_sssp_u32_pull(apspie_ctx ctx, int src, int64_t nnz, int m,
                         const int *d_ptr, const int *d_ind, const uint32_t *d_w,
                         const int *d_tptr, const int *d_tind, const uint32_t *d_tw,
                         uint32_t *d_dist, int max_rounds);
int apspie_sssp_f32_pull(apspie_ctx ctx, int src, int64_t nnz, int m,
                         const int *d_ptr, const int *d_ind, const float *d_w,
                         const int *d_tptr, const int *d_tind, const float *d_tw,
                         float *d_dist, int max_rounds);
int apspie_sssp_set_pull(apspie_ctx ctx, int alpha);

typedef struct {
  int32_t rounds;            /* frontier rounds run */
  int32_t phases;            /* near-far phases (0 without near-far) */
  int64_t vertices_reached;  /* |R| */
  int64_t edges_traversed;   /* E_R = sum of out-degrees of reached vertices */
  int64_t relaxations;       /* edges scanned over all rounds (>= E_R) */
} apspie_sssp_stats;

/* Near-far schedule of apspie_sssp_*: a vertex whose distance drops below
 * the threshold T joins the next frontier, one at or above it waits in a far
 * list until the frontier runs dry and T grows by delta.  delta 0 (the
 * default) = T infinite, i.e. frontier Bellman-Ford.  The distances do not
 * depend on delta (same fixpoint); the work and the number of rounds do. */
int apspie_sssp_set_params(apspie_ctx ctx, uint32_t delta_u32, float delta_f32);

/* Per-round trace of the last SSSP (synchronises), expansion rounds only
 * (at most 64): frontier vertices, their out-edges, device ns of the round
 * and ns until the last block finished its share (the rest is the grid
 * barrier).  *n_out = rounds written; the arrays may be NULL. */
int apspie_sssp_get_trace(apspie_ctx ctx, int max_rounds, int *n_out,
                          int64_t *h_frontier, int64_t *h_frontier_edges,
                          int64_t *h_ns, int64_t *h_work_last_ns);

/* Statistics of the last SSSP on this context (synchronises). */
int apspie_sssp_get_stats(apspie_ctx ctx, apspie_sssp_stats *out);

/* ---------------------------------------------------------------- MIS ---
 * Replaces spmspvMis<V>() (src/spmspvMis.cuh:150-344).  d_prio holds one
 * uint32 priority per vertex (mt19937 draws, apspie_mt19937_fill_host).  A
 * vertex joins when it beats every undecided neighbour in key
 * (prio << 32 | id): the result is the greedy MIS in descending key order,
 * independent of delta, which only sets how fast the candidate threshold
 * falls (the reference's `minimum -= delta`, src/spmspvMis.cuh:235-236;
 * delta <= 0 means 1).  d_mis[v] = 1 (in the set) or 0.  Self-loops are
 * ignored.  The graph must be symmetric. */
int apspie_mis(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr,
               const int *d_ind, const uint32_t *d_prio, int32_t *d_mis,
               float delta);
/* Rounds used by the last apspie_mis (synchronises). */
int apspie_mis_get_rounds(apspie_ctx ctx, int *rounds);

/* Neighbour flags: d_out[v] = 1 if v is an out-neighbour of some u with
 * d_in[u] != 0, else 0.  Replaces spmspvCsr() (src/spmspvMis.cuh:81-147),
 * the SpMSpV behind the reference's MIS check (test/mis/main.cu:217-221). */
int apspie_neighbor_flags(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr,
                          const int *d_ind, const int32_t *d_in,
                          int32_t *d_out);

/* ------------------------------------------------------ batched traversal ---
 * Many BFS / SSSP traversals, on graphs of different sizes, in one
 * persistent launch (no reference counterpart: the reference runs one query
 * per driver invocation).  A BFS job runs up to 64 sources of a graph as one
 * multi-source BFS (64-bit per-vertex source masks); more sources are split
 * into several device jobs.  An SSSP job relaxes (source, vertex) items with
 * uint32 weights.  Per source the results equal apspie_bfs / apspie_sssp_u32:
 * d_out holds nsrc rows of m entries (depths, -1 unreached; or distances,
 * UINT32_MAX unreached).  alpha / beta < 0 take the context's defaults (the
 * autotuner sets them per graph); alpha 0 never pulls.  At most 64 device jobs per call; nsrc * m
 * must stay below 2^31 for SSSP jobs.  max_steps > 0 caps the super-steps. */
typedef enum { APSPIE_JOB_BFS = 0, APSPIE_JOB_SSSP_U32 = 1 } apspie_job_type;
typedef struct {
  int type;             /* apspie_job_type */
  int m;
  int64_t nnz;
  const int *d_ptr, *d_ind;    /* out-adjacency */
  const int *d_tptr, *d_tind;  /* in-adjacency for pull, or NULL */
  const uint32_t *d_w;         /* SSSP weights */
  int symmetric;               /* 1: pull may use d_ptr / d_ind */
  int nsrc;
  const int *h_src;            /* host array of nsrc sources */
  int32_t *d_out;              /* nsrc x m results */
  int alpha, beta;             /* BFS direction thresholds, < 0 = default */
  /* SSSP only, may be NULL: the in-adjacency with its weights; then steps
   * whose frontier out-edges times the context's batch pull switch
   * (apspie_batch_set_sssp_pull; default 0 = never) exceed nnz are pull
   * steps */
  const int *d_stptr, *d_stind;
  const uint32_t *d_stw;
} apspie_job;
typedef struct {
  int32_t super_steps;
  int32_t pad;
  int64_t frontier_edges;  /* sum of frontier out-edges over all jobs and steps */
} apspie_batch_stats;

int apspie_batch_run(apspie_ctx ctx, int njobs, const apspie_job *jobs,
                     int max_steps);
/* Jobs on graphs whose BFS takes more than 64 levels (found by one probe BFS
 * per new graph, cached by fingerprint) are latency bound per level and
 * share little between sources: their sources run as single-source
 * traversals (apspie_bfs / apspie_sssp_u32, SSSP near-far with the
 * context's step or 1024), up to max_concurrent (default 48, at most 64)
 * at a time on sub-contexts of this context (own streams and workspaces),
 * next to the multi-source launch of the other jobs; deep_blocks = their
 * blocks in all (0: half the resident blocks).  The call stays
 * stream-ordered on the context's stream.  max_concurrent = 0 puts every
 * job in the multi-source launch instead; max_steps > 0 always does. */
int apspie_batch_set_params(apspie_ctx ctx, int deep_blocks);
int apspie_batch_set_deep_mode(apspie_ctx ctx, int max_concurrent);
/* Pull switch of the multi-source SSSP steps (0 = never pull, the
 * default: on R-MAT 20 / 22 with 8 .. 32 sources the pull steps were 3 - 30 %
 * slower than the push steps, each reading a distance row per in-edge). */
int apspie_batch_set_sssp_pull(apspie_ctx ctx, int alpha);
/* Statistics of the last batch (synchronises; reports a barrier timeout). */
int apspie_batch_get_stats(apspie_ctx ctx, apspie_batch_stats *out);

/* ------------------------------------------------------------- serving ---
 * A query server over device-resident graphs (no reference counterpart).
 * Queries arrive at any time; a worker thread admits them in arrival order
 * while their device state fits state_budget_bytes and the device memory
 * the server can use: what its lanes' workspaces and result buffers already
 * hold (admitted queries reuse it) plus the device's free memory, less a
 * 2 GiB reserve (read when a batch forms, at most every 10 ms; the
 * first query of an idle server is always admitted),
 * coalesces the admitted
 * BFS / SSSP queries by (graph, kind) into one apspie_batch_run launch, runs
 * MIS queries after it, and copies each result row into the caller's host
 * buffer.  Two batch slots (each its own context and stream) keep a new batch
 * queued on the GPU while the previous one is still running.  Query kinds:
 * 0 = BFS (int32 depths), 1 = SSSP over the graph's uint32 weights (uint32
 * distances), 2 = MIS with mt19937(seed) priorities (int32 membership).
 * h_result must hold m 32-bit entries and stay valid until the query is done.
 * The graphs' device arrays must outlive the server. */
typedef struct apspie_server *apspie_server_t;
typedef struct {
  uint64_t completed, batches, jobs, pending;
  uint64_t in_flight_bytes;
  double p50_ms, p99_ms, max_ms;  /* submit -> result in host memory */
  uint64_t admission_waits;  /* times admission stopped at the budget / memory cap */
  uint64_t memory_cap_bytes; /* held + free device memory less the reserve, last read */
  double max_launch_ms;      /* longest host time the worker spent launching one batch */
} apspie_server_stats;

int apspie_server_create(int device, size_t state_budget_bytes, int max_batch,
                         apspie_server_t *out);
int apspie_server_add_graph(apspie_server_t s, int m, int64_t nnz,
                            const int *d_ptr, const int *d_ind,
                            const int *d_tptr, const int *d_tind,
                            const uint32_t *d_w, int symmetric, int *graph_id);
/* Registers graph's in-adjacency with its uint32 weights (e.g. from
 * apspie_csr_transpose): its SSSP queries then run push/pull rounds
 * (apspie_sssp_u32_pull).  Call before submitting queries on the graph. */
int apspie_server_set_sssp_in(apspie_server_t s, int graph, const int *d_tptr,
                              const int *d_tind, const uint32_t *d_tw);
/* Non-blocking; APSPIE_ERR_BUSY when the pending queue is full. */
int apspie_server_submit(apspie_server_t s, int type, int graph, int source,
                         uint32_t seed, void *h_result, uint64_t *req_id);
/* As apspie_server_submit, with the result row copied into d_result (device
 * memory, m 32-bit entries) instead; d_result == NULL drops the result once it
 * is computed (load tests: only the latency is recorded). */
int apspie_server_submit_device(apspie_server_t s, int type, int graph,
                                int source, uint32_t seed, int32_t *d_result,
                                uint64_t *req_id);
/* One query of a timed stream: kind and arguments as for submit, arrival
 * time in microseconds from the start of the stream (non-decreasing). */
typedef struct {
  int32_t type, graph, source;
  uint32_t seed;
  double t_us;
} apspie_query;
/* Open-loop replay: submits query i at its arrival time and waits for all;
 * lat_ms[i] = arrival -> result in host memory (to_host != 0: each result
 * row is copied into the server's pinned staging memory) or on the device
 * (to_host == 0); results are not kept.  *wall_ms = stream start -> last
 * completion. */
int apspie_server_replay(apspie_server_t s, int n, const apspie_query *q,
                         int to_host, double *lat_ms, double *wall_ms);
/* apspie_server_replay that keeps answers: d_keep (may be NULL) holds one
 * device pointer per query, NULL or a row of m 32-bit entries on the
 * server's device into which that query's result is copied (device to
 * device, on the query's stream, before its completion is recorded), so a
 * sample of the served answers can be checked after a timed replay. */
int apspie_server_replay_keep(apspie_server_t s, int n, const apspie_query *q, int to_host,
                              int32_t *const *d_keep, double *lat_ms, double *wall_ms);
/* The same stream one query at a time, in arrival order, through
 * apspie_bfs / apspie_sssp_u32 / apspie_mis on a stream and context of its
 * own, kept by the server across calls (the plain single-query path);
 * latencies likewise from the arrival times.  Not to be called from two
 * threads at once. */
int apspie_server_replay_plain(apspie_server_t s, int n, const apspie_query *q,
                               int to_host, double *lat_ms, double *wall_ms);
/* *done = 1 once the result is in h_result (the request is then retired and
 * its status returned). */
int apspie_server_poll(apspie_server_t s, uint64_t req_id, int *done,
                       double *latency_ms);
/* Blocks until the query is done (at most 600 s, else APSPIE_ERR_TIMEOUT). */
int apspie_server_wait(apspie_server_t s, uint64_t req_id, double *latency_ms);
int apspie_server_get_stats(apspie_server_t s, apspie_server_stats *out);
int apspie_server_reset_stats(apspie_server_t s);
/* Finishes the queued queries, then stops the worker and frees the server. */
int apspie_server_destroy(apspie_server_t s);

/* ----------------------------------------------------------- autotuner ---
 * The reference hard-codes its launch shapes and table sizes (NTHREADS,
 * TABLE_SIZE, partSize from an "aggro" factor: src/spgemm.cuh:15,
 * src/spgemmKernel.cuh:9-26, test/spgemm/main.cu:362-377).  Here the
 * data-dependent choices are context settings, measured per graph by the
 * autotuners below and cached under a fingerprint of the graph (m, nnz,
 * sampled row offsets; for SpGEMM of both operands, for a batch of every
 * job's graph and source count): a graph seen again is not re-measured, the
 * cached choice is applied to the context again. */
typedef struct {
  int32_t bfs_alpha, bfs_beta;     /* BFS switch points (alpha 0: never pull) */
  int32_t bfs_blocks_per_sm;       /* persistent BFS launch, blocks per SM (0: as many as fit, 3) */
  int32_t sssp_blocks_per_sm;      /* persistent SSSP launch (0: as many as fit) */
  int32_t sssp_pull_alpha;         /* SSSP pull rounds (0: push only; see apspie_sssp_set_pull) */
  int32_t batch_blocks_per_sm;     /* batched multi-source launch (0: as many as fit, 2) */
  int32_t batch_deep_blocks;       /* blocks of the deep-graph sources in a batch (0: default share) */
  int32_t spgemm_table_load;       /* SpGEMM hash tables hold >= load x entries: 2 or 4 */
  int32_t spgemm_warp_max_prod;    /* SpGEMM rows of <= this many products are one warp's (16..256) */
  int64_t spgemm_bitmap_max_cols;  /* see apspie_spgemm_set_params */
  double spmspv_sort_factor;       /* see apspie_spmspv_set_params */
} apspie_tuning;
int apspie_ctx_get_tuning(apspie_ctx ctx, apspie_tuning *out);
/* Sets every field (validated: APSPIE_ERR_INVALID when out of range). */
int apspie_ctx_set_tuning(apspie_ctx ctx, const apspie_tuning *in);

/* Measures the BFS direction thresholds on the given sample sources (a grid
 * of alpha / beta values and push-only, timed with CUDA events: ranked on
 * the first half of the sources, the four best timed again on the second
 * half together with the reference point alpha 32 / beta 128, the pick by
 * the sum over both halves and kept only if it beats the reference point by
 * more than 2 %), then the blocks per SM of the persistent launch (3, 2, 1
 * with the chosen switch points on all sources; fewer blocks kept only when
 * more than 2 % faster).  Stores the result in the context (used by
 * apspie_bfs and, for jobs with alpha / beta < 0, by apspie_batch_run).
 * d_depth_scratch: m int32.  *ms_out (may be NULL) = mean ms per BFS. */
int apspie_autotune_bfs(apspie_ctx ctx, int nsrc, const int *h_src, int64_t nnz,
                        int m, const int *d_ptr, const int *d_ind,
                        const int *d_tptr, const int *d_tind,
                        int32_t *d_depth_scratch, int *alpha_out, int *beta_out,
                        float *ms_out);
/* Finds the frontier density at which the SpMSpV bitmap path beats the
 * radix-sort path on this matrix and sets the context's sort factor (see
 * apspie_spmspv_set_params).  Scratch: m ints (x), m ints + m floats (y);
 * the frontiers are timed with unit values, so d_xval_scratch is not
 * written and may be NULL. */
int apspie_autotune_spmspv(apspie_ctx ctx, int m, int64_t nnz, const int *d_ptr,
                           const int *d_ind, const float *d_val,
                           int *d_xind_scratch, float *d_xval_scratch,
                           int *d_yind_scratch, float *d_yval_scratch,
                           double *factor_out);
/* Measures the persistent SSSP launch's blocks per SM (as many as fit, then
 * fewer) and, when the in-adjacency is given (d_tptr / d_tind / d_tw, or
 * all NULL), the pull-round switch alpha (0, 2, 8), on uint32 weights from
 * the given sources (two sweeps in opposite orders, each candidate scored by
 * its better time; a choice other than the current default is kept only
 * when more than 2 % faster).  d_dist_scratch: m uint32.  *ms_out (may be
 * NULL) = mean ms per SSSP of the pick; *cached_out (may be NULL) = 1 when
 * the graph was in the cache. */
int apspie_autotune_sssp(apspie_ctx ctx, int nsrc, const int *h_src, int64_t nnz, int m,
                         const int *d_ptr, const int *d_ind, const uint32_t *d_w,
                         const int *d_tptr, const int *d_tind, const uint32_t *d_tw,
                         uint32_t *d_dist_scratch, float *ms_out, int *cached_out);
/* Measures the batched launch's blocks per SM (as many as fit, then one)
 * and, when some job runs on a deep graph (see apspie_batch_set_params),
 * the deep sources' block share (a quarter, half, three quarters of the
 * resident blocks), running apspie_batch_run on the given jobs (their
 * d_out rows are written).  Same scoring and caching as
 * apspie_autotune_sssp; the fingerprint covers every job's graph, type and
 * source count. */
int apspie_autotune_batch(apspie_ctx ctx, int njobs, const apspie_job *jobs, float *ms_out,
                          int *cached_out);

/* --------------------------------------------------------- test hooks ---
 * For the tests of the timeout paths (no reference counterpart).  Every
 * device-side wait is bounded and reports APSPIE_ERR_TIMEOUT when it runs
 * out; a hook makes one run out without a fault or an unbounded wait.
 * One-shot: APSPIE_INJECT_BFS_BARRIER -- the next BFS launch on ctx (ctx NULL:
 * the next apspie_bfs_noalloc on the current device) loses its last block
 * before the first grid barrier; the others' wait gives up (about 1.7 s) and
 * apspie_bfs_get_stats (or the no-alloc status word) reports the timeout.
 * APSPIE_INJECT_SORT_LOOKBACK -- the first tile of the next multi-tile radix
 * sort pass on ctx withholds its look-back status; its successors give up
 * (about half a second), write their keys in bounds, and the next call that
 * reads the sort's give-up word (apspie_spmspv, apspie_tc_prepare, the device
 * graph build) reports the timeout.  APSPIE_INJECT_ALLOC_FAIL -- the next
 * workspace growth on ctx fails on the host as an exhausted cudaMalloc would:
 * the call returns APSPIE_ERR_OOM and the context stays usable. */
enum {
  APSPIE_INJECT_BFS_BARRIER = 1,
  APSPIE_INJECT_SORT_LOOKBACK = 2,
  APSPIE_INJECT_ALLOC_FAIL = 3
};
int apspie_debug_inject(apspie_ctx ctx, int what);
/* The next query group of the given kind (0 BFS, 1 SSSP, 2 MIS) that the
 * server launches completes with APSPIE_ERR_CUDA without running: its
 * requests' waits return the error, the other groups are unaffected. */
int apspie_server_debug_fail_next(apspie_server_t s, int kind);

/* ------------------------------------------------------------- SpMSpV ---
 * Semirings of the reference's three SpMSpV variants. */
typedef enum {
  APSPIE_PLUS_TIMES = 0, /* mXv (src/mXv.cuh:106 multiply, :201 ReduceByKey plus) */
  APSPIE_MIN_PLUS = 1,   /* spmspvSssp (src/spmspvSssp.cuh:87 add, :232 minimum) */
  APSPIE_MAX_TIMES = 2,  /* spmspvMis (src/spmspvMis.cuh:289 maximum) */
  APSPIE_OR_AND = 3      /* Boolean reachability (keys-only spmspvBfs) */
} apspie_semiring;

/* Sparse x (d_xind ascending-unique, d_xval or NULL = ones) times A, where
 * d_ptr / d_ind / d_val (NULL = ones) list A's columns: y[r] = (+) over x's
 * entries j of A(r, j) (x) x[j].  Replaces the sparse mXv<T>()
 * (src/mXv.cuh:250-389).  y comes back sorted by row with one entry per
 * touched row (structural, as the reference's ReduceByKey); d_yind / d_yval
 * must hold m entries.  *h_ynnz = nnz(y); *h_expanded (may be NULL) = number
 * of products.  PLUS_TIMES sums in double and rounds once; MIN_PLUS and
 * MAX_TIMES form each term with one float op, as the reference does.
 * Synchronises (the output size goes to the host, as in the reference). */
int apspie_spmspv(apspie_ctx ctx, int semiring, int m, int64_t nnz,
                  const int *d_ptr, const int *d_ind, const float *d_val,
                  int xnnz, const int *d_xind, const float *d_xval, int *d_yind,
                  float *d_yval, int *h_ynnz, int64_t *h_expanded);

/* Dense SpMV over every row: y[r] = (+) over row r's entries k of
 * A(r, ind[k]) (x) x[ind[k]] (d_val NULL = ones), for all m rows; an empty
 * row gets the (+) identity (0, or +/-FLT_MAX for MIN_PLUS / MAX_TIMES).
 * Replaces the dense spmv() (mgpu::SpmvCsrBinary, src/bfs.cuh:12-14) and
 * cuspmv() (cusparseScsrmv, src/tc.cuh:18-59).  PLUS_TIMES sums in double
 * and rounds once; each row is reduced in a fixed order.  No sync. */
int apspie_spmv(apspie_ctx ctx, int semiring, int m, int64_t nnz,
                const int *d_ptr, const int *d_ind, const float *d_val,
                const float *d_x, float *d_y);

/* Dense x in, dense y out: the dense mXv<T>() (src/mXv.cuh:111-247) and
 * spmspvSssp (src/spmspvSssp.cuh:92).  The frontier is {j : x[j] > 0.5}
 * for PLUS_TIMES (bitify, src/mXv.cuh:50), {j : -1 < x[j] < 1e38} for
 * MIN_PLUS (src/spmspvSssp.cuh:31) and {j : x[j] != 0} otherwise; untouched
 * y entries are 0 (1.70141e38 for MIN_PLUS), as preprocessFlag sets them.
 * *h_expanded (may be NULL) = the reference's return value `total`. */
int apspie_mxv_dense(apspie_ctx ctx, int semiring, int m, int64_t nnz,
                     const int *d_ptr, const int *d_ind, const float *d_val,
                     const float *d_x, float *d_y, int64_t *h_expanded);

/* SpMSpV path choice: the bitmap (dense accumulator) path is used when
 * products * sort_factor > m, else the radix-sort path.  Default 4. */
int apspie_spmspv_set_params(apspie_ctx ctx, double sort_factor);

/* ------------------------------------------------------------- SpGEMM ---
 * The reference's d_matrix (src/matrix.hpp:6-37) reduced to its CSR part:
 * int32 row offsets (m + 1), int32 column indices and float values, all
 * device pointers.  d_val may be NULL (all ones) for inputs. */
typedef struct {
  int m, n;
  int64_t nnz;
  int *d_ptr;
  int *d_ind;
  float *d_val;
} apspie_csr;

/* C = A * B (A->n == B->m).  Replaces the hash SpGEMM
 * spgemm(d_matrix *C, d_matrix *A, d_matrix *B, partSize, partNum, ctx)
 * (src/spgemm.cuh:132-342) and the column-by-column mXm
 * (src/tc.cuh:315-375).  C's structure is the symbolic product (an entry for
 * every (i, j) with some A(i,k) B(k,j), cancellations kept), columns
 * ascending in each row; values are the double-accumulated sums rounded to
 * float.  C's arrays are allocated by the library, as the reference's are;
 * release them with apspie_csr_free.  Synchronises. */
int apspie_spgemm(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                  apspie_csr *C);
/* The two phases of apspie_spgemm with caller-owned C (the reference's
 * spgemm does both inside one call, src/spgemm.cuh:132-342).
 * apspie_spgemm_symbolic writes C's m + 1 row offsets into d_Cptr and nnz(C)
 * into *h_nnz (synchronises once to read it); apspie_spgemm_numeric then
 * fills d_Cind / d_Cval (nnz(C) entries each) for the same A and B on the
 * same context, stream-ordered and without synchronising.  The row bins
 * and accumulators of the symbolic phase stay in the context's workspace
 * (slots of their own), so the numeric phase may be repeated for new
 * values of A and B as long as their structure is unchanged; the next
 * symbolic phase, or apspie_spgemm, replaces the plan (a numeric call for
 * other matrices then returns APSPIE_ERR_INVALID).  A numeric call after
 * the structure changed in place (same pointers) is not detected: its C is
 * wrong, but every write stays inside C's rows and the library's buffers. */
int apspie_spgemm_symbolic(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                           int *d_Cptr, int64_t *h_nnz);
int apspie_spgemm_numeric(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                          const int *d_Cptr, int *d_Cind, float *d_Cval);
/* Rows of A with more than 4096 products (2048 at table load 4) are
 * accumulated over a shared-memory bitmap of C's columns (one bit per
 * column of B, the position of each product in the column-ordered row is a
 * prefix popcount) when B has at most bitmap_max_cols columns (default
 * 262144, limited to 262144 by shared memory; 0 = always the hash tables). */
int apspie_spgemm_set_params(apspie_ctx ctx, int64_t bitmap_max_cols);
/* Measures the SpGEMM table load (2, 4), the warp-row limit (256, 64
 * products) and, when B has at most 262144 columns, bitmap versus hash
 * tables for the long rows, timing apspie_spgemm_symbolic +
 * apspie_spgemm_numeric of A * B (C is allocated and freed inside); keeps
 * the fastest (a choice other than the defaults only when more than 2 %
 * faster) in the context's tuning (apspie_ctx_get_tuning).  Leaves no
 * SpGEMM plan in the context. */
int apspie_autotune_spgemm(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                           float *ms_out, int *cached_out);
int apspie_csr_free(apspie_ctx ctx, apspie_csr *C);
/* Stream-ordered device-to-device copy of a library-owned CSR into caller
 * buffers (m + 1 offsets, nnz indices, nnz values; d_ind / d_val may be
 * NULL). */
int apspie_csr_copy_out(apspie_ctx ctx, const apspie_csr *C, int *d_ptr,
                        int *d_ind, float *d_val);

/* ----------------------------------------------------- triangle count ---
 * L of a symmetric graph (no self-loops counted): vertices relabelled by
 * ascending (degree, id) -- d_perm[v] = new id -- and L(new(u), :) = the new
 * ids of u's neighbours below new(u), rows sorted.  test/tc/main.cu:40-55,
 * 172-175 builds the strict triangles on the host.  d_Lptr holds m + 1
 * entries, d_Lind at least nnz / 2; *h_lnnz = nnz(L).  A graph that is not
 * symmetric is refused with APSPIE_ERR_INVALID: the wrapping sums of a
 * 64-bit hash of every edge (u, v) and of (v, u) must agree (equal edge
 * multisets; a different one passes with probability 2^-64), as must the
 * counts of entries below and above the new order.  Synchronises. */
int apspie_tc_prepare(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr,
                      const int *d_ind, int *d_perm, int *d_Lptr, int *d_Lind,
                      int64_t *h_lnnz);
/* Triangles = sum over (i, k) in L of |L(i,:) n L(k,:)|, as the masked
 * product (L * L) .* L, counted in int64.  Replaces cuSPARSE U * L
 * (src/tc.cuh:63-165) + ewiseMultTc (src/tc.cuh:169-199) + the float
 * reduction of test/tc/main.cu:249.  Synchronises. */
int apspie_tc(apspie_ctx ctx, int m, int64_t lnnz, const int *d_Lptr,
              const int *d_Lind, int64_t *h_count);

/* ------------------------------------------------- host graph builders ---
 * Synthetic inputs of the benchmark configurations (no reference
 * counterpart: the reference reads .mtx files, src/util.cuh:355-430).
 * Results are malloc'ed; release them with apspie_host_free.
 *
 * R-MAT (a,b,c,d) = (0.57,0.19,0.19,0.05), edge_factor * 2^scale samples,
 * self-loops and duplicates removed, optionally symmetrised; vertex ids are
 * scrambled by a seeded bijection when scramble != 0. */
int apspie_gen_rmat_host(int scale, int edge_factor, uint64_t seed,
                         int symmetric, int scramble, int *m_out,
                         int64_t *nnz_out, int **h_ptr, int **h_ind);
/* Erdos-Renyi: n*mean_degree/2 uniform vertex pairs, symmetrised, deduped. */
int apspie_gen_er_host(int n, int mean_degree, uint64_t seed, int64_t *nnz_out,
                       int **h_ptr, int **h_ind);
/* The same R-MAT / Erdos-Renyi graphs built on the device: samples drawn
 * with the host builders' counter-based hash, packed (row, col) keys radix
 * sorted, repeats and self-loops dropped, CSR offsets from row counts.  The
 * result equals apspie_gen_*_host bit for bit; *out is library-owned
 * (apspie_csr_copy_out / apspie_csr_free).  Scratch: 16 bytes per sample
 * (x2 when symmetrised) of context workspace.  Synchronises once (for nnz). */
int apspie_gen_rmat_device(apspie_ctx ctx, int scale, int edge_factor,
                           uint64_t seed, int symmetric, int scramble,
                           apspie_csr *out);
int apspie_gen_er_device(apspie_ctx ctx, int n, int mean_degree, uint64_t seed,
                         apspie_csr *out);
/* apspie_gen_weights_*_host on device arrays (same values). */
int apspie_gen_weights_u32_device(apspie_ctx ctx, int m, const int *d_ptr,
                                  const int *d_ind, uint64_t seed, uint32_t lo,
                                  uint32_t hi, uint32_t *d_w);
int apspie_gen_weights_f32_device(apspie_ctx ctx, int m, const int *d_ptr,
                                  const int *d_ind, uint64_t seed, float *d_w);
/* rows x cols 2-D 5-point grid, vertex id = r*cols + c. */
int apspie_gen_grid_host(int rows, int cols, int64_t *nnz_out, int **h_ptr,
                         int **h_ind);
/* Edge weights as a function of (row, col, seed), so they do not depend on
 * the CSR build order.  u32: uniform in [lo, hi].  f32: uniform in (0, 1]
 * on the grid k * 2^-24. */
int apspie_gen_weights_u32_host(int m, const int *h_ptr, const int *h_ind,
                                uint64_t seed, uint32_t lo, uint32_t hi,
                                uint32_t *h_w);
int apspie_gen_weights_f32_host(int m, const int *h_ptr, const int *h_ind,
                                uint64_t seed, float *h_w);
/* m x n matrix whose row lengths follow a power law: k = floor(X), X a
 * Pareto(alpha, x_min) truncated at max_deg + 1, with x_min solved by
 * bisection so that E[k] = mean (written to *xmin_out); k uniform columns
 * per row (duplicates dropped, so rows can be shorter), values uniform in
 * [-1, 1) on the 2^-23 grid.  The SpGEMM benchmark input (2^18 x 2^18,
 * alpha 2.1, mean 16, max 4096). */
int apspie_gen_powerlaw_host(int m, int n, double alpha, double mean,
                             int max_deg, uint64_t seed, double *xmin_out,
                             int64_t *nnz_out, int **h_ptr, int **h_ind,
                             float **h_val);
/* MT19937 priorities: n outputs of genrand_int32() after init_genrand(seed)
 * (src/mt19937ar.cpp:57-150), the generator the reference uses for its hash
 * constants (src/spgemmKernel.cuh:173-177). */
int apspie_mt19937_fill_host(uint32_t seed, int64_t n, uint32_t *h_out);
/* Matrix Market ingest with the reference's orientation: readEdge/readMtx
 * (src/util.cuh:355-430) store a line's first index as the column and the
 * second as the row; buildMatrix (src/matrix.cpp:56-111) keeps file order
 * inside a row.  undirected != 0 symmetrises as makeSymmetric
 * (src/util.cuh:573-643): mirrors added, sorted by (row, col), repeats
 * dropped, self-loops kept.  h_val may be NULL.  The header's entry count
 * is a bound, not a size: a file with fewer entries is read as far as it
 * goes.  Returns APSPIE_ERR_INVALID for a missing file or an index outside
 * [1, m], APSPIE_ERR_OVERFLOW past 2^31 - 1 entries, APSPIE_ERR_OOM when host
 * memory runs out. */
int apspie_read_mtx_host(const char *path, int undirected, int *m_out,
                         int64_t *nnz_out, int **h_ptr, int **h_ind,
                         float **h_val, int *weighted_out);
void apspie_host_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* APSPIE_H */
