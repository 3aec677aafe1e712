/*
 * graphone_b200.h -- C ABI of the B200 graph engines (libgraphone_b200.so).
 *
 * Plain C types only: opaque handles, raw pointers and sizes, a cudaStream_t
 * passed as void*.  Pointers to CSR arrays and result vectors may be host
 * memory (pageable or pinned) or device memory of the graph's GPU; the
 * library detects which with cudaPointerGetAttributes and copies as needed.
 * Every call returns a g1_status; g1_last_error() gives the message of the
 * last failure on the calling thread.  Nothing is printed, nothing exits.
 *
 * Each entry point names the GraphOne interface it replaces (paths inside
 * the GraphOne source tree).  The functor-templated engines of the
 * GraphOne-compatible headers (include/GraphOne/) call the g1_mem_* / plan /
 * launch-configuration entry points below for all of their host work.
 *
 * Threading: calls on different graphs may run concurrently; calls on one
 * graph are serialised by the graph's own lock (they share its workspace).
 */
#ifndef GRAPHONE_B200_H_
#define GRAPHONE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    G1_OK = 0,
    G1_ERR_INVALID = 1,     /* bad argument or malformed CSR */
    G1_ERR_OOM = 2,         /* device allocation failed / admission refused */
    G1_ERR_DEVICE = 3,      /* a CUDA call failed */
    G1_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
    G1_ERR_UNSUPPORTED = 5, /* combination not available */
    G1_ERR_OVERFLOW = 6     /* a device queue would have overflowed */
} g1_status;

typedef enum { G1_U32 = 0, G1_F32 = 1 } g1_dtype;

typedef enum {
    G1_SR_MINPLUS_U32 = 0,   /* sssp_blas functor, u32 distances */
    G1_SR_MINPLUS_F32 = 1,   /* sssp_blas functor as the app builds it (float) */
    G1_SR_PLUSTIMES_F32 = 2, /* pagerank_blas functor */
    G1_SR_BFS_U32 = 3        /* min-plus with unit weights */
} g1_semiring;

typedef enum {
    G1_SCHED_AUTO = 0,   /* per-graph choice (autotuned when g1_autotune ran) */
    G1_SCHED_MERGE = 1,  /* merge-path row/nonzero split */
    G1_SCHED_VECTOR = 2  /* CSR-vector, lanes per row from the mean degree */
} g1_schedule;

typedef enum {
    G1_ENGINE_BLAS = 0,    /* pull SpMV per iteration (BlasGcEngine, sparse frontier);
                              from 2^20 edges, steps whose frontier is small are computed
                              from the frontier's out-edges (same results) */
    G1_ENGINE_ADVANCE = 1, /* push advance/filter (AdvanceGC); BFS on graphs of small uniform
                              degree runs its rounds in one persistent launch */
    G1_ENGINE_AUTO = 2,    /* near-far on graphs of small uniform degree; else push while
                              the frontier is small and pull when it is large (below 2^24
                              edges: the BLAS engine with its sparse steps) */
    G1_ENGINE_NEARFAR = 3  /* distance-ordered near/far queues in one persistent launch
                              (no GraphOne counterpart; for high-diameter graphs) */
} g1_engine;

typedef enum {
    G1_PR_REFERENCE = 0, /* (1-a)/N + sum: dangling mass dropped, as pagerank_blas */
    G1_PR_DANGLING = 1   /* dangling mass a*sum(rank[dangling])/N added to every vertex */
} g1_pr_mode;

/* Graph creation flags. */
#define G1_GRAPH_SYMMETRIC 0x1u      /* CSR equals its transpose: one copy serves both */
#define G1_GRAPH_INPUT_TRANSPOSE 0x2u /* the arrays given are the in-edge CSR */
#define G1_GRAPH_BUILD_OTHER 0x4u    /* also build the other orientation on the GPU */
#define G1_GRAPH_NO_VALIDATE 0x8u    /* skip the device check of the CSR */
#define G1_GRAPH_RELABEL 0x10u       /* store vertices in decreasing out-degree order
                                        internally (results stay in caller order) */

typedef struct g1_graph g1_graph;

/* ------------------------------------------------------------- basics */
const char* g1_status_string(g1_status s);
const char* g1_last_error(void);
/* Library version string and the compiled architecture ("sm_100a"). */
const char* g1_version(void);

/* Device memory for the header engines' Buffer / DenseVec
 * (replaces archi::memalloc/memfree/memset/memcpy, archi/mem/cuda.cuh:11-59).
 * Allocations are padded to 256 bytes; g1_mem_alloc zero-fills. */
g1_status g1_mem_alloc(void** ptr, size_t bytes);
g1_status g1_mem_free(void* ptr);
/* kind: 0 = host->device, 1 = device->host, 2 = device->device. */
g1_status g1_mem_copy(void* dst, const void* src, size_t bytes, int kind, void* stream);
/* The library keeps the device blocks of closed graphs, plans and engines
 * (up to a quarter of the device's memory) for reuse by later ones of about
 * the same size.  This returns the current device's kept blocks to the
 * driver, after waiting for the device; *released_bytes (may be NULL) gets
 * their total.  No GraphOne counterpart (GraphOne frees at once). */
g1_status g1_release_cached_memory(size_t* released_bytes);
g1_status g1_mem_fill_u32(void* dst, uint32_t value, size_t count, void* stream);
g1_status g1_stream_sync(void* stream);

/* Number of kernels this library has launched since it was loaded (all
 * devices, all threads).  No GraphOne counterpart: measurement support. */
uint64_t g1_kernel_launches(void);
/* Adds n to that counter: the functor-templated engines of the GraphOne
 * headers launch their kernels from the application and report them here. */
void g1_count_user_launches(uint64_t n);
/* For tests of the timeout paths: every bounded device wait launched after
 * this call (the near-far engine's grid barrier, the waits on bulk copies of
 * the TMA-staged SpMV variants) gives up after `polls` polls (0: at the
 * first poll) and the call reports G1_ERR_TIMEOUT; a negative value
 * restores the defaults (a few seconds each).  Copies already in flight are
 * still waited for before a kernel leaves.  Process-wide.  No GraphOne
 * counterpart (GraphOne's kernels never wait on one another). */
g1_status g1_test_set_wait_polls(int64_t polls);
/* Random loads served to the SMs per second, on the current device: gathers
 * of item_bytes (4 or 16) at random positions of a buffer of footprint_bytes
 * (a power of two, 64 KiB .. 4 GiB; by its size the buffer sits in L1, L2 or
 * HBM), blocks_per_sm (1 or 2) 1024-thread blocks per SM, in_flight (1, 4, 8,
 * 16 or 32) independent loads per thread.  From L2 each load is one request,
 * and on B200 an SM gets about one served per cycle whatever the item size,
 * the loads in flight or the warps: the ceiling of the pull SpMV's x gathers
 * that miss the shared-memory copy of x.  No GraphOne counterpart:
 * measurement support. */
g1_status g1_measure_gather_rate(uint32_t item_bytes, uint32_t in_flight, uint32_t blocks_per_sm,
                                 uint64_t footprint_bytes, double* gathers_per_s, void* stream);
/* Random 4-byte loads served per second from shared memory, on the current
 * device: one 1024-thread block per SM with 128 KB of shared memory, in
 * thread-block clusters of cluster_size (1, 2, 4, 8 or 16) blocks, all
 * resident at once; each thread gathers from its own block's shared memory
 * (remote 0) or from a random block of its cluster (remote 1, distributed
 * shared memory).  *blocks (may be NULL): the blocks that ran.  With the L2
 * rate of g1_measure_gather_rate beside it, this shows whether a
 * cluster-wide copy of the SpMV's x could serve the gathers that miss a
 * block's own copy.  No GraphOne counterpart. */
g1_status g1_measure_smem_gather_rate(uint32_t cluster_size, int remote, double* gathers_per_s,
                                      uint32_t* blocks, void* stream);
/* Kernel timing of the SpMV launches (main merge / vector kernels only):
 * between g1_profile_begin and g1_profile_end every such launch is
 * bracketed by CUDA events on its own stream; g1_profile_end synchronises
 * and returns the summed milliseconds and the launch count.  No GraphOne
 * counterpart: measurement support for the roofline figures. */
g1_status g1_profile_begin(void);
g1_status g1_profile_end(double* spmv_ms, uint64_t* spmv_launches);

/* ------------------------------------------------------------- graphs */
/* Makes a device-resident graph from one CSR (row_ptr n+1 entries, col and
 * val m entries, val of `vtype`).  Replaces graph::build + EdgeCache::ToCsr
 * (graph/builder.h:9-46, loader/edge_cache.h:50-105): the other orientation
 * is built on the GPU when G1_GRAPH_BUILD_OTHER is set.  With
 * G1_GRAPH_INPUT_TRANSPOSE the arrays are the in-edge CSR (what
 * graph::build<BlasViews> keeps). */
g1_status g1_graph_create(const uint32_t* row_ptr, const uint32_t* col, const void* val,
                          g1_dtype vtype, uint32_t n, uint32_t m, uint32_t flags,
                          void* stream, g1_graph** out);
g1_status g1_graph_destroy(g1_graph* g);
/* n, m, and whether the out-edge (normal) and in-edge (transpose) CSRs exist. */
g1_status g1_graph_info(const g1_graph* g, uint32_t* n, uint32_t* m, int* has_normal,
                        int* has_transpose);
/* Device pointers of one orientation (0 = out-edges, 1 = in-edges), for the
 * header engines' GraphArchRef (graph/graph_arch_ref.h:23-116). */
g1_status g1_graph_arrays(const g1_graph* g, int transpose, const uint32_t** row_ptr,
                          const uint32_t** col, const void** val);
/* Bytes of device memory the graph holds (CSRs, plans, workspaces). */
size_t g1_graph_device_bytes(const g1_graph* g);

/* ------------------------------------------------------------- SpMV */
/* Merge-path partition of one orientation into tiles of `items_per_tile`
 * merge items (rows + nonzeros; 0 = the orientation's current default),
 * cached in the graph (replaces the SpmvDispatcher<SpmvCudaCsrMergeBased>
 * constructor's SegmentSearch, archi/blas/spmv/cuda/cuda.cuh:75-92).
 * The arrays stay owned by the graph: tile_row/tile_nnz have n_tiles+1
 * entries; carry/tail have room for n_tiles+1 values of up to 16 bytes. */
g1_status g1_spmv_plan(g1_graph* g, int transpose, uint32_t items_per_tile,
                       uint32_t* n_tiles, const uint32_t** tile_row,
                       const uint32_t** tile_nnz, void** carry, void** tail);
/* The nnz-split plan of one orientation (built once per graph): tiles of
 * 256 nonzeros, the rank of the row holding each tile's first nonzero
 * (tile_seg, n_tiles+1), the row-start bitmap over the nonzeros (sbits),
 * the non-empty rows in order followed by the empty rows (rows, n_rows), the
 * tiles in which a row begun in an earlier tile ends (fix_tiles, n_fix) with
 * {tile, row, first tile of the row, 0} per such tile (fix_info, 16 bytes
 * each; the first n_fix_short end in the tile after their first), and
 * carry/tail (room for n_tiles+1 values of up to 16 bytes).  The arrays stay
 * owned by the graph.  For GraphOne-API engines that instantiate the nnz
 * kernels with their own functors (replaces the merge-path plan of
 * SpmvDispatcher<SpmvCudaCsrMergeBased>, archi/blas/spmv/cuda/cuda.cuh:75-92). */
typedef struct g1_nnz_plan {
    uint32_t n_rows, nnz, n_tiles, n_nonempty, n_empty, n_fix, n_fix_short;
    const uint32_t* tile_seg;
    const uint32_t* sbits;
    const uint32_t* rows;
    const uint32_t* row_ptr;
    const uint32_t* fix_tiles;
    const void* fix_info;
    void* carry;
    void* tail;
} g1_nnz_plan;
g1_status g1_spmv_nnz_plan(g1_graph* g, int transpose, g1_nnz_plan* out);
/* y = A (semiring) x over one orientation (replaces SpmvDispatcher::operator(),
 * archi/blas/spmv/cuda/cuda.cuh:94-99; y stays on the device stream, no
 * device synchronisation). x, y device pointers of n entries. */
g1_status g1_spmv(g1_graph* g, int transpose, g1_semiring sr, g1_schedule sched,
                  const void* x, void* y, void* stream);
/* Fixes the schedule G1_SCHED_AUTO resolves to for one orientation:
 * G1_SCHED_MERGE with a merge kernel variant, or G1_SCHED_VECTOR;
 * G1_SCHED_AUTO restores the default.  Merge variants (all on the
 * merge-path partition): warp tiles of 32 x k items loaded into registers
 * (0: k=11, 8 warps/block; 1: k=7, 8 warps; 2: k=7, 32 warps + x[0,16384)
 * cached in shared memory; 5: k=11, 32 warps + cache), block tiles of
 * 256 x 7 items staged by TMA bulk copies (3: two staging buffers, 4: one),
 * warp tiles staged by per-warp TMA bulk copies (6: k=15, 24 warps + cache;
 * 7: k=31, 16 warps; 8: k=15, 32 warps; 9: k=23, 16 warps + cache).
 * No GraphOne counterpart (GraphOne hard-wires the merge schedule,
 * engine/blas_gc.h:130-132). */
g1_status g1_graph_set_schedule(g1_graph* g, int transpose, g1_schedule sched, int variant);
/* y = A (semiring) x like g1_spmv, for callers that cannot allocate device
 * memory: a process whose device memory comes only from its own arena or
 * caching pool (a cudaMalloc outside it breaks the pool's accounting), a
 * plugin loaded into such a host, or a latency-critical loop that cannot
 * afford cudaMalloc's implicit device synchronisation.  No GraphOne
 * counterpart: it has no equivalent in the reference.  The CSR
 * (row_ptr n+1, col and val m entries, 4-byte values), x and y are the
 * caller's device buffers; nothing is allocated and no g1_graph is needed.
 * Scratch (merge-path partition and per-tile carries) lives in one
 * file-scope device array of 4 MiB per GPU, held until the process exits:
 * n + m may be at most 58,720,256 (G1_ERR_INVALID beyond).  Each call
 * looks up that array's device address on the current device.  The first
 * call on a device (in a CUDA context) loads the library module holding the
 * array: the driver then allocates its 4 MiB and the module's code there.
 * Make that first call at set-up time, before any stream capture, or set
 * CUDA_MODULE_LOADING=EAGER.  Every call shares the array and it keeps the
 * last call's contents (each call rewrites what it reads, nothing needs
 * zeroing); calls that overlap on the GPU race on it: serialise them (one
 * stream). */
g1_status g1_spmv_noalloc(const uint32_t* row_ptr, const uint32_t* col, const void* val,
                          uint32_t n, uint32_t m, g1_semiring sr, const void* x, void* y,
                          void* stream);
/* Times the merge schedule at each tile size and the CSR-vector schedule on
 * this graph and keeps the fastest for G1_SCHED_AUTO.  Results (may be
 * NULL): the best merge time and the vector time in ms, the winning merge
 * variant. */
g1_status g1_autotune(g1_graph* g, float* merge_ms, float* vector_ms, int* merge_variant,
                      void* stream);
/* Picks this graph's push/pull thresholds by timing SSSP from n_sources
 * (0: 16, at most 64) sources spread over the vertices with out-edges: the
 * single-source AUTO engine pushes while the frontier's out-degree sum is
 * below m / push_div (candidates 4 .. 128, default 16), and the batched
 * engines list the next iteration's rows while the changed vertices'
 * out-edges are below (m + n) / slot_div (candidates 2 .. 32, default 8).
 * The chosen divisors are returned (may be NULL) and kept for the graph.
 * Results never depend on them.  No GraphOne counterpart (GraphOne has no
 * direction switch: AdvanceGC always pushes, BlasGcEngine always pulls). */
g1_status g1_autotune_traversal(g1_graph* g, uint32_t n_sources, uint32_t* push_div,
                                uint32_t* slot_div, void* stream);
/* Sets those divisors by hand (0 keeps one).  push_div also sets where the
 * G1_ENGINE_BLAS loop (on graphs of 2^20 edges or more with the out-edge
 * CSR) computes a step from the frontier's out-edges alone instead of
 * pulling every row: while the frontier's out-degree sum is below
 * m / push_div; and where g1_ppr's sparse steps end (same graphs: while
 * the rows a step reaches have fewer than m / push_div in-edges).  BFS and
 * SSSP results and iteration counts never depend on them; PPR ranks only
 * in rounding (a listed row sums its in-edges in another order).  No
 * GraphOne counterpart. */
g1_status g1_set_traversal_thresholds(g1_graph* g, uint32_t push_div, uint32_t slot_div);

/* PageRank's column layout on this graph.  The pull SpMV gathers x[u] once
 * per out-edge of u and its tile kernel keeps a prefix of x in shared
 * memory, so it runs fastest when the vertices with the most out-edges come
 * first.  G1_GRAPH_RELABEL gets that by rebuilding both CSRs in degree order
 * (about 11 ms on a 65 M-edge graph).  On a graph kept in the caller's order,
 * g1_pagerank instead renames only the in-edge CSR's columns (vertices by
 * decreasing out-degree), into a copy of the column array (4 bytes per edge
 * more on the device, built on the first call, about 0.5 ms on 65 M edges)
 * and keeps x in that order.  Each row's nonzeros keep their order: the ranks
 * are the same bits either way.  g1_ppr uses the same copy (built by it
 * first, the order is by out-degree).  AUTO (the default): on graphs of 2^22
 * edges or more that are not relabelled, have a row of more than 64 in-edges
 * (skewed degrees) and are not on the CSR-vector schedule; OFF: never; ON:
 * always.  No GraphOne counterpart. */
typedef enum {
    G1_HOT_COLUMNS_AUTO = 0,
    G1_HOT_COLUMNS_OFF = 1,
    G1_HOT_COLUMNS_ON = 2
} g1_hot_columns;
g1_status g1_graph_set_hot_columns(g1_graph* g, g1_hot_columns mode);

/* ------------------------------------------------------------- algorithms */
/* PageRank for a fixed iteration count (Run<PRFunctor> over
 * AllActiveFrontier with BlasGcEngine<ALL_ACTIVE>, engine/blas_gc.h:353-434,
 * apps/pagerank_blas.cu:36-123).  rank_out: n floats, host or device. */
g1_status g1_pagerank(g1_graph* g, float alpha, int iters, g1_pr_mode mode, float* rank_out,
                      void* stream);
/* Single-source shortest paths, u32 weights, UINT32_MAX = unreachable
 * (Run<SSSPFunctor> with BlasGcEngine<SPARSE_BASED>, engine/blas_gc.h:171-247,
 * apps/sssp_blas.cu; or AdvanceGC, engine/advance_gc.h:162-283,
 * apps/sssp_adv.cu).  dist_out: n u32, host or device.  iters_out may be NULL. */
g1_status g1_sssp(g1_graph* g, uint32_t src, g1_engine engine, uint32_t* dist_out,
                  uint32_t* iters_out, void* stream);
/* BFS hop levels from src, UINT32_MAX = unreachable. */
g1_status g1_bfs(g1_graph* g, uint32_t src, g1_engine engine, uint32_t* level_out,
                 uint32_t* iters_out, void* stream);

/* One push step of the advance/filter engine (replaces AdvanceGC::Forward,
 * engine/advance_gc.h:162-283, with the relax functor of apps/sssp_adv.cu:
 * 48-72; unit != 0 relaxes with weight 1, i.e. BFS levels).  For each vertex
 * u of frontier[0, n_frontier) and out-edge (u, v, w): dist[v] =
 * min(dist[v], dist[u] + w); a vertex whose distance dropped joins
 * out_frontier once per step (visited[v] is set to iter).  frontier, dist
 * (n), visited (n) and out_frontier (room for n) are device arrays; pass a
 * new iter for each step (visited starting at 0, iter from 1).
 * *out_size (host) gets the new frontier's length; the call synchronises
 * `stream`.  Needs the out-edge CSR and a graph created without
 * G1_GRAPH_RELABEL (ids are the caller's). */
g1_status g1_advance_run(g1_graph* g, int unit, const uint32_t* frontier, uint32_t n_frontier,
                         uint32_t* dist, uint32_t* visited, uint32_t iter, uint32_t* out_frontier,
                         uint32_t* out_size, void* stream);

/* ----------------------------------------------------- batched queries */
/* k sources as one multi-source pass (no GraphOne counterpart: GraphOne
 * runs one source per Run, apps/sssp_blas.cu:87-136).  srcs: k vertex ids
 * (host or device); out: k*n u32 in source-major order (out[s*n + v]) --
 * the layout of k g1_bfs / g1_sssp calls, and bit-identical to them.  Up to
 * 256 sources iterate together; when one finishes, the next source takes its
 * slot while the others keep iterating.  Needs the in-edge CSR.
 * iters_out: iterations of the longest query (may be NULL). */
g1_status g1_bfs_batch(g1_graph* g, const uint32_t* srcs, uint32_t k, uint32_t* levels_out,
                       uint32_t* iters_out, void* stream);
g1_status g1_sssp_batch(g1_graph* g, const uint32_t* srcs, uint32_t k, uint32_t* dist_out,
                        uint32_t* iters_out, void* stream);

/* Personalized PageRank of src (no GraphOne app; the pagerank_blas
 * iteration, apps/pagerank_blas.cu:86-125, restarted at src): rank starts as
 * the indicator of src and `iters` times
 *     rank'[v] = sum_{u->v} rank[u] * alpha / outdeg(u)
 *                + [v == src] * ((1 - alpha) + alpha * sum_{outdeg(u)=0} rank[u]).
 * Transition weights are 1/out-degree (edge values are not used).  fp32.
 * Runs on the SpMV schedules (one pass over the in-edge CSR per iteration,
 * 4 bytes per edge), except while rank is still confined near src: on
 * graphs of 2^20 edges or more with the out-edge CSR (or symmetric), a step
 * whose reachable rows have fewer than m / push_div in-edges computes only
 * those rows (every step of a short query on a grid; the first few on
 * RMAT).  g1_ppr_batch runs the slot engine, whose per-slot
 * results are the same bits wherever a query sits in a batch.  Both agree
 * with an FP64 evaluation within 1e-6 relative L1; they are not bit-identical
 * to each other (different summation orders).  rank_out: n f32, host or
 * device.  Needs the in-edge CSR. */
g1_status g1_ppr(g1_graph* g, uint32_t src, float alpha, uint32_t iters, float* rank_out,
                 void* stream);
/* k personalized PageRanks, rank_out: k*n f32 source-major. */
g1_status g1_ppr_batch(g1_graph* g, const uint32_t* srcs, uint32_t k, float alpha, uint32_t iters,
                       float* rank_out, void* stream);

/* --------------------------------------------------------- serving loop */
/* A request loop (one host thread, one CUDA stream per graph and query
 * kind) over resident graphs.  Queries on the same graph and of the same
 * kind share a multi-source engine of up to max_batch slots: a query is
 * admitted into a free slot between two iterations of the engine and its
 * result is written as soon as its own traversal completes, while the rest
 * of the batch keeps running (continuous batching).  Batching pays only for
 * dozens of queries at once, so while an executor's slots are empty and
 * fewer than 32 queries wait (or the waiting ones would finish within
 * solo_queue_ms one by one), its queries take the server's solo lanes:
 * worker threads (solo_lanes) each running one query at a time, shortest
 * expected first across graphs and kinds with waiting time counted in
 * (lane_stretch), never two of one graph at once, on the
 * single-source engines (the results of g1_sssp / g1_bfs with
 * G1_ENGINE_AUTO and of g1_ppr).  SSSP and BFS on graphs of small uniform
 * degree -- grids -- always take a lane (the near-far engine).  Executors of different graphs / kinds run
 * concurrently on their own streams.  An engine's state is allocated when
 * its first batch arrives, sized by the free device memory (slots halve
 * until it fits, down to 32; otherwise queries wait for memory to be
 * released), and kept until another engine needs the memory (or, with
 * idle_release_ms set, released after that long without queries).  No
 * GraphOne counterpart. */
typedef struct g1_server g1_server;
typedef enum { G1_QUERY_BFS = 0, G1_QUERY_SSSP = 1, G1_QUERY_PPR = 2 } g1_query_kind;
typedef struct {
    uint32_t max_batch;       /* slots per engine, 1..256 (rounded up to 32s); 0 = 256 */
    uint64_t reserve_bytes;   /* device memory admission leaves free */
    uint64_t memory_limit;    /* cap on engine state bytes; 0 = none */
    float ppr_alpha;          /* PPR damping; 0 = 0.85 */
    uint32_t ppr_iters;       /* PPR iterations; 0 = 20 */
    uint32_t idle_release_ms; /* release idle engine state after this; 0 = keep it
                                 until another engine needs the memory */
    int32_t solo_queue_ms;    /* queries run one at a time on the single-source engines
                                 while fewer than 32 wait or the waiting ones would
                                 finish within this many ms that way (estimated),
                                 batched beyond; 0 = 20; negative = always batched
                                 (grid SSSP / BFS stay on the near-far engine) */
    uint32_t solo_lanes;      /* worker threads running such queries, one each, never two
                                 of one graph at a time; 0 = 1, at most 16 */
    float lane_stretch;       /* which waiting query a free lane takes: the lowest
                                 expected_ms - waited_ms / lane_stretch, expected_ms being
                                 the moving average of that graph and kind's lane queries
                                 (short ones first; a query expected T ms longer than the
                                 others waits at most about lane_stretch * T); 0 = 2;
                                 negative = oldest first */
} g1_server_config;
typedef struct {
    uint64_t submitted, completed, failed;
    double p50_ms, p99_ms, mean_ms, max_ms; /* latency: submit -> result written */
    double queries_per_s;                   /* completed / (last completion - first submit) */
    uint64_t steps;                         /* engine steps launched */
    uint32_t max_occupancy;                 /* most slots busy in one engine step */
    uint32_t engines;                       /* engines holding device state now */
    uint64_t device_bytes;                  /* their device bytes */
} g1_server_metrics;

/* cfg may be NULL (defaults). */
g1_status g1_server_create(int device, const g1_server_config* cfg, g1_server** out);
/* Registers a resident graph (not owned; it must outlive the server and must
 * not be destroyed while registered).  Needs the in-edge CSR. */
g1_status g1_server_add_graph(g1_server* srv, g1_graph* g, uint32_t* graph_id);
/* Queues one query; returns at once.  out: n u32 (BFS levels, SSSP
 * distances) or n f32 (PPR ranks) -- device memory, pinned host memory or
 * pageable host memory (slowest); it must stay valid until the query is
 * done. */
g1_status g1_server_submit(g1_server* srv, uint32_t graph_id, g1_query_kind kind, uint32_t src,
                           void* out, uint64_t* ticket);
/* done = 1 once the result is written; then returns the query's status and
 * forgets the ticket.  latency_ms may be NULL. */
g1_status g1_server_poll(g1_server* srv, uint64_t ticket, int* done, double* latency_ms);
/* Blocks until the query is done (G1_ERR_TIMEOUT after timeout_ms; 0 = no
 * limit), then behaves like g1_server_poll. */
g1_status g1_server_wait(g1_server* srv, uint64_t ticket, uint32_t timeout_ms, double* latency_ms);
/* Latency percentiles over the queries completed since creation or the
 * last reset (reset != 0 clears them after reading). */
g1_status g1_server_stats(g1_server* srv, int reset, g1_server_metrics* out);
/* Stops the loop: queued queries fail, running ones finish first. */
g1_status g1_server_destroy(g1_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* GRAPHONE_B200_H_ */
