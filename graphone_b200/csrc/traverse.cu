// Single-source SSSP and BFS on the two GraphOne engines.
//
// * BLAS engine (pull): GraphOne's BlasGcEngine<SPARSE_BASED>
//   (engine/blas_gc.h:171-247) per iteration fills x with default_info over
//   N, scatters construct_each of the frontier, runs the merge SpMV over all
//   rows, transforms y over N into flags and copy_ifs the next frontier, with
//   two host synchronisations.  Here x stays default_info between
//   iterations and only the frontier's entries are set and reset (O(|F|)),
//   apply + frontier compaction run in the SpMV epilogue (warp-aggregated
//   appends), and one 8-byte read-back per iteration tells the host the next
//   frontier size.  Per-iteration results are those of the reference.
// * Advance engine (push): GraphOne's AdvanceGC (engine/advance_gc.h:162-283)
//   sizes an invalid-padded output by a degree-sum reduction, launches the
//   advance kernel, synchronises, then filters duplicates in a second pass.
//   Here the advance relaxes with atomicMin, deduplicates at emission time
//   with the visited stamp of the sssp_adv filter (apps/sssp_adv.cu:62-71,
//   made atomic) and appends compactly: one kernel per iteration.
// * AUTO: push while the frontier's out-degree sum is below m/16, pull
//   otherwise (direction-optimising); on graphs of small uniform degree
//   (grids) the near-far engine (nearfar.cu) instead.  Final distances are
//   the unique shortest-path distances whichever engine runs, so all agree
//   bit-exactly with the oracle.
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "g1/semiring.cuh"
#include "g1/spmv.cuh"
#include "internal.h"
#include "spmv_launch.cuh"

namespace g1 {

// apply_each of the sssp_blas functor under the engine's guard
// (blas_gc.h:230-237): res != default_result && res < dist[v] -> update,
// activate.  The degree sum of activated vertices feeds the push/pull choice.
struct SparseApplyEpilogue {
    static constexpr bool kRowsIndependent = true;
    uint32_t* dist;
    uint32_t* out;
    uint32_t* out_count;
    unsigned long long* deg_sum;
    const uint32_t* out_rp;  // out-edge offsets (for the degree sum)
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t v, const uint32_t& res) {
        if (res != kU32Max && res < dist[v]) {
            dist[v] = res;
            append_sum(out, out_count, deg_sum, v, out_rp[v + 1] - out_rp[v]);
        }
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

__global__ void tr_init_kernel(uint32_t n, uint32_t src, uint32_t* dist, uint32_t* x,
                               uint32_t* visited, uint32_t* frontier) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        dist[v] = v == src ? 0u : kU32Max;
        x[v] = kU32Max;
        visited[v] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) frontier[0] = src;
}

// x[f] = dist[f] (construct_each of sssp_blas) or MAX (reset) over F.
__global__ void tr_scatter_kernel(const uint32_t* F, uint32_t nF, const uint32_t* dist,
                                  uint32_t* x, int reset) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nF; i += stride) {
        const uint32_t f = F[i];
        x[f] = reset ? kU32Max : dist[f];
    }
}

// Push relaxation of one edge; emits v once per iteration.
template <bool UNIT>
__device__ __forceinline__ void relax(uint32_t du, uint32_t v, uint32_t w, uint32_t* dist,
                                      uint32_t* visited, uint32_t iter, uint32_t* out,
                                      uint32_t* out_count, const uint32_t* rp,
                                      unsigned long long* deg_sum) {
    const uint32_t cand = UNIT ? du + 1u : du + w;
    if (cand < dist[v]) {  // cheap pre-check; atomicMin decides
        const uint32_t old = atomicMin(&dist[v], cand);
        if (cand < old && atomicExch(&visited[v], iter) != iter)
            append_sum(out, out_count, deg_sum, v, rp[v + 1] - rp[v]);
    }
}

// A frontier entry the advance may expand: an id below n (otherwise the
// device error word records kDevInvalid and the entry is skipped; frontiers
// the engines build are always in range, g1_advance_run's come from the
// caller) whose distance is finite (an unreached vertex has nothing to push:
// MAX + w would wrap).
__device__ __forceinline__ bool frontier_vertex_ok(uint32_t u, uint32_t n, uint32_t* err) {
    if (u < n) return true;
    set_error(err, kDevInvalid);
    return false;
}

// Advance over the frontier: TPV lanes per vertex for short adjacency lists
// (TPV the power of two at or above the frontier's mean degree, so a small
// frontier of low-degree vertices still gets about a thread per edge), the
// whole warp for lists of 32 or more edges (coalesced col/val reads).
template <bool UNIT, int TPV>
__global__ void __launch_bounds__(256)
tr_advance_kernel(const uint32_t* F, uint32_t nF, uint32_t n, const uint32_t* rp, const uint32_t* col,
                  const uint32_t* val, uint32_t* dist, uint32_t* visited, uint32_t iter,
                  uint32_t* out, uint32_t* out_count, unsigned long long* deg_sum, uint32_t* err) {
    constexpr uint32_t VPW = 32 / TPV;  // vertices per warp and round
    const uint32_t lane = lane_id();
    const uint32_t sub = lane % TPV, grp = lane / TPV;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t rounds = (uint32_t)ceil_div(nF, (uint64_t)warps * VPW);
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t i = (r * warps + wid) * VPW + grp;
        uint32_t u = 0, b = 0, e = 0, du = 0;
        if (i < nF) {
            u = F[i];
            if (frontier_vertex_ok(u, n, err)) {
                du = dist[u];
                if (du != kU32Max) {
                    b = rp[u];
                    e = rp[u + 1];
                }
            }
        }
        // long lists: cooperative, one list at a time
        unsigned big = __ballot_sync(0xffffffffu, sub == 0 && e - b >= 32);
        while (big) {
            const int src_lane = __ffs(big) - 1;
            big &= big - 1;
            const uint32_t bb = __shfl_sync(0xffffffffu, b, src_lane);
            const uint32_t ee = __shfl_sync(0xffffffffu, e, src_lane);
            const uint32_t dd = __shfl_sync(0xffffffffu, du, src_lane);
            for (uint32_t k = bb + lane; k < ee; k += 32)
                relax<UNIT>(dd, col[k], UNIT ? 1u : val[k], dist, visited, iter, out, out_count,
                            rp, deg_sum);
        }
        if (e - b < 32) {
            for (uint32_t k = b + sub; k < e; k += TPV)
                relax<UNIT>(du, col[k], UNIT ? 1u : val[k], dist, visited, iter, out, out_count, rp,
                            deg_sum);
        }
    }
}

// Out-degrees of the frontier (deg[nF] = 0) for the edge-balanced advance;
// 0 for an entry the advance skips (out of range, or unreached).
__global__ void tr_frontier_degrees_kernel(const uint32_t* F, uint32_t nF, uint32_t n,
                                           const uint32_t* rp, const uint32_t* dist, uint32_t* deg,
                                           uint32_t* err) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= nF; i += stride) {
        uint32_t d = 0;
        if (i < nF) {
            const uint32_t u = F[i];
            if (frontier_vertex_ok(u, n, err) && dist[u] != kU32Max) d = rp[u + 1] - rp[u];
        }
        deg[i] = d;
    }
}

// Edge-balanced advance: the frontier's edges are numbered by the
// exclusive prefix of its degrees; warps take 32 consecutive edge numbers and
// each lane finds its frontier vertex by binary search, so a hub's edges are
// spread over as many warps as the rest of the frontier's.
template <bool UNIT>
__global__ void __launch_bounds__(256)
tr_advance_lb_kernel(const uint32_t* F, uint32_t nF, const uint32_t* prefix, const uint32_t* rp,
                     const uint32_t* col, const uint32_t* val, uint32_t* dist, uint32_t* visited,
                     uint32_t iter, uint32_t* out, uint32_t* out_count,
                     unsigned long long* deg_sum) {
    const uint32_t total = prefix[nF];
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; (uint64_t)c * 32 < total;
         c += warps) {
        const uint32_t r = c * 32 + lane;
        if (r >= total) continue;
        uint32_t lo = 0, hi = nF;  // last i with prefix[i] <= r
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= r) lo = mid; else hi = mid - 1;
        }
        // entries the degree pass skipped have degree 0, so edge number r
        // never lands on one: F[lo] is in range with a finite distance
        const uint32_t u = F[lo];
        const uint32_t k = rp[u] + (r - prefix[lo]);
        relax<UNIT>(dist[u], col[k], UNIT ? 1u : val[k], dist, visited, iter, out, out_count, rp,
                    deg_sum);
    }
}

// ------------------------------------------------ device-driven advance
// The push engine for graphs whose out-degrees are all at most 32 (grids,
// meshes, road-like graphs: thousands of small-frontier iterations).  One
// kernel per iteration with everything the host loop decided between
// iterations moved onto the device -- the frontier size and its degree sum
// are read from device counters, the lanes per vertex follow from them --
// so iterations are captured as CUDA graphs of 2^i step pairs and the host
// reads the frontier size back only between graphs.  Per iteration the
// result is that of GraphOne's AdvanceGC step (engine/advance_gc.h:162-283
// with apps/sssp_adv.cu:49-71): relax every out-edge of the frontier with
// atomicMin, emit each improved vertex once (the visited stamp of the
// sssp_adv filter).  Appends go to a per-block shared-memory queue flushed
// with one global atomic per block (a single global counter bumped by
// every warp serialises at one L2 slice when frontiers hold hundreds of
// thousands of vertices).

// Frontier size and out-degree sum of one frontier buffer.
struct AgCounter {
    uint32_t n;
    uint32_t pad;
    unsigned long long deg;
};

// Store layout (4-byte words): dist[n], visited[n], F0[n], F1[n], then the
// control words: [0] completed iterations, [1] block ticket, and the two
// counters at words 4 and 8.
struct AgState {
    uint32_t *dist, *visited, *F[2], *ctl;
    AgCounter* c[2];
};

inline size_t ag_words(uint32_t n) { return 4 * (size_t)n + 16; }

inline AgState ag_layout(uint32_t* store, uint32_t n) {
    AgState a;
    a.dist = store;
    a.visited = store + n;
    a.F[0] = store + 2 * (size_t)n;
    a.F[1] = store + 3 * (size_t)n;
    a.ctl = store + 4 * (size_t)n;
    a.c[0] = reinterpret_cast<AgCounter*>(a.ctl + 4);
    a.c[1] = reinterpret_cast<AgCounter*>(a.ctl + 8);
    return a;
}

constexpr int kAgBlock = 256;
constexpr int kAgQueue = 2048;  // shared-memory queue entries per block

// Shared-memory side of a block's appends: the queue, its fill count, the
// block's base in the global frontier and the warps' degree sums.
struct AgBlockQueue {
    uint32_t q[kAgQueue];
    uint32_t cnt, base;
    unsigned long long deg[kAgBlock / 32];
};

// Push relaxation of edge (u -> v) of weight w from distance du: atomicMin;
// an improved vertex is emitted once per iteration (the visited stamp) into
// the block's queue (straight to F_out when the queue is full).
template <bool UNIT>
__device__ __forceinline__ void ag_relax(uint32_t du, uint32_t v, uint32_t w, uint32_t* dist,
                                         uint32_t* visited, uint32_t it, const uint32_t* rp,
                                         unsigned long long& my_deg, AgBlockQueue& bq, uint32_t* F_out,
                                         AgCounter* c_out) {
    const uint32_t cand = UNIT ? du + 1u : du + w;
    if (cand < dist[v]) {  // cheap pre-check; atomicMin decides
        const uint32_t old = atomicMin(&dist[v], cand);
        if (cand < old && atomicExch(&visited[v], it) != it) {
            my_deg += rp[v + 1] - rp[v];
            const uint32_t p = atomicAdd(&bq.cnt, 1u);
            if (p < (uint32_t)kAgQueue) bq.q[p] = v;
            else F_out[atomicAdd(&c_out->n, 1u)] = v;  // queue full: straight out
        }
    }
}

// Publishes a block's appends: one global atomic for the count, one for the
// degree sum.  All threads of the block; bq.cnt was zeroed before the block's
// relaxations.
__device__ __forceinline__ void ag_flush(AgBlockQueue& bq, unsigned long long my_deg, uint32_t* F_out,
                                         AgCounter* c_out) {
    my_deg = warp_sum(my_deg);
    if (lane_id() == 0) bq.deg[threadIdx.x >> 5] = my_deg;
    __syncthreads();
    const uint32_t cnt = min(bq.cnt, (uint32_t)kAgQueue);
    if (threadIdx.x == 0) {
        unsigned long long d = 0ull;
        for (int w = 0; w < kAgBlock / 32; ++w) d += bq.deg[w];
        if (d) atomicAdd(&c_out->deg, d);
        bq.base = cnt ? atomicAdd(&c_out->n, cnt) : 0u;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < cnt; q += kAgBlock) F_out[bq.base + q] = bq.q[q];
}

// Lanes per frontier vertex: the power of two at or above the mean degree.
__device__ __forceinline__ uint32_t ag_tpv(uint32_t nF, unsigned long long degF) {
    const unsigned long long mean = (degF + nF - 1) / nF;
    uint32_t tpv = 1;
    while (tpv < 32 && tpv < mean) tpv <<= 1;
    return tpv;
}

__global__ void ag_init_kernel(uint32_t n, uint32_t src, const uint32_t* rp, AgState a) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        a.dist[v] = v == src ? 0u : kU32Max;
        a.visited[v] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.F[0][0] = src;
        a.ctl[0] = 0u;
        a.ctl[1] = 0u;
        a.c[0]->n = 1u;
        a.c[0]->deg = rp[src + 1] - rp[src];
        a.c[1]->n = 0u;
        a.c[1]->deg = 0ull;
    }
}

// Last block of a step (every block calls this once, thread 0): zeroes c_in
// (it is the next step's c_out) and `also` when given, and advances the
// iteration count when the step had a frontier.
__device__ __forceinline__ void ag_last_block_rotate(AgCounter* c_in, uint32_t* ctl, uint32_t nF,
                                                     AgCounter* also = nullptr) {
    __threadfence();
    if (atomicAdd(&ctl[1], 1u) == gridDim.x - 1) {
        // every block has read c_in and published its appends
        if (nF) ctl[0] += 1u;
        c_in->n = 0u;
        c_in->deg = 0ull;
        if (also) {
            also->n = 0u;
            also->pad = 0u;
            also->deg = 0ull;
        }
        ctl[1] = 0u;
        __threadfence();
    }
}

// One advance step: frontier F_in (size and degree sum in c_in) -> F_out
// (counted in c_out, zero on entry); out-degrees at most 32.  The last block
// to finish zeroes c_in and bumps the iteration count.  An empty frontier
// makes the step a no-op, so graphs may run past convergence.
template <bool UNIT>
__global__ void __launch_bounds__(kAgBlock)
ag_step_kernel(const uint32_t* F_in, uint32_t* F_out, AgCounter* c_in, AgCounter* c_out,
               uint32_t* ctl, uint32_t n, const uint32_t* rp, const uint32_t* col, const uint32_t* val,
               uint32_t* dist, uint32_t* visited, uint32_t* err) {
    __shared__ AgBlockQueue bq;
    const uint32_t nF = c_in->n;
    if (nF == 0) return;  // the same for every block
    const uint32_t it = ctl[0] + 1u;  // visited stamp of this iteration
    const uint32_t tpv = ag_tpv(nF, c_in->deg);
    if (threadIdx.x == 0) bq.cnt = 0u;
    __syncthreads();
    const uint32_t lane = lane_id();
    const uint32_t sub = lane & (tpv - 1u), grp = lane / tpv, vpw = 32u / tpv;
    const uint64_t warps = (uint64_t)gridDim.x * (kAgBlock / 32);
    const uint64_t wid = ((uint64_t)blockIdx.x * kAgBlock + threadIdx.x) >> 5;
    unsigned long long my_deg = 0ull;
    for (uint64_t first = wid * vpw; first < nF; first += warps * vpw) {
        const uint64_t i = first + grp;
        uint32_t b = 0, e = 0, du = 0;
        if (i < nF) {
            const uint32_t u = F_in[i];
            if (frontier_vertex_ok(u, n, err)) {
                du = dist[u];
                if (du != kU32Max) {
                    b = rp[u];
                    e = rp[u + 1];
                }
            }
        }
        for (uint32_t k = b + sub; k < e; k += tpv)
            ag_relax<UNIT>(du, col[k], UNIT ? 1u : val[k], dist, visited, it, rp, my_deg, bq, F_out, c_out);
    }
    ag_flush(bq, my_deg, F_out, c_out);
    if (threadIdx.x == 0) ag_last_block_rotate(c_in, ctl, nF);
}

template <bool UNIT>
static void ag_enqueue_pairs(const g1_graph* g, const AgState& a, uint32_t pairs, uint32_t grid,
                             cudaStream_t s) {
    const Orientation& o = g->o[0];
    const auto* val = static_cast<const uint32_t*>(o.val);
    for (uint32_t p = 0; p < pairs; ++p)
        for (int h = 0; h < 2; ++h)
            ag_step_kernel<UNIT><<<grid, kAgBlock, 0, s>>>(a.F[h], a.F[h ^ 1], a.c[h], a.c[h ^ 1], a.ctl, g->n,
                                                           o.rp, o.col, val, a.dist, a.visited, g->err_word);
}

inline bool advance_graph_suits(const g1_graph* g) {
    return g->o[0].present && g->o[0].max_deg <= 32 && g->n > 0;
}

template <bool UNIT>
static g1_status advance_graph_traverse(g1_graph* g, uint32_t src, uint32_t* out, uint32_t* iters_out,
                                        cudaStream_t s) {
    const uint32_t n = g->n;
    const int mode = UNIT ? 1 : 0;
    uint32_t* store = nullptr;
    G1_TRY(g->ws.get("ag_store", ag_words(n), &store));
    const AgState a = ag_layout(store, n);
    G1_TRY(g->ws.pinned.ensure(64));
    uint32_t* host = g->ws.pinned.as<uint32_t>();
    if (!g->adv_graphs) g->adv_graphs.reset(new AdvGraphs());
    AdvGraphs& ag = *g->adv_graphs;
    if (ag.key[mode] != store) ag.reset(mode);  // captured on another store
    if (!ag.capture) G1_CUDA(cudaStreamCreateWithFlags(&ag.capture, cudaStreamNonBlocking));
    static int occ = [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, ag_step_kernel<UNIT>, kAgBlock, 0) != cudaSuccess) {
            cudaGetLastError();
            b = 1;
        }
        return std::max(1, b);
    }();
    const uint32_t grid = (uint32_t)g->sm_count * (uint32_t)occ;
    const uint32_t gi = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, 256), grid));
    ag_init_kernel<<<gi, 256, 0, s>>>(n, src, g->o[0].rp, a);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    // graphs of 2^i pairs, i growing to kSizes - 1: few read-backs on long
    // traversals, little overshoot on short ones
    int i = 2;
    for (;;) {
        cudaGraphExec_t& gx = ag.exec[mode][i];
        if (!gx) {
            cudaGraph_t graph = nullptr;
            CaptureScope cs;
            G1_CUDA(cudaStreamBeginCapture(ag.capture, cudaStreamCaptureModeThreadLocal));
            ag_enqueue_pairs<UNIT>(g, a, 1u << i, grid, ag.capture);
            const cudaError_t e = cudaStreamEndCapture(ag.capture, &graph);
            if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture(advance steps)");
            const cudaError_t ei = cudaGraphInstantiate(&gx, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) {
                gx = nullptr;
                return fail_cuda(ei, "cudaGraphInstantiate(advance steps)");
            }
            ag.key[mode] = store;
        }
        G1_CUDA(cudaGraphLaunch(gx, s));
        count_launches(2ull << i);
        G1_CUDA(cudaMemcpyAsync(host, a.ctl, 16, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaMemcpyAsync(host + 4, a.c[0], 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        if (host[4] == 0) break;  // frontier empty after the last pair
        // Bellman-Ford settles within n rounds; more means corrupted state.
        if (host[0] > n + 1) return fail(G1_ERR_TIMEOUT, "traversal did not converge within n rounds");
        if (host[4] > n) return fail(G1_ERR_OVERFLOW, "frontier larger than the vertex count");
        if (i < AdvGraphs::kSizes - 1) ++i;
    }
    if (iters_out) *iters_out = host[0];
    G1_TRY(copy_out_vertices(g, out, a.dist, s));
    return check_device_error(g, s);
}

// ------------------------------------------------ device-driven BLAS engine
// GraphOne's sparse-frontier BLAS engine loop (engine/blas_gc.h:199-245,
// apps/sssp_blas.cu:48-84) with every per-iteration decision on the device,
// so that iterations are captured as CUDA graphs like the advance engine's:
//   1. x[f] = dist[f] over the frontier (construct_each), frontier size read
//      from its device counter;
//   2. the min-plus SpMV over all rows with apply_each fused in its epilogue
//      (res != MAX && res < dist[v] -> update, append v to the next
//      frontier);
//   3. x[f] = MAX over the frontier again; the last block zeroes the
//      frontier's counter and advances the iteration count.
// A step whose frontier is empty is a no-op in all its kernels (the SpMV's
// epilogue reports itself inactive), so graphs may run past convergence.
// Per iteration the results are those of the reference loop, iteration
// count included.

// Store: the advance engine's (ag_layout), then x[n], the sparse step's
// listed rows cand[n], its counter (8 words: rows in n, heavy frontier
// vertices in pad), row values res[n] and heavy frontier vertices heavy[n].
inline size_t bg_words(uint32_t n) { return ag_words(n) + 4 * (size_t)n + 8; }

struct BgSparse {
    uint32_t* cand;
    AgCounter* c_cand;
    uint32_t* res;
    uint32_t* heavy;
};

inline BgSparse bg_sparse_layout(uint32_t* store, uint32_t n) {
    BgSparse b;
    uint32_t* p = store + ag_words(n) + n;  // after x
    b.cand = p;
    b.c_cand = reinterpret_cast<AgCounter*>(p + n);  // 8-byte aligned: the store is, and 6n + 16 words precede
    b.res = p + n + 8;
    b.heavy = p + 2 * (size_t)n + 8;
    return b;
}

// Frontier vertices with more out-edges than this are left to the whole grid
// (bg_spmspv_heavy_kernel) instead of one warp.
constexpr uint32_t kSparseHeavy = 2048;

__global__ void bg_x_init_kernel(uint32_t* x, uint32_t n, BgSparse sp) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        x[v] = kU32Max;
        sp.res[v] = kU32Max;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sp.c_cand->n = 0u;
        sp.c_cand->pad = 0u;
        sp.c_cand->deg = 0ull;
    }
}

// Sparse step.  A row's min-plus value is the reduce of combine(w, x[u])
// over its in-edges, and x is MAX (the identity of every combine) except on
// the frontier, so only the frontier's out-edges contribute.  While they sum
// below `limit` the step computes exactly those contributions -- each out-edge
// (u -> v, w) of each frontier vertex u folds combine(w, x[u]) into res[v]
// with atomicMin (min is order-free: the same value as the full pull's
// row fold) -- and applies the rows it reached, as the full pull's epilogue
// does.  Results and iteration counts are the full pull's; the work is the
// frontier's out-edges instead of all m.
constexpr uint32_t kSparseStepMinEdges = 1u << 20;
constexpr uint32_t kAutoDeviceEdges = 1u << 24;

__device__ __forceinline__ bool bg_sparse_step(const AgCounter* c_in, unsigned long long limit) {
    return c_in->n != 0u && c_in->deg < limit;
}

// Folds out-edge k of a frontier vertex (value xu) into res[v]; a row is
// listed by the edge that first lowers its value from MAX.
template <class SR>
__device__ __forceinline__ void bg_spmspv_edge(uint32_t k, uint32_t xu, const uint32_t* out_col,
                                               const uint32_t* out_val, const BgSparse& sp, AgBlockQueue& bq) {
    const uint32_t v = out_col[k];
    const uint32_t c = SR::combine(reads_weight<SR>::value ? out_val[k] : 0u, xu);
    if (c == kU32Max || c >= sp.res[v]) return;  // cheap pre-check; atomicMin decides
    if (atomicMin(&sp.res[v], c) != kU32Max) return;  // listed already
    const uint32_t p = atomicAdd(&bq.cnt, 1u);
    if (p < (uint32_t)kAgQueue) bq.q[p] = v;
    else sp.cand[atomicAdd(&sp.c_cand->n, 1u)] = v;  // queue full: straight out
}

// Publishes a block's listed rows (all threads of the block).
__device__ __forceinline__ void bg_list_flush(AgBlockQueue& bq, const BgSparse& sp) {
    __syncthreads();
    const uint32_t cnt = min(bq.cnt, (uint32_t)kAgQueue);
    if (threadIdx.x == 0) bq.base = cnt ? atomicAdd(&sp.c_cand->n, cnt) : 0u;
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < cnt; q += kAgBlock) sp.cand[bq.base + q] = bq.q[q];
}

// Sparse step, part 1: one warp per frontier vertex, lanes over its out-edges;
// vertices of more than kSparseHeavy out-edges are listed for part 2.
template <class SR>
__global__ void __launch_bounds__(kAgBlock)
bg_spmspv_kernel(const uint32_t* F_in, const AgCounter* c_in, unsigned long long limit, uint32_t n,
                 const uint32_t* out_rp, const uint32_t* out_col, const uint32_t* out_val, const uint32_t* x,
                 BgSparse sp, uint32_t* err) {
    __shared__ AgBlockQueue bq;
    if (!bg_sparse_step(c_in, limit)) return;  // the same for every block
    const uint32_t nF = c_in->n;
    if (threadIdx.x == 0) bq.cnt = 0u;
    __syncthreads();
    const uint32_t lane = lane_id();
    const uint64_t warps = (uint64_t)gridDim.x * (kAgBlock / 32);
    for (uint64_t i = ((uint64_t)blockIdx.x * kAgBlock + threadIdx.x) >> 5; i < nF; i += warps) {
        const uint32_t u = F_in[i];
        if (!frontier_vertex_ok(u, n, err)) continue;
        const uint32_t b = out_rp[u], e = out_rp[u + 1];
        if (e - b > kSparseHeavy) {
            if (lane == 0) sp.heavy[atomicAdd(&sp.c_cand->pad, 1u)] = u;
            continue;
        }
        const uint32_t xu = x[u];
        for (uint32_t k = b + lane; k < e; k += 32) bg_spmspv_edge<SR>(k, xu, out_col, out_val, sp, bq);
    }
    bg_list_flush(bq, sp);
}

// Sparse step, part 2: the heavy frontier vertices' out-edges, spread over
// the whole grid one vertex after another.
template <class SR>
__global__ void __launch_bounds__(kAgBlock)
bg_spmspv_heavy_kernel(const AgCounter* c_in, unsigned long long limit, const uint32_t* out_rp,
                       const uint32_t* out_col, const uint32_t* out_val, const uint32_t* x, BgSparse sp) {
    __shared__ AgBlockQueue bq;
    if (!bg_sparse_step(c_in, limit)) return;
    const uint32_t nh = sp.c_cand->pad;
    if (nh == 0) return;  // the same for every block
    if (threadIdx.x == 0) bq.cnt = 0u;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * kAgBlock;
    for (uint32_t h = 0; h < nh; ++h) {
        const uint32_t u = sp.heavy[h];
        const uint32_t xu = x[u];
        const uint32_t b = out_rp[u], e = out_rp[u + 1];
        for (uint64_t k = b + (uint64_t)blockIdx.x * kAgBlock + threadIdx.x; k < e; k += stride)
            bg_spmspv_edge<SR>((uint32_t)k, xu, out_col, out_val, sp, bq);
    }
    bg_list_flush(bq, sp);
}

// Sparse step, part 3: one thread per listed row applies its value as the
// full pull's epilogue does (BgApplyEpilogue) and resets it to MAX.
__global__ void __launch_bounds__(kAgBlock)
bg_spmspv_apply_kernel(const AgCounter* c_in, unsigned long long limit, BgSparse sp, uint32_t* dist,
                       uint32_t* F_out, AgCounter* c_out, const uint32_t* out_rp) {
    __shared__ AgBlockQueue bq;
    if (!bg_sparse_step(c_in, limit)) return;
    const uint32_t nc = sp.c_cand->n;
    if (threadIdx.x == 0) bq.cnt = 0u;
    __syncthreads();
    unsigned long long my_deg = 0ull;
    const uint64_t stride = (uint64_t)gridDim.x * kAgBlock;
    for (uint64_t i = (uint64_t)blockIdx.x * kAgBlock + threadIdx.x; i < nc; i += stride) {
        const uint32_t v = sp.cand[i];
        const uint32_t r = sp.res[v];
        sp.res[v] = kU32Max;
        if (r < dist[v]) {
            dist[v] = r;
            my_deg += out_rp[v + 1] - out_rp[v];
            const uint32_t p = atomicAdd(&bq.cnt, 1u);
            if (p < (uint32_t)kAgQueue) bq.q[p] = v;
            else F_out[atomicAdd(&c_out->n, 1u)] = v;
        }
    }
    ag_flush(bq, my_deg, F_out, c_out);
}

// x[f] = dist[f] (reset: MAX) over the frontier of c_in; with reset, the
// last block also rotates the counters (ag_last_block_rotate) and zeroes
// the sparse step's row count.
__global__ void __launch_bounds__(kAgBlock)
bg_frontier_x_kernel(const uint32_t* F_in, AgCounter* c_in, uint32_t* ctl, const uint32_t* dist,
                     uint32_t* x, int reset, AgCounter* c_cand) {
    const uint32_t nF = c_in->n;
    if (nF == 0) return;
    const uint64_t stride = (uint64_t)gridDim.x * kAgBlock;
    for (uint64_t i = (uint64_t)blockIdx.x * kAgBlock + threadIdx.x; i < nF; i += stride) {
        const uint32_t f = F_in[i];
        x[f] = reset ? kU32Max : dist[f];
    }
    if (reset && threadIdx.x == 0) ag_last_block_rotate(c_in, ctl, nF, c_cand);
}

// apply_each of the sssp_blas functor under the engine's guard, for the
// device-driven loop: inactive (the SpMV kernels return at once) when the
// step's frontier is empty.
struct BgApplyEpilogue {
    static constexpr bool kRowsIndependent = true;
    uint32_t* dist;
    uint32_t* out;
    AgCounter* c_out;
    const AgCounter* c_in;
    const uint32_t* out_rp;  // out-edge offsets (for the degree sum)
    unsigned long long sparse_limit;  // the sparse step runs instead below it
    __device__ __forceinline__ bool active() const {
        return c_in->n != 0u && !bg_sparse_step(c_in, sparse_limit);
    }
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t v, const uint32_t& res) {
        if (res != kU32Max && res < dist[v]) {
            dist[v] = res;
            append_sum(out, &c_out->n, &c_out->deg, v, out_rp[v + 1] - out_rp[v]);
        }
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

// Builds the SpMV's plan and its kernels' launch facts outside of any capture
// (they may allocate and query the device).
template <class SR, class Epi>
static g1_status bg_prepare_spmv(g1_graph* g, int t) {
    if (resolve_schedule(g, t, G1_SCHED_AUTO) == G1_SCHED_VECTOR) {
        (void)vector_grid<SR, Epi>(g);
        return G1_OK;
    }
    uint32_t mg = 0, fg = 0;
    return merge_grids<SR, Epi>(g, t, &mg, &fg);
}

template <bool UNIT>
static g1_status bg_enqueue_pairs(g1_graph* g, const AgState& a, uint32_t* x, const BgSparse& sp,
                                  unsigned long long limit, const uint32_t* out_rp, uint32_t pairs,
                                  uint32_t grid, cudaStream_t s) {
    using SR = typename std::conditional<UNIT, BfsU32, MinPlusU32>::type;
    const int pull_t = 1;
    for (uint32_t p = 0; p < pairs; ++p)
        for (int h = 0; h < 2; ++h) {
            bg_frontier_x_kernel<<<grid, kAgBlock, 0, s>>>(a.F[h], a.c[h], a.ctl, a.dist, x, 0, sp.c_cand);
            if (limit) {
                const Orientation& o = g->o[0];
                bg_spmspv_kernel<SR><<<grid, kAgBlock, 0, s>>>(a.F[h], a.c[h], limit, g->n, o.rp, o.col,
                                                               static_cast<const uint32_t*>(o.val), x, sp,
                                                               g->err_word);
                bg_spmspv_heavy_kernel<SR><<<grid, kAgBlock, 0, s>>>(a.c[h], limit, o.rp, o.col,
                                                                     static_cast<const uint32_t*>(o.val), x, sp);
                bg_spmspv_apply_kernel<<<grid, kAgBlock, 0, s>>>(a.c[h], limit, sp, a.dist, a.F[h ^ 1], a.c[h ^ 1],
                                                                 out_rp);
                count_launches(3);
            }
            BgApplyEpilogue e{a.dist, a.F[h ^ 1], a.c[h ^ 1], a.c[h], out_rp, limit};
            G1_TRY((run_spmv<SR>(g, pull_t, G1_SCHED_AUTO, x, e, s)));
            bg_frontier_x_kernel<<<grid, kAgBlock, 0, s>>>(a.F[h], a.c[h], a.ctl, a.dist, x, 1, sp.c_cand);
            count_launches(2);
        }
    return G1_OK;
}

template <bool UNIT>
static g1_status blas_graph_traverse(g1_graph* g, uint32_t src, uint32_t* out, uint32_t* iters_out,
                                     cudaStream_t s) {
    const uint32_t n = g->n;
    const int mode = 2 + (UNIT ? 1 : 0);
    const int pull_t = 1;
    const uint32_t* out_rp = g->o[0].present ? g->o[0].rp : g->o[pull_t].rp;
    if (UNIT)
        G1_TRY((bg_prepare_spmv<BfsU32, BgApplyEpilogue>(g, pull_t)));
    else
        G1_TRY((bg_prepare_spmv<MinPlusU32, BgApplyEpilogue>(g, pull_t)));
    uint32_t* store = nullptr;
    G1_TRY(g->ws.get("bg_store", bg_words(n), &store));
    const AgState a = ag_layout(store, n);
    uint32_t* x = store + ag_words(n);
    const BgSparse sp = bg_sparse_layout(store, n);
    // sparse steps while the frontier's out-edges sum below m / push_div (the
    // AUTO engine's push/pull switch); they need the out-edge CSR, and below
    // kSparseStepMinEdges a full pull costs a few microseconds, no more than
    // the sparse step's own two launches
    const unsigned long long limit =
        g->o[0].present && g->m >= kSparseStepMinEdges
            ? (unsigned long long)g->m / std::max<uint32_t>(1, g->push_div)
            : 0ull;
    G1_TRY(g->ws.pinned.ensure(64));
    uint32_t* host = g->ws.pinned.as<uint32_t>();
    if (!g->adv_graphs) g->adv_graphs.reset(new AdvGraphs());
    AdvGraphs& ag = *g->adv_graphs;
    // captured on another store, or with another sparse-pull limit
    if (ag.key[mode] != store || ag.param[mode] != limit) ag.reset(mode);
    if (!ag.capture) G1_CUDA(cudaStreamCreateWithFlags(&ag.capture, cudaStreamNonBlocking));
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, kAgBlock), (uint64_t)g->sm_count * 4));
    const uint32_t gi = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, 256), grid));
    ag_init_kernel<<<gi, 256, 0, s>>>(n, src, out_rp, a);
    bg_x_init_kernel<<<gi, 256, 0, s>>>(x, n, sp);
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    // kernels per pair of steps (counted per graph launch): x set and
    // reset, the SpMV's one or two, the sparse step's three
    const uint64_t per_pair =
        2ull * (2 + (resolve_schedule(g, pull_t, G1_SCHED_AUTO) == G1_SCHED_VECTOR ? 1 : 2) + (limit ? 3 : 0));
    int i = 1;
    for (;;) {
        cudaGraphExec_t& gx = ag.exec[mode][i];
        if (!gx) {
            cudaGraph_t graph = nullptr;
            CaptureScope cs;
            G1_CUDA(cudaStreamBeginCapture(ag.capture, cudaStreamCaptureModeThreadLocal));
            const g1_status st = bg_enqueue_pairs<UNIT>(g, a, x, sp, limit, out_rp, 1u << i, grid, ag.capture);
            const cudaError_t e = cudaStreamEndCapture(ag.capture, &graph);
            if (st != G1_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture(BLAS steps)");
            const cudaError_t ei = cudaGraphInstantiate(&gx, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) {
                gx = nullptr;
                return fail_cuda(ei, "cudaGraphInstantiate(BLAS steps)");
            }
            ag.key[mode] = store;
            ag.param[mode] = limit;
        }
        G1_CUDA(cudaGraphLaunch(gx, s));
        count_launches(per_pair << i);
        G1_CUDA(cudaMemcpyAsync(host, a.ctl, 16, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaMemcpyAsync(host + 4, a.c[0], 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        if (host[4] == 0) break;  // frontier empty after the last pair
        if (host[0] > n + 1) return fail(G1_ERR_TIMEOUT, "traversal did not converge within n rounds");
        if (host[4] > n) return fail(G1_ERR_OVERFLOW, "frontier larger than the vertex count");
        if (i < AdvGraphs::kSizes - 1) ++i;
    }
    if (iters_out) *iters_out = host[0];
    G1_TRY(copy_out_vertices(g, out, a.dist, s));
    return check_device_error(g, s);
}

struct TrState {
    uint32_t* dist;
    uint32_t* x;
    uint32_t* visited;
    uint32_t* F[2];
    uint32_t* cnt;  // [0] next frontier size, [2..3] degree sum (u64)
    uint32_t* host;  // pinned
    uint32_t* deg;     // frontier degrees (n + 1)
    uint32_t* prefix;  // their exclusive prefix (n + 1)
};

template <bool UNIT>
static g1_status traverse(g1_graph* g, uint32_t src_caller, g1_engine engine, uint32_t* out,
                          uint32_t* iters_out, cudaStream_t s) {
    const uint32_t n = g->n;
    if (src_caller >= n) return fail(G1_ERR_INVALID, "source vertex out of range");
    uint32_t src = src_caller;
    G1_TRY(internal_vertex(g, src_caller, &src, s));
    if (engine == G1_ENGINE_AUTO && nearfar_suits(g)) engine = G1_ENGINE_NEARFAR;
    // BFS on the advance engine on graphs of small uniform degree (grids,
    // meshes): thousands of small frontiers, so one persistent launch whose
    // rounds are the advance/filter steps (every vertex the last round
    // reached pushes its out-edges; the newly reached ones, once each, form
    // the next frontier), separated by a grid barrier instead of launches:
    // 4096^2 grid 57-63 -> 35 ms.  Not for SSSP: without distance buckets,
    // Bellman-Ford's correction waves make large frontiers, where the
    // edge-balanced push of the captured steps below is faster (745 against
    // 314 ms on that grid).
    const bool frontier = UNIT && engine == G1_ENGINE_ADVANCE && nearfar_suits(g);
    if (engine == G1_ENGINE_NEARFAR || frontier) {
        if (!UNIT && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
        uint32_t* dist = nullptr;
        uint32_t rounds = 0;
        G1_TRY(nearfar_traverse(g, src, UNIT, &dist, &rounds, s, frontier));
        if (iters_out) *iters_out = rounds;
        G1_TRY(copy_out_vertices(g, out, dist, s));
        return check_device_error(g, s);
    }
    if ((engine == G1_ENGINE_BLAS || engine == G1_ENGINE_AUTO) && !g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "pull engine needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if ((engine == G1_ENGINE_ADVANCE || engine == G1_ENGINE_AUTO) && !g->o[0].present)
        return fail(G1_ERR_UNSUPPORTED, "push engine needs the out-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (!UNIT && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
    if (engine == G1_ENGINE_ADVANCE && advance_graph_suits(g))
        return advance_graph_traverse<UNIT>(g, src, out, iters_out, s);
    // AUTO below kAutoDeviceEdges: the device-driven BLAS engine, whose sparse
    // steps (from 2^20 edges) are the same push/pull switch with no host round
    // trip per iteration, is the faster one there (SSSP p50, relabelled RMAT:
    // 0.24 against 0.37 ms at scale 14, 0.57 against 0.66 ms at 18); above it
    // the host-driven loop's edge-balanced push wins by a few percent (RMAT-20
    // and -22).  Distances are the same on every engine.
    if (engine == G1_ENGINE_BLAS || (engine == G1_ENGINE_AUTO && g->m < kAutoDeviceEdges))
        return blas_graph_traverse<UNIT>(g, src, out, iters_out, s);
    Workspace& ws = g->ws;
    TrState st;
    G1_TRY(ws.get("tr_dist", n, &st.dist));
    G1_TRY(ws.get("tr_x", n, &st.x));
    G1_TRY(ws.get("tr_visited", n, &st.visited));
    G1_TRY(ws.get("tr_f0", n, &st.F[0]));
    G1_TRY(ws.get("tr_f1", n, &st.F[1]));
    G1_TRY(ws.get("tr_cnt", 8, &st.cnt));
    G1_TRY(ws.get("tr_deg", (size_t)n + 1, &st.deg));
    G1_TRY(ws.get("tr_prefix", (size_t)n + 1, &st.prefix));
    size_t scan_bytes = 0;
    G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, st.deg, st.prefix, (int)n + 1, s));
    unsigned char* scan_tmp = nullptr;
    G1_TRY(ws.get("tr_scan", scan_bytes + 16, &scan_tmp));
    G1_TRY(ws.pinned.ensure(64));
    st.host = ws.pinned.as<uint32_t>();
    unsigned long long* deg_sum = reinterpret_cast<unsigned long long*>(st.cnt + 2);
    const uint32_t g_n = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
    tr_init_kernel<<<g_n, 256, 0, s>>>(n, src, st.dist, st.x, st.visited, st.F[0]);
    count_launches(1);
    G1_CUDA(cudaGetLastError());

    const int pull_t = 1, push_t = 0;
    const uint32_t* push_rp = g->o[push_t].present ? g->o[push_t].rp : g->o[pull_t].rp;
    uint32_t nF = 1;
    uint64_t degF = 0;
    {
        // out-degree of the source, for the first push/pull decision
        uint32_t h[2];
        G1_CUDA(cudaMemcpyAsync(h, push_rp + src, 8, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        degF = h[1] - h[0];
    }
    uint32_t it = 0;
    int cur = 0;
    const uint64_t push_limit = std::max<uint64_t>(1, g->m / std::max<uint32_t>(1, g->push_div));
    while (nF > 0) {
        ++it;
        // Bellman-Ford settles within n rounds; more means corrupted state.
        if (it > n + 1) return fail(G1_ERR_TIMEOUT, "traversal did not converge within n rounds");
        G1_CUDA(cudaMemsetAsync(st.cnt, 0, 16, s));
        const bool push = engine == G1_ENGINE_ADVANCE || (engine == G1_ENGINE_AUTO && degF < push_limit);
        const uint32_t gf = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(ceil_div(nF, 256), (uint64_t)g->sm_count * 8));
        if (push) {
            const Orientation& o = g->o[push_t];
            if (o.max_deg <= 32) {  // short lists only: TPV lanes per frontier vertex
                const uint64_t mean = ceil_div(std::max<uint64_t>(degF, 1), nF);
                int tpv = 1;
                while (tpv < 32 && (uint64_t)tpv < mean) tpv <<= 1;
                const uint32_t gt = (uint32_t)std::max<uint64_t>(
                    1, std::min<uint64_t>(ceil_div((uint64_t)nF * tpv, 256), (uint64_t)g->sm_count * 8));
                count_launches(1);
#define G1_TR_ADV(T)                                                                                    \
    tr_advance_kernel<UNIT, T><<<gt, 256, 0, s>>>(st.F[cur], nF, n, o.rp, o.col, static_cast<const uint32_t*>(o.val), \
                                                  st.dist, st.visited, it, st.F[cur ^ 1], st.cnt, deg_sum, g->err_word)
                switch (tpv) {
                    case 1: G1_TR_ADV(1); break;
                    case 2: G1_TR_ADV(2); break;
                    case 4: G1_TR_ADV(4); break;
                    case 8: G1_TR_ADV(8); break;
                    case 16: G1_TR_ADV(16); break;
                    default: G1_TR_ADV(32); break;
                }
#undef G1_TR_ADV
            } else {
                tr_frontier_degrees_kernel<<<gf, 256, 0, s>>>(st.F[cur], nF, n, o.rp, st.dist, st.deg,
                                                              g->err_word);
                size_t tb = scan_bytes;
                G1_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, tb, st.deg, st.prefix, (int)nF + 1, s));
                const uint32_t ga = (uint32_t)std::max<uint64_t>(
                    1, std::min<uint64_t>(ceil_div(degF, 256), (uint64_t)g->sm_count * 8));
                tr_advance_lb_kernel<UNIT><<<ga, 256, 0, s>>>(
                    st.F[cur], nF, st.prefix, o.rp, o.col, static_cast<const uint32_t*>(o.val),
                    st.dist, st.visited, it, st.F[cur ^ 1], st.cnt, deg_sum);
                count_launches(3);
            }
        } else {
            tr_scatter_kernel<<<gf, 256, 0, s>>>(st.F[cur], nF, st.dist, st.x, 0);
            count_launches(2);
            SparseApplyEpilogue e{st.dist, st.F[cur ^ 1], st.cnt, deg_sum, push_rp};
            if (UNIT)
                G1_TRY((run_spmv<BfsU32>(g, pull_t, G1_SCHED_AUTO, st.x, e, s)));
            else
                G1_TRY((run_spmv<MinPlusU32>(g, pull_t, G1_SCHED_AUTO, st.x, e, s)));
            tr_scatter_kernel<<<gf, 256, 0, s>>>(st.F[cur], nF, st.dist, st.x, 1);
        }
        G1_CUDA(cudaGetLastError());
        G1_CUDA(cudaMemcpyAsync(st.host, st.cnt, 16, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        nF = st.host[0];
        degF = (uint64_t)st.host[2] | ((uint64_t)st.host[3] << 32);
        cur ^= 1;
        if (nF > n) return fail(G1_ERR_OVERFLOW, "frontier larger than the vertex count");
    }
    if (iters_out) *iters_out = it;
    G1_TRY(copy_out_vertices(g, out, st.dist, s));
    return check_device_error(g, s);
}

// One push step over caller-owned device arrays (g1_advance_run): the push
// branch of traverse() on a given frontier.  The TPV choice uses the graph's
// mean degree (the frontier's is not known without a pass over it); the
// edge-balanced kernel grid-strides over the frontier's edges, so its grid
// needs no degree sum either.
template <bool UNIT>
static g1_status advance_step(g1_graph* g, const uint32_t* F, uint32_t nF, uint32_t* dist,
                              uint32_t* visited, uint32_t iter, uint32_t* out, uint32_t* out_size,
                              cudaStream_t s) {
    const Orientation& o = g->o[0];
    Workspace& ws = g->ws;
    uint32_t* cnt = nullptr;
    G1_TRY(ws.get("adv_cnt", 8, &cnt));
    G1_TRY(ws.pinned.ensure(64));
    uint32_t* host = ws.pinned.as<uint32_t>();
    unsigned long long* deg_sum = reinterpret_cast<unsigned long long*>(cnt + 2);
    G1_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
    const uint64_t cap = (uint64_t)g->sm_count * 8;
    const auto* val = static_cast<const uint32_t*>(o.val);
    if (o.max_deg <= 32) {
        const double mean = g->n ? (double)g->m / g->n : 1.0;
        int tpv = 1;
        while (tpv < 32 && tpv < mean) tpv <<= 1;
        const uint32_t gt =
            (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div((uint64_t)nF * tpv, 256), cap));
        count_launches(1);
#define G1_ADV_STEP(T)                                                                              \
    tr_advance_kernel<UNIT, T><<<gt, 256, 0, s>>>(F, nF, g->n, o.rp, o.col, val, dist, visited, iter, out, \
                                                  cnt, deg_sum, g->err_word)
        switch (tpv) {
            case 1: G1_ADV_STEP(1); break;
            case 2: G1_ADV_STEP(2); break;
            case 4: G1_ADV_STEP(4); break;
            case 8: G1_ADV_STEP(8); break;
            case 16: G1_ADV_STEP(16); break;
            default: G1_ADV_STEP(32); break;
        }
#undef G1_ADV_STEP
    } else {
        uint32_t *deg = nullptr, *prefix = nullptr;
        G1_TRY(ws.get("adv_deg", (size_t)nF + 1, &deg));
        G1_TRY(ws.get("adv_prefix", (size_t)nF + 1, &prefix));
        size_t scan_bytes = 0;
        G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, deg, prefix, (int)nF + 1, s));
        unsigned char* scan_tmp = nullptr;
        G1_TRY(ws.get("adv_scan", scan_bytes + 16, &scan_tmp));
        const uint32_t gf = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div((uint64_t)nF + 1, 256), cap));
        tr_frontier_degrees_kernel<<<gf, 256, 0, s>>>(F, nF, g->n, o.rp, dist, deg, g->err_word);
        G1_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, deg, prefix, (int)nF + 1, s));
        tr_advance_lb_kernel<UNIT><<<(uint32_t)cap, 256, 0, s>>>(F, nF, prefix, o.rp, o.col, val, dist, visited,
                                                                 iter, out, cnt, deg_sum);
        count_launches(3);
    }
    G1_CUDA(cudaGetLastError());
    G1_CUDA(cudaMemcpyAsync(host, cnt, 16, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    if (host[0] > g->n) return fail(G1_ERR_OVERFLOW, "frontier larger than the vertex count");
    *out_size = host[0];
    return check_device_error(g, s);
}

g1_status traverse_locked(g1_graph* g, uint32_t src, g1_engine engine, bool unit, uint32_t* out,
                          uint32_t* iters_out, cudaStream_t s) {
    return unit ? traverse<true>(g, src, engine, out, iters_out, s)
                : traverse<false>(g, src, engine, out, iters_out, s);
}

}  // namespace g1

using namespace g1;

extern "C" g1_status g1_advance_run(g1_graph* g, int unit, const uint32_t* frontier, uint32_t n_frontier,
                                    uint32_t* dist, uint32_t* visited, uint32_t iter, uint32_t* out_frontier,
                                    uint32_t* out_size, void* stream) {
    if (!g || !dist || !visited || !out_frontier || !out_size || (n_frontier && !frontier))
        return fail(G1_ERR_INVALID, "g1_advance_run: null argument");
    if (n_frontier > g->n) return fail(G1_ERR_INVALID, "g1_advance_run: frontier larger than the vertex count");
    if (!g->o[0].present)
        return fail(G1_ERR_UNSUPPORTED, "g1_advance_run: needs the out-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (g->relabeled) return fail(G1_ERR_UNSUPPORTED, "g1_advance_run: graph was created with G1_GRAPH_RELABEL");
    if (!unit && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "g1_advance_run: SSSP needs u32 edge weights");
    if (!is_device_ptr(frontier ? (const void*)frontier : (const void*)dist) || !is_device_ptr(dist) ||
        !is_device_ptr(visited) || !is_device_ptr(out_frontier))
        return fail(G1_ERR_INVALID, "g1_advance_run: frontier, dist, visited and out_frontier must be device memory");
    *out_size = 0;
    if (n_frontier == 0) return G1_OK;
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStream_t s = as_stream(stream);
    return unit ? advance_step<true>(g, frontier, n_frontier, dist, visited, iter, out_frontier, out_size, s)
                : advance_step<false>(g, frontier, n_frontier, dist, visited, iter, out_frontier, out_size, s);
}

extern "C" g1_status g1_sssp(g1_graph* g, uint32_t src, g1_engine engine, uint32_t* dist_out,
                             uint32_t* iters_out, void* stream) {
    if (!g || !dist_out) return fail(G1_ERR_INVALID, "g1_sssp: bad argument");
    if (engine < G1_ENGINE_BLAS || engine > G1_ENGINE_NEARFAR)
        return fail(G1_ERR_INVALID, "g1_sssp: unknown engine");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    return traverse<false>(g, src, engine, dist_out, iters_out, as_stream(stream));
}

extern "C" g1_status g1_bfs(g1_graph* g, uint32_t src, g1_engine engine, uint32_t* level_out,
                            uint32_t* iters_out, void* stream) {
    if (!g || !level_out) return fail(G1_ERR_INVALID, "g1_bfs: bad argument");
    if (engine < G1_ENGINE_BLAS || engine > G1_ENGINE_NEARFAR)
        return fail(G1_ERR_INVALID, "g1_bfs: unknown engine");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    return traverse<true>(g, src, engine, level_out, iters_out, as_stream(stream));
}
