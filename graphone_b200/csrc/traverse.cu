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
    if (engine == G1_ENGINE_NEARFAR) {
        if (!UNIT && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
        uint32_t* dist = nullptr;
        uint32_t rounds = 0;
        G1_TRY(nearfar_traverse(g, src, UNIT, &dist, &rounds, s));
        if (iters_out) *iters_out = rounds;
        G1_TRY(copy_out_vertices(g, out, dist, s));
        return check_device_error(g, s);
    }
    if ((engine == G1_ENGINE_BLAS || engine == G1_ENGINE_AUTO) && !g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "pull engine needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if ((engine == G1_ENGINE_ADVANCE || engine == G1_ENGINE_AUTO) && !g->o[0].present)
        return fail(G1_ERR_UNSUPPORTED, "push engine needs the out-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (!UNIT && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
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
    const uint64_t push_limit = std::max<uint64_t>(1, g->m / 16);
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
