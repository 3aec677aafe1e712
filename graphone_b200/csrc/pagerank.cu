// PageRank on the plus-times SpMV with the apply/construct step fused into
// the SpMV epilogue.
//
// GraphOne's all-active engine runs, per iteration, the merge SpMV over the
// in-edge CSR, then apply_construct_kernel over all N vertices
// (engine/blas_gc.h:377-428): rank'[v] = (1-a)/N + y[v] (apply_each,
// apps/pagerank_blas.cu:115-121) and x'[v] = rank'[v] * iweights[v]
// (construct_each, :95-101).  Here each completed row of the SpMV applies and
// constructs in registers, so y never reaches HBM and there is no N-sized
// second pass.  x and rank are double-buffered across iterations.
//
// Writes an iteration does not need are left out: rank only in the last
// iteration (earlier ones need only x'), x' never for a vertex without
// out-weight (0 in both x buffers from the start), and under the nnz
// schedule the fixup skips isolated vertices (no in- or out-edges) until
// the last iteration, adding their dangling share as a count (exact in the
// fixed-point sum below).  The final ranks are the same bits.
//
// G1_PR_DANGLING adds a*sum(rank[dangling])/N; that sum is reduced on the
// device by the epilogues themselves, so no host round trip.  It is an exact
// integer sum of the ranks in 2^-56 fixed point (one 64-bit atomic per
// block): the result does not depend on which block emits which row, nor on
// the order of the atomics, so every schedule gives the same bits.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "g1/semiring.cuh"
#include "g1/spmv.cuh"
#include "internal.h"
#include "spmv_launch.cuh"

namespace g1 {

// Dangling sums in fixed point: rank r >= 0 (the ranks sum to at most 1)
// as floor(r * 2^56), from the float's bits with integer shifts only; 64-bit
// integer sums are exact and order-free.
constexpr double kDangScale = 72057594037927936.0;  // 2^56
__device__ __forceinline__ unsigned long long dang_fixed(float r) {
    const uint32_t b = __float_as_uint(r);
    const int e = (int)((b >> 23) & 0xFFu);
    if (e == 0) return 0ull;  // zero or subnormal: below the 2^-56 resolution
    const unsigned long long m = (unsigned long long)((b & 0x7FFFFFu) | 0x800000u);
    const int sh = e - 94;  // r * 2^56 = m * 2^(e - 150 + 56); sh <= 33 for r <= 1
    return sh >= 0 ? (m << min(sh, 39)) : (sh > -24 ? (m >> -sh) : 0ull);
}

// Adds the block's fixed-point dangling sum to *out.
template <int BLOCK>
__device__ __forceinline__ void dang_block_add(unsigned long long v, unsigned long long* out,
                                               char* smem) {
    const unsigned long long sum =
        block_sum<unsigned long long, BLOCK>(v, reinterpret_cast<unsigned long long*>(smem));
    if (threadIdx.x == 0 && sum) atomicAdd(out, sum);
}

struct PrEpilogue {
    static constexpr bool kRowsIndependent = true;
    float* rank_next;
    float* x_next;
    const float* iw;
    // dangling sums (fixed point) rotate through three words: this
    // iteration reads dang_in, adds into dang_out (zero on entry) and the
    // main kernel's first thread zeroes dang_clear (read one iteration ago)
    const unsigned long long* dang_in;
    unsigned long long* dang_out;
    unsigned long long* dang_clear;  // null in the fixup
    double alpha_over_n;
    float base0;           // (float)((1 - alpha) / N), the reference's alpha_div_v
    int dangling;          // G1_PR_DANGLING
    int write_rank;        // last iteration: rank_next is the result
    // hot-column layout: x is stored by hot id (row v's entry at xperm[v]);
    // null: by vertex id
    const uint32_t* xperm = nullptr;
    // nnz fixup: the empty rows to emit when set (those with out-weight);
    // the n_iso isolated vertices left out add n_iso * base to the
    // dangling sum (block 0, thread 0)
    const uint32_t* empty_list = nullptr;
    uint32_t n_empty_list = 0;
    uint32_t n_iso = 0;

    float base;
    unsigned long long dang_local;

    __device__ __forceinline__ void begin() {
        dang_local = 0ull;
        if (dang_clear && blockIdx.x == 0 && threadIdx.x == 0) *dang_clear = 0ull;
        // under programmatic dependent launch the fixup runs this before its
        // dependency wait: dang_in was written by a grid that completed
        // before this one launched (the previous fixup)
        base = dangling ? (float)((double)base0 + alpha_over_n * ((double)(*dang_in) / kDangScale))
                        : base0;
        if (n_iso && dangling && blockIdx.x == 0 && threadIdx.x == 0)
            dang_local = (unsigned long long)n_iso * dang_fixed(base);
    }
    struct Pre {
        float w;
        uint32_t xi;
    };
    __device__ __forceinline__ void emit(uint32_t v, const float& y) {
        emit_prepared(v, y, prepare(v));
    }
    // iweights[v] and x's slot for v do not depend on the row's value:
    // loaded ahead
    __device__ __forceinline__ Pre prepare(uint32_t v) const {
        return Pre{__ldg(iw + v), xperm ? __ldg(xperm + v) : v};
    }
    __device__ __forceinline__ void emit_prepared(uint32_t v, const float& y, const Pre& p) {
        const float r = base + y;
        if (write_rank) rank_next[v] = r;
        if (p.w != 0.0f) x_next[p.xi] = r * p.w;
        else if (dangling) dang_local += dang_fixed(r);
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char* smem) {
        if (dangling) dang_block_add<BLOCK>(dang_local, dang_out, smem);
    }
};

// Out-weight sums from the in-edge CSR only (no out-edge CSR built): a
// weighted histogram of the column indices.  The lowest PRIV vertex ids get
// block-private shared-memory bins (RMAT hubs sit at low ids), the rest go
// straight to global atomics.  Few, large blocks (two per SM): each block
// adds its PRIV bins to global memory once at the end.  Four edges per
// thread and step (col and val 16-byte aligned).
template <int PRIV, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
pr_outw_from_transpose_kernel(const uint32_t* tcol, const float* tval, uint32_t m, uint32_t n,
                              float* outw) {
    __shared__ float bins[PRIV];
    for (int i = threadIdx.x; i < PRIV; i += BLOCK) bins[i] = 0.0f;
    __syncthreads();
    auto add = [&](uint32_t u, float w) {
        if (u < PRIV) atomicAdd(&bins[u], w);
        else if (u < n) atomicAdd(&outw[u], w);  // ids are validated after an eager upload
    };
    const uint64_t stride = (uint64_t)gridDim.x * BLOCK;
    const uint64_t m4 = m / 4;
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < m4; i += stride) {
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(tcol) + i);
        const float4 w = __ldg(reinterpret_cast<const float4*>(tval) + i);
        add(u.x, w.x);
        add(u.y, w.y);
        add(u.z, w.z);
        add(u.w, w.w);
    }
    for (uint64_t k = m4 * 4 + (uint64_t)blockIdx.x * BLOCK + threadIdx.x; k < m; k += stride)
        add(__ldg(tcol + k), __ldg(tval + k));
    __syncthreads();
    for (int i = threadIdx.x; i < PRIV && i < (int)n; i += BLOCK)
        if (bins[i] != 0.0f) atomicAdd(&outw[i], bins[i]);
}

// iweights = alpha / out-weight (0 for a vertex without out-weight,
// apps/pagerank_blas.cu:41-53), the initial ranks 1/N, x0 = rank0 * iw,
// x1 = 0 where there is no out-weight (never written after), and the
// dangling sum of rank0.  x is indexed by xperm[v] when set.
__global__ void pr_init_from_outw_kernel(const float* outw, uint32_t n, float alpha, float* iw,
                                         float* rank0, float* x0, float* x1,
                                         unsigned long long* dang_out, const uint32_t* xperm) {
    __shared__ alignas(16) char smem[64 * 8];
    const float r0 = (float)(1.0 / (double)n);
    unsigned long long dl = 0ull;
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    for (uint64_t v = (uint64_t)blockIdx.x * 256 + threadIdx.x; v < n; v += stride) {
        const float s = outw[v];
        const float w = s != 0.0f ? alpha / s : 0.0f;
        iw[v] = w;
        rank0[v] = r0;
        const uint32_t xi = xperm ? xperm[v] : (uint32_t)v;
        x0[xi] = r0 * w;
        if (w == 0.0f) {
            x1[xi] = 0.0f;
            dl += dang_fixed(r0);
        }
    }
    dang_block_add<256>(dl, dang_out, smem);
}

struct HasOutWeight {
    const float* outw;
    __device__ __forceinline__ bool operator()(uint32_t v) const { return outw[v] != 0.0f; }
};

// The empty in-edge rows with out-weight, in plan order (the nnz fixup
// emits only these before the last iteration) and the number of isolated
// vertices; once per graph.
static g1_status pr_empty_active(g1_graph* g, const NnzPlan& p, const float* outw, cudaStream_t s) {
    uint32_t* list = nullptr;
    uint32_t* count = nullptr;
    G1_TRY(g->ws.get("pr_empty_active", (size_t)p.n_empty + 1, &list));
    G1_TRY(g->ws.get("pr_empty_count", 4, &count));
    const uint32_t* empty = p.rows.as<uint32_t>() + p.n_nonempty;
    uint32_t active = 0;
    if (p.n_empty > 0) {
        size_t tb = 0;
        G1_CUDA(cub::DeviceSelect::If(nullptr, tb, empty, list, count, (int)p.n_empty,
                                      HasOutWeight{outw}, s));
        unsigned char* temp = nullptr;  // kept in the graph's workspace: no free
        G1_TRY(g->ws.get("pr_select_tmp", tb + 16, &temp));
        G1_CUDA(cub::DeviceSelect::If(temp, tb, empty, list, count, (int)p.n_empty,
                                      HasOutWeight{outw}, s));
        G1_CUDA(cudaMemcpyAsync(&active, count, 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
    }
    g->pr_active_empty = active;
    g->pr_isolated = p.n_empty - active;
    g->pr_empty_ready = true;
    return G1_OK;
}

struct PrBuffers {
    float* iw;
    float* rank[2];
    float* x[2];
    unsigned long long* dang;  // [3], fixed point
    int t;                     // the in-edge CSR: 1, or its hot-column copy 2
    const uint32_t* xperm;     // with 2: vertex id -> hot id (x's index)
};

// Hot-column layout.  The pull SpMV gathers x[u] once per out-edge of u,
// and its tile kernel caches a prefix of x in shared memory.  A graph
// relabelled by degree (G1_GRAPH_RELABEL) has its hot vertices in that
// prefix, but the relabelling rebuilds both CSRs (about 11 ms on RMAT-22).
// For a graph kept in the caller's order PageRank instead renames only the
// columns: hot id k is the k-th vertex by decreasing out-degree (ties by
// id), x is stored by hot id, and a copy of the in-edge CSR's column array
// holds hot ids (orientation 2; rows, values and plans stay orientation
// 1's).  The order is by out-weight, which PageRank computes anyway (for
// weights of similar size it follows the out-degree; any order gives the
// same results).  Each row's nonzeros keep their order, so every row sums
// the same values in the same order: the ranks are the same bits.  Built
// once per graph, from 2^22 edges (RMAT-22: 0.265 -> 0.181 ms per SpMV,
// against 0.215 ms relabelled).
__global__ void pr_iota_kernel(uint32_t* ids, uint32_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        ids[i] = (uint32_t)i;
}

__global__ void pr_hot_rank_kernel(const uint32_t* order, uint32_t n, uint32_t* hot) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        hot[order[i]] = (uint32_t)i;
}

// out[k] = hot[col[k]], four columns per thread (col and out 16-byte aligned).
__global__ void pr_hot_cols_kernel(const uint32_t* col, uint32_t m, const uint32_t* hot, uint32_t* out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t m4 = m / 4;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m4; i += stride) {
        const uint4 c = __ldg(reinterpret_cast<const uint4*>(col) + i);
        reinterpret_cast<uint4*>(out)[i] = make_uint4(__ldg(hot + c.x), __ldg(hot + c.y), __ldg(hot + c.z),
                                                      __ldg(hot + c.w));
    }
    for (uint64_t k = m4 * 4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
        out[k] = __ldg(hot + col[k]);
}

constexpr uint32_t kHotLayoutMinEdges = 1u << 22;
constexpr uint32_t kHotLayoutMinMaxDegree = 64;

// Builds orientation 2 and the hot ids (workspace "pr_hot") if the graph
// qualifies, ordering by `keys` (PageRank: the out-weights, non-negative
// floats whose bits sort as unsigned integers; personalized PageRank: the
// out-degrees); *t the orientation the SpMV runs on.  A layout built by one
// serves the other (any order gives the same results).  Caller holds g->mu.
static g1_status pr_hot_layout(g1_graph* g, const uint32_t* keys, cudaStream_t s, int* t,
                               const uint32_t** xperm) {
    *t = 1;
    *xperm = nullptr;
    const Orientation& in = g->o[1];
    if (g->hot_mode == G1_HOT_COLUMNS_OFF) return G1_OK;
    // AUTO: large graphs in the caller's order with skewed degrees (where a
    // few vertices take most gathers; on a grid every vertex is as hot)
    if (g->hot_mode == G1_HOT_COLUMNS_AUTO &&
        (g->relabeled || g->m < kHotLayoutMinEdges || in.max_deg <= kHotLayoutMinMaxDegree ||
         resolve_schedule(g, 1, G1_SCHED_AUTO) == G1_SCHED_VECTOR))
        return G1_OK;
    const uint32_t n = g->n, m = g->m;
    Orientation& h = g->o[2];
    uint32_t* hot = nullptr;
    if (!h.present) {
        const uint32_t* deg = keys;
        DevBuf sorted, ids, order, temp;
        size_t tb = 0;
        G1_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, deg, sorted.as<uint32_t>(),
                                                          ids.as<uint32_t>(), order.as<uint32_t>(),
                                                          (int)n, 0, 32, s));
        // all memory first: under AUTO a graph that does not fit its copy of
        // the columns runs on the plain layout instead (same results)
        g1_status st = g->ws.get("pr_hot", n, &hot);
        if (st == G1_OK) st = sorted.ensure((size_t)n * 4 + 16);
        if (st == G1_OK) st = ids.ensure((size_t)n * 4 + 16);
        if (st == G1_OK) st = order.ensure((size_t)n * 4 + 16);
        if (st == G1_OK) st = temp.ensure(tb + 16);
        // the same zeroed pad as the other column arrays
        if (st == G1_OK) st = h.b_col.ensure(((size_t)m + kWarpTilePad + 64) * 4);
        if (st != G1_OK) {
            h.b_col.release();
            if (st == G1_ERR_OOM && g->hot_mode == G1_HOT_COLUMNS_AUTO) return G1_OK;
            return st;
        }
        const size_t nz_used = (size_t)m * 4;
        G1_CUDA(cudaMemsetAsync(h.b_col.as<char>() + nz_used, 0, h.b_col.bytes - nz_used, s));
        const uint32_t grid = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
        pr_iota_kernel<<<grid, 256, 0, s>>>(ids.as<uint32_t>(), n);
        G1_CUDA(cub::DeviceRadixSort::SortPairsDescending(temp.p, tb, deg, sorted.as<uint32_t>(),
                                                          ids.as<uint32_t>(), order.as<uint32_t>(),
                                                          (int)n, 0, 32, s));
        pr_hot_rank_kernel<<<grid, 256, 0, s>>>(order.as<uint32_t>(), n, hot);
        pr_hot_cols_kernel<<<(uint32_t)g->sm_count * 8, 256, 0, s>>>(in.col, m, hot, h.b_col.as<uint32_t>());
        count_launches(3);
        G1_CUDA(cudaGetLastError());
        // the temporaries are released (to the block cache) when this returns
        G1_CUDA(cudaStreamSynchronize(s));
        h.rp = in.rp;
        h.col = h.b_col.as<uint32_t>();
        h.val = in.val;
        h.max_deg = in.max_deg;
        h.present = true;
    } else {
        G1_TRY(g->ws.get("pr_hot", n, &hot));
    }
    h.max_deg = in.max_deg;
    h.tuned_sched = in.tuned_sched;
    h.tuned_variant = in.tuned_variant;
    *t = 2;
    *xperm = hot;
    return G1_OK;
}

constexpr int kEagerOutwChunks = 8;
// the chunks whose out-weights order the hot-column layout built during an upload
constexpr int kEagerHotChunks = 6;

__global__ void pr_max_row_kernel(const uint32_t* rp, uint32_t n, uint32_t* out) {
    uint32_t mx = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        mx = max(mx, rp[v + 1] - rp[v]);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31u) == 0 && mx) atomicMax(out, mx);
}

// Uploads the in-edge CSR's columns and f32 values from host memory in
// chunks on s; a second stream sums each chunk's out-weights as soon as it
// has arrived (workspace "pr_outw", what PageRank's first call would
// otherwise compute after the whole copy), so only the last chunk's
// histogram is left when the copy ends.  Where PageRank would build its
// hot-column layout (degrees skewed: a row of more than 64 in-edges), the
// second stream also builds it: once the first kEagerHotChunks chunks are
// summed it orders the vertices by those partial out-weights (any order
// gives the same ranks), remaps the arrived chunks' columns while the rest
// are copied, and each later chunk as it arrives.  s waits for all of it.
g1_status upload_transpose_with_outw(g1_graph* g, const uint32_t* col, const void* val, cudaStream_t s) {
    Orientation& o = g->o[1];
    const uint32_t n = g->n, m = g->m;
    float* outw = nullptr;
    G1_TRY(g->ws.get("pr_outw", n, &outw));
    G1_CUDA(cudaMemsetAsync(outw, 0, (size_t)n * 4, s));
    // chunk starts at multiples of 1024 edges: 16-byte aligned for the
    // kernels' vector loads
    const size_t chunk = (ceil_div((size_t)m, (size_t)kEagerOutwChunks) + 1023) & ~size_t(1023);
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
    // the largest in-degree (the row offsets are on the device already),
    // read back without holding up the chunks queued after it
    const bool may_hot = g->hot_mode != G1_HOT_COLUMNS_OFF && m >= kHotLayoutMinEdges &&
                         (size_t)(kEagerHotChunks + 1) * chunk <= m;
    uint32_t* d_max = nullptr;
    cudaEvent_t ev_max = nullptr;
    if (may_hot) {
        G1_TRY(g->ws.get("pr_up_max", 4, &d_max));
        G1_TRY(g->ws.pinned.ensure(64));
        G1_CUDA(cudaMemsetAsync(d_max, 0, 4, s));
        pr_max_row_kernel<<<grid, 256, 0, s>>>(o.rp, n, d_max);
        count_launches(1);
        G1_CUDA(cudaGetLastError());
        G1_CUDA(cudaMemcpyAsync(g->ws.pinned.p, d_max, 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaEventCreateWithFlags(&ev_max, cudaEventDisableTiming));
        G1_CUDA(cudaEventRecord(ev_max, s));
    }
    cudaStream_t h = nullptr;
    G1_CUDA(cudaStreamCreateWithFlags(&h, cudaStreamNonBlocking));
    cudaEvent_t ev[kEagerOutwChunks + 1] = {};
    g1_status st = G1_OK;
    auto check = [&](cudaError_t e, const char* what) {
        if (st == G1_OK && e != cudaSuccess) st = fail_cuda(e, what);
        return st == G1_OK;
    };
    Orientation& hc = g->o[2];
    uint32_t* hot = nullptr;
    DevBuf sorted, ids, order, temp;  // released to the block cache (reused after a device sync)
    bool build_hot = false;
    auto remap = [&](size_t lo, size_t cnt) {
        pr_hot_cols_kernel<<<(uint32_t)g->sm_count * 8, 256, 0, h>>>(o.col + lo, (uint32_t)cnt, hot,
                                                                     hc.b_col.as<uint32_t>() + lo);
        count_launches(1);
        check(cudaGetLastError(), "pr_hot_cols_kernel");
    };
    int used = 0;
    for (int c = 0; c < kEagerOutwChunks && st == G1_OK; ++c) {
        const size_t lo = (size_t)c * chunk;
        if (lo >= m) break;
        const size_t cnt = std::min(chunk, (size_t)m - lo);
        if (!check(cudaMemcpyAsync(o.col + lo, col + lo, cnt * 4, cudaMemcpyHostToDevice, s), "upload col"))
            break;
        if (!check(cudaMemcpyAsync(static_cast<char*>(o.val) + lo * 4, static_cast<const char*>(val) + lo * 4,
                                   cnt * 4, cudaMemcpyHostToDevice, s),
                   "upload val"))
            break;
        if (!check(cudaEventCreateWithFlags(&ev[c], cudaEventDisableTiming), "event")) break;
        used = c + 1;
        if (!check(cudaEventRecord(ev[c], s), "event record")) break;
        if (!check(cudaStreamWaitEvent(h, ev[c], 0), "stream wait")) break;
        pr_outw_from_transpose_kernel<8192, 1024><<<(uint32_t)g->sm_count * 2, 1024, 0, h>>>(
            o.col + lo, static_cast<const float*>(o.val) + lo, (uint32_t)cnt, n, outw);
        count_launches(1);
        if (!check(cudaGetLastError(), "pr_outw_from_transpose_kernel")) break;
        if (build_hot) remap(lo, cnt);
        if (may_hot && c == kEagerHotChunks - 1) {
            // the copies queued so far keep the copy engine busy meanwhile
            if (!check(cudaEventSynchronize(ev_max), "event sync")) break;
            const uint32_t max_in = *g->ws.pinned.as<uint32_t>();
            if (max_in <= kHotLayoutMinMaxDegree && g->hot_mode == G1_HOT_COLUMNS_AUTO) continue;
            size_t tb = 0;
            if (!check(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, (const uint32_t*)nullptr,
                                                                 (uint32_t*)nullptr, (const uint32_t*)nullptr,
                                                                 (uint32_t*)nullptr, (int)n, 0, 32, h),
                       "sort size"))
                break;
            // all memory first: a graph without room for the copy simply
            // gets it (or not) at PageRank's first call
            g1_status a = g->ws.get("pr_hot", n, &hot);
            if (a == G1_OK) a = sorted.ensure((size_t)n * 4 + 16);
            if (a == G1_OK) a = ids.ensure((size_t)n * 4 + 16);
            if (a == G1_OK) a = order.ensure((size_t)n * 4 + 16);
            if (a == G1_OK) a = temp.ensure(tb + 16);
            if (a == G1_OK) a = hc.b_col.ensure(((size_t)m + kWarpTilePad + 64) * 4);
            if (a != G1_OK) {
                hc.b_col.release();
                continue;
            }
            const size_t nz_used = (size_t)m * 4;
            if (!check(cudaMemsetAsync(hc.b_col.as<char>() + nz_used, 0, hc.b_col.bytes - nz_used, h), "pad"))
                break;
            const uint32_t* keys = reinterpret_cast<const uint32_t*>(outw);
            pr_iota_kernel<<<grid, 256, 0, h>>>(ids.as<uint32_t>(), n);
            if (!check(cub::DeviceRadixSort::SortPairsDescending(temp.p, tb, keys, sorted.as<uint32_t>(),
                                                                 ids.as<uint32_t>(), order.as<uint32_t>(),
                                                                 (int)n, 0, 32, h),
                       "sort"))
                break;
            pr_hot_rank_kernel<<<grid, 256, 0, h>>>(order.as<uint32_t>(), n, hot);
            count_launches(2);
            if (!check(cudaGetLastError(), "hot ids")) break;
            build_hot = true;
            remap(0, lo + cnt);  // the chunks that have arrived
        }
    }
    // s continues after the histograms (and the remaps), whatever happened above
    cudaEvent_t& done = ev[kEagerOutwChunks];
    if (check(cudaEventCreateWithFlags(&done, cudaEventDisableTiming), "event") &&
        check(cudaEventRecord(done, h), "event record"))
        check(cudaStreamWaitEvent(s, done, 0), "stream wait");
    else
        cudaStreamSynchronize(h);
    for (int c = 0; c < used; ++c) cudaEventDestroy(ev[c]);
    if (done) cudaEventDestroy(done);
    if (ev_max) cudaEventDestroy(ev_max);
    cudaStreamDestroy(h);  // released once its work completes
    if (st != G1_OK) return st;
    g->outw_ready = true;
    if (build_hot) {
        hc.rp = o.rp;
        hc.col = hc.b_col.as<uint32_t>();
        hc.val = o.val;
        hc.present = true;
    }
    return G1_OK;
}

static g1_status pr_setup(g1_graph* g, float alpha, PrBuffers& b, uint32_t* grids,
                          cudaStream_t s) {
    const uint32_t n = g->n;
    Workspace& ws = g->ws;
    G1_TRY(ws.get("pr_iw", n, &b.iw));
    G1_TRY(ws.get("pr_rank0", n, &b.rank[0]));
    G1_TRY(ws.get("pr_rank1", n, &b.rank[1]));
    G1_TRY(ws.get("pr_x0", n, &b.x[0]));
    G1_TRY(ws.get("pr_x1", n, &b.x[1]));
    G1_TRY(ws.get("pr_dang", 4, &b.dang));
    // grids[3] init; grids[0] main merge, grids[1] fixup, grids[2] vector below
    grids[3] = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
    G1_CUDA(cudaMemsetAsync(b.dang, 0, 4 * sizeof(unsigned long long), s));
    float* outw = nullptr;
    G1_TRY(ws.get("pr_outw", n, &outw));
    if (!g->outw_ready) {
        if (g->o[0].present) {
            // row sums of the out-edge CSR = plus-times SpMV against ones
            float* ones = nullptr;
            G1_TRY(ws.get("pr_ones", n, &ones));
            G1_TRY(g1_mem_fill_u32(ones, 0x3f800000u, n, s));
            G1_TRY((run_spmv<PlusTimesF32>(g, 0, G1_SCHED_AUTO, ones, StoreEpilogue<float>{outw}, s)));
        } else {
            G1_CUDA(cudaMemsetAsync(outw, 0, (size_t)n * 4, s));
            pr_outw_from_transpose_kernel<8192, 1024><<<(uint32_t)g->sm_count * 2, 1024, 0, s>>>(
                g->o[1].col, static_cast<const float*>(g->o[1].val), g->m, n, outw);
            count_launches(1);
        }
        G1_CUDA(cudaGetLastError());
        g->outw_ready = true;
    }
    G1_TRY(pr_hot_layout(g, reinterpret_cast<const uint32_t*>(outw), s, &b.t, &b.xperm));
    const int t = b.t;
    G1_TRY((merge_grids<PlusTimesF32, PrEpilogue>(g, t, &grids[0], &grids[1])));
    grids[2] = vector_grid<PlusTimesF32, PrEpilogue>(g);
    pr_init_from_outw_kernel<<<grids[3], 256, 0, s>>>(outw, n, alpha, b.iw, b.rank[0], b.x[0],
                                                      b.x[1], &b.dang[0], b.xperm);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    const int v = merge_variant(g, t);
    if ((kMergeVariants[v].kind == 3 || kMergeVariants[v].kind == 5) && !g->pr_empty_ready) {
        NnzPlan* p = nullptr;
        G1_TRY(ensure_nnz_plan(g, t, &p));
        G1_TRY(pr_empty_active(g, *p, outw, s));
    }
    return G1_OK;
}

// PageRank iteration `it` of `iters`: reads x[cur], writes x[nxt] (cur =
// it & 1) and, in the last iteration, rank[nxt]; reads dang[it % 3], adds
// into dang[(it + 1) % 3], zeroes dang[(it + 2) % 3].
static g1_status pr_iterate(g1_graph* g, const PrBuffers& b, const uint32_t* grids, float alpha,
                            g1_pr_mode mode, int it, int iters, g1_schedule sched, cudaStream_t s) {
    const bool last = it == iters - 1;
    const int cur = it & 1, nxt = cur ^ 1;
    PrEpilogue e;
    e.rank_next = b.rank[nxt];
    e.x_next = b.x[nxt];
    e.iw = b.iw;
    e.dang_in = &b.dang[it % 3];
    e.dang_out = &b.dang[(it + 1) % 3];
    e.dang_clear = &b.dang[(it + 2) % 3];
    e.alpha_over_n = (double)alpha / (double)g->n;
    e.base0 = (float)((1.0 - (double)alpha) / (double)g->n);
    e.dangling = mode == G1_PR_DANGLING;
    e.write_rank = last ? 1 : 0;
    e.xperm = b.xperm;
    const int t = b.t;
    if (resolve_schedule(g, t, sched) == G1_SCHED_VECTOR)
        return launch_vector<PlusTimesF32>(g, t, b.x[cur], e, s);
    PrEpilogue f = e;
    f.dang_clear = nullptr;
    const int kind = kMergeVariants[merge_variant(g, t)].kind;
    if (!last && g->pr_empty_ready && (kind == 3 || kind == 5)) {
        uint32_t* list = nullptr;  // allocated by pr_empty_active, at least this large
        G1_TRY(g->ws.get("pr_empty_active", (size_t)g->pr_active_empty + 1, &list));
        f.empty_list = list;
        f.n_empty_list = g->pr_active_empty;
        f.n_iso = g->pr_isolated;
    }
    return launch_merge<PlusTimesF32>(g, t, b.x[cur], e, f, s);
}

// ------------------------------------------------ personalized PageRank
//
// Single-source PPR (the pagerank_blas iteration restarted at src, as the
// batched slot engine runs it) on the same SpMV schedules: x[u] = rank[u] *
// alpha / outdeg(u) is built by the previous iteration's epilogue, the SpMV
// sums x over each row's in-edges with every edge weight taken as 1 (the
// edge values are not read: 4 bytes per nonzero instead of 8), and the
// epilogue adds the teleport (1 - alpha) + alpha * sum(rank[dangling]) at
// src, writes x' and accumulates the next dangling sum (fixed point, as
// PageRank's).  Every vertex other than src without in-edges has rank 0 from
// the first iteration on, so before the last iteration the nnz fixup emits
// no empty row: only src, when its own row is empty, is emitted by the
// fixup's first thread.
struct PprEpilogue {
    static constexpr bool kRowsIndependent = true;
    float* rank_next;
    float* x_next;
    const float* iw;
    const uint32_t* src_p;  // internal id of the source
    const unsigned long long* dang_in;
    unsigned long long* dang_out;
    unsigned long long* dang_clear;  // null in the fixup
    double alpha;
    int write_rank;
    // nnz fixup before the last iteration: an empty list (no empty row
    // emitted) and the in-edge row pointers, to emit src if its row is empty
    const uint32_t* empty_list = nullptr;
    uint32_t n_empty_list = 0;
    const uint32_t* src_rows = nullptr;
    // sparse steps: the word that says this iteration is one (its kernels
    // then return at once), or null
    const uint32_t* sparse_now = nullptr;
    // hot-column layout: x is stored by hot id (row v's entry at xperm[v]);
    // null: by vertex id
    const uint32_t* xperm = nullptr;

    uint32_t src;
    float tele;
    unsigned long long dang_local;

    __device__ __forceinline__ bool active() const { return !sparse_now || *sparse_now == 0u; }
    __device__ __forceinline__ void begin() {
        dang_local = 0ull;
        if (dang_clear && blockIdx.x == 0 && threadIdx.x == 0) *dang_clear = 0ull;
        src = *src_p;
        tele = (float)((1.0 - alpha) + alpha * ((double)(*dang_in) / kDangScale));
        if (src_rows && blockIdx.x == 0 && threadIdx.x == 0 && src_rows[src] == src_rows[src + 1])
            emit_prepared(src, 0.0f, prepare(src));
    }
    struct Pre {
        float w;
        uint32_t xi;
    };
    __device__ __forceinline__ void emit(uint32_t v, const float& y) {
        emit_prepared(v, y, prepare(v));
    }
    __device__ __forceinline__ Pre prepare(uint32_t v) const {
        return Pre{__ldg(iw + v), xperm ? __ldg(xperm + v) : v};
    }
    __device__ __forceinline__ void emit_prepared(uint32_t v, const float& y, const Pre& p) {
        const float r = v == src ? y + tele : y;
        if (write_rank) rank_next[v] = r;
        if (p.w != 0.0f) x_next[p.xi] = r * p.w;
        else dang_local += dang_fixed(r);
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char* smem) {
        dang_block_add<BLOCK>(dang_local, dang_out, smem);
    }
};

// iw[v] = alpha / outdeg(v), 0 without out-edges (the slot engine's
// transition weights, bit for bit).
__global__ void ppr_iw_kernel(const uint32_t* deg, uint32_t n, double alpha, float* iw) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        iw[v] = deg[v] ? (float)(alpha / (double)deg[v]) : 0.0f;
}

// rank0 = e_src, x0 = rank0 * iw, the dangling sum of rank0 (fixed point:
// 1.0 is 2^56); x0 and x1 are zero elsewhere (cleared by the caller).
__global__ void ppr_init_kernel(const uint32_t* perm, uint32_t src, const float* iw, uint32_t* src_out,
                                float* rank0, float* x0, unsigned long long* dang, const uint32_t* xperm) {
    const uint32_t v = perm ? perm[src] : src;
    *src_out = v;
    rank0[v] = 1.0f;
    x0[xperm ? xperm[v] : v] = iw[v];
    dang[0] = iw[v] == 0.0f ? (1ull << 56) : 0ull;
    dang[1] = 0ull;
    dang[2] = 0ull;
}

// Sparse steps of single-source PPR.  x is zero off the vertices its last
// step reached (x0 off src), and a row's value sums x over its in-edges, so
// a step only has to compute the rows the nonzeros of x reach (their
// out-neighbours, and src for the teleport): every other row is 0 (its rank
// and x stay 0).  A step lists those rows and folds each over all its
// in-edges while
//   - their in-edges sum below a limit and none has more than kPprRowCap
//     (a row is one warp's loop), and
//   - the vertices it expands have out-edges summing below the limit and
//     none more than kPprRowCap (checked before any is expanded, from the
//     sums the previous step took of its rows);
// once a step is not sparse every later one is a full SpMV (a sticky flag).
// The lists rotate through three buffers: F the nonzeros of x (this step's
// input), C the rows being listed (the next F), Z the nonzeros x' still
// holds from two steps ago (zeroed first; a full SpMV overwrites them all
// anyway).  No host round trip: each kernel reads the decision from the
// control words.
constexpr uint32_t kPprRowCap = 1024;

struct PprSparse {
    // [0] dense from now on, [1] this step is sparse, [2..3] in-edge sum of
    // C (u64), [4..6] list counts, [7] block ticket, [8] the max in-degree
    // in C; [12 + 4p .. 15 + 4p] for p = step parity: the out-edge sum (u64)
    // and max out-degree of the rows listed in the step of that parity
    uint32_t* ctl;
    uint32_t* bits;  // a bit per vertex: listed in this step
    uint32_t* list[3];
    const uint32_t* out_rp;
    const uint32_t* out_col;
    const uint32_t* in_rp;
    const uint32_t* xperm;  // hot-column layout: row v's x entry at xperm[v]; null: at v
    unsigned long long limit;
};

__device__ __forceinline__ uint32_t warp_max_u32(uint32_t v) { return __reduce_max_sync(0xffffffffu, v); }

// Checks the step can be sparse, zeroes x' on Z, then lists C: the
// out-neighbours of F's vertices and src, each once, with their in- and
// out-edge sums and maxima; the last block decides.
__global__ void __launch_bounds__(256)
ppr_sparse_expand_kernel(PprSparse sp, uint32_t it, const uint32_t* src_p, uint32_t n, float* x_next) {
    __shared__ unsigned long long part[8];
    __shared__ uint32_t smax[2];
    if (sp.ctl[0]) return;  // dense from now on: the same for every block
    const uint32_t fi = it % 3;
    const uint32_t src = *src_p;
    unsigned long long fout;
    uint32_t fmax;
    if (it == 0) {
        fout = fmax = sp.out_rp[src + 1] - sp.out_rp[src];
    } else {
        const uint32_t* p = sp.ctl + 12 + 4 * (it & 1u);
        fout = (unsigned long long)p[0] | ((unsigned long long)p[1] << 32);
        fmax = p[2];
    }
    if (fout >= sp.limit || fmax > kPprRowCap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sp.ctl[1] = 0u;
            sp.ctl[0] = 1u;
        }
        return;
    }
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t threads = (uint64_t)gridDim.x * blockDim.x;
    {
        const uint32_t zi = (fi + 2) % 3;
        const uint32_t nz = sp.ctl[4 + zi];
        for (uint64_t i = tid; i < nz; i += threads) {
            const uint32_t v = sp.list[zi][i];
            x_next[sp.xperm ? sp.xperm[v] : v] = 0.0f;
        }
    }
    if (threadIdx.x < 2) smax[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t* F = sp.list[fi];
    uint32_t* C = sp.list[(fi + 1) % 3];
    const uint32_t nf = sp.ctl[4 + fi];
    uint32_t* nc = &sp.ctl[4 + (fi + 1) % 3];
    unsigned long long in_sum = 0ull, out_sum = 0ull;
    uint32_t in_max = 0u, out_max = 0u;
    auto list = [&](uint32_t v) {
        const uint32_t bit = 1u << (v & 31u);
        if (atomicOr(&sp.bits[v >> 5], bit) & bit) return;
        C[atomicAdd(nc, 1u)] = v;
        const uint32_t di = sp.in_rp[v + 1] - sp.in_rp[v];
        const uint32_t dout = sp.out_rp[v + 1] - sp.out_rp[v];
        in_sum += di;
        out_sum += dout;
        in_max = max(in_max, di);
        out_max = max(out_max, dout);
    };
    if (tid == 0) list(src);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint64_t i = tid >> 5; i < nf; i += threads >> 5) {
        const uint32_t u = F[i];
        if (u >= n) continue;
        for (uint32_t k = sp.out_rp[u] + lane; k < sp.out_rp[u + 1]; k += 32) list(sp.out_col[k]);
    }
    in_max = warp_max_u32(in_max);
    out_max = warp_max_u32(out_max);
    if (lane == 0) {
        if (in_max) atomicMax(&smax[0], in_max);
        if (out_max) atomicMax(&smax[1], out_max);
    }
    const unsigned long long bin = block_sum<unsigned long long, 256>(in_sum, part);
    const unsigned long long bout = block_sum<unsigned long long, 256>(out_sum, part);
    if (threadIdx.x == 0) {
        unsigned long long* g_in = reinterpret_cast<unsigned long long*>(sp.ctl + 2);
        uint32_t* nxt = sp.ctl + 12 + 4 * ((it + 1) & 1u);
        if (bin) atomicAdd(g_in, bin);
        if (bout) atomicAdd(reinterpret_cast<unsigned long long*>(nxt), bout);
        if (smax[0]) atomicMax(&sp.ctl[8], smax[0]);
        if (smax[1]) atomicMax(&nxt[2], smax[1]);
        __threadfence();
        if (atomicAdd(&sp.ctl[7], 1u) == gridDim.x - 1) {
            // every block has listed its rows and added its sums; atomic
            // reads, as this block's L1 may hold the line from its reads of
            // ctl above
            const bool sparse = atomicAdd(g_in, 0ull) < sp.limit && atomicMax(&sp.ctl[8], 0u) <= kPprRowCap;
            sp.ctl[1] = sparse ? 1u : 0u;
            if (!sparse) sp.ctl[0] = 1u;
            sp.ctl[7] = 0u;
            __threadfence();
        }
    }
}

// The listed rows, one warp each: the sum of x over all the row's in-edges
// (each lane in edge order, four loads in flight, then a shuffle tree: a
// fixed order), then the epilogue's arithmetic (teleport at src, x', rank
// in the last step, the dangling sum); clears the rows' bits and, for the
// next step, Z's count (its C), the in-edge sum and maximum and the
// out-edge sums this step read.
__global__ void __launch_bounds__(256)
ppr_sparse_rows_kernel(PprSparse sp, uint32_t it, const uint32_t* in_col, const float* x, const float* iw,
                       const uint32_t* src_p, const unsigned long long* dang_in, unsigned long long* dang_out,
                       unsigned long long* dang_clear, double alpha, float* x_next, float* rank_next, int write_rank) {
    __shared__ alignas(16) char smem[64 * 8];
    if (!sp.ctl[1]) return;
    const uint32_t fi = it % 3;
    const uint32_t ci = (fi + 1) % 3;
    const uint32_t nc = sp.ctl[4 + ci];
    const uint32_t* C = sp.list[ci];
    const uint32_t src = *src_p;
    const float tele = (float)((1.0 - alpha) + alpha * ((double)(*dang_in) / kDangScale));
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    unsigned long long dl = 0ull;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += warps) {
        const uint32_t v = C[i];
        const uint32_t end = sp.in_rp[v + 1];
        float acc = 0.0f;
        for (uint32_t k = sp.in_rp[v] + lane; k < end; k += 128) {
            float a[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t kk = k + 32u * j;
                a[j] = kk < end ? x[in_col[kk]] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) acc += a[j];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) {
            atomicAnd(&sp.bits[v >> 5], ~(1u << (v & 31u)));
            const float r = v == src ? acc + tele : acc;
            if (write_rank) rank_next[v] = r;
            const float w = iw[v];
            if (w != 0.0f) x_next[sp.xperm ? sp.xperm[v] : v] = r * w;
            else dl += dang_fixed(r);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < 8) {
        uint32_t* cur = sp.ctl + 12 + 4 * (it & 1u);
        switch (threadIdx.x) {
            case 0: *dang_clear = 0ull; break;
            case 1: sp.ctl[4 + (fi + 2) % 3] = 0u; break;  // Z becomes the next step's C
            case 2: sp.ctl[2] = 0u; break;
            case 3: sp.ctl[3] = 0u; break;
            case 4: sp.ctl[8] = 0u; break;
            case 5: cur[0] = 0u; break;  // the next step accumulates here
            case 6: cur[1] = 0u; break;
            case 7: cur[2] = 0u; break;
        }
    }
    dang_block_add<256>(dl, dang_out, smem);
}

namespace {

constexpr size_t kPprAlign = 64;  // words (256 bytes)
size_t ppr_round(size_t w) { return (w + kPprAlign - 1) / kPprAlign * kPprAlign; }

struct PprLayout {
    unsigned long long* dang;
    uint32_t* src;
    float *iw, *rank[2], *x[2], *carry, *tail;
    uint32_t *ctl, *bits, *list[3];  // sparse steps
};

PprLayout ppr_layout(uint32_t n, const NnzPlan* plan, uint32_t* store) {
    PprLayout L;
    size_t w = 0;
    auto take = [&](size_t words) {
        uint32_t* p = store + w;
        w += ppr_round(words);
        return p;
    };
    L.dang = reinterpret_cast<unsigned long long*>(take(8));
    L.src = take(1);
    L.iw = reinterpret_cast<float*>(take(n));
    for (int i = 0; i < 2; ++i) L.rank[i] = reinterpret_cast<float*>(take(n));
    for (int i = 0; i < 2; ++i) L.x[i] = reinterpret_cast<float*>(take(n));
    const size_t nt = plan ? (size_t)plan->n_tiles + 1 : 1;
    L.carry = reinterpret_cast<float*>(take(nt));
    L.tail = reinterpret_cast<float*>(take(nt));
    L.ctl = take(32);
    L.bits = take((size_t)n / 32 + 1);
    for (int i = 0; i < 3; ++i) L.list[i] = take(n);
    return L;
}

}  // namespace

size_t ppr_state_words(uint32_t n, const NnzPlan* plan) {
    const size_t nt = plan ? (size_t)plan->n_tiles + 1 : 1;
    return ppr_round(8) + ppr_round(1) + 5 * ppr_round(n) + 2 * ppr_round(nt) + ppr_round(32) +
           ppr_round((size_t)n / 32 + 1) + 3 * ppr_round(n);
}

g1_status ppr_prepare(g1_graph* g, cudaStream_t s, PprPlan* out) {
    if (!g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "personalized PageRank needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    uint32_t* deg = nullptr;
    G1_TRY(out_degrees(g, &deg, s));
    out->deg = deg;
    out->plan = nullptr;
    // the SpMV on the hot-column copy of the in-edge CSR where it applies
    // (a graph kept in the caller's order), x by hot id
    G1_TRY(pr_hot_layout(g, deg, s, &out->t, &out->xperm));
    if (resolve_schedule(g, 1, G1_SCHED_AUTO) != G1_SCHED_VECTOR) {
        NnzPlan* p = nullptr;
        G1_TRY(ensure_nnz_plan(g, 1, &p));
        out->plan = p;
    }
    out->words = ppr_state_words(g->n, out->plan);
    // sparse steps need the out-edges (the in-edge CSR itself when symmetric),
    // on graphs of 2^20 edges or more (below, a full SpMV costs a few
    // microseconds); the limit on the listed rows' in-edges is m / push_div,
    // the BLAS traversal loop's threshold
    out->out_rp = g->o[0].present ? g->o[0].rp : (g->symmetric ? g->o[1].rp : nullptr);
    out->out_col = g->o[0].present ? g->o[0].col : (g->symmetric ? g->o[1].col : nullptr);
    out->sparse_limit = out->out_rp && g->m >= (1u << 20)
                            ? (unsigned long long)g->m / std::max<uint32_t>(1, g->push_div)
                            : 0ull;
    // with rows or out-lists longer than kPprRowCap (hubs), a query reaches
    // one within a step or two and runs dense from there: its sparse
    // kernels are launched for the first three steps only
    const uint32_t out_max = g->o[0].present ? g->o[0].max_deg : g->o[1].max_deg;
    out->sparse_steps = std::max(g->o[1].max_deg, out_max) > kPprRowCap ? 3u : UINT32_MAX;
    return G1_OK;
}

g1_status ppr_enqueue(g1_graph* g, const PprPlan& pl, uint32_t* store, uint32_t src, float alpha,
                      uint32_t iters, const uint32_t* perm, cudaStream_t s, const float** rank_out) {
    const uint32_t n = g->n;
    const int t = pl.t;  // 1, or the hot-column copy 2 (same rows, plans and values)
    const PprLayout L = ppr_layout(n, pl.plan, store);
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
    ppr_iw_kernel<<<grid, 256, 0, s>>>(pl.deg, n, (double)alpha, L.iw);
    G1_CUDA(cudaMemsetAsync(L.x[0], 0, (size_t)n * 4, s));
    G1_CUDA(cudaMemsetAsync(L.x[1], 0, (size_t)n * 4, s));
    if (iters == 0) G1_CUDA(cudaMemsetAsync(L.rank[0], 0, (size_t)n * 4, s));
    ppr_init_kernel<<<1, 1, 0, s>>>(perm, src, L.iw, L.src, L.rank[0], L.x[0], L.dang, pl.xperm);
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    PprSparse sp{};
    const bool sparse = pl.sparse_limit != 0;
    if (sparse) {
        sp.ctl = L.ctl;
        sp.bits = L.bits;
        for (int i = 0; i < 3; ++i) sp.list[i] = L.list[i];
        sp.out_rp = pl.out_rp;
        sp.out_col = pl.out_col;
        sp.in_rp = g->o[t].rp;
        sp.xperm = pl.xperm;
        sp.limit = pl.sparse_limit;
        // F0 = {src} (ctl[4] = 1), the other counts, sums, flags and bits zero
        G1_CUDA(cudaMemsetAsync(L.ctl, 0, 32 * 4, s));
        G1_CUDA(cudaMemsetAsync(L.bits, 0, ((size_t)n / 32 + 1) * 4, s));
        G1_CUDA(cudaMemcpyAsync(L.list[0], L.src, 4, cudaMemcpyDeviceToDevice, s));
        G1_TRY(g1_mem_fill_u32(L.ctl + 4, 1u, 1, s));
    }
    const uint32_t sgrid = (uint32_t)g->sm_count * 2;
    for (uint32_t it = 0; it < iters; ++it) {
        const bool last = it + 1 == iters;
        const int cur = it & 1, nxt = cur ^ 1;
        const bool sparse_it = sparse && it < pl.sparse_steps;
        if (sparse_it) {
            // a sparse last step writes only its rows' ranks
            if (last) G1_CUDA(cudaMemsetAsync(L.rank[nxt], 0, (size_t)n * 4, s));
            ppr_sparse_expand_kernel<<<sgrid, 256, 0, s>>>(sp, it, L.src, n, L.x[nxt]);
            ppr_sparse_rows_kernel<<<sgrid, 256, 0, s>>>(sp, it, g->o[t].col, L.x[cur], L.iw, L.src,
                                                         &L.dang[it % 3], &L.dang[(it + 1) % 3],
                                                         &L.dang[(it + 2) % 3], (double)alpha, L.x[nxt],
                                                         L.rank[nxt], last ? 1 : 0);
            count_launches(2);
            G1_CUDA(cudaGetLastError());
        }
        PprEpilogue e;
        e.rank_next = L.rank[nxt];
        e.x_next = L.x[nxt];
        e.iw = L.iw;
        e.src_p = L.src;
        e.dang_in = &L.dang[it % 3];
        e.dang_out = &L.dang[(it + 1) % 3];
        e.dang_clear = &L.dang[(it + 2) % 3];
        e.alpha = (double)alpha;
        e.write_rank = last ? 1 : 0;
        e.sparse_now = sparse_it ? L.ctl + 1 : nullptr;
        e.xperm = pl.xperm;
        if (!pl.plan) {
            G1_TRY((launch_vector<PlusPatternF32>(g, t, L.x[cur], e, s)));
            continue;
        }
        PprEpilogue f = e;
        f.dang_clear = nullptr;
        if (!last) {
            f.empty_list = L.src;  // never read: the list is empty
            f.n_empty_list = 0;
            f.src_rows = g->o[t].rp;
        }
        G1_TRY((launch_nnz<PlusPatternF32, PprEpilogue, 32, 1, 32768>(g, t, *pl.plan, L.x[cur], e, f, s,
                                                                      L.carry, L.tail)));
    }
    *rank_out = L.rank[iters & 1];
    return G1_OK;
}

}  // namespace g1

using namespace g1;

extern "C" g1_status g1_graph_set_hot_columns(g1_graph* g, g1_hot_columns mode) {
    if (!g || (mode != G1_HOT_COLUMNS_AUTO && mode != G1_HOT_COLUMNS_OFF && mode != G1_HOT_COLUMNS_ON))
        return fail(G1_ERR_INVALID, "g1_graph_set_hot_columns: bad argument");
    std::lock_guard<std::mutex> lk(g->mu);
    g->hot_mode = mode;
    return G1_OK;
}

extern "C" g1_status g1_pagerank(g1_graph* g, float alpha, int iters, g1_pr_mode mode,
                                 float* rank_out, void* stream) {
    if (!g || !rank_out || iters < 0) return fail(G1_ERR_INVALID, "g1_pagerank: bad argument");
    if (g->vtype != G1_F32) return fail(G1_ERR_INVALID, "g1_pagerank: needs fp32 edge values");
    if (mode != G1_PR_REFERENCE && mode != G1_PR_DANGLING)
        return fail(G1_ERR_INVALID, "g1_pagerank: unknown mode");
    if (!g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "g1_pagerank: needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (g->n == 0) return G1_OK;
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStream_t s = as_stream(stream);
    PrBuffers b;
    uint32_t grids[4];
    G1_TRY(pr_setup(g, alpha, b, grids, s));
    for (int it = 0; it < iters; ++it)
        G1_TRY(pr_iterate(g, b, grids, alpha, mode, it, iters, G1_SCHED_AUTO, s));
    G1_TRY(copy_out_vertices(g, rank_out, b.rank[iters & 1], s));
    return check_device_error(g, s);
}

namespace g1 {

g1_status ppr_locked(g1_graph* g, uint32_t src, float alpha, uint32_t iters, float* rank_out,
                     cudaStream_t s) {
    if (src >= g->n) return fail(G1_ERR_INVALID, "source vertex out of range");
    PprPlan pl;
    G1_TRY(ppr_prepare(g, s, &pl));
    uint32_t* store = nullptr;
    G1_TRY(g->ws.get("ppr_store", pl.words, &store));
    const float* rank = nullptr;
    const uint32_t* perm = g->relabeled ? g->perm.as<uint32_t>() : nullptr;
    G1_TRY(ppr_enqueue(g, pl, store, src, alpha, iters, perm, s, &rank));
    G1_TRY(copy_out_vertices(g, rank_out, rank, s));
    return check_device_error(g, s);
}

}  // namespace g1

extern "C" g1_status g1_ppr(g1_graph* g, uint32_t src, float alpha, uint32_t iters, float* rank_out,
                            void* stream) {
    if (!g || !rank_out) return fail(G1_ERR_INVALID, "g1_ppr: bad argument");
    if (!(alpha > 0.0f && alpha < 1.0f))
        return fail(G1_ERR_INVALID, "personalized PageRank: damping must be in (0, 1)");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    return ppr_locked(g, src, alpha, iters, rank_out, as_stream(stream));
}
