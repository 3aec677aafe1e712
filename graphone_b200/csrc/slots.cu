// Slot engine: multi-source BFS / SSSP / personalized PageRank with
// per-source slots that are admitted and retired between iterations.
//
// Each iteration is one pull over the in-edge CSR, cut into row pieces of at
// most kPieceEdges edges (one warp each):
//   BFS : lanes = (neighbour, word); OR of the in-neighbours' frontier rows,
//         new = that & ~seen; levels of new bits are stored row-wise;
//   SSSP: lane l owns slots 32j + l; for every in-neighbour whose changed row
//         has a bit in word j the warp reads 128 bytes of its distance row
//         and relaxes min(dist + w) in registers; improvements set changed
//         bits for the next iteration;
//   PPR : lane l accumulates slots 32j + l over the row's in-edges,
//         rank'[v] = sum rank[u] * alpha / outdeg(u); hub rows (several
//         pieces) are summed from per-piece partials in piece order, then
//         the teleport (1 - alpha) and the dangling mass alpha * sum of the
//         ranks of out-degree-0 vertices go to each slot's source.
// The frontier / changed bit rows are triple-buffered: iteration i reads
// buffer i, fills buffer i+1 and clears buffer i+2, so no buffer is memset
// between iterations.  BFS / SSSP iterations are dense (every row piece) or
// sparse (only the pieces of vertices with an in-neighbour changed by the
// previous iteration, listed by that iteration through the out-edges while
// few vertices change -- the push/pull switch of a frontier engine).  A
// dense iteration clears buffer i+2 through the first piece of every row, a
// sparse one through the list of vertices changed in iteration i-2.  The
// slots that changed in iteration i are OR-ed into one of two 8-word arrays;
// the host reads the last one after a step.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "g1/common.cuh"
#include "internal.h"
#include "slots.cuh"

namespace g1 {

// ------------------------------------------------------- per-graph arrays

// Pieces per vertex: max(1, ceil(deg / kPieceEdges)).
__global__ void piece_count_kernel(const uint32_t* rp, uint32_t n, uint32_t* cnt) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint32_t d = rp[v + 1] - rp[v];
        cnt[v] = d == 0 ? 1u : (d + kPieceEdges - 1) / kPieceEdges;
    }
}

__global__ void piece_fill_kernel(const uint32_t* rp, uint32_t n, const uint32_t* off,
                                  uint32_t* piece_v, uint32_t* piece_e) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint32_t rs = rp[v], re = rp[v + 1];
        uint32_t p = off[v];
        uint32_t e = rs;
        do {
            piece_v[p] = (uint32_t)v;
            piece_e[p] = e;
            ++p;
            e += kPieceEdges;
        } while (e < re);
    }
}

// Hub rows: flag and piece count of every row with more than one piece.
__global__ void hub_flag_kernel(const uint32_t* rp, uint32_t n, uint32_t* flag, uint32_t* pieces) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint32_t d = rp[v + 1] - rp[v];
        const bool hub = d > kPieceEdges;
        flag[v] = hub ? 1u : 0u;
        pieces[v] = hub ? (d + kPieceEdges - 1) / kPieceEdges : 0u;
    }
}

__global__ void hub_fill_kernel(const uint32_t* rp, uint32_t n, const uint32_t* piece_off,
                                const uint32_t* hub_idx, const uint32_t* hp0, uint32_t* hub_v,
                                uint32_t* hub_hp, uint32_t* piece_hp) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint32_t d = rp[v + 1] - rp[v];
        const uint32_t p0 = piece_off[v];
        if (d > kPieceEdges) {
            const uint32_t h = hub_idx[v];
            hub_v[h] = (uint32_t)v;
            hub_hp[h] = hp0[v];
            const uint32_t cnt = (d + kPieceEdges - 1) / kPieceEdges;
            for (uint32_t i = 0; i < cnt; ++i) piece_hp[p0 + i] = hp0[v] + i;
        } else {
            piece_hp[p0] = kU32Max;
        }
    }
}

__global__ void out_degree_from_csr_kernel(const uint32_t* rp, uint32_t n, uint32_t* deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        deg[v] = rp[v + 1] - rp[v];
}

__global__ void out_degree_from_transpose_kernel(const uint32_t* col, uint32_t m, uint32_t* deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride)
        atomicAdd(&deg[col[e]], 1u);
}

namespace {

uint32_t grid_for(const g1_graph* g, uint64_t n) {
    return (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 16));
}

g1_status exclusive_scan(uint32_t* in, uint32_t* out, uint32_t count, cudaStream_t s) {
    size_t tb = 0;
    G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)count, s));
    DevBuf temp;
    G1_TRY(temp.ensure(tb + 16));
    G1_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, in, out, (int)count, s));
    G1_CUDA(cudaStreamSynchronize(s));  // temp is freed on return
    return G1_OK;
}

g1_status read_u32(const uint32_t* dev, uint32_t* out, cudaStream_t s) {
    G1_CUDA(cudaMemcpyAsync(out, dev, 4, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    return G1_OK;
}

}  // namespace

g1_status out_degrees(g1_graph* g, uint32_t** deg, cudaStream_t s) {
    const uint32_t n = g->n;
    G1_TRY(g->ws.get("slot_outdeg", (size_t)n + 1, deg));
    if (!g->outdeg_ready) {
        if (g->o[0].present) {
            out_degree_from_csr_kernel<<<grid_for(g, n), 256, 0, s>>>(g->o[0].rp, n, *deg);
        } else {
            G1_CUDA(cudaMemsetAsync(*deg, 0, (size_t)n * 4, s));
            out_degree_from_transpose_kernel<<<grid_for(g, g->m), 256, 0, s>>>(g->o[1].col, g->m, *deg);
        }
        count_launches(1);
        G1_CUDA(cudaGetLastError());
        G1_CUDA(cudaStreamSynchronize(s));
        g->outdeg_ready = true;
    }
    return G1_OK;
}

g1_status slot_graph(g1_graph* g, int kind, cudaStream_t s, SlotGraph* out) {
    if (!g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "multi-source traversal needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (kind == kSlotSssp && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
    Workspace& ws = g->ws;
    const uint32_t n = g->n;
    const Orientation& o = g->o[1];
    const uint32_t grid = grid_for(g, n);
    uint32_t *cnt = nullptr, *off = nullptr, *piece_v = nullptr, *piece_e = nullptr;
    G1_TRY(ws.get("pc_off", (size_t)n + 1, &off));
    if (!g->pieces_ready) {
        G1_TRY(ws.get("pc_cnt", (size_t)n + 1, &cnt));
        piece_count_kernel<<<grid, 256, 0, s>>>(o.rp, n, cnt);
        G1_CUDA(cudaMemsetAsync(cnt + n, 0, 4, s));
        G1_TRY(exclusive_scan(cnt, off, n + 1, s));
        uint32_t h = 0;
        G1_TRY(read_u32(off + n, &h, s));
        G1_TRY(ws.get("pc_v", (size_t)h + 1, &piece_v));
        G1_TRY(ws.get("pc_e", (size_t)h + 1, &piece_e));
        piece_fill_kernel<<<grid, 256, 0, s>>>(o.rp, n, off, piece_v, piece_e);
        count_launches(2);
        G1_CUDA(cudaGetLastError());
        G1_CUDA(cudaStreamSynchronize(s));
        g->n_pieces = h;
        g->pieces_ready = true;
    }
    G1_TRY(ws.get("pc_v", (size_t)g->n_pieces + 1, &piece_v));
    G1_TRY(ws.get("pc_e", (size_t)g->n_pieces + 1, &piece_e));
    SlotGraph sg;
    sg.rp = o.rp;
    sg.col = o.col;
    sg.val = g->vtype == G1_U32 ? static_cast<const uint32_t*>(o.val) : nullptr;
    sg.piece_v = piece_v;
    sg.piece_e = piece_e;
    sg.piece_off = off;
    // out-edges list the next iteration's rows; a symmetric graph's in-edge
    // CSR is its out-edge CSR
    const Orientation* out_o = g->o[0].present ? &g->o[0] : (g->symmetric ? &g->o[1] : nullptr);
    sg.out_rp = out_o ? out_o->rp : nullptr;
    sg.out_col = out_o ? out_o->col : nullptr;
    sg.n = n;
    sg.m = g->m;
    sg.n_pieces = g->n_pieces;
    sg.sm_count = g->sm_count;
    sg.perm = g->relabeled ? g->perm.as<uint32_t>() : nullptr;
    sg.sparse_div = g->slot_div;
    if (kind == kSlotPpr) {
        uint32_t *flag = nullptr, *hpc = nullptr, *hidx = nullptr, *hp0 = nullptr, *hub_v = nullptr,
                 *hub_hp = nullptr, *piece_hp = nullptr, *deg = nullptr;
        if (!g->hubs_ready) {
            G1_TRY(ws.get("hub_flag", (size_t)n + 1, &flag));
            G1_TRY(ws.get("hub_pcs", (size_t)n + 1, &hpc));
            G1_TRY(ws.get("hub_idx", (size_t)n + 1, &hidx));
            G1_TRY(ws.get("hub_hp0", (size_t)n + 1, &hp0));
            hub_flag_kernel<<<grid, 256, 0, s>>>(o.rp, n, flag, hpc);
            G1_CUDA(cudaMemsetAsync(flag + n, 0, 4, s));
            G1_CUDA(cudaMemsetAsync(hpc + n, 0, 4, s));
            G1_TRY(exclusive_scan(flag, hidx, n + 1, s));
            G1_TRY(exclusive_scan(hpc, hp0, n + 1, s));
            uint32_t nh = 0, nhp = 0;
            G1_TRY(read_u32(hidx + n, &nh, s));
            G1_TRY(read_u32(hp0 + n, &nhp, s));
            G1_TRY(ws.get("hub_v", (size_t)nh + 1, &hub_v));
            G1_TRY(ws.get("hub_hp", (size_t)nh + 1, &hub_hp));
            G1_TRY(ws.get("piece_hp", (size_t)g->n_pieces + 1, &piece_hp));
            hub_fill_kernel<<<grid, 256, 0, s>>>(o.rp, n, off, hidx, hp0, hub_v, hub_hp, piece_hp);
            count_launches(2);
            G1_CUDA(cudaGetLastError());
            G1_CUDA(cudaStreamSynchronize(s));
            g->n_hubs = nh;
            g->n_hub_pieces = nhp;
            g->hubs_ready = true;
        }
        G1_TRY(ws.get("hub_v", (size_t)g->n_hubs + 1, &hub_v));
        G1_TRY(ws.get("hub_hp", (size_t)g->n_hubs + 1, &hub_hp));
        G1_TRY(ws.get("piece_hp", (size_t)g->n_pieces + 1, &piece_hp));
        G1_TRY(out_degrees(g, &deg, s));
        sg.hub_v = hub_v;
        sg.hub_hp = hub_hp;
        sg.piece_hp = piece_hp;
        sg.out_deg = deg;
        sg.n_hubs = g->n_hubs;
        sg.n_hub_pieces = g->n_hub_pieces;
    }
    *out = sg;
    return G1_OK;
}

// ------------------------------------------------------------- iteration

// Frontier state of one BFS / SSSP iteration `it` (all rotating buffers
// already resolved by the host).  ctr holds 4 groups of 4 words; group
// x % 4 describes what iteration x - 1 left for iteration x:
//   [0] row pieces in iteration x's list,
//   [1] iteration x - 1 built that list and recorded its changed vertices,
//   [2] how many changed vertices it recorded,
//   [3] sum of (out-degree + 1) over the vertices it changed.
//
// The iteration number is it + *it_base when it_base is set: a step
// captured in a CUDA graph bakes in offsets and the buffers of its rotation
// phase, and reads the iterations completed before it from the device.
struct Frontier {
    uint32_t* mark;             // n: iteration a vertex was listed for
    const uint32_t* plist_in;   // this iteration's row pieces (when valid)
    uint32_t* plist_out;        // the next iteration's row pieces
    uint32_t* clist_out;        // vertices this iteration changes
    const uint32_t* clist_old;  // vertices changed two iterations ago
    uint32_t* ctr;
    const uint32_t* it_base;    // device word added to `it`, or null
    uint32_t it;
    uint32_t thresh;  // the next list is built while the changed degree sum is below
};

__device__ __forceinline__ uint32_t frontier_iter(const Frontier& f) {
    return f.it + (f.it_base ? *f.it_base : 0u);
}

// Bit j: word j of the occupied slots (device words) is not empty.
__device__ __forceinline__ uint32_t occ_word_mask(const uint32_t* occ, uint32_t W) {
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if ((uint32_t)j < W && __ldg(occ + j) != 0u) m |= 1u << j;
    return m;
}

struct IterCtl {
    bool dense;      // pull every row piece
    bool mark;       // build the next iteration's list
    uint32_t total;  // pieces to pull
    uint32_t* cout;  // the next iteration's counters
};

// Reads this iteration's counters, zeroes the group two ahead and, in a
// sparse iteration, clears the bit rows of the vertices changed two
// iterations ago (a dense iteration clears every row through the first
// piece of each vertex instead).  An iteration is sparse only when the
// previous one listed its pieces and the one before recorded its changed
// vertices; it builds the next list only while few edges leave the
// vertices the previous iteration changed.
__device__ __forceinline__ IterCtl iter_begin(const SlotGraph& sg, const Frontier& f, uint32_t it,
                                              uint32_t W, uint32_t* clear) {
    const uint32_t* cin = f.ctr + 4 * (it & 3u);
    uint32_t* cout = f.ctr + 4 * ((it + 1) & 3u);
    uint32_t* cz = f.ctr + 4 * ((it + 2) & 3u);
    const uint32_t* cold = f.ctr + 4 * ((it + 3) & 3u);
    IterCtl c;
    c.dense = cin[1] == 0u || cold[1] == 0u;
    c.mark = sg.out_rp != nullptr && cin[3] < f.thresh;
    c.total = c.dense ? sg.n_pieces : cin[0];
    c.cout = cout;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cz[0] = cz[1] = cz[2] = cz[3] = 0u;
        cout[1] = c.mark ? 1u : 0u;
    }
    if (!c.dense) {
        const uint64_t tot = (uint64_t)cold[2] * W;
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += stride)
            clear[(size_t)f.clist_old[i / W] * W + i % W] = 0u;
    }
    return c;
}

// Appends the row pieces of v's out-neighbours not yet listed for
// iteration `tag` to `list` (count *cnt).  Warp-uniform call.
__device__ void list_out_neighbours(const SlotGraph& sg, uint32_t* mark, uint32_t tag, uint32_t* list,
                                    uint32_t* cnt, uint32_t v) {
    const uint32_t lane = lane_id();
    const uint32_t os = sg.out_rp[v], oe = sg.out_rp[v + 1];
    for (uint32_t e0 = os; e0 < oe; e0 += 32) {
        const uint32_t e = e0 + lane;
        uint32_t np = 0, first = 0;
        if (e < oe) {
            const uint32_t w = __ldg(sg.out_col + e);
            if (mark[w] != tag && atomicExch(&mark[w], tag) != tag) {
                first = sg.piece_off[w];
                np = sg.piece_off[w + 1] - first;
            }
        }
        uint32_t incl = np;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (total == 0) continue;
        uint32_t base = 0;
        if (lane == 31) base = atomicAdd(cnt, total);
        base = __shfl_sync(0xffffffffu, base, 31);
        for (uint32_t k = 0; k < np; ++k) list[base + incl - np + k] = first + k;
    }
}

// v changed in this iteration (warp-uniform call): its out-degree joins the
// warp's total; while the next list is built it is recorded for the
// clearing two iterations on and its out-neighbours are listed.
__device__ __forceinline__ void note_changed(const SlotGraph& sg, const Frontier& f, uint32_t it,
                                             const IterCtl& c, uint32_t v, uint32_t& deg_acc) {
    deg_acc += 1u + (sg.out_rp ? sg.out_rp[v + 1] - sg.out_rp[v] : 0u);
    if (!c.mark) return;
    if (lane_id() == 0) f.clist_out[atomicAdd(&c.cout[2], 1u)] = v;
    list_out_neighbours(sg, f.mark, it + 1, f.plist_out, &c.cout[0], v);
}

__device__ __forceinline__ void iter_end(const IterCtl& c, uint32_t deg_acc) {
    if (lane_id() == 0 && deg_acc) atomicAdd(&c.cout[3], deg_acc);
}

template <int WP>  // words per vertex rounded up to a power of two (1..8)
__global__ void __launch_bounds__(256)
slot_bfs_kernel(SlotGraph sg, Frontier f, uint32_t W, uint32_t K, const uint32_t* occ, const uint32_t* front,
                uint32_t* seen, uint32_t* next, uint32_t* clear, uint32_t* lv, const uint32_t* start,
                uint32_t* chw, uint32_t* chw_clear) {
    constexpr int SLOTS = 32 / WP;  // neighbours per warp step
    const uint32_t lane = lane_id();
    const uint32_t w = lane % WP, q = lane / WP;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t it = frontier_iter(f);
    const uint32_t depth = it;
    if (blockIdx.x == 0 && threadIdx.x < 8) chw_clear[threadIdx.x] = 0u;
    const IterCtl c = iter_begin(sg, f, it, W, clear);
    const bool has_word = w < W;
    const uint32_t lw = has_word ? __ldg(occ + w) : 0u;
    uint32_t new_acc = 0, deg_acc = 0;
    for (uint32_t idx = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; idx < c.total; idx += warps) {
        const uint32_t p = c.dense ? idx : f.plist_in[idx];
        const uint32_t v = sg.piece_v[p];
        const uint32_t rs = sg.rp[v], re = sg.rp[v + 1];
        const bool multi = re - rs > kPieceEdges;
        const uint32_t e0 = sg.piece_e[p], e1 = min(e0 + kPieceEdges, re);
        if (c.dense && e0 == rs && q == 0 && has_word) clear[(size_t)v * W + w] = 0u;
        uint32_t raw = 0, sn = 0xffffffffu;  // seen, with the bits of idle slots set
        if (has_word) {
            raw = seen[(size_t)v * W + w];
            sn = raw | ~lw;
        }
        if (__all_sync(0xffffffffu, sn == 0xffffffffu)) continue;
        uint32_t acc = 0;
        if (sn != 0xffffffffu) {
            for (uint32_t e = e0 + q; e < e1; e += SLOTS) {
                const uint32_t u = __ldg(sg.col + e);
                acc |= __ldg(front + (size_t)u * W + w);
            }
        }
#pragma unroll
        for (int off = WP; off < 32; off <<= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, off);
        uint32_t nw = acc & ~sn;
        if (has_word && q == 0 && nw) {
            if (multi) {
                // several pieces of this row: keep the bits first claimed here
                nw &= ~atomicOr(&seen[(size_t)v * W + w], nw);
                if (nw) atomicOr(&next[(size_t)v * W + w], nw);
            } else {
                next[(size_t)v * W + w] = nw;
                seen[(size_t)v * W + w] = raw | nw;
            }
            new_acc |= nw;
        }
        bool any_new = false;
        for (uint32_t j = 0; j < W; ++j) {
            const uint32_t bits = __shfl_sync(0xffffffffu, nw, (int)j);
            if (bits == 0) continue;
            any_new = true;
            const uint32_t s = 32 * j + lane;
            if ((bits >> lane) & 1u) lv[(size_t)v * K + s] = depth - __ldg(start + s);
        }
        if (any_new) note_changed(sg, f, it, c, v, deg_acc);
    }
    iter_end(c, deg_acc);
    if (q == 0 && has_word && new_acc) atomicOr(&chw[w], new_acc);
}

__global__ void __launch_bounds__(256)
slot_sssp_kernel(SlotGraph sg, Frontier f, uint32_t W, uint32_t K, const uint32_t* occ, uint32_t* dist,
                 const uint32_t* chg, uint32_t* chg_next, uint32_t* clear, uint32_t* chw,
                 uint32_t* chw_clear) {
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t it = frontier_iter(f);
    const uint32_t wmask = occ_word_mask(occ, W);
    if (blockIdx.x == 0 && threadIdx.x < 8) chw_clear[threadIdx.x] = 0u;
    const IterCtl c = iter_begin(sg, f, it, W, clear);
    const bool my_word = lane < W && ((wmask >> lane) & 1u);
    uint32_t deg_acc = 0;
    uint32_t changed[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) changed[j] = 0u;
    for (uint32_t idx = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; idx < c.total; idx += warps) {
        const uint32_t p = c.dense ? idx : f.plist_in[idx];
        const uint32_t v = sg.piece_v[p];
        const uint32_t rs = sg.rp[v], re = sg.rp[v + 1];
        const bool multi = re - rs > kPieceEdges;
        const uint32_t e0 = sg.piece_e[p], e1 = min(e0 + kPieceEdges, re);
        if (c.dense && e0 == rs && lane < W) clear[(size_t)v * W + lane] = 0u;
        uint32_t best[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) best[j] = kU32Max;
        for (uint32_t c0 = e0; c0 < e1; c0 += 32) {
            // 32 in-edges at a time: lane t holds edge c0 + t and the changed
            // row of its source (W <= 8 words, one 32-byte sector)
            const uint32_t ec = c0 + lane;
            const bool valid = ec < e1;
            const uint32_t cu = valid ? __ldg(sg.col + ec) : 0u;
            const uint32_t cw = valid ? __ldg(sg.val + ec) : 0u;
            const uint32_t* cr = chg + (size_t)cu * W;
            uint32_t m[8];
            uint32_t wm = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                m[j] = (valid && (uint32_t)j < W && ((wmask >> j) & 1u)) ? __ldg(cr + j) : 0u;
                wm |= (m[j] != 0u ? 1u : 0u) << j;
            }
            // edges whose source changed, two at a time so that both
            // sources' distance rows are in flight together
            unsigned todo = __ballot_sync(0xffffffffu, wm != 0u);
            while (todo) {
                const int ta = __ffs(todo) - 1;
                todo &= todo - 1;
                const bool two = todo != 0u;
                const int tb = two ? __ffs(todo) - 1 : ta;
                if (two) todo &= todo - 1;
                const uint32_t ua = __shfl_sync(0xffffffffu, cu, ta);
                const uint32_t ub = __shfl_sync(0xffffffffu, cu, tb);
                const uint32_t wa = __shfl_sync(0xffffffffu, cw, ta);
                const uint32_t wb = __shfl_sync(0xffffffffu, cw, tb);
                const uint32_t ma = __shfl_sync(0xffffffffu, wm, ta);
                const uint32_t mb = two ? __shfl_sync(0xffffffffu, wm, tb) : 0u;
                const uint32_t* da = dist + (size_t)ua * K + lane;
                const uint32_t* db = dist + (size_t)ub * K + lane;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t ba = __shfl_sync(0xffffffffu, m[j], ta);
                    const uint32_t bb = __shfl_sync(0xffffffffu, m[j], tb);
                    // a changed entry is finite: the sum cannot wrap for
                    // distances below 2^32 - max weight
                    uint32_t xa = kU32Max, xb = kU32Max;
                    if (((ma >> j) & 1u) && ((ba >> lane) & 1u)) xa = da[32 * j] + wa;
                    if (((mb >> j) & 1u) && ((bb >> lane) & 1u)) xb = db[32 * j] + wb;
                    best[j] = min(best[j], min(xa, xb));
                }
            }
        }
        uint32_t* dv = dist + (size_t)v * K;
        uint32_t vbits = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if ((uint32_t)j >= W) break;
            const uint32_t s = 32 * j + lane;
            bool imp = false;
            if (best[j] != kU32Max) {
                if (multi) {
                    imp = best[j] < atomicMin(&dv[s], best[j]);
                } else {
                    const uint32_t old = dv[s];
                    if (best[j] < old) {
                        dv[s] = best[j];
                        imp = true;
                    }
                }
            }
            const unsigned bits = __ballot_sync(0xffffffffu, imp);
            if (lane == 0 && bits) {
                if (multi)
                    atomicOr(&chg_next[(size_t)v * W + j], bits);
                else
                    chg_next[(size_t)v * W + j] = bits;
            }
            changed[j] |= bits;
            vbits |= bits;
        }
        if (vbits) note_changed(sg, f, it, c, v, deg_acc);
    }
    iter_end(c, deg_acc);
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (lane == (uint32_t)j && changed[j]) atomicOr(&chw[j], changed[j]);
}

// rank' = A^T (rank * iw) over the row's in-edges; hub rows go to
// per-piece partials; per-warp dangling partial sums of the current rank.
__global__ void __launch_bounds__(256)
slot_ppr_pull_kernel(SlotGraph sg, uint32_t W, uint32_t K, const uint32_t* occ, const float* iw,
                     const float* rank, float* rank_next, float* hub_part, float* dang_part) {
    const uint32_t wmask = occ_word_mask(occ, W);
    const uint32_t lane = lane_id();
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    float dang[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) dang[j] = 0.0f;
    for (uint32_t p = gw; p < sg.n_pieces; p += warps) {
        const uint32_t v = sg.piece_v[p];
        const uint32_t rs = sg.rp[v], re = sg.rp[v + 1];
        const uint32_t e0 = sg.piece_e[p], e1 = min(e0 + kPieceEdges, re);
        float acc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = 0.0f;
        for (uint32_t c0 = e0; c0 < e1; c0 += 32) {
            const uint32_t ec = c0 + lane;
            const uint32_t cu = ec < e1 ? __ldg(sg.col + ec) : 0u;
            const float cf = ec < e1 ? __ldg(iw + cu) : 0.0f;
            const uint32_t ne = min(32u, e1 - c0);
#pragma unroll 4
            for (uint32_t t = 0; t < ne; ++t) {
                const uint32_t u = __shfl_sync(0xffffffffu, cu, (int)t);
                const float f = __shfl_sync(0xffffffffu, cf, (int)t);
                const float* ru = rank + (size_t)u * K + lane;
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if ((uint32_t)j < W && ((wmask >> j) & 1u)) acc[j] = fmaf(__ldg(ru + 32 * j), f, acc[j]);
            }
        }
        const uint32_t hp = sg.piece_hp[p];
        float* dst = hp == kU32Max ? rank_next + (size_t)v * K : hub_part + (size_t)hp * K;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if ((uint32_t)j < W && ((wmask >> j) & 1u)) dst[32 * j + lane] = acc[j];
        if (e0 == rs && __ldg(sg.out_deg + v) == 0u) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if ((uint32_t)j < W && ((wmask >> j) & 1u)) dang[j] += rank[(size_t)v * K + 32 * j + lane];
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if ((uint32_t)j < W && ((wmask >> j) & 1u)) dang_part[(size_t)gw * K + 32 * j + lane] = dang[j];
}

// Hub rows: sum of their pieces' partials in piece order.
__global__ void __launch_bounds__(256)
slot_ppr_hub_kernel(SlotGraph sg, uint32_t W, uint32_t K, const uint32_t* occ, const float* hub_part,
                    float* rank_next) {
    const uint32_t wmask = occ_word_mask(occ, W);
    const uint32_t t = threadIdx.x;
    if (t >= K || !((wmask >> (t >> 5)) & 1u)) return;
    for (uint32_t h = blockIdx.x; h < sg.n_hubs; h += gridDim.x) {
        const uint32_t v = sg.hub_v[h], hp = sg.hub_hp[h];
        const uint32_t d = sg.rp[v + 1] - sg.rp[v];
        const uint32_t cnt = (d + kPieceEdges - 1) / kPieceEdges;
        float s = 0.0f;
        for (uint32_t i = 0; i < cnt; ++i) s += hub_part[(size_t)(hp + i) * K + t];
        rank_next[(size_t)v * K + t] = s;
    }
}

// One block per slot: the dangling mass (per-warp partials folded in a
// fixed order) and the teleport go to the slot's source.
__global__ void __launch_bounds__(256)
slot_ppr_teleport_kernel(uint32_t K, const uint32_t* occ, const uint32_t* slot_src, const float* dang_part,
                         uint32_t n_warps, double alpha, float* rank_next) {
    __shared__ double red[8];
    const uint32_t s = blockIdx.x;
    if (s >= K || !((__ldg(occ + (s >> 5)) >> (s & 31)) & 1u)) return;
    double d = 0.0;
    for (uint32_t i = threadIdx.x; i < n_warps; i += blockDim.x) d += (double)dang_part[(size_t)i * K + s];
    d = block_sum<double, 256>(d, red);
    if (threadIdx.x == 0) {
        const uint32_t v = slot_src[s];
        rank_next[(size_t)v * K + s] += (float)((1.0 - alpha) + alpha * d);
    }
}

// The last node of a captured step: the step's iterations are done.
__global__ void slot_it_advance_kernel(uint32_t* it_base, uint32_t n) { *it_base += n; }

// The occupied slots, by value into the device words the kernels read.
__global__ void slot_set_occ_kernel(uint32_t* occ, Bits256 b) {
    if (threadIdx.x < 8) occ[threadIdx.x] = b.w[threadIdx.x];
}

__global__ void slot_ppr_iw_kernel(const uint32_t* deg, uint32_t n, double alpha, float* iw) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        iw[v] = deg[v] ? (float)(alpha / (double)deg[v]) : 0.0f;
}

// ------------------------------------------------------------- admission

// Resets the admitted slots' columns to `init` and (BFS) their seen bits.
__global__ void slot_reset_kernel(uint32_t n, uint32_t K, uint32_t W, uint32_t cnt,
                                  const uint32_t* slots, uint32_t init, uint32_t* rows,
                                  uint32_t* seen, Bits256 amask) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t total = (uint64_t)n * cnt;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const uint64_t v = i / cnt;
        const uint32_t c = (uint32_t)(i - v * cnt);
        rows[v * K + slots[c]] = init;
    }
    if (seen) {
        const uint64_t nw = (uint64_t)n * W;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += stride) {
            const uint32_t m = amask.w[i % W];
            if (m) seen[i] &= ~m;
        }
    }
}

// One warp per admitted source.  BFS / SSSP seeds also enter the frontier
// state of the next iteration (it + 1): the source counts as changed by
// iteration it, and its out-neighbours join the next list when that list
// is being built.
__global__ void slot_seed_kernel(int kind, SlotGraph sg, uint32_t W, uint32_t K, uint32_t cnt,
                                 const uint32_t* slots, const uint32_t* srcs, uint32_t* rows,
                                 uint32_t* front, uint32_t* seen, uint32_t* slot_src, Frontier f) {
    const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= cnt) return;
    const uint32_t s = slots[c];
    const uint32_t v = sg.perm ? sg.perm[srcs[c]] : srcs[c];
    const uint32_t bit = 1u << (s & 31);
    if (kind == kSlotPpr) {
        if (lane_id() == 0) {
            rows[(size_t)v * K + s] = 0x3f800000u;  // 1.0f
            slot_src[s] = v;
        }
        return;
    }
    if (lane_id() == 0) {
        rows[(size_t)v * K + s] = 0u;
        atomicOr(&front[(size_t)v * W + (s >> 5)], bit);
        if (kind == kSlotBfs) atomicOr(&seen[(size_t)v * W + (s >> 5)], bit);
    }
    // the frontier's iteration is the one that comes next; its counters are
    // group it % 4
    const uint32_t it = frontier_iter(f);
    uint32_t* cnext = f.ctr + 4 * (it & 3u);
    if (lane_id() == 0)
        atomicAdd(&cnext[3], 1u + (sg.out_rp ? sg.out_rp[v + 1] - sg.out_rp[v] : 0u));
    if (cnext[1] == 0u) return;  // the next iteration is dense
    if (lane_id() == 0) f.clist_out[atomicAdd(&cnext[2], 1u)] = v;
    list_out_neighbours(sg, f.mark, it, f.plist_out, &cnext[0], v);
}

// out_c[v] = rows[perm(v)][slots[c]]: 32 vertices x 32 slots per block.
__global__ void slot_extract_kernel(const uint32_t* rows, uint32_t n, uint32_t K, uint32_t cnt,
                                    const uint32_t* slots, const uint32_t* perm, uint32_t* const* outs) {
    __shared__ uint32_t tile[32][33];
    const uint32_t v0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t v = v0 + i, c = c0 + tx;
        if (v < n && c < cnt) {
            const uint32_t row = perm ? perm[v] : v;
            tile[i][tx] = rows[(size_t)row * K + slots[c]];
        }
    }
    __syncthreads();
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t c = c0 + i, v = v0 + tx;
        if (v < n && c < cnt) outs[c][v] = tile[tx][i];
    }
}

// ------------------------------------------------------------- host side

namespace {

// Layout of slot_dev_ (u32 words): admission slots, admission sources,
// extraction slots, internal sources of the slots, BFS start iterations.
// Then the iteration counter and the occupied slots (8 words).
constexpr size_t kDevAdmSlots = 0, kDevAdmSrcs = kMaxSlots, kDevExtSlots = 2 * kMaxSlots,
                 kDevSlotSrc = 3 * kMaxSlots, kDevStart = 4 * kMaxSlots, kDevIt = 5 * kMaxSlots,
                 kDevOcc = 5 * kMaxSlots + 8, kDevWords = 5 * kMaxSlots + 16;
// Layout of host_ (pinned, u32 words): chw mirror, admission staging,
// extraction staging, start staging; then K output pointers.
constexpr size_t kHostChw = 0, kHostAdm = 16, kHostExt = 16 + 2 * kMaxSlots,
                 kHostStart = 16 + 3 * kMaxSlots, kHostWords = 16 + 4 * kMaxSlots;

uint32_t pull_grid(const SlotGraph& sg) {
    const uint64_t want = ceil_div(sg.n_pieces, 8);  // 8 warps per block
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sg.sm_count * 8));
}

}  // namespace

Frontier SlotEngine::frontier(uint32_t it) {
    Frontier f;
    f.mark = mark_.as<uint32_t>();
    f.plist_in = plist_[it % 2].as<uint32_t>();
    f.plist_out = plist_[(it + 1) % 2].as<uint32_t>();
    f.clist_out = clist_[it % 3].as<uint32_t>();
    f.clist_old = clist_[(it + 1) % 3].as<uint32_t>();  // iteration it - 2's
    f.ctr = ctr_.as<uint32_t>();
    f.it_base = nullptr;
    f.it = it;
    // the next list is built while fewer than 1/sparse_div (by default 1/8)
    // of the graph's edges leave the changed vertices: listing costs at most
    // that many marks, and a sparse pull never reads more rows than a dense one
    f.thresh = (uint32_t)std::max<uint64_t>(
        64, std::min<uint64_t>(0xFFFFFFFFull, ((uint64_t)sg_.m + sg_.n) / std::max<uint32_t>(1, sg_.sparse_div)));
    return f;
}

size_t SlotEngine::bytes(const SlotGraph& sg, int kind, uint32_t K) {
    K = std::min<uint32_t>(kMaxSlots, (K + 31) / 32 * 32);
    const uint64_t n = sg.n, W = K / 32;
    uint64_t b = n * K * 4 + kDevWords * 4 + 64 + kMaxSlots * 8;
    if (kind == kSlotBfs) b += 4 * n * W * 4;
    if (kind == kSlotSssp) b += 3 * n * W * 4;
    if (kind != kSlotPpr) b += n * 4 + (5 * (uint64_t)sg.n_pieces + 3 * kMaxSlots) * 4 + 64 + 6 * 256;
    if (kind == kSlotPpr)
        b += n * K * 4 + n * 4 + (uint64_t)std::max<uint32_t>(1, sg.n_hub_pieces) * K * 4 +
             (uint64_t)pull_grid(sg) * 8 * K * 4;
    return b + 16 * 256;  // allocation rounding
}

size_t SlotEngine::device_bytes() const {
    size_t b = rows_.bytes + rows2_.bytes + seen_.bytes + iw_.bytes + hub_part_.bytes + dang_part_.bytes +
               slot_dev_.bytes + chw_.bytes + ptrs_.bytes + mark_.bytes + ctr_.bytes;
    for (auto& x : bits_) b += x.bytes;
    for (auto& x : plist_) b += x.bytes;
    for (auto& x : clist_) b += x.bytes;
    return b;
}

void SlotEngine::drop_graphs() {
    for (auto& row : graphs_)
        for (auto& gx : row) {
            if (gx) cudaGraphExecDestroy(gx);  // one still running is freed when it completes
            gx = nullptr;
        }
}

void SlotEngine::release() {
    drop_graphs();
    if (capture_) {
        cudaStreamDestroy(capture_);
        capture_ = nullptr;
    }
    occ_dev_valid_ = false;
    rows_.release();
    rows2_.release();
    for (auto& x : bits_) x.release();
    seen_.release();
    mark_.release();
    for (auto& x : plist_) x.release();
    for (auto& x : clist_) x.release();
    ctr_.release();
    iw_.release();
    hub_part_.release();
    dang_part_.release();
    slot_dev_.release();
    chw_.release();
    ptrs_.release();
    K_ = W_ = 0;
    n_used_ = 0;
    used_.clear();
}

g1_status SlotEngine::init(const SlotGraph& sg, int kind, uint32_t K, float alpha, uint32_t ppr_iters,
                           cudaStream_t s) {
    release();
    if (K == 0 || K > kMaxSlots) return fail(G1_ERR_INVALID, "slot count must be 1..256");
    sg_ = sg;
    kind_ = kind;
    K_ = (K + 31) / 32 * 32;
    W_ = K_ / 32;
    WP_ = W_ <= 1 ? 1 : W_ <= 2 ? 2 : W_ <= 4 ? 4 : 8;
    it_ = 0;
    alpha_ = alpha;
    ppr_iters_ = ppr_iters;
    n_used_ = 0;
    used_.assign(K_, 0);
    start_.assign(K_, 0);
    pull_grid_ = pull_grid(sg);
    const uint64_t n = sg.n;
    const uint64_t nk = n * K_, nw = n * W_;
    G1_TRY(rows_.ensure(nk * 4 + 16));
    if (kind == kSlotBfs || kind == kSlotSssp) {
        for (auto& x : bits_) {
            G1_TRY(x.ensure(nw * 4 + 16));
            G1_CUDA(cudaMemsetAsync(x.p, 0, nw * 4, s));
        }
        if (kind == kSlotBfs) {
            G1_TRY(seen_.ensure(nw * 4 + 16));
            G1_CUDA(cudaMemsetAsync(seen_.p, 0, nw * 4, s));
        }
        G1_TRY(mark_.ensure(n * 4 + 16));
        G1_CUDA(cudaMemsetAsync(mark_.p, 0, n * 4, s));
        for (auto& x : plist_) G1_TRY(x.ensure((uint64_t)sg.n_pieces * 4 + 16));
        // a changed vertex is recorded once per row piece, admitted sources once more
        for (auto& x : clist_) G1_TRY(x.ensure(((uint64_t)sg.n_pieces + kMaxSlots) * 4 + 16));
        G1_TRY(ctr_.ensure(16 * 4));
        G1_CUDA(cudaMemsetAsync(ctr_.p, 0, 16 * 4, s));
        // iteration 1 starts from a valid, empty list (byte fill: nonzero =
        // valid) when out-edges can list the seeds' neighbours
        if (sg.out_rp) {
            G1_CUDA(cudaMemsetAsync(ctr_.as<uint32_t>() + 4 * 0 + 1, 1, 4, s));
            G1_CUDA(cudaMemsetAsync(ctr_.as<uint32_t>() + 4 * 1 + 1, 1, 4, s));
        }
    } else {
        G1_TRY(rows2_.ensure(nk * 4 + 16));
        G1_TRY(iw_.ensure(n * 4 + 16));
        G1_TRY(hub_part_.ensure((uint64_t)std::max<uint32_t>(1, sg.n_hub_pieces) * K_ * 4));
        G1_TRY(dang_part_.ensure((uint64_t)pull_grid_ * 8 * K_ * 4));
        slot_ppr_iw_kernel<<<std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, 256), sg.sm_count * 16)),
                             256, 0, s>>>(sg.out_deg, sg.n, (double)alpha, iw_.as<float>());
        count_launches(1);
        G1_CUDA(cudaGetLastError());
    }
    G1_TRY(slot_dev_.ensure(kDevWords * 4));
    G1_CUDA(cudaMemsetAsync(slot_dev_.p, 0, kDevWords * 4, s));
    G1_TRY(chw_.ensure(16 * 4));
    G1_CUDA(cudaMemsetAsync(chw_.p, 0, 16 * 4, s));
    G1_TRY(ptrs_.ensure(kMaxSlots * sizeof(void*)));
    G1_TRY(host_.ensure(kHostWords * 4 + kMaxSlots * sizeof(void*)));
    std::memset(host_.p, 0, kHostWords * 4);
    return G1_OK;
}

g1_status SlotEngine::set_alpha(float alpha, uint32_t ppr_iters, cudaStream_t s) {
    ppr_iters_ = ppr_iters;
    if (kind_ != kSlotPpr || alpha == alpha_) return G1_OK;
    if (n_used_) return fail(G1_ERR_INVALID, "damping changed while queries run");
    alpha_ = alpha;
    drop_graphs();  // the teleport nodes hold the damping
    slot_ppr_iw_kernel<<<std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(sg_.n, 256), sg_.sm_count * 16)),
                         256, 0, s>>>(sg_.out_deg, sg_.n, (double)alpha, iw_.as<float>());
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

int SlotEngine::take_slot() {
    for (uint32_t i = 0; i < K_; ++i)
        if (!used_[i]) {
            used_[i] = 1;
            ++n_used_;
            return (int)i;
        }
    return -1;
}

void SlotEngine::free_slot(uint32_t slot) {
    if (slot < K_ && used_[slot]) {
        used_[slot] = 0;
        --n_used_;
    }
}

Bits256 SlotEngine::occupied_bits() const {
    Bits256 b;
    std::memset(&b, 0, sizeof(b));
    for (uint32_t i = 0; i < K_; ++i)
        if (used_[i]) b.w[i >> 5] |= 1u << (i & 31);
    return b;
}

g1_status SlotEngine::admit(const uint32_t* slots, const uint32_t* srcs, uint32_t cnt, cudaStream_t s) {
    if (cnt == 0) return G1_OK;
    if (cnt > K_) return fail(G1_ERR_INVALID, "more admissions than slots");
    uint32_t* h = host_.as<uint32_t>();
    Bits256 amask;
    std::memset(&amask, 0, sizeof(amask));
    for (uint32_t c = 0; c < cnt; ++c) {
        h[kHostAdm + c] = slots[c];
        h[kHostAdm + kMaxSlots + c] = srcs[c];
        amask.w[slots[c] >> 5] |= 1u << (slots[c] & 31);
        start_[slots[c]] = it_;
    }
    for (uint32_t i = 0; i < K_; ++i) h[kHostStart + i] = start_[i];
    uint32_t* d = slot_dev_.as<uint32_t>();
    G1_CUDA(cudaMemcpyAsync(d + kDevAdmSlots, h + kHostAdm, (size_t)cnt * 4, cudaMemcpyHostToDevice, s));
    G1_CUDA(cudaMemcpyAsync(d + kDevAdmSrcs, h + kHostAdm + kMaxSlots, (size_t)cnt * 4,
                            cudaMemcpyHostToDevice, s));
    if (kind_ == kSlotBfs)
        G1_CUDA(cudaMemcpyAsync(d + kDevStart, h + kHostStart, (size_t)K_ * 4, cudaMemcpyHostToDevice, s));
    // the buffers the next iteration (it_ + 1) reads
    uint32_t* rows = (kind_ == kSlotPpr && (it_ & 1)) ? rows2_.as<uint32_t>() : rows_.as<uint32_t>();
    uint32_t* front = kind_ == kSlotPpr ? nullptr : bits_[(it_ + 1) % 3].as<uint32_t>();
    const uint32_t init = kind_ == kSlotPpr ? 0u : kU32Max;
    const uint64_t work = (uint64_t)sg_.n * cnt;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(std::max<uint64_t>(work, (uint64_t)sg_.n * W_), 256),
                              (uint64_t)sg_.sm_count * 16));
    if (cnt == K_) {
        // every slot: whole rows (init is a repeated byte)
        G1_CUDA(cudaMemsetAsync(rows, init ? 0xFF : 0, (size_t)sg_.n * K_ * 4, s));
        if (kind_ == kSlotBfs) G1_CUDA(cudaMemsetAsync(seen_.p, 0, (size_t)sg_.n * W_ * 4, s));
    } else {
        slot_reset_kernel<<<grid, 256, 0, s>>>(sg_.n, K_, W_, cnt, d + kDevAdmSlots, init, rows,
                                               kind_ == kSlotBfs ? seen_.as<uint32_t>() : nullptr, amask);
    }
    // seeds count as changed by iteration it_ and feed iteration it_ + 1's list
    Frontier f;
    std::memset(&f, 0, sizeof(f));
    if (kind_ != kSlotPpr) {
        f = frontier(it_ + 1);
        f.clist_out = clist_[it_ % 3].as<uint32_t>();
        f.plist_out = plist_[(it_ + 1) % 2].as<uint32_t>();
    }
    slot_seed_kernel<<<(unsigned)ceil_div(cnt, 8), 256, 0, s>>>(
        kind_, sg_, W_, K_, cnt, d + kDevAdmSlots, d + kDevAdmSrcs, rows, front,
        kind_ == kSlotBfs ? seen_.as<uint32_t>() : nullptr, d + kDevSlotSrc, f);
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

uint32_t SlotEngine::max_step(uint32_t want) const {
    if (kind_ != kSlotPpr) return std::max<uint32_t>(1, want);
    uint32_t m = want ? want : 1;
    for (uint32_t i = 0; i < K_; ++i)
        if (used_[i]) m = std::min(m, ppr_iters_ - std::min(ppr_iters_, it_ - start_[i]));
    return std::max<uint32_t>(1, m);
}

g1_status SlotEngine::enqueue_iterations(uint32_t n, uint32_t phase, cudaStream_t s) {
    uint32_t* d = slot_dev_.as<uint32_t>();
    uint32_t* chw = chw_.as<uint32_t>();
    const uint32_t* occ = d + kDevOcc;
    const uint32_t grid = pull_grid_;
    for (uint32_t k = 1; k <= n; ++k) {
        // buffers of iteration base + k, base = phase (mod 6); its number
        // comes from the device counter
        const uint32_t v = phase + k;
        uint32_t* c_now = chw + 8 * (v & 1);
        uint32_t* c_next = chw + 8 * ((v + 1) & 1);
        if (kind_ == kSlotBfs) {
            Frontier f = frontier(v);
            f.it_base = d + kDevIt;
            f.it = k;
            const uint32_t* front = bits_[v % 3].as<uint32_t>();
            uint32_t* next = bits_[(v + 1) % 3].as<uint32_t>();
            uint32_t* clr = bits_[(v + 2) % 3].as<uint32_t>();
#define G1_SLOT_BFS(WPV)                                                                              \
    slot_bfs_kernel<WPV><<<grid, 256, 0, s>>>(sg_, f, W_, K_, occ, front, seen_.as<uint32_t>(), next, clr, \
                                              rows_.as<uint32_t>(), d + kDevStart, c_now, c_next)
            switch (WP_) {
                case 1: G1_SLOT_BFS(1); break;
                case 2: G1_SLOT_BFS(2); break;
                case 4: G1_SLOT_BFS(4); break;
                default: G1_SLOT_BFS(8); break;
            }
#undef G1_SLOT_BFS
        } else if (kind_ == kSlotSssp) {
            Frontier f = frontier(v);
            f.it_base = d + kDevIt;
            f.it = k;
            slot_sssp_kernel<<<grid, 256, 0, s>>>(sg_, f, W_, K_, occ, rows_.as<uint32_t>(),
                                                  bits_[v % 3].as<uint32_t>(), bits_[(v + 1) % 3].as<uint32_t>(),
                                                  bits_[(v + 2) % 3].as<uint32_t>(), c_now, c_next);
        } else {
            // iteration it reads the rank block of parity (it - 1) and writes the other
            const float* cur = ((v - 1) & 1) ? rows2_.as<float>() : rows_.as<float>();
            float* nxt = ((v - 1) & 1) ? rows_.as<float>() : rows2_.as<float>();
            slot_ppr_pull_kernel<<<grid, 256, 0, s>>>(sg_, W_, K_, occ, iw_.as<float>(), cur, nxt,
                                                      hub_part_.as<float>(), dang_part_.as<float>());
            if (sg_.n_hubs)
                slot_ppr_hub_kernel<<<std::min<uint32_t>(sg_.n_hubs, sg_.sm_count * 8), 256, 0, s>>>(
                    sg_, W_, K_, occ, hub_part_.as<float>(), nxt);
            slot_ppr_teleport_kernel<<<K_, 256, 0, s>>>(K_, occ, d + kDevSlotSrc, dang_part_.as<float>(),
                                                        grid * 8, (double)alpha_, nxt);
        }
        G1_CUDA(cudaGetLastError());
    }
    slot_it_advance_kernel<<<1, 1, 0, s>>>(d + kDevIt, n);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status SlotEngine::step_graph(int i, uint32_t phase, cudaGraphExec_t* out) {
    cudaGraphExec_t& gx = graphs_[i][phase];
    if (!gx) {
        if (!capture_) G1_CUDA(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        G1_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
        g1_status st;
        cudaError_t e;
        {
            CaptureScope cs;  // counted per launch in step()
            st = enqueue_iterations(1u << i, phase, capture_);
            e = cudaStreamEndCapture(capture_, &graph);
        }
        if (st != G1_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture(slot step)");
        const cudaError_t ei = cudaGraphInstantiate(&gx, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            gx = nullptr;
            return fail_cuda(ei, "cudaGraphInstantiate(slot step)");
        }
    }
    *out = gx;
    return G1_OK;
}

g1_status SlotEngine::step(uint32_t iters, cudaStream_t s) {
    if (!ready()) return fail(G1_ERR_INVALID, "slot engine not initialised");
    uint32_t* d = slot_dev_.as<uint32_t>();
    const Bits256 occ = occupied_bits();
    if (!occ_dev_valid_ || std::memcmp(&occ, &occ_dev_, sizeof(occ)) != 0) {
        slot_set_occ_kernel<<<1, 32, 0, s>>>(d + kDevOcc, occ);
        count_launches(1);
        G1_CUDA(cudaGetLastError());
        occ_dev_ = occ;
        occ_dev_valid_ = true;
    }
    // iters as a sum of powers of two, each a captured graph
    const uint32_t per_iter = kind_ == kSlotPpr ? (sg_.n_hubs ? 3u : 2u) : 1u;
    for (int i = kStepGraphs - 1; i >= 0; --i) {
        const uint32_t n = 1u << i;
        while (iters >= n) {
            cudaGraphExec_t gx = nullptr;
            G1_TRY(step_graph(i, it_ % kPhases, &gx));
            G1_CUDA(cudaGraphLaunch(gx, s));
            count_launches((uint64_t)n * per_iter + 1);
            iters -= n;
            it_ += n;
        }
    }
    if (kind_ != kSlotPpr)
        G1_CUDA(cudaMemcpyAsync(host_.as<uint32_t>() + kHostChw, chw_.as<uint32_t>() + 8 * (it_ & 1), 8 * 4,
                                cudaMemcpyDeviceToHost, s));
    return G1_OK;
}

void SlotEngine::finished(std::vector<uint32_t>* out) const {
    out->clear();
    const uint32_t* h = host_.as<uint32_t>() + kHostChw;
    for (uint32_t i = 0; i < K_; ++i) {
        if (!used_[i]) continue;
        if (kind_ == kSlotPpr) {
            if (it_ - start_[i] >= ppr_iters_) out->push_back(i);
        } else if (it_ > start_[i] && !((h[i >> 5] >> (i & 31)) & 1u)) {
            out->push_back(i);
        }
    }
}

g1_status SlotEngine::extract(const uint32_t* slots, uint32_t cnt, void* const* outs, cudaStream_t s) {
    if (cnt == 0) return G1_OK;
    uint32_t* h = host_.as<uint32_t>();
    void** hp = reinterpret_cast<void**>(h + kHostWords);
    for (uint32_t c = 0; c < cnt; ++c) {
        h[kHostExt + c] = slots[c];
        hp[c] = outs[c];
    }
    uint32_t* d = slot_dev_.as<uint32_t>();
    G1_CUDA(cudaMemcpyAsync(d + kDevExtSlots, h + kHostExt, (size_t)cnt * 4, cudaMemcpyHostToDevice, s));
    G1_CUDA(cudaMemcpyAsync(ptrs_.p, hp, (size_t)cnt * sizeof(void*), cudaMemcpyHostToDevice, s));
    const uint32_t* rows = (kind_ == kSlotPpr && (it_ & 1)) ? rows2_.as<uint32_t>() : rows_.as<uint32_t>();
    dim3 grid((unsigned)ceil_div(sg_.n, 32), (unsigned)ceil_div(cnt, 32)), block(32, 8);
    if (sg_.n)
        slot_extract_kernel<<<grid, block, 0, s>>>(rows, sg_.n, K_, cnt, d + kDevExtSlots, sg_.perm,
                                                   ptrs_.as<uint32_t* const>());
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

}  // namespace g1
