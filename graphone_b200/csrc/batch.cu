// Batched multi-source BFS and SSSP: k sources (k <= 256 per pass) run as
// one pass over the graph per iteration instead of k independent traversals.
//
// Layout (vertex-major, so one vertex's state for all sources is one
// contiguous row and every access below is coalesced):
//   BFS : frontier / seen / next bit rows of W = ceil(k/32) words per vertex
//         (bit s of word s/32), levels[v][s] rows of k u32;
//   SSSP: dist[v][s] rows of k u32, changed[v] / changed_next[v] bit rows.
// Each iteration is a pull over the in-edge CSR with one warp per vertex:
//   BFS : OR of the in-neighbours' frontier rows (lanes = (neighbour slot,
//         word)); new = that & ~seen; levels of the new bits are stored as
//         one coalesced 128-byte row segment per word;
//   SSSP: lane l owns sources l, l+32, ...; for every in-neighbour u whose
//         changed row has a bit in word j, the warp reads dist[u][32j..]
//         (128 bytes) and relaxes min(dist + w) in registers; improved
//         sources set their bits in changed_next[v] by ballot.  No atomics.
// A device flag says whether anything changed; the host reads it once per
// iteration.  Results are transposed at the end into source-major rows
// (out[s*n + v]), the layout of k single-source calls.  Min-plus is
// order-independent, so levels and distances are bit-exact with k plain
// traversals.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "g1/common.cuh"
#include "internal.h"

namespace g1 {

constexpr uint32_t kMaxBatch = 256;

// ------------------------------------------------------------------ BFS
// Row pieces: every vertex's in-edge range cut into pieces of at most
// kPieceEdges edges, so a hub's row is pulled by many warps (its pieces merge
// with atomics) while ordinary rows stay one warp each (plain stores).
constexpr uint32_t kPieceEdges = 1024;

template <int WP>  // words per vertex rounded up to a power of two (1..8)
__global__ void __launch_bounds__(256)
msbfs_pull_kernel(const uint32_t* rp, const uint32_t* col, const uint32_t* piece_v,
                  const uint32_t* piece_e, uint32_t n_pieces, uint32_t W, uint32_t k,
                  const uint32_t* frontier, uint32_t* seen, uint32_t* next, uint32_t* lvm,
                  uint32_t depth, uint32_t* changed) {
    constexpr int SLOTS = 32 / WP;  // neighbours per warp step
    const uint32_t lane = lane_id();
    const uint32_t w = lane % WP, q = lane / WP;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    uint32_t any = 0;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_pieces; p += warps) {
        const uint32_t v = piece_v[p];
        const uint32_t rs = rp[v], re = rp[v + 1];
        const bool multi = re - rs > kPieceEdges;
        const uint32_t e0 = piece_e[p], e1 = min(e0 + kPieceEdges, re);
        uint32_t sn = 0xffffffffu;
        if (w < W) {
            sn = seen[(size_t)v * W + w];
            const uint32_t live = (w == W - 1 && (k & 31)) ? ((1u << (k & 31)) - 1u) : 0xffffffffu;
            sn |= ~live;  // sources beyond k count as seen
        }
        if (__all_sync(0xffffffffu, sn == 0xffffffffu)) continue;  // next[v] stays 0
        uint32_t acc = 0;
        for (uint32_t e = e0 + q; e < e1; e += SLOTS) {
            const uint32_t u = __ldg(col + e);
            if (w < W) acc |= __ldg(frontier + (size_t)u * W + w);
        }
#pragma unroll
        for (int off = WP; off < 32; off <<= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, off);
        uint32_t nw = acc & ~sn;
        if (w < W && q == 0 && nw) {
            if (multi) {
                // several pieces of this row: claim the bits first set here
                nw &= ~atomicOr(&seen[(size_t)v * W + w], nw);
                if (nw) atomicOr(&next[(size_t)v * W + w], nw);
            } else {
                next[(size_t)v * W + w] = nw;
                seen[(size_t)v * W + w] = sn | nw;
            }
        }
        // levels of the new bits: row segment j written by all 32 lanes
        for (uint32_t j = 0; j < W; ++j) {
            const uint32_t bits = __shfl_sync(0xffffffffu, nw, (int)j);
            if (bits == 0) continue;
            any = 1;
            if ((bits >> lane) & 1u) lvm[(size_t)v * k + 32 * j + lane] = depth;
        }
    }
    if (any && lane == 0) atomicOr(changed, 1u);
}

__global__ void msbfs_init_kernel(uint32_t n, uint32_t W, uint32_t k, const uint32_t* srcs,
                                  uint32_t* frontier, uint32_t* seen, uint32_t* lvm) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nw = (uint64_t)n * W, nk = (uint64_t)n * k;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride) {
        lvm[i] = kU32Max;
        if (i < nw) {
            frontier[i] = 0u;
            seen[i] = 0u;
        }
    }
}

__global__ void msbfs_seed_kernel(uint32_t W, uint32_t k, const uint32_t* srcs, uint32_t* frontier,
                                  uint32_t* seen, uint32_t* lvm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    const uint32_t v = srcs[s];
    atomicOr(&frontier[(size_t)v * W + s / 32], 1u << (s % 32));
    atomicOr(&seen[(size_t)v * W + s / 32], 1u << (s % 32));
    lvm[(size_t)v * k + s] = 0u;
}

// ------------------------------------------------------------------ SSSP
// Lane l of the warp owns sources 32j + l (j < W).
__global__ void __launch_bounds__(256)
mssssp_pull_kernel(const uint32_t* rp, const uint32_t* col, const uint32_t* val,
                   const uint32_t* piece_v, const uint32_t* piece_e, uint32_t n_pieces,
                   uint32_t W, uint32_t k, uint32_t* dist, const uint32_t* chg,
                   uint32_t* chg_next, uint32_t* changed) {
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    uint32_t any = 0;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_pieces; p += warps) {
        const uint32_t v = piece_v[p];
        const uint32_t rs = rp[v], re = rp[v + 1];
        const bool multi = re - rs > kPieceEdges;
        const uint32_t e0 = piece_e[p], e1 = min(e0 + kPieceEdges, re);
        uint32_t best[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) best[j] = kU32Max;
        for (uint32_t e = e0; e < e1; ++e) {
            const uint32_t u = __ldg(col + e);
            // the changed row of u (W <= 8 words) is read by every lane
            const uint32_t mine = lane < W ? __ldg(chg + (size_t)u * W + lane) : 0u;
            unsigned words = __ballot_sync(0xffffffffu, mine != 0u);
            if (!words) continue;
            const uint32_t w = __ldg(val + e);
            const uint32_t* du = dist + (size_t)u * k;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (!((words >> j) & 1u)) continue;
                const uint32_t bits = __shfl_sync(0xffffffffu, mine, j);
                if ((bits >> lane) & 1u) {
                    const uint32_t d = du[32 * j + lane];
                    best[j] = min(best[j], d + w);  // d is finite: it changed
                }
            }
        }
        uint32_t* dv = dist + (size_t)v * k;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if ((uint32_t)j >= W) break;
            const uint32_t s = 32 * j + lane;
            bool imp = false;
            if (s < k && best[j] != kU32Max) {
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
            any |= bits;
        }
    }
    if (any && lane == 0) atomicOr(changed, 1u);
}

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

__global__ void mssssp_init_kernel(uint32_t n, uint32_t W, uint32_t k, uint32_t* dist,
                                   uint32_t* chg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nk = (uint64_t)n * k, nw = (uint64_t)n * W;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += stride) {
        dist[i] = kU32Max;
        if (i < nw) chg[i] = 0u;
    }
}

__global__ void mssssp_seed_kernel(uint32_t W, uint32_t k, const uint32_t* srcs, uint32_t* dist,
                                   uint32_t* chg) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    const uint32_t v = srcs[s];
    dist[(size_t)v * k + s] = 0u;
    atomicOr(&chg[(size_t)v * W + s / 32], 1u << (s % 32));
}

// ------------------------------------------------------------- shared parts
// out[s*n + v] = in[v*k + s] (vertex rows -> source rows), 32x32 tiles;
// with a relabelled graph `perm` maps the caller's v to the internal row.
__global__ void transpose_out_kernel(const uint32_t* in, uint32_t n, uint32_t k, const uint32_t* perm,
                                     uint32_t* out) {
    __shared__ uint32_t tile[32][33];
    const uint32_t v0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t v = v0 + i, s = s0 + tx;
        if (v < n && s < k) {
            const uint32_t row = perm ? perm[v] : v;
            tile[i][tx] = in[(size_t)row * k + s];
        }
    }
    __syncthreads();
    for (uint32_t i = ty; i < 32; i += 8) {
        const uint32_t s = s0 + i, v = v0 + tx;
        if (v < n && s < k) out[(size_t)s * n + v] = tile[tx][i];
    }
}

__global__ void map_sources_kernel(const uint32_t* in, uint32_t k, const uint32_t* perm,
                                   uint32_t n, uint32_t* out, uint32_t* bad) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    const uint32_t v = in[s];
    if (v >= n) {
        atomicOr(bad, 1u);
        out[s] = 0;
        return;
    }
    out[s] = perm ? perm[v] : v;
}

namespace {

// The in-edge CSR's row pieces, built once per graph.
g1_status ensure_pieces(g1_graph* g, cudaStream_t s, const uint32_t** pv, const uint32_t** pe,
                        uint32_t* np) {
    Workspace& ws = g->ws;
    uint32_t *cnt = nullptr, *off = nullptr, *piece_v = nullptr, *piece_e = nullptr, *tot = nullptr;
    const uint32_t n = g->n;
    const Orientation& o = g->o[1];
    if (!g->pieces_ready) {
        G1_TRY(ws.get("pc_cnt", (size_t)n + 1, &cnt));
        G1_TRY(ws.get("pc_off", (size_t)n + 1, &off));
        const uint32_t grid = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
        piece_count_kernel<<<grid, 256, 0, s>>>(o.rp, n, cnt);
        G1_CUDA(cudaMemsetAsync(cnt + n, 0, 4, s));
        size_t tb = 0;
        G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)n + 1, s));
        DevBuf temp;
        G1_TRY(temp.ensure(tb + 16));
        G1_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, cnt, off, (int)n + 1, s));
        uint32_t h = 0;
        G1_CUDA(cudaMemcpyAsync(&h, off + n, 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
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
    (void)tot;
    *pv = piece_v;
    *pe = piece_e;
    *np = g->n_pieces;
    return G1_OK;
}

uint32_t grid_warps(const g1_graph* g, uint64_t n) {
    const uint64_t want = ceil_div(n, 8);  // 8 warps per 256-thread block
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->sm_count * 8));
}

uint32_t grid_elems(const g1_graph* g, uint64_t n) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 16));
}

template <bool BFS>
g1_status run_batch(g1_graph* g, const uint32_t* srcs_in, uint32_t k, uint32_t* out,
                    uint32_t* iters_out, cudaStream_t s) {
    const uint32_t n = g->n;
    if (k == 0) return G1_OK;
    if (k > kMaxBatch) return fail(G1_ERR_INVALID, "batch size above 256 per call");
    if (!g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "batched traversal needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    if (!BFS && g->vtype != G1_U32) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
    const uint32_t W = (k + 31) / 32;
    Workspace& ws = g->ws;
    uint32_t *srcs = nullptr, *srcs_raw = nullptr, *a = nullptr, *b = nullptr, *c = nullptr,
             *rows = nullptr, *flag = nullptr;
    G1_TRY(ws.get("mb_srcs", kMaxBatch, &srcs));
    G1_TRY(ws.get("mb_srcs_raw", kMaxBatch, &srcs_raw));
    G1_TRY(ws.get("mb_a", (size_t)n * W, &a));
    G1_TRY(ws.get("mb_b", (size_t)n * W, &b));
    if (BFS) G1_TRY(ws.get("mb_c", (size_t)n * W, &c));
    G1_TRY(ws.get("mb_rows", (size_t)n * k, &rows));
    G1_TRY(ws.get("mb_flag", 4, &flag));
    G1_TRY(ws.pinned.ensure(64));
    uint32_t* host = ws.pinned.as<uint32_t>();

    G1_CUDA(cudaMemcpyAsync(srcs_raw, srcs_in, (size_t)k * 4,
                            is_device_ptr(srcs_in) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            s));
    G1_CUDA(cudaMemsetAsync(flag, 0, 4, s));
    map_sources_kernel<<<1, 256, 0, s>>>(srcs_raw, k, g->relabeled ? g->perm.as<uint32_t>() : nullptr,
                                         n, srcs, flag);
    G1_CUDA(cudaMemcpyAsync(host, flag, 4, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    if (host[0]) return fail(G1_ERR_INVALID, "source vertex out of range");

    const Orientation& o = g->o[1];
    const uint64_t nk = (uint64_t)n * k;
    if (BFS) {
        msbfs_init_kernel<<<grid_elems(g, nk), 256, 0, s>>>(n, W, k, srcs, a, c, rows);
        msbfs_seed_kernel<<<1, 256, 0, s>>>(W, k, srcs, a, c, rows);
    } else {
        mssssp_init_kernel<<<grid_elems(g, nk), 256, 0, s>>>(n, W, k, rows, a);
        mssssp_seed_kernel<<<1, 256, 0, s>>>(W, k, srcs, rows, a);
    }
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    const uint32_t *pv = nullptr, *pe = nullptr;
    uint32_t np = 0;
    G1_TRY(ensure_pieces(g, s, &pv, &pe, &np));
    uint32_t it = 0;
    uint32_t* cur = a;
    uint32_t* nxt = b;
    const uint32_t gw = grid_warps(g, np);
    for (;;) {
        ++it;
        if (it > n + 2) return fail(G1_ERR_TIMEOUT, "batched traversal did not converge");
        G1_CUDA(cudaMemsetAsync(flag, 0, 4, s));
        G1_CUDA(cudaMemsetAsync(nxt, 0, (size_t)n * W * 4, s));
        if (BFS) {
            switch (W <= 1 ? 1 : W <= 2 ? 2 : W <= 4 ? 4 : 8) {
                case 1: msbfs_pull_kernel<1><<<gw, 256, 0, s>>>(o.rp, o.col, pv, pe, np, W, k, cur, c, nxt, rows, it, flag); break;
                case 2: msbfs_pull_kernel<2><<<gw, 256, 0, s>>>(o.rp, o.col, pv, pe, np, W, k, cur, c, nxt, rows, it, flag); break;
                case 4: msbfs_pull_kernel<4><<<gw, 256, 0, s>>>(o.rp, o.col, pv, pe, np, W, k, cur, c, nxt, rows, it, flag); break;
                default: msbfs_pull_kernel<8><<<gw, 256, 0, s>>>(o.rp, o.col, pv, pe, np, W, k, cur, c, nxt, rows, it, flag); break;
            }
        } else {
            mssssp_pull_kernel<<<gw, 256, 0, s>>>(o.rp, o.col, static_cast<const uint32_t*>(o.val), pv,
                                                  pe, np, W, k, rows, cur, nxt, flag);
        }
        count_launches(1);
        G1_CUDA(cudaGetLastError());
        G1_CUDA(cudaMemcpyAsync(host, flag, 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        std::swap(cur, nxt);
        if (!host[0]) break;
    }
    if (iters_out) *iters_out = it;
    // source-major result
    uint32_t* tout = nullptr;
    const bool dev_out = is_device_ptr(out);
    if (dev_out)
        tout = out;
    else
        G1_TRY(ws.get("mb_out", nk, &tout));
    dim3 grid((unsigned)ceil_div(n, 32), (unsigned)ceil_div(k, 32)), block(32, 8);
    transpose_out_kernel<<<grid, block, 0, s>>>(rows, n, k,
                                                g->relabeled ? g->perm.as<uint32_t>() : nullptr, tout);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    if (!dev_out) {
        G1_CUDA(cudaMemcpyAsync(out, tout, nk * 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
    }
    return check_device_error(g, s);
}

template <bool BFS>
g1_status batch_entry(g1_graph* g, const uint32_t* srcs, uint32_t k, uint32_t* out,
                      uint32_t* iters_out, void* stream) {
    if (!g || (k && (!srcs || !out))) return fail(G1_ERR_INVALID, "batched traversal: bad argument");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStream_t s = as_stream(stream);
    // more than 256 sources: consecutive passes of 256
    uint32_t total_it = 0;
    const bool dev_src = is_device_ptr(srcs);
    for (uint32_t b0 = 0; b0 < k; b0 += kMaxBatch) {
        const uint32_t kb = std::min(kMaxBatch, k - b0);
        uint32_t it = 0;
        const uint32_t* sp = srcs + b0;
        std::vector<uint32_t> hs;
        if (!dev_src) hs.assign(sp, sp + kb);
        G1_TRY(run_batch<BFS>(g, dev_src ? sp : hs.data(), kb, out + (size_t)b0 * g->n, &it, s));
        total_it = std::max(total_it, it);
    }
    if (iters_out) *iters_out = total_it;
    return G1_OK;
}

}  // namespace
}  // namespace g1

using namespace g1;

extern "C" g1_status g1_bfs_batch(g1_graph* g, const uint32_t* srcs, uint32_t k,
                                  uint32_t* levels_out, uint32_t* iters_out, void* stream) {
    return batch_entry<true>(g, srcs, k, levels_out, iters_out, stream);
}

extern "C" g1_status g1_sssp_batch(g1_graph* g, const uint32_t* srcs, uint32_t k,
                                   uint32_t* dist_out, uint32_t* iters_out, void* stream) {
    return batch_entry<false>(g, srcs, k, dist_out, iters_out, stream);
}
