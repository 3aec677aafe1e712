#pragma once
// Semiring SpMV schedules over CSR for sm_100a.
//
// y[r] = reduce_{k in row r} combine(val[k], x[col[k]]), folded from
// SR::identity().  This is the contract of GraphOne's SpMV adapter
// (engine/blas_gc.h:113-128: initialize = default_result, combine =
// gather_combine, reduce = gather_reduce) and of SpMV_cpu_navie
// (archi/blas/spmv/cpu/naive.hpp:8-20).  Every completed row is handed to an
// epilogue functor `epi.emit(row, value)` instead of being stored, so the
// engines fuse apply_each / construct_each / frontier compaction into the
// SpMV (GraphOne runs those as separate N-sized passes: blas_gc.h:224-245,
// 27-76).
//
// Two schedules:
//  * merge-path (Merrill & Garland, SC'16, "Merge-based parallel sparse
//    matrix-vector multiplication"): the (row-end, nonzero) merge of a tile
//    of ITEMS = BLOCK*IPT items per CTA is staged in shared memory; each
//    thread folds IPT consecutive merge items, then a block-wide segmented
//    scan stitches rows that cross threads.  Rows that cross tiles are
//    finished by `spmv_fixup_kernel`, one thread per tile, folding the
//    per-tile carries in tile order (deterministic, no atomics).  Balanced
//    for any degree distribution.
//  * CSR-vector: TPR lanes per row with a shuffle reduction, for graphs with
//    uniformly small degrees (grids), where the merge bookkeeping costs more
//    than it saves.
//
// Semiring concept (all members static, device-callable):
//   using value_t;  // gather type (y)
//   using x_t;      // info type (x)
//   using w_t;      // edge value type
//   value_t identity();
//   value_t combine(const w_t&, const x_t&);
//   value_t reduce(const value_t& earlier, const value_t& later);
//
// Epilogue concept:
//   __device__ void begin();                                    // all threads, once
//   __device__ void emit(uint32_t row, const value_t& v);
//   template <int BLOCK> __device__ void block_end(char* smem);  // all threads, once

#include "g1/common.cuh"

namespace g1 {

// Merge-path partition of one CSR for tiles of `items` merge items.
// tile t spans merge diagonals [t*items, min((t+1)*items, n_rows+nnz)); its
// start coordinate is (tile_row[t], tile_nnz[t]).  n_tiles+1 entries.
struct MergePlanView {
    uint32_t n_rows;
    uint32_t nnz;
    uint32_t items;
    uint32_t n_tiles;
    const uint32_t* row_ptr;   // n_rows + 1
    const uint32_t* tile_row;  // n_tiles + 1
    const uint32_t* tile_nnz;  // n_tiles + 1
};

// Merge-path search of diagonal d over A = row_ptr[1..] (row ends) and
// B = 0..nnz-1: row-end i is merged before nonzero j iff A[i] <= j.
__device__ __forceinline__ void merge_path_search(uint64_t d, const uint32_t* row_end,
                                                  uint32_t n_rows, uint32_t nnz,
                                                  uint32_t* i_out, uint32_t* j_out) {
    uint64_t lo = d > nnz ? d - nnz : 0;
    uint64_t hi = d < n_rows ? d : n_rows;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if ((uint64_t)row_end[mid] <= d - 1 - mid)
            lo = mid + 1;
        else
            hi = mid;
    }
    *i_out = (uint32_t)lo;
    *j_out = (uint32_t)(d - lo);
}

// Block-wide inclusive/exclusive segmented scan of (head, value) pairs in
// thread order.  A head starts a new segment with its own value.  `excl` is
// the inclusive result of the previous thread (identity for thread 0).
template <class SR, int BLOCK>
__device__ __forceinline__ void block_seg_scan(bool head, typename SR::value_t val,
                                               typename SR::value_t& incl,
                                               typename SR::value_t& excl,
                                               typename SR::value_t* s_wval, int* s_wflag,
                                               typename SR::value_t* s_wpre) {
    using V = typename SR::value_t;
    constexpr int NW = BLOCK / 32;
    const unsigned full = 0xffffffffu;
    const int lane = (int)lane_id();
    const int w = threadIdx.x >> 5;
    V s = val;
    int f = head ? 1 : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        V su = shfl_up_any(full, s, off);
        int fu = __shfl_up_sync(full, f, off);
        if (lane >= off) {
            if (!f) s = SR::reduce(su, s);
            f |= fu;
        }
    }
    if (lane == 31) {
        s_wval[w] = s;
        s_wflag[w] = f;
    }
    __syncthreads();
    if (w == 0) {
        V ws = lane < NW ? s_wval[lane] : SR::identity();
        int wf = lane < NW ? s_wflag[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            V su = shfl_up_any(full, ws, off);
            int fu = __shfl_up_sync(full, wf, off);
            if (lane >= off) {
                if (!wf) ws = SR::reduce(su, ws);
                wf |= fu;
            }
        }
        V ex = shfl_up_any(full, ws, 1);
        if (lane == 0) ex = SR::identity();
        if (lane < NW) s_wpre[lane] = ex;
    }
    __syncthreads();
    const V pre = s_wpre[w];
    incl = f ? s : SR::reduce(pre, s);
    V e = shfl_up_any(full, incl, 1);
    excl = lane == 0 ? pre : e;
}

template <class SR>
struct MergeArgs {
    MergePlanView plan;
    const uint32_t* col;           // readable (padded) up to round_up(nnz, 4) entries
    const typename SR::w_t* val;   // readable (padded) up to round_up(nnz, 16 / sizeof(w_t))
    const typename SR::x_t* x;
    typename SR::value_t* carry;   // n_tiles: partial of the row open at tile end
    typename SR::value_t* tail;    // n_tiles: in-tile partial of a row begun earlier
    uint32_t* err;                 // device error word (kDevTimeout on a stalled copy)
};

// Dynamic shared memory of the pipelined merge kernel: two staging buffers
// (row_ptr window, col, val of one tile each), the combined values of the
// tile being folded, the scan scratch, epilogue scratch and two mbarriers.
template <class SR, int BLOCK, int IPT>
struct MergeLayout {
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    static_assert(sizeof(W) == 4 || sizeof(W) == 8, "edge values of 4 or 8 bytes");
    static constexpr int ITEMS = BLOCK * IPT;
    static constexpr int AW = 16 / (int)sizeof(W);  // val elements per 16 bytes
    static constexpr int SLOTS = ((ITEMS + 8 + 3) / 4) * 4;
    static constexpr int VSLOTS = ((ITEMS + 2 * AW + AW - 1) / AW) * AW;
    static constexpr size_t RE_OFF = 0;
    static constexpr size_t COL_OFF = RE_OFF + (size_t)SLOTS * 4;
    static constexpr size_t VAL_OFF = COL_OFF + (size_t)SLOTS * 4;
    static constexpr size_t STAGE_BYTES = VAL_OFF + (size_t)VSLOTS * sizeof(W);
    static constexpr size_t V_OFF = 2 * STAGE_BYTES;
    static constexpr size_t V_BYTES = ((ITEMS * sizeof(V) + 15) / 16) * 16;
    static constexpr size_t WVAL_OFF = V_OFF + V_BYTES;
    static constexpr size_t WPRE_OFF = WVAL_OFF + ((BLOCK / 32) * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t WFLAG_OFF = WPRE_OFF + ((BLOCK / 32) * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t EPI_OFF = WFLAG_OFF + ((BLOCK / 32) * 4 + 15) / 16 * 16;
    static constexpr size_t BAR_OFF = EPI_OFF + 512;
    static constexpr size_t BYTES = BAR_OFF + 16;
};

// Issues the bulk copies of tile `tile` into staging buffer `st` (one thread).
template <class SR, int BLOCK, int IPT>
__device__ __forceinline__ void merge_issue_tile(const MergeArgs<SR>& a, uint32_t tile,
                                                 unsigned char* st, uint64_t* bar) {
    using L = MergeLayout<SR, BLOCK, IPT>;
    using W = typename SR::w_t;
    const uint32_t i0 = a.plan.tile_row[tile], i1 = a.plan.tile_row[tile + 1];
    const uint32_t j0 = a.plan.tile_nnz[tile], j1 = a.plan.tile_nnz[tile + 1];
    const uint32_t r_lo = i0 & ~3u, r_hi = (i1 + 1 + 3) & ~3u;
    const uint32_t c_lo = j0 & ~3u, c_hi = (j1 + 3) & ~3u;
    const uint32_t v_lo = j0 & ~(uint32_t)(L::AW - 1);
    const uint32_t v_hi = (j1 + L::AW - 1) & ~(uint32_t)(L::AW - 1);
    const uint32_t br = (r_hi - r_lo) * 4, bc = (c_hi - c_lo) * 4;
    const uint32_t bv = (v_hi - v_lo) * (uint32_t)sizeof(W);
    mbar_arrive_expect_tx(bar, br + bc + bv);
    bulk_g2s(st + L::RE_OFF, a.plan.row_ptr + r_lo, br, bar);
    if (bc) bulk_g2s(st + L::COL_OFF, a.col + c_lo, bc, bar);
    if (bv) bulk_g2s(st + L::VAL_OFF, a.val + v_lo, bv, bar);
}

// Persistent merge-path SpMV: CTA b folds tiles b, b+grid, ...; while tile t
// is folded, the bulk copies of tile t+grid land in the other staging buffer.
template <class SR, class Epi, int BLOCK, int IPT>
__global__ void __launch_bounds__(BLOCK, 4)
spmv_merge_kernel(MergeArgs<SR> a, Epi epi) {
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    using L = MergeLayout<SR, BLOCK, IPT>;
    extern __shared__ __align__(16) unsigned char dsm[];
    V* sv = reinterpret_cast<V*>(dsm + L::V_OFF);
    V* s_wval = reinterpret_cast<V*>(dsm + L::WVAL_OFF);
    V* s_wpre = reinterpret_cast<V*>(dsm + L::WPRE_OFF);
    int* s_wflag = reinterpret_cast<int*>(dsm + L::WFLAG_OFF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(dsm + L::BAR_OFF);
    const uint32_t tid = threadIdx.x;
    epi.begin();

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && blockIdx.x < a.plan.n_tiles)
        merge_issue_tile<SR, BLOCK, IPT>(a, blockIdx.x, dsm, &bar[0]);

    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < a.plan.n_tiles; tile += gridDim.x, ++it) {
        const uint32_t stage = it & 1u;
        const uint32_t next = tile + gridDim.x;
        if (tid == 0 && next < a.plan.n_tiles) {
            fence_proxy_async_smem();
            merge_issue_tile<SR, BLOCK, IPT>(a, next, dsm + (stage ^ 1u) * L::STAGE_BYTES,
                                             &bar[stage ^ 1u]);
        }
        const uint32_t i0 = a.plan.tile_row[tile], i1 = a.plan.tile_row[tile + 1];
        const uint32_t j0 = a.plan.tile_nnz[tile], j1 = a.plan.tile_nnz[tile + 1];
        const uint32_t na = i1 - i0, nb = j1 - j0;
        unsigned char* st = dsm + stage * L::STAGE_BYTES;
        const uint32_t* RE = reinterpret_cast<const uint32_t*>(st + L::RE_OFF) + (i0 & 3u);
        const uint32_t* CO = reinterpret_cast<const uint32_t*>(st + L::COL_OFF) + (j0 & 3u);
        const W* VA = reinterpret_cast<const W*>(st + L::VAL_OFF) + (j0 & (uint32_t)(L::AW - 1));

        const bool arrived = mbar_wait_bounded(&bar[stage], (it >> 1) & 1u);
        if (__syncthreads_or(!arrived)) {
            // A copy never completed: record it, let the copy already issued
            // for the next tile land (bounded), and stop; the host sees the
            // error word and discards this launch's results.
            if (tid == 0) {
                set_error(a.err, kDevTimeout);
                if (next < a.plan.n_tiles) mbar_wait_bounded(&bar[stage ^ 1u], ((it + 1) >> 1) & 1u);
            }
            break;
        }

        // Gather x for the tile (IPT independent loads per thread), combine.
        typename SR::x_t xv[IPT];
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = (uint32_t)u * BLOCK + tid;
            if (k < nb) xv[u] = ldg_any(a.x + CO[k]);
        }
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = (uint32_t)u * BLOCK + tid;
            if (k < nb) sv[k] = SR::combine(VA[k], xv[u]);
        }
        __syncthreads();

        // Per-thread merge-path start: row-end i precedes nonzero j iff
        // row_ptr[i0+1+i] - j0 <= j.
        const uint32_t total = na + nb;
        const uint32_t d = min(tid * (uint32_t)IPT, total);
        uint32_t lo = d > nb ? d - nb : 0;
        uint32_t hi = min(d, na);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (RE[1 + mid] - j0 <= d - 1 - mid)
                lo = mid + 1;
            else
                hi = mid;
        }
        uint32_t i = lo, j = d - lo;
        const uint32_t dend = min(d + (uint32_t)IPT, total);

        V acc = SR::identity();
        bool has_first = false;
        uint32_t first_row = 0;
        V first_val = acc;
#pragma unroll
        for (int s = 0; s < IPT; ++s) {
            if (d + (uint32_t)s < dend) {
                if (i < na && RE[1 + i] - j0 <= j) {
                    if (!has_first) {
                        has_first = true;
                        first_row = i0 + i;
                        first_val = acc;
                    } else {
                        epi.emit(i0 + i, acc);
                    }
                    acc = SR::identity();
                    ++i;
                } else {
                    acc = SR::reduce(acc, sv[j]);
                    ++j;
                }
            }
        }

        V incl, excl;
        block_seg_scan<SR, BLOCK>(has_first, acc, incl, excl, s_wval, s_wflag, s_wpre);

        if (has_first) {
            const V val = SR::reduce(excl, first_val);
            // the tile's first row began in an earlier tile: the fixup owns it
            const bool deferred = first_row == i0 && j0 > RE[0];
            if (deferred)
                a.tail[tile] = val;
            else
                epi.emit(first_row, val);
        }
        if (tid == BLOCK - 1 && tile + 1 < a.plan.n_tiles) a.carry[tile] = incl;
        __syncthreads();  // staging buffer and sv are reused next
    }
    epi.template block_end<BLOCK>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

// Finishes rows that cross tiles: for every tile T whose first row began in
// an earlier tile and ends inside T, folds carry[first..T-1] and tail[T] in
// tile order and emits the row.  One thread per tile.
template <class SR, class Epi, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
spmv_fixup_kernel(MergeArgs<SR> a, Epi epi) {
    using V = typename SR::value_t;
    __shared__ alignas(16) char epi_smem[64 * 8];
    const uint32_t t = blockIdx.x * BLOCK + threadIdx.x;
    epi.begin();
    if (t < a.plan.n_tiles) {
        const uint32_t i0 = a.plan.tile_row[t];
        const uint32_t j0 = a.plan.tile_nnz[t];
        const uint32_t i1 = a.plan.tile_row[t + 1];
        if (i1 > i0 && i0 < a.plan.n_rows) {
            const uint32_t rs = a.plan.row_ptr[i0];
            if (j0 > rs) {  // spanning row, completed in tile t (t >= 1 here)
                V acc = a.tail[t];
                uint32_t k = t - 1;
                for (;;) {
                    acc = SR::reduce(a.carry[k], acc);
                    if (k > 0 && a.plan.tile_row[k] == i0 && a.plan.tile_nnz[k] > rs)
                        --k;
                    else
                        break;
                }
                epi.emit(i0, acc);
            }
        }
    }
    epi.template block_end<BLOCK>(epi_smem);
}

// CSR-vector schedule: TPR lanes per row (TPR in {1,2,4,8,16,32}).
template <class SR, class Epi, int BLOCK, int TPR>
__global__ void __launch_bounds__(BLOCK)
spmv_vector_kernel(uint32_t n_rows, const uint32_t* row_ptr, const uint32_t* col,
                   const typename SR::w_t* val, const typename SR::x_t* x, Epi epi) {
    using V = typename SR::value_t;
    __shared__ alignas(16) char epi_smem[64 * 8];
    const uint32_t g = (blockIdx.x * BLOCK + threadIdx.x);
    epi.begin();
    const uint32_t lane = g % TPR;
    const uint32_t groups = gridDim.x * (BLOCK / TPR);
    // Rows are strided so that every lane of a group sees the same trip count.
    const uint32_t rounds = (uint32_t)ceil_div(n_rows, groups);
    for (uint32_t rr = 0; rr < rounds; ++rr) {
        const uint32_t row = rr * groups + g / TPR;
        V acc = SR::identity();
        if (row < n_rows) {
            const uint32_t rs = row_ptr[row], re = row_ptr[row + 1];
            for (uint32_t k = rs + lane; k < re; k += TPR)
                acc = SR::reduce(acc, SR::combine(ldg_any(val + k), ldg_any(x + __ldg(col + k))));
        }
        if constexpr (TPR > 1) {
#pragma unroll
            for (int off = TPR / 2; off > 0; off >>= 1) {
                constexpr int W = (sizeof(V) + 3) / 4;
                uint32_t w[W] = {};
                memcpy(w, &acc, sizeof(V));
#pragma unroll
                for (int q = 0; q < W; ++q) w[q] = __shfl_down_sync(0xffffffffu, w[q], off, TPR);
                V other;
                memcpy(&other, w, sizeof(V));
                acc = SR::reduce(acc, other);
            }
        }
        if (lane == 0 && row < n_rows) epi.emit(row, acc);
    }
    epi.template block_end<BLOCK>(epi_smem);
}

// ----------------------------------------------------------- epilogues

// Plain SpMV: y[row] = value.
template <class V>
struct StoreEpilogue {
    V* y;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t row, const V& v) { y[row] = v; }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

}  // namespace g1
