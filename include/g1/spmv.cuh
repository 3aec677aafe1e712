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
    const uint32_t* col;
    const typename SR::w_t* val;
    const typename SR::x_t* x;
    typename SR::value_t* carry;  // n_tiles: partial of the row open at tile end
    typename SR::value_t* tail;   // n_tiles: in-tile partial of a row begun earlier
};

// Shared memory of one merge tile.
template <class SR, int BLOCK, int IPT>
struct MergeSmem {
    static constexpr int ITEMS = BLOCK * IPT;
    uint32_t row_end[ITEMS + 1];
    typename SR::value_t v[ITEMS];
    typename SR::value_t wval[BLOCK / 32];
    typename SR::value_t wpre[BLOCK / 32];
    int wflag[BLOCK / 32];
    alignas(16) char epi[64 * 8];
};

template <class SR, class Epi, int BLOCK, int IPT>
__global__ void __launch_bounds__(BLOCK)
spmv_merge_kernel(MergeArgs<SR> a, Epi epi) {
    using V = typename SR::value_t;
    __shared__ MergeSmem<SR, BLOCK, IPT> sm;
    const uint32_t tid = threadIdx.x;
    epi.begin();

    for (uint32_t tile = blockIdx.x; tile < a.plan.n_tiles; tile += gridDim.x) {
        const uint32_t i0 = a.plan.tile_row[tile];
        const uint32_t j0 = a.plan.tile_nnz[tile];
        const uint32_t i1 = a.plan.tile_row[tile + 1];
        const uint32_t j1 = a.plan.tile_nnz[tile + 1];
        const uint32_t na = i1 - i0;
        const uint32_t nb = j1 - j0;

        // Stage the tile's row ends (relative to j0) and combined values.
        for (uint32_t k = tid; k < na; k += BLOCK) sm.row_end[k] = a.plan.row_ptr[i0 + 1 + k] - j0;
        if (tid == 0) sm.row_end[na] = kU32Max;
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = (uint32_t)u * BLOCK + tid;
            if (k < nb) {
                const uint32_t j = j0 + k;
                const uint32_t c = __ldg(a.col + j);
                sm.v[k] = SR::combine(a.val[j], a.x[c]);
            }
        }
        __syncthreads();

        // Per-thread merge-path start.
        const uint32_t total = na + nb;
        const uint32_t d = min(tid * (uint32_t)IPT, total);
        uint32_t lo = d > nb ? d - nb : 0;
        uint32_t hi = min(d, na);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.row_end[mid] <= d - 1 - mid)
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
                if (sm.row_end[i] <= j) {
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
                    acc = SR::reduce(acc, sm.v[j]);
                    ++j;
                }
            }
        }

        V incl, excl;
        block_seg_scan<SR, BLOCK>(has_first, acc, incl, excl, sm.wval, sm.wflag, sm.wpre);

        if (has_first) {
            const V val = SR::reduce(excl, first_val);
            bool deferred = false;
            if (first_row == i0) {
                const uint32_t rs = a.plan.row_ptr[i0];
                deferred = j0 > rs;  // the row began in an earlier tile
            }
            if (deferred)
                a.tail[tile] = val;
            else
                epi.emit(first_row, val);
        }
        if (tid == BLOCK - 1 && tile + 1 < a.plan.n_tiles) a.carry[tile] = incl;
        __syncthreads();  // smem reuse by the next tile
    }
    epi.template block_end<BLOCK>(sm.epi);
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
                acc = SR::reduce(acc, SR::combine(val[k], x[__ldg(col + k)]));
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
