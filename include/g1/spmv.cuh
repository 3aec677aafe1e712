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

#include <type_traits>
#include <utility>

#include "g1/common.cuh"
#include "g1/semiring.cuh"

namespace g1 {

// Epilogues may declare `bool active() const`: when it returns false every
// SpMV kernel returns at once (a step of a captured CUDA graph that has
// nothing to do, decided on the device).
template <class E, class = void>
struct has_active : std::false_type {};
template <class E>
struct has_active<E, std::void_t<decltype(std::declval<const E&>().active())>> : std::true_type {};
template <class E>
__device__ __forceinline__ bool epi_active(const E& e) {
    if constexpr (has_active<E>::value) return e.active();
    else return true;
}

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

template <class SR>
struct MergeArgs {
    MergePlanView plan;
    const uint32_t* col;           // readable (padded) up to round_up(nnz, 4) entries
    const typename SR::w_t* val;   // readable (padded) up to round_up(nnz, 16 / sizeof(w_t))
    const typename SR::x_t* x;
    typename SR::value_t* carry;   // n_tiles: partial of the row open at tile end
    typename SR::value_t* tail;    // n_tiles: in-tile partial of a row begun earlier
    uint32_t* err;                 // device error word (kDevTimeout on a stalled copy)
    uint32_t wait_limit = kWaitPolls;  // polls before a wait on a bulk copy gives up
};

// (row, partial) pair carried by the tile scan: the row a segment belongs
// to travels with its partial value.
template <class V>
struct RowPartial {
    uint32_t row;
    V val;
};

// Block-wide segmented scan of (head, row, value) in thread order: a head
// thread starts a new segment with its own (row, value); other threads
// extend the segment of the nearest head before them.  Rows of segments
// that began before thread 0 read as kU32Max.
template <class SR, int BLOCK>
__device__ __forceinline__ void block_seg_scan_rows(bool head, RowPartial<typename SR::value_t> v,
                                                    RowPartial<typename SR::value_t>& incl,
                                                    RowPartial<typename SR::value_t>& excl,
                                                    RowPartial<typename SR::value_t>* s_w,
                                                    int* s_wflag,
                                                    RowPartial<typename SR::value_t>* s_wpre) {
    using P = RowPartial<typename SR::value_t>;
    constexpr int NW = BLOCK / 32;
    const unsigned full = 0xffffffffu;
    const int lane = (int)lane_id();
    const int w = threadIdx.x >> 5;
    P s = v;
    int f = head ? 1 : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        P su = shfl_up_any(full, s, off);
        int fu = __shfl_up_sync(full, f, off);
        if (lane >= off) {
            if (!f) {
                s.val = SR::reduce(su.val, s.val);
                s.row = su.row;
            }
            f |= fu;
        }
    }
    if (lane == 31) {
        s_w[w] = s;
        s_wflag[w] = f;
    }
    __syncthreads();
    if (w == 0) {
        P ws;
        ws.row = kU32Max;
        ws.val = SR::identity();
        int wf = 0;
        if (lane < NW) {
            ws = s_w[lane];
            wf = s_wflag[lane];
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            P su = shfl_up_any(full, ws, off);
            int fu = __shfl_up_sync(full, wf, off);
            if (lane >= off) {
                if (!wf) {
                    ws.val = SR::reduce(su.val, ws.val);
                    ws.row = su.row;
                }
                wf |= fu;
            }
        }
        P ex = shfl_up_any(full, ws, 1);
        if (lane == 0) {
            ex.row = kU32Max;
            ex.val = SR::identity();
        }
        if (lane < NW) s_wpre[lane] = ex;
    }
    __syncthreads();
    const P pre = s_wpre[w];
    incl = s;
    if (!f) {
        incl.val = SR::reduce(pre.val, s.val);
        incl.row = pre.row;
    }
    P e = shfl_up_any(full, incl, 1);
    excl = lane == 0 ? pre : e;
}

// Dynamic shared memory of the merge kernel: STAGES staging buffers (row_ptr
// window, col, val of one tile each) plus scan/epilogue scratch and the
// mbarriers.  With 4-byte values the combined values overwrite the staged
// col slots and the per-item row-start marks overwrite the staged val slots
// (each thread rewrites only the slots it read), so a stage is all the
// per-tile memory; other sizes get their own arrays.
template <class SR, int BLOCK, int IPT, int STAGES>
struct MergeLayout {
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    static_assert(sizeof(W) == 4 || sizeof(W) == 8, "edge values of 4 or 8 bytes");
    static constexpr int ITEMS = BLOCK * IPT;
    static constexpr int AW = 16 / (int)sizeof(W);  // val elements per 16 bytes
    static constexpr int SLOTS = ((ITEMS + 8 + 3) / 4) * 4;
    static constexpr int VSLOTS = ((ITEMS + 2 * AW + AW - 1) / AW) * AW;
    static constexpr bool SV_ALIAS = sizeof(V) == 4;
    static constexpr bool SROW_ALIAS = sizeof(W) == 4;
    static constexpr size_t RE_OFF = 0;
    static constexpr size_t COL_OFF = RE_OFF + (size_t)SLOTS * 4;
    static constexpr size_t VAL_OFF = COL_OFF + (size_t)SLOTS * 4;
    static constexpr size_t STAGE_BYTES = ((VAL_OFF + (size_t)VSLOTS * sizeof(W)) + 15) / 16 * 16;
    static constexpr size_t SV_OFF = STAGES * STAGE_BYTES;
    static constexpr size_t SV_BYTES = SV_ALIAS ? 0 : ((ITEMS * sizeof(V) + 15) / 16) * 16;
    static constexpr size_t SROW_OFF = SV_OFF + SV_BYTES;
    static constexpr size_t SROW_BYTES = SROW_ALIAS ? 0 : (size_t)SLOTS * 4;
    using P = RowPartial<V>;
    static constexpr size_t W_OFF = SROW_OFF + SROW_BYTES;
    static constexpr size_t WP_BYTES = ((BLOCK / 32) * sizeof(P) + 15) / 16 * 16;
    static constexpr size_t WPRE_OFF = W_OFF + WP_BYTES;
    static constexpr size_t WFLAG_OFF = WPRE_OFF + WP_BYTES;
    static constexpr size_t EPI_OFF = WFLAG_OFF + ((BLOCK / 32) * 4 + 15) / 16 * 16;
    static constexpr size_t BAR_OFF = EPI_OFF + 512;
    static constexpr size_t BYTES = BAR_OFF + 16;
};

// Issues the bulk copies of tile `tile` into staging buffer `st` (one
// thread): row_ptr[i0 .. i1+1], col and val of nonzeros [j0, j1), each range
// widened to 16-byte boundaries (the arrays are padded for that).
template <class L, class SR>
__device__ __forceinline__ void merge_issue_tile(const MergeArgs<SR>& a, uint32_t tile,
                                                 unsigned char* st, uint64_t* bar) {
    using W = typename SR::w_t;
    const uint32_t i0 = a.plan.tile_row[tile], i1 = a.plan.tile_row[tile + 1];
    const uint32_t j0 = a.plan.tile_nnz[tile], j1 = a.plan.tile_nnz[tile + 1];
    const uint32_t r_lo = i0 & ~3u, r_hi = (i1 + 2 + 3) & ~3u;
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

// Persistent merge-path SpMV.  CTA b folds tiles b, b+grid, ... (tile
// boundaries from the merge-path partition, so rows + nonzeros are balanced
// across tiles whatever the degree distribution).  Per tile:
//   1. wait for the tile's bulk copies (with STAGES == 2 the next tile's
//      copies are already in flight into the other buffer);
//   2. each thread gathers x for IPT strided nonzeros and combines them;
//   3. rows are walked: empty rows emit identity at once, every non-empty
//      row that starts inside the tile marks its first nonzero with its id;
//   4. each thread folds IPT consecutive nonzeros, closing a segment at
//      every mark (independent shared-memory reads: no search, no chain);
//   5. a (row, value) segmented scan carries open segments across threads;
//      the first segment of each thread and the tile's last segment are
//      emitted after it.  A row that began in an earlier tile is finished by
//      spmv_fixup_kernel from the tiles' carries (tail holds its in-tile part).
template <class SR, class Epi, int BLOCK, int IPT, int STAGES>
__global__ void __launch_bounds__(BLOCK, STAGES == 1 ? 6 : 4)
spmv_merge_kernel(MergeArgs<SR> a, Epi epi) {
    if (!epi_active(epi)) return;
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    using L = MergeLayout<SR, BLOCK, IPT, STAGES>;
    using P = RowPartial<V>;
    extern __shared__ __align__(16) unsigned char dsm[];
    P* s_w = reinterpret_cast<P*>(dsm + L::W_OFF);
    P* s_wpre = reinterpret_cast<P*>(dsm + L::WPRE_OFF);
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
        merge_issue_tile<L>(a, blockIdx.x, dsm, &bar[0]);

    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < a.plan.n_tiles; tile += gridDim.x, ++it) {
        const uint32_t stage = STAGES == 2 ? (it & 1u) : 0u;
        const uint32_t parity = STAGES == 2 ? ((it >> 1) & 1u) : (it & 1u);
        const uint32_t next = tile + gridDim.x;
        if (STAGES == 2 && tid == 0 && next < a.plan.n_tiles) {
            fence_proxy_async_smem();
            merge_issue_tile<L>(a, next, dsm + (stage ^ 1u) * L::STAGE_BYTES, &bar[stage ^ 1u]);
        }
        const uint32_t i0 = a.plan.tile_row[tile], i1 = a.plan.tile_row[tile + 1];
        const uint32_t j0 = a.plan.tile_nnz[tile], j1 = a.plan.tile_nnz[tile + 1];
        const uint32_t nb = j1 - j0;
        unsigned char* st = dsm + stage * L::STAGE_BYTES;
        const uint32_t* RE = reinterpret_cast<const uint32_t*>(st + L::RE_OFF) + (i0 & 3u);
        const uint32_t* CO = reinterpret_cast<const uint32_t*>(st + L::COL_OFF) + (j0 & 3u);
        const W* VA = reinterpret_cast<const W*>(st + L::VAL_OFF) + (j0 & (uint32_t)(L::AW - 1));
        V* sv = L::SV_ALIAS ? reinterpret_cast<V*>(const_cast<uint32_t*>(CO))
                            : reinterpret_cast<V*>(dsm + L::SV_OFF);
        uint32_t* srow = L::SROW_ALIAS ? reinterpret_cast<uint32_t*>(const_cast<W*>(VA))
                                       : reinterpret_cast<uint32_t*>(dsm + L::SROW_OFF);

        const bool arrived = mbar_wait_bounded(&bar[stage], parity, a.wait_limit);
        if (__syncthreads_or(!arrived)) {
            // A copy did not complete in time: record it, let this tile's
            // copy and the one already issued for the next tile land
            // (bounded) before the block leaves its shared memory, and stop;
            // the host sees the error word and discards this launch's results.
            if (tid == 0) {
                set_error(a.err, kDevTimeout);
                mbar_wait_bounded(&bar[stage], parity);
                if (STAGES == 2 && next < a.plan.n_tiles)
                    mbar_wait_bounded(&bar[stage ^ 1u], ((it + 1) >> 1) & 1u);
            }
            __syncthreads();
            break;
        }

        // 2. gather + combine; clear the row-start marks of the same slots
        typename SR::x_t xv[IPT];
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = (uint32_t)u * BLOCK + tid;
            if (k < nb) xv[u] = ldg_any(a.x + CO[k]);
        }
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = (uint32_t)u * BLOCK + tid;
            if (k < nb) {
                const V c = SR::combine(VA[k], xv[u]);
                sv[k] = c;
                srow[k] = kU32Max;
            }
        }
        __syncthreads();

        // 3. rows of the tile: i0 .. i1 (i1 may only start here).  The first
        // row is "spanning" when some of its nonzeros lie in earlier tiles.
        const bool spanning = j0 > RE[0];
        for (uint32_t r = i0 + tid; r <= i1; r += BLOCK) {
            const uint32_t rs = RE[r - i0], re = RE[r - i0 + 1];
            if (r == i0 && spanning) {
                // completes here with no nonzero in this tile: in-tile part is empty
                if (i1 > i0 && re == j0) a.tail[tile] = SR::identity();
                continue;
            }
            if (r < i1 && re == rs) {
                epi.emit(r, SR::identity());  // empty row
            } else if (rs < j1) {
                srow[rs - j0] = r;  // non-empty row starting in this tile
            }
        }
        __syncthreads();

        // 4. per-thread fold of IPT consecutive nonzeros
        const uint32_t k0 = tid * (uint32_t)IPT;
        V acc = SR::identity();
        bool head = false;
        uint32_t open_row = kU32Max;
        V first_val = acc;
        uint32_t lead = 0;  // nonzeros folded before the first mark
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            const uint32_t k = k0 + (uint32_t)u;
            if (k < nb) {
                const uint32_t mark = srow[k];
                const V val = sv[k];
                if (mark != kU32Max) {
                    if (!head) {
                        head = true;
                        first_val = acc;
                        lead = (uint32_t)u;
                    } else {
                        epi.emit(open_row, acc);
                    }
                    open_row = mark;
                    acc = SR::identity();
                }
                acc = SR::reduce(acc, val);
            }
        }

        // 5. stitch segments across threads
        P mine;
        mine.row = open_row;
        mine.val = acc;
        P incl, excl;
        block_seg_scan_rows<SR, BLOCK>(head, mine, incl, excl, s_w, s_wflag, s_wpre);

        if (head && !(tid == 0 && lead == 0)) {
            // the segment open at this thread's start ends before its first mark
            const V val = SR::reduce(excl.val, first_val);
            if (excl.row == kU32Max) {
                if (spanning) a.tail[tile] = val;  // first row began in an earlier tile
            } else {
                epi.emit(excl.row, val);
            }
        }
        if (tid == BLOCK - 1) {
            // the tile's last segment
            uint32_t lr = incl.row;
            if (lr == kU32Max && spanning) lr = i0;
            V carry = SR::identity();
            if (lr != kU32Max) {
                if (lr < i1) {  // completes at the tile's end
                    if (lr == i0 && spanning)
                        a.tail[tile] = incl.val;
                    else
                        epi.emit(lr, incl.val);
                } else {
                    carry = incl.val;  // row i1 continues in the next tile
                }
            }
            if (tile + 1 < a.plan.n_tiles) a.carry[tile] = carry;
        }
        __syncthreads();  // staging buffer reuse
        if (STAGES == 1 && tid == 0 && next < a.plan.n_tiles) {
            fence_proxy_async_smem();
            merge_issue_tile<L>(a, next, dsm, &bar[0]);
        }
    }
    epi.template block_end<BLOCK>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

// Warp-level (row, value) segmented scan, same contract as the block scan.
template <class SR>
__device__ __forceinline__ void warp_seg_scan_rows(bool head, RowPartial<typename SR::value_t> v,
                                                   RowPartial<typename SR::value_t>& incl,
                                                   RowPartial<typename SR::value_t>& excl) {
    using P = RowPartial<typename SR::value_t>;
    const unsigned full = 0xffffffffu;
    const int lane = (int)lane_id();
    P s = v;
    int f = head ? 1 : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        P su = shfl_up_any(full, s, off);
        int fu = __shfl_up_sync(full, f, off);
        if (lane >= off) {
            if (!f) {
                s.val = SR::reduce(su.val, s.val);
                s.row = su.row;
            }
            f |= fu;
        }
    }
    incl = s;
    P e = shfl_up_any(full, s, 1);
    if (lane == 0) {
        e.row = kU32Max;
        e.val = SR::identity();
    }
    excl = e;
}

// Warp-tile merge-path SpMV: the merge-path partition is cut into tiles of
// 32*IPT items and every warp folds its own tiles with no block barrier.
// Lane l loads nonzeros l, l+32, ... of the tile (coalesced), gathers x and
// combines into the warp's shared-memory slice; rows of the tile are walked
// the same way (empty rows emit identity, row starts are marked); then lane
// l folds items [l*IPT, (l+1)*IPT) (odd IPT: bank-conflict free), a warp
// (row, value) segmented scan carries open segments across lanes, and rows
// that cross tiles are finished by spmv_fixup_kernel.
// Shared memory of the warp-tile kernel: an optional cache of x[0, HOT)
// (the hottest vertices when the graph is degree-ordered) and, per warp, the
// (combined value, row-start mark) of each item and the value of each row
// completed in the tile.
// x[c] from the shared-memory copy of x[0, hot) or from global x.  For
// 4-byte values one generic-address load (a shared and a global load would
// both issue for almost every warp); otherwise the two-way select.
template <class X>
__device__ __forceinline__ X gather_x(const X* xc, const X* x, uint32_t c, uint32_t hot) {
    if constexpr (sizeof(X) == 4) {
        const uint32_t bits = ld_generic_u32((c < hot ? xc : x) + c);
        X v;
        memcpy(&v, &bits, 4);
        return v;
    } else {
        return c < hot ? xc[c] : ldg_any(x + c);
    }
}

template <class V>
struct alignas(8) ItemSlot {
    V val;
    uint32_t mark;
};

template <class SR, int WARPS, int IPT, int HOT>
struct WarpMergeLayout {
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    using S = ItemSlot<V>;
    static constexpr int WITEMS = 32 * IPT;
    static constexpr size_t XC_OFF = 0;
    static constexpr size_t XC_BYTES = ((size_t)HOT * sizeof(X) + 15) / 16 * 16;
    static constexpr size_t S_OFF = XC_OFF + XC_BYTES;
    static constexpr size_t S_BYTES = ((size_t)WARPS * WITEMS * sizeof(S) + 15) / 16 * 16;
    static constexpr size_t Y_OFF = S_OFF + S_BYTES;
    static constexpr size_t Y_BYTES = ((size_t)WARPS * WITEMS * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t EPI_OFF = Y_OFF + Y_BYTES;
    static constexpr size_t BYTES = EPI_OFF + 512;
};

// Items each warp tile may read past its last nonzero (the col/val arrays
// are padded with this many zero entries): loads need no bounds checks.
constexpr uint32_t kWarpTilePad = 1024;

// BOUNDED: col/val loads stay inside [0, nnz) (for CSR arrays without the
// tile padding); otherwise loads run past the tile into the padding.
template <class SR, class Epi, int WARPS, int IPT, int MINB, int HOT, bool BOUNDED = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
spmv_wmerge_kernel(MergeArgs<SR> a, Epi epi) {
    if (!epi_active(epi)) return;
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    using W = typename SR::w_t;
    using P = RowPartial<V>;
    using L = WarpMergeLayout<SR, WARPS, IPT, HOT>;
    using S = ItemSlot<V>;
    constexpr int WITEMS = L::WITEMS;
    static_assert(WITEMS <= (int)kWarpTilePad, "tile larger than the array padding");
    extern __shared__ __align__(16) unsigned char dsm[];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    X* xc = reinterpret_cast<X*>(dsm + L::XC_OFF);
    S* slot = reinterpret_cast<S*>(dsm + L::S_OFF) + (size_t)w * WITEMS;
    V* sy = reinterpret_cast<V*>(dsm + L::Y_OFF) + (size_t)w * WITEMS;
    epi.begin();
    // x[0, HOT) is read once per CTA and served from shared memory.
    const uint32_t hot = HOT < a.plan.n_rows ? (uint32_t)HOT : a.plan.n_rows;
    if constexpr (HOT > 0) {
        fill_x_cache<WARPS * 32>(xc, a.x, hot);
        __syncthreads();
    }
    const uint32_t total_warps = gridDim.x * WARPS;
    uint32_t tile = blockIdx.x * WARPS + w;
    // tile coordinates are fetched one tile ahead
    uint32_t c_i0 = 0, c_i1 = 0, c_j0 = 0, c_j1 = 0;
    if (tile < a.plan.n_tiles) {
        c_i0 = a.plan.tile_row[tile];
        c_i1 = a.plan.tile_row[tile + 1];
        c_j0 = a.plan.tile_nnz[tile];
        c_j1 = a.plan.tile_nnz[tile + 1];
    }
    for (; tile < a.plan.n_tiles; tile += total_warps) {
        const uint32_t i0 = c_i0, i1 = c_i1, j0 = c_j0, j1 = c_j1;
        const uint32_t nxt = tile + total_warps;
        if (nxt < a.plan.n_tiles) {
            c_i0 = a.plan.tile_row[nxt];
            c_i1 = a.plan.tile_row[nxt + 1];
            c_j0 = a.plan.tile_nnz[nxt];
            c_j1 = a.plan.tile_nnz[nxt + 1];
        }
        const uint32_t nb = j1 - j0;
        // items u*32 + lane exist for u < nv (col/val are loaded regardless:
        // the arrays are padded, and padding columns are 0)
        const uint32_t nv = nb > lane ? (nb - lane + 31) >> 5 : 0u;
        const uint32_t* colp = a.col + j0 + lane;
        const W* valp = a.val + j0 + lane;
        uint32_t cv[IPT];
        W wv[IPT];
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if (!BOUNDED || (uint32_t)u < nv) {
                cv[u] = __ldg(colp + u * 32);
                wv[u] = ldg_any(valp + u * 32);
            }
        }
        const uint32_t r_lane = i0 + lane;
        uint32_t ra = 0, rb = 0;
        if (r_lane <= i1) {
            ra = __ldg(a.plan.row_ptr + r_lane);
            // row_ptr[n + 1] exists only in padded arrays
            rb = (!BOUNDED || r_lane < a.plan.n_rows) ? __ldg(a.plan.row_ptr + r_lane + 1) : ra;
        }
        X xv[IPT];
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nv) {
                if constexpr (HOT > 0)
                    xv[u] = gather_x(xc, a.x, cv[u], hot);
                else
                    xv[u] = ldg_any(a.x + cv[u]);
            }
        }
        const bool spanning = j0 > __shfl_sync(0xffffffffu, ra, 0);
        S* sl = slot + lane;
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nv) {
                S e;
                e.val = SR::combine(wv[u], xv[u]);
                e.mark = kU32Max;
                sl[u * 32] = e;
            }
        }
        __syncwarp();
        // Rows i0..i1 of the tile: empty rows get identity, starts are marked.
        for (uint32_t r = r_lane; r <= i1; r += 32) {
            uint32_t rs = ra, re = rb;
            if (r != r_lane) {
                rs = __ldg(a.plan.row_ptr + r);
                re = (!BOUNDED || r < a.plan.n_rows) ? __ldg(a.plan.row_ptr + r + 1) : rs;
            }
            if (r == i0 && spanning) {
                if (i1 > i0 && re == j0) a.tail[tile] = SR::identity();
                continue;
            }
            if (r < i1) {
                if (re == rs)
                    sy[r - i0] = SR::identity();  // empty row
                else
                    slot[rs - j0].mark = r;
            } else if (rs < j1) {
                slot[rs - j0].mark = r;  // row i1 starts here and continues
            }
        }
        __syncwarp();

        // Fold IPT consecutive items; a closed segment is a finished row.
        const uint32_t k0 = lane * (uint32_t)IPT;
        const uint32_t nk = nb > k0 ? min(nb - k0, (uint32_t)IPT) : 0u;
        const S* sk = slot + k0;
        V acc = SR::identity();
        bool head = false;
        uint32_t open_row = kU32Max;
        V first_val = acc;
        uint32_t lead = 0;
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nk) {
                const S e = sk[u];
                if (e.mark != kU32Max) {
                    if (!head) {
                        head = true;
                        first_val = acc;
                        lead = (uint32_t)u;
                    } else {
                        sy[open_row - i0] = acc;
                    }
                    open_row = e.mark;
                    acc = SR::identity();
                }
                acc = SR::reduce(acc, e.val);
            }
        }
        P mine;
        mine.row = open_row;
        mine.val = acc;
        P incl, excl;
        warp_seg_scan_rows<SR>(head, mine, incl, excl);
        if (head && !(lane == 0 && lead == 0)) {
            const V val = SR::reduce(excl.val, first_val);
            if (excl.row == kU32Max) {
                if (spanning) a.tail[tile] = val;
            } else {
                sy[excl.row - i0] = val;
            }
        }
        if (lane == 31) {
            uint32_t lr = incl.row;
            if (lr == kU32Max && spanning) lr = i0;
            V carry = SR::identity();
            if (lr != kU32Max) {
                if (lr < i1) {
                    if (lr == i0 && spanning)
                        a.tail[tile] = incl.val;
                    else
                        sy[lr - i0] = incl.val;
                } else {
                    carry = incl.val;
                }
            }
            if (tile + 1 < a.plan.n_tiles) a.carry[tile] = carry;
        }
        __syncwarp();
        // Coalesced epilogue over the rows completed in this tile.
        for (uint32_t r = i0 + (spanning ? 1u : 0u) + lane; r < i1; r += 32) epi.emit(r, sy[r - i0]);
        __syncwarp();
    }
    epi.template block_end<WARPS * 32>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

// Per-warp shared memory of the bulk-staged warp-tile kernel: the tile's
// col and val (4-byte values) land in `stage` by one bulk copy and the same
// bytes are then reused as the tile's (value, mark) slots; `y` holds the
// values of the rows completed in the tile.
template <class SR, int IPT>
struct WarpTmaSlice {
    using V = typename SR::value_t;
    static constexpr int WITEMS = 32 * IPT;
    static constexpr size_t COL_OFF = 0;
    static constexpr size_t VAL_OFF = ((size_t)(WITEMS + 8) * 4 + 15) / 16 * 16;
    static constexpr size_t STAGE_BYTES = VAL_OFF + ((size_t)(WITEMS + 8) * 4 + 15) / 16 * 16;
    static constexpr size_t SLOT_BYTES = (size_t)WITEMS * sizeof(ItemSlot<V>);
    static constexpr size_t BUF_BYTES = STAGE_BYTES > SLOT_BYTES ? STAGE_BYTES : SLOT_BYTES;
    static constexpr size_t Y_OFF = BUF_BYTES;
    static constexpr size_t BAR_OFF = Y_OFF + ((size_t)WITEMS * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t BYTES = BAR_OFF + 16;
};

template <class SR, int WARPS, int IPT, int HOT>
struct WarpTmaLayout {
    using X = typename SR::x_t;
    using S = WarpTmaSlice<SR, IPT>;
    static constexpr size_t XC_BYTES = ((size_t)HOT * sizeof(X) + 15) / 16 * 16;
    static constexpr size_t SLICE_OFF = XC_BYTES;
    static constexpr size_t EPI_OFF = SLICE_OFF + (size_t)WARPS * S::BYTES;
    static constexpr size_t BYTES = EPI_OFF + 512;
};

// One lane issues the bulk copies of a warp tile's col/val ranges widened to
// 16-byte boundaries (the arrays are padded for that).
template <class SR, int IPT>
__device__ __forceinline__ void warp_tile_issue(const MergeArgs<SR>& a, uint32_t j0, uint32_t j1,
                                                unsigned char* slice, uint64_t* bar) {
    using S = WarpTmaSlice<SR, IPT>;
    const uint32_t c_lo = j0 & ~3u, c_hi = (j1 + 3) & ~3u;
    const uint32_t bytes = (c_hi - c_lo) * 4;
    if (bytes == 0) {
        mbar_arrive_expect_tx(bar, 0);
        return;
    }
    mbar_arrive_expect_tx(bar, 2 * bytes);
    bulk_g2s(slice + S::COL_OFF, a.col + c_lo, bytes, bar);
    bulk_g2s(slice + S::VAL_OFF, a.val + c_lo, bytes, bar);
}

// Warp-tile merge SpMV with bulk-staged tiles: as spmv_wmerge_kernel, but the
// tile's col/val arrive by a bulk copy into the warp's shared memory (no
// registers tied up by in-flight loads), which allows tiles of 32*IPT items
// with IPT up to 31 and so amortises the per-tile scan, row walk and
// epilogue over many more items.  4-byte edge values only.
template <class SR, class Epi, int WARPS, int IPT, int HOT>
__global__ void __launch_bounds__(WARPS * 32, 1)
spmv_wtma_kernel(MergeArgs<SR> a, Epi epi) {
    if (!epi_active(epi)) return;
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    using W = typename SR::w_t;
    using P = RowPartial<V>;
    using L = WarpTmaLayout<SR, WARPS, IPT, HOT>;
    using SL = WarpTmaSlice<SR, IPT>;
    using S = ItemSlot<V>;
    static_assert(sizeof(W) == 4, "bulk-staged tiles need 4-byte edge values");
    
    extern __shared__ __align__(16) unsigned char dsm[];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    X* xc = reinterpret_cast<X*>(dsm);
    unsigned char* slice = dsm + L::SLICE_OFF + (size_t)w * SL::BYTES;
    S* slot = reinterpret_cast<S*>(slice);
    V* sy = reinterpret_cast<V*>(slice + SL::Y_OFF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(slice + SL::BAR_OFF);
    epi.begin();
    if (lane == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    const uint32_t hot = HOT < a.plan.n_rows ? (uint32_t)HOT : a.plan.n_rows;
    if constexpr (HOT > 0)
        fill_x_cache<WARPS * 32>(xc, a.x, hot);
    __syncthreads();

    const uint32_t total_warps = gridDim.x * WARPS;
    uint32_t tile = blockIdx.x * WARPS + w;
    uint32_t c_i0 = 0, c_i1 = 0, c_j0 = 0, c_j1 = 0;
    if (tile < a.plan.n_tiles) {
        c_i0 = a.plan.tile_row[tile];
        c_i1 = a.plan.tile_row[tile + 1];
        c_j0 = a.plan.tile_nnz[tile];
        c_j1 = a.plan.tile_nnz[tile + 1];
        if (lane == 0) warp_tile_issue<SR, IPT>(a, c_j0, c_j1, slice, bar);
    }
    uint32_t phase = 0;
    bool failed = false;
    for (; tile < a.plan.n_tiles; tile += total_warps, phase ^= 1u) {
        const uint32_t i0 = c_i0, i1 = c_i1, j0 = c_j0, j1 = c_j1;
        const uint32_t nxt = tile + total_warps;
        if (nxt < a.plan.n_tiles) {
            c_i0 = a.plan.tile_row[nxt];
            c_i1 = a.plan.tile_row[nxt + 1];
            c_j0 = a.plan.tile_nnz[nxt];
            c_j1 = a.plan.tile_nnz[nxt + 1];
        }
        const uint32_t nb = j1 - j0;
        const uint32_t nv = nb > lane ? (nb - lane + 31) >> 5 : 0u;
        const uint32_t r_lane = i0 + lane;
        uint32_t ra = 0, rb = 0;
        if (r_lane <= i1) {
            ra = __ldg(a.plan.row_ptr + r_lane);
            rb = __ldg(a.plan.row_ptr + r_lane + 1);
        }
        const bool arrived = mbar_wait_bounded(bar, phase, a.wait_limit);
        if (!__all_sync(0xffffffffu, arrived)) {
            // let the copy in flight land (bounded) before the warp leaves
            // its shared memory
            if (lane == 0) {
                set_error(a.err, kDevTimeout);
                mbar_wait_bounded(bar, phase);
            }
            __syncwarp();
            failed = true;
            break;
        }
        const uint32_t* CO = reinterpret_cast<const uint32_t*>(slice + SL::COL_OFF) + (j0 & 3u);
        const W* VA = reinterpret_cast<const W*>(slice + SL::VAL_OFF) + (j0 & 3u);
        V vv[IPT];
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nv) {
                const uint32_t c = CO[u * 32 + lane];
                X xval;
                if constexpr (HOT > 0)
                    xval = gather_x(xc, a.x, c, hot);
                else
                    xval = ldg_any(a.x + c);
                vv[u] = SR::combine(VA[u * 32 + lane], xval);
            }
        }
        const bool spanning = j0 > __shfl_sync(0xffffffffu, ra, 0);
        __syncwarp();  // every lane is done with the staged col/val
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nv) {
                S e;
                e.val = vv[u];
                e.mark = kU32Max;
                slot[u * 32 + lane] = e;
            }
        }
        __syncwarp();
        for (uint32_t r = r_lane; r <= i1; r += 32) {
            uint32_t rs = ra, re = rb;
            if (r != r_lane) {
                rs = __ldg(a.plan.row_ptr + r);
                re = __ldg(a.plan.row_ptr + r + 1);
            }
            if (r == i0 && spanning) {
                if (i1 > i0 && re == j0) a.tail[tile] = SR::identity();
                continue;
            }
            if (r < i1) {
                if (re == rs)
                    sy[r - i0] = SR::identity();
                else
                    slot[rs - j0].mark = r;
            } else if (rs < j1) {
                slot[rs - j0].mark = r;
            }
        }
        __syncwarp();

        const uint32_t k0 = lane * (uint32_t)IPT;
        const uint32_t nk = nb > k0 ? min(nb - k0, (uint32_t)IPT) : 0u;
        const S* sk = slot + k0;
        V acc = SR::identity();
        bool head = false;
        uint32_t open_row = kU32Max;
        V first_val = acc;
        uint32_t lead = 0;
#pragma unroll
        for (int u = 0; u < IPT; ++u) {
            if ((uint32_t)u < nk) {
                const S e = sk[u];
                if (e.mark != kU32Max) {
                    if (!head) {
                        head = true;
                        first_val = acc;
                        lead = (uint32_t)u;
                    } else {
                        sy[open_row - i0] = acc;
                    }
                    open_row = e.mark;
                    acc = SR::identity();
                }
                acc = SR::reduce(acc, e.val);
            }
        }
        P mine;
        mine.row = open_row;
        mine.val = acc;
        P incl, excl;
        warp_seg_scan_rows<SR>(head, mine, incl, excl);
        if (head && !(lane == 0 && lead == 0)) {
            const V val = SR::reduce(excl.val, first_val);
            if (excl.row == kU32Max) {
                if (spanning) a.tail[tile] = val;
            } else {
                sy[excl.row - i0] = val;
            }
        }
        if (lane == 31) {
            uint32_t lr = incl.row;
            if (lr == kU32Max && spanning) lr = i0;
            V carry = SR::identity();
            if (lr != kU32Max) {
                if (lr < i1) {
                    if (lr == i0 && spanning)
                        a.tail[tile] = incl.val;
                    else
                        sy[lr - i0] = incl.val;
                } else {
                    carry = incl.val;
                }
            }
            if (tile + 1 < a.plan.n_tiles) a.carry[tile] = carry;
        }
        __syncwarp();  // slots are dead: the next tile's bulk copy may land
        if (lane == 0 && nxt < a.plan.n_tiles) {
            fence_proxy_async_smem();
            warp_tile_issue<SR, IPT>(a, c_j0, c_j1, slice, bar);
        }
        for (uint32_t r = i0 + (spanning ? 1u : 0u) + lane; r < i1; r += 32) epi.emit(r, sy[r - i0]);
        __syncwarp();
    }
    (void)failed;
    epi.template block_end<WARPS * 32>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

// Finishes rows that cross tiles.  For every tile T whose first row i0
// began in an earlier tile and ends inside T, the row's value is
// carry[first..T-1] (partials of the row in the tiles it spans) folded with
// tail[T] (its part inside T).  The common case -- the row began in tile
// T-1 -- is one load per thread; rows spanning more tiles (hubs) are folded
// by the whole warp: a binary search over tile_row finds the first tile of
// the row, then the lanes fold the carries strided and combine them with a
// shuffle tree.  The emit goes through the same epilogue as the main kernel.
template <class SR, class Epi, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
spmv_fixup_kernel(MergeArgs<SR> a, Epi epi) {
    if (!epi_active(epi)) return;
    using V = typename SR::value_t;
    __shared__ alignas(16) char epi_smem[64 * 8];
    const uint32_t t = blockIdx.x * BLOCK + threadIdx.x;
    const uint32_t lane = lane_id();
    epi.begin();
    bool longc = false;
    uint32_t i0 = 0, rs = 0;
    V acc = SR::identity();
    if (t < a.plan.n_tiles) {
        i0 = a.plan.tile_row[t];
        const uint32_t j0 = a.plan.tile_nnz[t];
        const uint32_t i1 = a.plan.tile_row[t + 1];
        if (i1 > i0 && i0 < a.plan.n_rows) {
            rs = a.plan.row_ptr[i0];
            if (j0 > rs) {  // spanning row, completed in tile t (t >= 1 here)
                acc = SR::reduce(a.carry[t - 1], a.tail[t]);
                const uint32_t k = t - 1;
                if (k > 0 && a.plan.tile_row[k] == i0 && a.plan.tile_nnz[k] > rs)
                    longc = true;  // the row also spans tile t-2 or earlier
                else
                    epi.emit(i0, acc);
            }
        }
    }
    unsigned pending = __ballot_sync(0xffffffffu, longc);
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const uint32_t r = __shfl_sync(0xffffffffu, i0, src);
        const uint32_t rsv = __shfl_sync(0xffffffffu, rs, src);
        const uint32_t tt = blockIdx.x * BLOCK + (threadIdx.x & ~31u) + (uint32_t)src;
        // first tile whose start lies in row r
        uint32_t lo = 0, hi = tt - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (a.plan.tile_row[mid] < r) lo = mid + 1; else hi = mid;
        }
        // the row began inside tile lo-1 unless tile lo starts exactly at it
        const uint32_t first = (lo > 0 && a.plan.tile_nnz[lo] > rsv) ? lo - 1 : lo;
        V part = SR::identity();
        for (uint32_t k = first + lane; k + 1 < tt; k += 32)
            part = SR::reduce(part, a.carry[k]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            part = SR::reduce(part, shfl_down_any(0xffffffffu, part, off));
        part = shfl_any(0xffffffffu, part, 0);  // the fold's total sits in lane 0
        if ((int)lane == src) epi.emit(i0, SR::reduce(part, acc));
    }
    epi.template block_end<BLOCK>(epi_smem);
}

// ------------------------------------------------------ nnz-split tiles
//
// Tile t covers the nonzeros [t*256, (t+1)*256): lane l of the tile's warp
// folds the 8 consecutive nonzeros from t*256 + 8l, read with two 16-byte
// loads of col and two of val.  Row starts come from a bitmap over the
// nonzeros (bit k: nonzero k is the first of its row), so a lane finds its
// segment boundaries with one word load and no search; rows are numbered by
// their rank among the non-empty rows.  Per tile:
//   1. lane-local fold of the 8 products; every segment that starts and ends
//      inside the lane is stored (by its number within the tile) in shared
//      memory; the lane keeps its head (items before its first start) and
//      its tail (items from its last start);
//   2. a warp segmented scan of the tails joins segments that cross lanes;
//   3. the tile's complete rows are emitted in row order, 32 at a time
//      (coalesced row-id loads and epilogue stores);
//   4. a row open at the tile end leaves its partial in carry[t]; the part
//      of a row begun in an earlier tile goes to tail[t]; rows that cross
//      tiles and the empty rows are finished by spmv_nnz_fixup_kernel.
// Work per tile is exactly 256 nonzeros whatever the degree distribution;
// empty rows cost nothing here.

constexpr uint32_t kNnzIpt = 8;
constexpr uint32_t kNnzTile = 32 * kNnzIpt;

struct NnzPlanView {
    uint32_t n_rows;
    uint32_t nnz;
    uint32_t n_tiles;   // ceil(nnz / 256)
    uint32_t n_nonempty;
    uint32_t n_empty;
    const uint32_t* tile_seg;    // n_tiles + 1: rank of the row holding nonzero t*256
    const uint32_t* sbits;       // row-start bitmap, zero-padded to n_tiles*8 + 1 words
    const uint32_t* nz_rows;     // non-empty rows in order
    const uint32_t* empty_rows;  // n_empty
    const uint32_t* row_ptr;     // n_rows + 1
    uint32_t n_fix;
    const uint32_t* fix_tiles;   // tiles in which a row begun in an earlier tile ends
    const uint4* fix_info;       // per such tile: {tile, row, tile of the row's first nonzero, 0}
    uint32_t n_fix_short;        // fix_info[0, n_fix_short): rows begun in the previous tile;
                                 // the rest: rows that span more tiles
};

template <class SR>
struct NnzArgs {
    NnzPlanView plan;
    const uint32_t* col;          // padded by at least kNnzTile entries
    const typename SR::w_t* val;  // padded likewise
    const typename SR::x_t* x;
    typename SR::value_t* carry;  // n_tiles: partial of the row open at the tile end
    typename SR::value_t* tail;   // n_tiles: in-tile partial of a row begun earlier
    uint32_t* err = nullptr;      // device error word (bounded waits of the bulk variant)
    uint32_t wait_limit = kWaitPolls;  // polls before a wait on a bulk copy gives up
};

// Epilogues may split emit into prepare(row) -- the loads that depend only
// on the row, issued before the row's value is known -- and
// emit_prepared(row, value, prepared).
template <class E, class = void>
struct has_prepare : std::false_type {};
template <class E>
struct has_prepare<E, std::void_t<decltype(std::declval<E&>().prepare(0u))>> : std::true_type {};

// Shared memory of one block: the x cache, the per-warp segment values,
// with BULK the per-warp staging buffer of one tile's col (BULK 2) or col
// and val (BULK 1), filled by bulk copies, and the warps' mbarriers, then
// the epilogue's scratch.
template <class SR, int WARPS, int HOT, int BULK = 0>
struct NnzLayout {
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    static constexpr size_t XC_OFF = 0;
    static constexpr size_t XC_BYTES = ((size_t)HOT * sizeof(X) + 15) / 16 * 16;
    static constexpr size_t SY_OFF = XC_OFF + XC_BYTES;
    static constexpr size_t SY_BYTES = ((size_t)WARPS * kNnzTile * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t ST_OFF = SY_OFF + SY_BYTES;
    static constexpr size_t ST_WARP = (BULK == 2 ? 1 : 2) * kNnzTile * 4;  // col [then val]
    static constexpr size_t ST_BYTES = BULK ? (size_t)WARPS * ST_WARP : 0;
    static constexpr size_t BAR_OFF = ST_OFF + ST_BYTES;
    static constexpr size_t BAR_BYTES = BULK ? (size_t)WARPS * 8 : 0;
    static constexpr size_t EPI_OFF = BAR_OFF + BAR_BYTES;
    static constexpr size_t BYTES = EPI_OFF + 512;
};

// Epilogues whose emit(v) touches only row v's outputs (plus block-local
// partials and atomics) declare `static constexpr bool kRowsIndependent =
// true`: the fixup then emits the empty rows while the main kernel still
// runs.
template <class E, class = void>
struct rows_independent : std::false_type {};
template <class E>
struct rows_independent<E, std::enable_if_t<E::kRowsIndependent>> : std::true_type {};

// Epilogues with members `const uint32_t* empty_list; uint32_t
// n_empty_list;` may narrow the empty rows the nnz fixup emits: when
// empty_list is set, only those rows are emitted (the epilogue accounts for
// the others itself).
template <class E, class = void>
struct has_empty_list : std::false_type {};
template <class E>
struct has_empty_list<E, std::void_t<decltype(std::declval<E&>().empty_list),
                                     decltype(std::declval<E&>().n_empty_list)>> : std::true_type {};

template <class E, bool = has_prepare<E>::value>
struct prepared_type {
    using type = int;
};
template <class E>
struct prepared_type<E, true> {
    using type = decltype(std::declval<E&>().prepare(0u));
};

// Stage 1 of a tile: its 16-byte col/val loads and bitmap / plan words.
struct NnzIn {
    uint4 c0, c1, v0, v1;
    uint32_t sw, endw, seg0;
};

// Stage 2: x gathered, rows the tile may emit (and their epilogue loads)
// requested.
template <class SR, class Epi>
struct NnzReady {
    typename SR::x_t x[kNnzIpt];
    uint32_t v[kNnzIpt];
    uint32_t sw, endw, seg_base, row_pre;
    typename prepared_type<Epi>::type pre;
};

template <class SR, bool HINTS>
__device__ __forceinline__ NnzIn nnz_load(const NnzArgs<SR>& a, uint32_t tile, uint64_t pol_stream) {
    const uint32_t lane = lane_id();
    const uint32_t j0 = tile * kNnzTile;
    const uint32_t jl = j0 + lane * kNnzIpt;
    NnzIn in;
    in.v0 = in.v1 = make_uint4(0u, 0u, 0u, 0u);
    if constexpr (HINTS) {
        in.c0 = ldg_v4_policy(a.col + jl, pol_stream);
        in.c1 = ldg_v4_policy(a.col + jl + 4, pol_stream);
        if constexpr (reads_weight<SR>::value) {
            in.v0 = ldg_v4_policy(a.val + jl, pol_stream);
            in.v1 = ldg_v4_policy(a.val + jl + 4, pol_stream);
        }
    } else {
        // a lane's 8 columns and values are 32 aligned bytes each (col and
        // val are 32-byte aligned; the host checks); read once, so they do
        // not displace the x lines the gathers reuse from L1
        ldg_v8_stream(a.col + jl, in.c0, in.c1);
        if constexpr (reads_weight<SR>::value) ldg_v8_stream(a.val + jl, in.v0, in.v1);
    }
    in.sw = __ldg(a.plan.sbits + (j0 >> 5) + (lane >> 2));
    in.endw = __ldg(a.plan.sbits + ((j0 + kNnzTile) >> 5));
    in.seg0 = __ldg(a.plan.tile_seg + tile);
    return in;
}

template <class SR, class Epi, int HOT, bool HINTS>
__device__ __forceinline__ NnzReady<SR, Epi> nnz_gather(const NnzArgs<SR>& a, const NnzIn& in,
                                                        const typename SR::x_t* xc, uint32_t hot,
                                                        uint64_t pol_keep, Epi& epi) {
    using X = typename SR::x_t;
    const uint32_t lane = lane_id();
    NnzReady<SR, Epi> r;
    const uint32_t cc[kNnzIpt] = {in.c0.x, in.c0.y, in.c0.z, in.c0.w, in.c1.x, in.c1.y, in.c1.z, in.c1.w};
    const uint32_t vv[kNnzIpt] = {in.v0.x, in.v0.y, in.v0.z, in.v0.w, in.v1.x, in.v1.y, in.v1.z, in.v1.w};
#pragma unroll
    for (int u = 0; u < (int)kNnzIpt; ++u) {
        r.v[u] = vv[u];
        if constexpr (HINTS && sizeof(X) == 4) {
            if (HOT > 0 && cc[u] < hot) {
                r.x[u] = xc[cc[u]];
            } else {
                const uint32_t bits = ldg_u32_policy(a.x + cc[u], pol_keep);
                memcpy(&r.x[u], &bits, 4);
            }
        } else if constexpr (HOT > 0) {
            r.x[u] = gather_x(xc, a.x, cc[u], hot);
        } else {
            r.x[u] = ldg_any(a.x + cc[u]);
        }
    }
    r.sw = in.sw;
    r.endw = in.endw;
    // the first 32 rows the tile may emit (rows past its last are unused);
    // bit 0 of the ballot is lane 0's: does the tile begin with a row
    const bool first_start = (__ballot_sync(0xffffffffu, in.sw & 1u) & 1u) != 0u;
    r.seg_base = in.seg0 + (first_start ? 0u : 1u);
    r.row_pre = r.seg_base + lane < a.plan.n_nonempty ? __ldg(a.plan.nz_rows + r.seg_base + lane) : 0u;
    if constexpr (has_prepare<Epi>::value) r.pre = epi.prepare(r.row_pre);
    else r.pre = 0;
    return r;
}

// FULL: the tile is not the last one (all 256 nonzeros exist, and the tile
// does not end the matrix).
template <class SR, class Epi, bool FULL = false>
__device__ __forceinline__ void nnz_finish(const NnzArgs<SR>& a, const NnzReady<SR, Epi>& r,
                                           uint32_t tile, typename SR::value_t* sy, Epi& epi) {
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    constexpr uint32_t IPT = kNnzIpt;
    const uint32_t lane = lane_id();
    const uint32_t nnz = a.plan.nnz;
    const uint32_t j0 = tile * kNnzTile;
    const uint32_t jl = j0 + lane * IPT;
    // nonzeros of this lane that exist (the last tile may be short);
    // padding past nnz has no start bits
    const uint32_t nv = FULL ? IPT : (jl < nnz ? min(nnz - jl, IPT) : 0u);
    const uint32_t sb = (r.sw >> ((lane & 3u) * 8u)) & 0xFFu;
    const bool first_start = (__ballot_sync(0xffffffffu, r.sw & 1u) & 1u) != 0u;
    V pv[IPT];
#pragma unroll
    for (int u = 0; u < (int)IPT; ++u) {
        W wv;
        memcpy(&wv, &r.v[u], 4);
        pv[u] = (uint32_t)u < nv ? SR::combine(wv, r.x[u]) : SR::identity();
    }
    // starts before this lane (exclusive prefix of the per-lane counts, 0..8)
    // and in the whole tile, from four bit-sliced ballots of the counts
    const uint32_t nst = __popc(sb);
    const uint32_t below = (1u << lane) - 1u;
    uint32_t excl = 0, nstarts = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const uint32_t bb = __ballot_sync(0xffffffffu, (nst >> b) & 1u);
        excl += (uint32_t)__popc(bb & below) << b;
        nstarts += (uint32_t)__popc(bb) << b;
    }
    // lanes at or below this one that hold a row start
    const uint32_t has_upto = __ballot_sync(0xffffffffu, nst != 0u) & ((2u << lane) - 1u);
    // 1. lane-local fold
    V head = SR::identity(), acc = SR::identity();
    uint32_t k = 0;
#pragma unroll
    for (int u = 0; u < (int)IPT; ++u) {
        if ((sb >> u) & 1u) {
            if (k == 0) head = acc;
            else sy[excl + k - 1] = acc;
            acc = SR::identity();
            ++k;
        }
        acc = SR::reduce(acc, pv[u]);
    }
    // 2. segmented scan of the lane tails: at offset `off`, s covers lanes
    // (lane - off, lane] unless a start lies there (then it is complete)
    V s = acc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const V su = shfl_up_any(0xffffffffu, s, off);
        const bool open = (int)lane >= off && (has_upto >> ((lane - off + 1) & 31u)) == 0u;
        if (open) s = SR::reduce(su, s);
    }
    V prev = shfl_up_any(0xffffffffu, s, 1);
    if (lane == 0) prev = SR::identity();
    if (nst) {
        const V val = SR::reduce(prev, head);
        if (excl > 0)
            sy[excl - 1] = val;  // segment begun in an earlier lane ends here
        else if (!first_start)
            a.tail[tile] = val;  // the row begun in an earlier tile ends here
    }
    const V last = shfl_any(0xffffffffu, s, 31);
    const bool closed = (!FULL && j0 + kNnzTile >= nnz) || (r.endw & 1u);
    if (lane == 0) {
        if (nstarts == 0) {
            a.tail[tile] = last;
            a.carry[tile] = last;
        } else if (closed) {
            sy[nstarts - 1] = last;
        } else {
            a.carry[tile] = last;
        }
    }
    __syncwarp();
    // 3. the tile's complete rows, in row order
    const uint32_t ncomplete = nstarts == 0 ? 0u : (closed ? nstarts : nstarts - 1);
    if (lane < ncomplete) {
        if constexpr (has_prepare<Epi>::value) epi.emit_prepared(r.row_pre, sy[lane], r.pre);
        else epi.emit(r.row_pre, sy[lane]);
    }
    for (uint32_t q = lane + 32; q < ncomplete; q += 32)
        epi.emit(__ldg(a.plan.nz_rows + r.seg_base + q), sy[q]);
    __syncwarp();
}

// Lane 0 of a warp: the bulk copies of one tile's col and, unless COL_ONLY,
// val (1 KB each; the arrays are padded past the last tile) into the warp's
// staging buffer.
template <class SR, bool COL_ONLY>
__device__ __forceinline__ void nnz_issue(const NnzArgs<SR>& a, uint32_t tile, unsigned char* st,
                                          uint64_t* bar) {
    constexpr uint32_t kBytes = kNnzTile * 4;
    const size_t j0 = (size_t)tile * kNnzTile;
    constexpr bool kVal = !COL_ONLY && reads_weight<SR>::value;
    mbar_arrive_expect_tx(bar, (kVal ? 2 : 1) * kBytes);
    bulk_g2s(st, a.col + j0, kBytes, bar);
    if constexpr (kVal) bulk_g2s(st + kBytes, a.val + j0, kBytes, bar);
}

// Lanes 0-3 of a warp: L2 prefetch of tile `tile`'s col and val (1 KB each,
// one bulk prefetch each), its row-start bitmap words and its tile_seg word,
// so that the tile's loads hit L2 instead of waiting for DRAM.
template <class SR>
__device__ __forceinline__ void nnz_prefetch_l2(const NnzArgs<SR>& a, uint32_t tile) {
    const uint32_t lane = lane_id();
    const size_t j0 = (size_t)tile * kNnzTile;
    if (lane == 0) prefetch_l2_bulk(a.col + j0, kNnzTile * 4);
    else if (lane == 1 && reads_weight<SR>::value) prefetch_l2_bulk(a.val + j0, kNnzTile * 4);
    else if (lane == 2) prefetch_l2(a.plan.sbits + (j0 >> 5));
    else if (lane == 3) prefetch_l2(a.plan.tile_seg + tile);
}

// HINTS: col/val are streamed with an evict-first L2 policy, x gathers use
// evict-last (x stays in L2 across the iteration).  PFL1: each warp
// prefetches its next tile's col/val lines into L1.  PIPE: a three-tile
// software pipeline per warp -- while tile A is folded, the x gathers of
// tile B and the col/val loads of tile C are in flight.  BULK: each warp's
// next tile of col (BULK 2) or col and val (BULK 1) is brought into its
// shared-memory staging buffer by bulk copies (the TMA engine, no load
// registers or LSU work) while the current tile is gathered and folded; with
// BULK 2 val is loaded at the tile start, its latency overlapping the x
// gathers.  The wait on the mbarrier is bounded and reports a timeout
// through the device error word.  PFL2 > 0: each warp prefetches into L2
// the tile it will fold PFL2 rounds later (nnz_prefetch_l2).
template <class SR, class Epi, int WARPS, int MINB, int HOT, bool HINTS = false, bool PIPE = false,
          bool PFL1 = false, int BULK = 0, int PFL2 = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB)
spmv_nnz_kernel(NnzArgs<SR> a, Epi epi) {
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    using W = typename SR::w_t;
    using L = NnzLayout<SR, WARPS, HOT, BULK>;
    static_assert(sizeof(W) == 4, "16-byte val loads assume 4-byte edge values");
    extern __shared__ __align__(16) unsigned char dsm[];
    // the fixup (launched with programmatic dependent launch) may start as
    // soon as every block is past this point
    grid_launch_dependents();
    if (!epi_active(epi)) return;
    const uint32_t w = threadIdx.x >> 5;
    X* xc = reinterpret_cast<X*>(dsm + L::XC_OFF);
    V* sy = reinterpret_cast<V*>(dsm + L::SY_OFF) + (size_t)w * kNnzTile;
    epi.begin();
    const uint32_t hot = HOT < a.plan.n_rows ? (uint32_t)HOT : a.plan.n_rows;
    const uint32_t total_warps = gridDim.x * WARPS;
    const uint32_t n_tiles = a.plan.n_tiles;
    if constexpr (BULK) {
        // the first tile's copies start before the x cache is filled
        unsigned char* st = dsm + L::ST_OFF + (size_t)w * L::ST_WARP;
        uint64_t* bar = reinterpret_cast<uint64_t*>(dsm + L::BAR_OFF) + w;
        const uint32_t lane = lane_id();
        uint32_t tile = blockIdx.x * WARPS + w;
        if (lane == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
            if (tile < n_tiles) nnz_issue<SR, BULK == 2>(a, tile, st, bar);
        }
        if constexpr (HOT > 0)
            fill_x_cache<WARPS * 32>(xc, a.x, hot);
        __syncthreads();
        const uint4* sc = reinterpret_cast<const uint4*>(st) + 2 * lane;
        const uint4* sv = reinterpret_cast<const uint4*>(st + kNnzTile * 4) + 2 * lane;
        uint32_t phase = 0;
        for (; tile < n_tiles; tile += total_warps, phase ^= 1u) {
            NnzIn in;
            const uint32_t j0 = tile * kNnzTile;
            in.sw = __ldg(a.plan.sbits + (j0 >> 5) + (lane >> 2));
            in.endw = __ldg(a.plan.sbits + ((j0 + kNnzTile) >> 5));
            in.seg0 = __ldg(a.plan.tile_seg + tile);
            in.v0 = in.v1 = make_uint4(0u, 0u, 0u, 0u);
            if constexpr (BULK == 2 && reads_weight<SR>::value) {
                in.v0 = __ldg(reinterpret_cast<const uint4*>(a.val + j0) + 2 * lane);
                in.v1 = __ldg(reinterpret_cast<const uint4*>(a.val + j0) + 2 * lane + 1);
            }
            const bool arrived = mbar_wait_bounded(bar, phase, a.wait_limit);
            if (!__all_sync(0xffffffffu, arrived)) {
                // let the copy in flight land (bounded) before the warp
                // leaves its shared memory
                if (lane == 0) {
                    set_error(a.err, kDevTimeout);
                    mbar_wait_bounded(bar, phase);
                }
                __syncwarp();
                break;
            }
            in.c0 = sc[0];
            in.c1 = sc[1];
            if constexpr (BULK == 1 && reads_weight<SR>::value) {
                in.v0 = sv[0];
                in.v1 = sv[1];
            }
            __syncwarp();  // the staging buffer is free: the next tile's copy may land
            const uint32_t nt = tile + total_warps;
            if (lane == 0 && nt < n_tiles) {
                fence_proxy_async_smem();
                nnz_issue<SR, BULK == 2>(a, nt, st, bar);
            }
            const NnzReady<SR, Epi> r = nnz_gather<SR, Epi, HOT, false>(a, in, xc, hot, 0, epi);
            nnz_finish<SR, Epi>(a, r, tile, sy, epi);
        }
        epi.template block_end<WARPS * 32>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
        return;
    }
    if constexpr (PFL2 > 0) {
        // the first rounds' tiles, before the x cache fill
        for (int d = 1; d < PFL2; ++d) {
            const uint64_t pt = blockIdx.x * WARPS + w + (uint64_t)d * total_warps;
            if (pt < n_tiles) nnz_prefetch_l2(a, (uint32_t)pt);
        }
    }
    if constexpr (HOT > 0) {
        fill_x_cache<WARPS * 32>(xc, a.x, hot);
        __syncthreads();
    }
    uint64_t pol_stream = 0, pol_keep = 0;
    if constexpr (HINTS) {
        pol_stream = l2_policy_evict_first();
        pol_keep = l2_policy_evict_last();
    }
    if constexpr (!PIPE) {
        for (uint32_t tile = blockIdx.x * WARPS + w; tile < n_tiles; tile += total_warps) {
            if constexpr (PFL2 > 0) {
                const uint64_t pt = tile + (uint64_t)PFL2 * total_warps;
                if (pt < n_tiles) nnz_prefetch_l2(a, (uint32_t)pt);
            }
            if constexpr (PFL1) {
                // the next tile's 8 col and 8 val lines into L1 while this one runs
                const uint32_t nt = tile + total_warps;
                const uint32_t lane = lane_id();
                if (nt < n_tiles && lane < (reads_weight<SR>::value ? 16u : 8u)) {
                    const uint32_t jn = nt * kNnzTile + (lane & 7u) * 32u;
                    prefetch_l1(lane < 8 ? (const void*)(a.col + jn) : (const void*)(a.val + jn));
                }
            }
            const NnzIn in = nnz_load<SR, HINTS>(a, tile, pol_stream);
            const NnzReady<SR, Epi> r = nnz_gather<SR, Epi, HOT, HINTS>(a, in, xc, hot, pol_keep, epi);
            if (tile + 1 < n_tiles)
                nnz_finish<SR, Epi, true>(a, r, tile, sy, epi);
            else
                nnz_finish<SR, Epi>(a, r, tile, sy, epi);
        }
    } else {
        uint32_t ta = blockIdx.x * WARPS + w;
        if (ta < n_tiles) {
            NnzReady<SR, Epi> ra =
                nnz_gather<SR, Epi, HOT, HINTS>(a, nnz_load<SR, HINTS>(a, ta, pol_stream), xc, hot, pol_keep, epi);
            uint32_t tb = ta + total_warps;
            NnzIn ib{};
            if (tb < n_tiles) ib = nnz_load<SR, HINTS>(a, tb, pol_stream);
            for (;;) {
                const uint32_t tc = tb + total_warps;
                if constexpr (PFL2 > 0) {
                    const uint64_t pt = tc + (uint64_t)PFL2 * total_warps;
                    if (pt < n_tiles) nnz_prefetch_l2(a, (uint32_t)pt);
                }
                NnzReady<SR, Epi> rb{};
                if (tb < n_tiles) rb = nnz_gather<SR, Epi, HOT, HINTS>(a, ib, xc, hot, pol_keep, epi);
                NnzIn ic{};
                if (tc < n_tiles) ic = nnz_load<SR, HINTS>(a, tc, pol_stream);
                nnz_finish<SR, Epi>(a, ra, ta, sy, epi);
                if (tb >= n_tiles) break;
                ra = rb;
                ta = tb;
                ib = ic;
                tb = tc;
            }
        }
    }
    epi.template block_end<WARPS * 32>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

// ------------------------------------------ nnz-split tiles, IPT per lane
// The same tiles as spmv_nnz_kernel with IPT consecutive nonzeros per lane
// (tiles of 32 * IPT nonzeros; the plan is built for that tile size).  A
// tile's fixed costs -- the plan-word loads, the start-count ballots, the
// warp segmented scan, the in-order emission and the loop -- are paid once
// per 32 * IPT nonzeros, so larger IPT cuts the instructions per nonzero; the
// per-nonzero work (gather, combine, lane-local fold) is unchanged.
template <int IPT>
constexpr int nnz_count_bits() {
    return IPT < 2 ? 1 : IPT < 4 ? 2 : IPT < 8 ? 3 : IPT < 16 ? 4 : IPT < 32 ? 5 : 6;
}

template <class SR, class Epi, int IPT>
struct Nnz2Ready {
    typename SR::x_t x[IPT];
    uint32_t v[IPT];
    uint32_t sb;    // this lane's start bits (bit u: nonzero jl + u starts a row)
    uint32_t endw;  // bitmap word whose bit 0 is the first nonzero after the tile
    uint32_t seg_base, row_pre;
    typename prepared_type<Epi>::type pre;
};

// Shared memory: the x cache, then per warp the values of the rows completed
// in its tile, then the epilogue's scratch.
template <class SR, int WARPS, int HOT, int IPT>
struct Nnz2Layout {
    using V = typename SR::value_t;
    using X = typename SR::x_t;
    static constexpr uint32_t TILE = 32 * IPT;
    static constexpr size_t XC_OFF = 0;
    static constexpr size_t XC_BYTES = ((size_t)HOT * sizeof(X) + 15) / 16 * 16;
    static constexpr size_t SY_OFF = XC_OFF + XC_BYTES;
    static constexpr size_t SY_BYTES = ((size_t)WARPS * TILE * sizeof(V) + 15) / 16 * 16;
    static constexpr size_t EPI_OFF = SY_OFF + SY_BYTES;
    static constexpr size_t BYTES = EPI_OFF + 512;
};

template <class SR, class Epi, int HOT, int IPT>
__device__ __forceinline__ Nnz2Ready<SR, Epi, IPT> nnz2_fetch(const NnzArgs<SR>& a, uint32_t tile,
                                                              const typename SR::x_t* xc, uint32_t hot,
                                                              Epi& epi) {
    static_assert(IPT % 8 == 0 && IPT <= 24, "IPT: 8, 16 or 24 nonzeros per lane");
    constexpr uint32_t TILE = 32 * IPT;
    const uint32_t lane = lane_id();
    const uint32_t j0 = tile * TILE;
    const uint32_t jl = j0 + lane * IPT;
    Nnz2Ready<SR, Epi, IPT> r;
    // a lane's start bits lie inside one 32-bit word when IPT divides 32;
    // for IPT = 24 they may straddle two
    const uint32_t w0 = __ldg(a.plan.sbits + (jl >> 5));
    if constexpr (32 % IPT == 0) {
        r.sb = (w0 >> (jl & 31u)) & ((1u << IPT) - 1u);
    } else {
        const uint32_t w1 = __ldg(a.plan.sbits + (jl >> 5) + 1);
        const uint64_t w = ((uint64_t)w1 << 32) | w0;
        r.sb = (uint32_t)(w >> (jl & 31u)) & ((1u << IPT) - 1u);
    }
    r.endw = __ldg(a.plan.sbits + ((j0 + TILE) >> 5));
    const uint32_t seg0 = __ldg(a.plan.tile_seg + tile);
    // all of the lane's col/val first (32-byte loads kept out of L1), then the gathers
    uint32_t cc[IPT];
#pragma unroll
    for (int c = 0; c < IPT / 8; ++c) {
        uint4 c0, c1, v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
        ldg_v8_stream(a.col + jl + 8 * c, c0, c1);
        if constexpr (reads_weight<SR>::value) ldg_v8_stream(a.val + jl + 8 * c, v0, v1);
        const uint32_t ci[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
        const uint32_t vi[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            cc[8 * c + u] = ci[u];
            r.v[8 * c + u] = vi[u];
        }
    }
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
        if constexpr (HOT > 0) r.x[u] = gather_x(xc, a.x, cc[u], hot);
        else r.x[u] = ldg_any(a.x + cc[u]);
    }
    const bool first_start = (__ballot_sync(0xffffffffu, r.sb & 1u) & 1u) != 0u;
    r.seg_base = seg0 + (first_start ? 0u : 1u);
    r.row_pre = r.seg_base + lane < a.plan.n_nonempty ? __ldg(a.plan.nz_rows + r.seg_base + lane) : 0u;
    if constexpr (has_prepare<Epi>::value) r.pre = epi.prepare(r.row_pre);
    else r.pre = 0;
    return r;
}

// FULL: the tile is not the last one.
template <class SR, class Epi, int IPT, bool FULL>
__device__ __forceinline__ void nnz2_finish(const NnzArgs<SR>& a, const Nnz2Ready<SR, Epi, IPT>& r,
                                            uint32_t tile, typename SR::value_t* sy, Epi& epi) {
    using V = typename SR::value_t;
    using W = typename SR::w_t;
    constexpr uint32_t TILE = 32 * IPT;
    const uint32_t lane = lane_id();
    const uint32_t nnz = a.plan.nnz;
    const uint32_t j0 = tile * TILE;
    const uint32_t jl = j0 + lane * IPT;
    const uint32_t nv = FULL ? (uint32_t)IPT : (jl < nnz ? min(nnz - jl, (uint32_t)IPT) : 0u);
    const uint32_t sb = r.sb;
    const bool first_start = (__ballot_sync(0xffffffffu, sb & 1u) & 1u) != 0u;
    // starts before this lane and in the whole tile, from bit-sliced ballots
    const uint32_t nst = __popc(sb);
    const uint32_t below = (1u << lane) - 1u;
    uint32_t excl = 0, nstarts = 0;
#pragma unroll
    for (int b = 0; b < nnz_count_bits<IPT>(); ++b) {
        const uint32_t bb = __ballot_sync(0xffffffffu, (nst >> b) & 1u);
        excl += (uint32_t)__popc(bb & below) << b;
        nstarts += (uint32_t)__popc(bb) << b;
    }
    const uint32_t has_upto = __ballot_sync(0xffffffffu, nst != 0u) & ((2u << lane) - 1u);
    // lane-local fold: segments that start and end in the lane go to sy
    V head = SR::identity(), acc = SR::identity();
    uint32_t k = 0;
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
        if ((sb >> u) & 1u) {
            if (k == 0) head = acc;
            else sy[excl + k - 1] = acc;
            acc = SR::identity();
            ++k;
        }
        W wv;
        memcpy(&wv, &r.v[u], 4);
        acc = SR::reduce(acc, (uint32_t)u < nv ? SR::combine(wv, r.x[u]) : SR::identity());
    }
    // warp segmented scan of the lane tails
    V s = acc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const V su = shfl_up_any(0xffffffffu, s, off);
        const bool open = (int)lane >= off && (has_upto >> ((lane - off + 1) & 31u)) == 0u;
        if (open) s = SR::reduce(su, s);
    }
    V prev = shfl_up_any(0xffffffffu, s, 1);
    if (lane == 0) prev = SR::identity();
    if (nst) {
        const V val = SR::reduce(prev, head);
        if (excl > 0)
            sy[excl - 1] = val;
        else if (!first_start)
            a.tail[tile] = val;
    }
    const V last = shfl_any(0xffffffffu, s, 31);
    const bool closed = (!FULL && j0 + TILE >= nnz) || (r.endw & 1u);
    if (lane == 0) {
        if (nstarts == 0) {
            a.tail[tile] = last;
            a.carry[tile] = last;
        } else if (closed) {
            sy[nstarts - 1] = last;
        } else {
            a.carry[tile] = last;
        }
    }
    __syncwarp();
    const uint32_t ncomplete = nstarts == 0 ? 0u : (closed ? nstarts : nstarts - 1);
    if (lane < ncomplete) {
        if constexpr (has_prepare<Epi>::value) epi.emit_prepared(r.row_pre, sy[lane], r.pre);
        else epi.emit(r.row_pre, sy[lane]);
    }
    for (uint32_t q = lane + 32; q < ncomplete; q += 32)
        epi.emit(__ldg(a.plan.nz_rows + r.seg_base + q), sy[q]);
    __syncwarp();
}

// CONTIG: block b folds the contiguous tile range [b * T, (b + 1) * T),
// T = ceil(n_tiles / blocks), its warps taking consecutive tiles, so that an
// SM streams one contiguous stretch of col/val and writes one stretch of
// rows; otherwise warp w of the grid takes tiles w, w + warps, ...
template <class SR, class Epi, int WARPS, int HOT, int IPT, bool CONTIG = false>
__global__ void __launch_bounds__(WARPS * 32, 1)
spmv_nnz2_kernel(NnzArgs<SR> a, Epi epi) {
    using X = typename SR::x_t;
    using V = typename SR::value_t;
    using L = Nnz2Layout<SR, WARPS, HOT, IPT>;
    static_assert(sizeof(typename SR::w_t) == 4, "32-byte val loads assume 4-byte edge values");
    extern __shared__ __align__(16) unsigned char dsm[];
    grid_launch_dependents();
    if (!epi_active(epi)) return;
    const uint32_t w = threadIdx.x >> 5;
    X* xc = reinterpret_cast<X*>(dsm + L::XC_OFF);
    V* sy = reinterpret_cast<V*>(dsm + L::SY_OFF) + (size_t)w * L::TILE;
    epi.begin();
    const uint32_t hot = HOT < a.plan.n_rows ? (uint32_t)HOT : a.plan.n_rows;
    if constexpr (HOT > 0) {
        fill_x_cache<WARPS * 32>(xc, a.x, hot);
        __syncthreads();
    }
    const uint32_t n_tiles = a.plan.n_tiles;
    uint32_t first, end, step;
    if constexpr (CONTIG) {
        const uint32_t per = (uint32_t)ceil_div(n_tiles, gridDim.x);
        first = blockIdx.x * per + w;
        end = min(n_tiles, (blockIdx.x + 1) * per);
        step = WARPS;
    } else {
        first = blockIdx.x * WARPS + w;
        end = n_tiles;
        step = gridDim.x * WARPS;
    }
    for (uint32_t tile = first; tile < end; tile += step) {
        const Nnz2Ready<SR, Epi, IPT> r = nnz2_fetch<SR, Epi, HOT, IPT>(a, tile, xc, hot, epi);
        if (tile + 1 < n_tiles) nnz2_finish<SR, Epi, IPT, true>(a, r, tile, sy, epi);
        else nnz2_finish<SR, Epi, IPT, false>(a, r, tile, sy, epi);
    }
    epi.template block_end<WARPS * 32>(reinterpret_cast<char*>(dsm + L::EPI_OFF));
}

__device__ __forceinline__ bool nnz_start_bit(const uint32_t* sbits, uint32_t k) {
    return (__ldg(sbits + (k >> 5)) >> (k & 31)) & 1u;
}

// Rows that cross nnz tiles, one per tile in which such a row ends (the
// plan lists them with the row and its first tile), and the empty rows
// (identity); grid-stride over all three kinds of work:
//   - empty rows: independent of the main kernel; with an epilogue whose
//     rows are independent they are emitted before grid_dependency_wait(),
//     overlapping the main kernel's tail under programmatic dependent launch;
//   - rows begun in the previous tile (the plan lists them first): one
//     thread each, carry[t-1] + tail[t];
//   - rows that span more tiles (hubs): one warp each, folding the carries
//     of the tiles they cover in tile order (lanes strided, four partials per
//     lane, shuffle tree), then + tail[t].  Per row the fold order is fixed,
//     so results do not depend on the grid.
template <class SR, class Epi, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
spmv_nnz_fixup_kernel(NnzArgs<SR> a, Epi epi) {
    if (!epi_active(epi)) return;
    using V = typename SR::value_t;
    constexpr bool kEarly = rows_independent<Epi>::value;
    __shared__ alignas(16) char epi_smem[64 * 8];
    const uint32_t i0 = blockIdx.x * BLOCK + threadIdx.x;
    const uint32_t stride = gridDim.x * BLOCK;
    const uint32_t lane = lane_id();
    const NnzPlanView& p = a.plan;
    if constexpr (!kEarly) grid_dependency_wait();
    epi.begin();
    const uint32_t* elist = p.empty_rows;
    uint32_t n_empty = p.n_empty;
    if constexpr (has_empty_list<Epi>::value) {
        if (epi.empty_list) {
            elist = epi.empty_list;
            n_empty = epi.n_empty_list;
        }
    }
    // empty rows four at a time: their row ids and epilogue loads are all in
    // flight before the first store
    uint32_t e = i0;
    for (; e + 3 * stride < n_empty; e += 4 * stride) {
        uint32_t v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = __ldg(elist + e + q * stride);
        if constexpr (has_prepare<Epi>::value) {
            typename prepared_type<Epi>::type pre[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) pre[q] = epi.prepare(v[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) epi.emit_prepared(v[q], SR::identity(), pre[q]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) epi.emit(v[q], SR::identity());
        }
    }
    for (; e < n_empty; e += stride) epi.emit(__ldg(elist + e), SR::identity());
    if constexpr (kEarly) grid_dependency_wait();
    grid_launch_dependents();
    // rows begun in the previous tile
    for (uint32_t i = i0; i < p.n_fix_short; i += stride) {
        const uint4 f = __ldg(p.fix_info + i);
        epi.emit(f.y, SR::reduce(a.carry[f.x - 1], a.tail[f.x]));
    }
    // longer chains, one warp each
    const uint32_t n_warps = stride >> 5;
    for (uint32_t j = p.n_fix_short + (i0 >> 5); j < p.n_fix; j += n_warps) {
        const uint4 f = __ldg(p.fix_info + j);
        const uint32_t tt = f.x, f0 = f.z;
        // carries of the tiles [f0, tt-1); tile tt-1's joins tail[tt] below
        V part = SR::identity(), p1 = SR::identity(), p2 = SR::identity(), p3 = SR::identity();
        uint32_t k = f0 + lane;
        for (; k + 96 + 1 < tt; k += 128) {
            part = SR::reduce(part, a.carry[k]);
            p1 = SR::reduce(p1, a.carry[k + 32]);
            p2 = SR::reduce(p2, a.carry[k + 64]);
            p3 = SR::reduce(p3, a.carry[k + 96]);
        }
        for (; k + 1 < tt; k += 32) part = SR::reduce(part, a.carry[k]);
        part = SR::reduce(SR::reduce(part, p1), SR::reduce(p2, p3));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            part = SR::reduce(part, shfl_down_any(0xffffffffu, part, off));
        if (lane == 0) epi.emit(f.y, SR::reduce(part, SR::reduce(a.carry[tt - 1], a.tail[tt])));
    }
    epi.template block_end<BLOCK>(epi_smem);
}

// CSR-vector schedule: TPR lanes per row (TPR in {1,2,4,8,16,32}).
template <class SR, class Epi, int BLOCK, int TPR>
__global__ void __launch_bounds__(BLOCK)
spmv_vector_kernel(uint32_t n_rows, const uint32_t* row_ptr, const uint32_t* col,
                   const typename SR::w_t* val, const typename SR::x_t* x, Epi epi) {
    if (!epi_active(epi)) return;
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
    static constexpr bool kRowsIndependent = true;
    V* y;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t row, const V& v) { y[row] = v; }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

}  // namespace g1
