// Host-side launch of the SpMV schedules for the prebuilt semirings.
#pragma once

#include <algorithm>

#include "g1/spmv.cuh"
#include "internal.h"

namespace g1 {

constexpr int kMergeBlock = 256;
constexpr int kVectorBlock = 256;

// Merge kernel variants the autotuner chooses from (all share the
// merge-path partition; items per lane odd so that consecutive lanes'
// shared-memory reads fall in distinct banks):
//   kind 0: warp tiles of 32*ipt items loaded into registers,
//   kind 1: block tiles of 256*ipt items staged by TMA bulk copies
//           (`stages` staging buffers),
//   kind 2: warp tiles staged by per-warp TMA bulk copies,
//   kind 3: nnz-split warp tiles of 256 nonzeros (16-byte loads, row-start
//           bitmap; its own plan instead of the merge-path partition);
//           stages: bit 0 = L2 cache policies, bit 1 = three-tile software
//           pipeline per warp, bit 2 = next-tile L1 prefetch, bit 3 / bit 4
//           = next tile's col and val / col only staged in shared memory by
//           bulk copies, stages / 32 = L2 prefetch distance in rounds;
//   kind 5: nnz-split warp tiles of 32 * ipt nonzeros (spmv_nnz2_kernel, the
//           nnz plan for that tile size); stages bit 0 = contiguous tile
//           ranges per block.
// `warps` per block (kind 0/2/3), `hot` x entries cached in shared memory,
// `minb` resident blocks per SM the register budget is sized for.
struct MergeVariant {
    int kind;
    int ipt;
    int stages;
    int warps;
    int hot;
    int minb;
};
constexpr MergeVariant kMergeVariants[] = {
    {0, 11, 0, 8, 0, 3},      {0, 7, 0, 8, 0, 4},       {0, 7, 0, 32, 16384, 1},
    {1, 7, 2, 8, 0, 4},       {1, 7, 1, 8, 0, 6},       {0, 11, 0, 32, 16384, 1},
    {2, 15, 0, 24, 16384, 1}, {2, 31, 0, 16, 0, 1},     {2, 15, 0, 32, 0, 1},
    {2, 23, 0, 16, 16384, 1}, {3, 8, 0, 32, 16384, 1},  {3, 8, 0, 16, 16384, 2},
    {3, 8, 0, 32, 0, 1},      {3, 8, 1, 32, 16384, 1},  {3, 8, 1, 16, 16384, 2},
    {3, 8, 1, 16, 8192, 3},   {3, 8, 0, 16, 8192, 3},   {3, 8, 0, 32, 32768, 1},
    {3, 8, 0, 32, 49152, 1},  {3, 8, 2, 24, 32768, 1},  {3, 8, 2, 16, 32768, 1},
    {3, 8, 3, 24, 32768, 1},  {3, 8, 4, 32, 32768, 1},  {3, 8, 4, 32, 16384, 1},
    {3, 8, 8, 32, 32768, 1},  {3, 8, 8, 32, 16384, 1},  {3, 8, 16, 32, 32768, 1},
    {3, 8, 16, 32, 24576, 1}, {3, 8, 32, 32, 32768, 1}, {3, 8, 64, 32, 32768, 1},
    {3, 8, 128, 32, 32768, 1}, {3, 8, 66, 24, 32768, 1}, {5, 8, 0, 32, 32768, 1},
    {5, 16, 0, 32, 32768, 1}, {5, 24, 0, 32, 32768, 1}, {5, 16, 0, 32, 16384, 1},
    {5, 8, 1, 32, 32768, 1},  {5, 8, 0, 32, 24576, 1},  {5, 8, 0, 32, 40960, 1},
    {5, 8, 1, 32, 24576, 1}};
constexpr int kNumMergeVariants = 40;
constexpr int kDefaultVariant = 17;

template <class K>
int blocks_per_sm(K kernel, int block, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, smem) != cudaSuccess) {
        cudaGetLastError();
        n = 1;
    }
    return std::max(1, n);
}

// Lanes per row of the CSR-vector schedule: the power of two >= mean degree.
inline int vector_tpr(const g1_graph* g) {
    const double mean = g->n ? (double)g->m / g->n : 0.0;
    int tpr = 1;
    while (tpr < 32 && tpr < mean) tpr <<= 1;
    return tpr;
}

inline g1_schedule resolve_schedule(const g1_graph* g, int t, g1_schedule sched) {
    if (sched != G1_SCHED_AUTO) return sched;
    const Orientation& o = g->o[t];
    if (o.tuned_sched) return (g1_schedule)o.tuned_sched;
    const double mean = g->n ? (double)g->m / g->n : 0.0;
    // Uniform small degrees on a small graph: one short row per lane group, no
    // merge bookkeeping.  From 2^22 nonzeros the nnz tiles win even there (a
    // 4096^2 grid: 170 against 337 us per SpMV; a 1024^2 grid: a tie).
    return (o.max_deg <= 64 && mean <= 16.0 && o.max_deg <= 8 * std::max(1.0, mean) && g->m < (1u << 22))
               ? G1_SCHED_VECTOR
               : G1_SCHED_MERGE;
}

inline int merge_variant(const g1_graph* g, int t) {
    const int v = g->o[t].tuned_variant;
    return (v >= 0 && v < kNumMergeVariants) ? v : kDefaultVariant;
}
inline uint32_t merge_items(int variant) {
    return (kMergeVariants[variant].kind == 1 ? kMergeBlock : 32) * kMergeVariants[variant].ipt;
}

template <class SR, class Epi, int WARPS, int IPT, int HOT>
struct WarpTmaKernel {
    using L = WarpTmaLayout<SR, WARPS, IPT, HOT>;
    static int occupancy() {
        static int occ = [] {
            auto k = spmv_wtma_kernel<SR, Epi, WARPS, IPT, HOT>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            return blocks_per_sm(k, WARPS * 32, L::BYTES);
        }();
        return occ;
    }
    static uint32_t grid(const g1_graph* g, uint32_t n_tiles) {
        const uint64_t want = ceil_div(n_tiles, WARPS);
        return (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occupancy()));
    }
};

template <class SR, class Epi, int WARPS, int IPT, int MINB, int HOT>
struct WarpMergeKernel {
    using L = WarpMergeLayout<SR, WARPS, IPT, HOT>;
    static int occupancy() {
        static int occ = [] {
            auto k = spmv_wmerge_kernel<SR, Epi, WARPS, IPT, MINB, HOT>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            return blocks_per_sm(k, WARPS * 32, L::BYTES);
        }();
        return occ;
    }
    static uint32_t grid(const g1_graph* g, uint32_t n_tiles) {
        const uint64_t want = ceil_div(n_tiles, WARPS);
        return (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occupancy()));
    }
};

template <class SR, class Epi, int WARPS, int MINB, int HOT, bool HINTS = false, bool PIPE = false,
          bool PFL1 = false, int BULK = 0, int PFL2 = 0>
struct NnzKernel {
    using L = NnzLayout<SR, WARPS, HOT, BULK>;
    static int occupancy() {
        static int occ = [] {
            auto k = spmv_nnz_kernel<SR, Epi, WARPS, MINB, HOT, HINTS, PIPE, PFL1, BULK, PFL2>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            return blocks_per_sm(k, WARPS * 32, L::BYTES);
        }();
        return occ;
    }
    static uint32_t grid(const g1_graph* g, uint32_t n_tiles) {
        const uint64_t want = ceil_div(n_tiles, WARPS);
        return (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occupancy()));
    }
};

template <class SR, class Epi, int WARPS, int HOT, int IPT, bool CONTIG = false>
struct Nnz2Kernel {
    using L = Nnz2Layout<SR, WARPS, HOT, IPT>;
    static int occupancy() {
        static int occ = [] {
            auto k = spmv_nnz2_kernel<SR, Epi, WARPS, HOT, IPT, CONTIG>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            return blocks_per_sm(k, WARPS * 32, L::BYTES);
        }();
        return occ;
    }
    static uint32_t grid(const g1_graph* g, uint32_t n_tiles) {
        const uint64_t want = ceil_div(n_tiles, WARPS);
        return (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occupancy()));
    }
};

// The nnz fixup runs grid-stride in one wave of resident blocks (blocks of
// a second wave would start their empty rows only after the main kernel).
template <class SR, class Epi>
uint32_t nnz_fix_grid(const g1_graph* g, const NnzPlan& p) {
    static const int occ =
        blocks_per_sm(spmv_nnz_fixup_kernel<SR, Epi, kMergeBlock>, kMergeBlock, 0);
    const uint64_t want = ceil_div(std::max(p.n_fix, p.n_empty), kMergeBlock);
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occ));
}

// Launch with programmatic stream serialization: the kernel may start while
// the preceding kernel in the stream finishes; it orders itself with
// grid_dependency_wait().
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), uint32_t grid, uint32_t block, size_t smem,
                       cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Per-instantiation launch facts of the merge kernel.
template <class SR, class Epi, int IPT, int STAGES>
struct MergeKernel {
    using L = MergeLayout<SR, kMergeBlock, IPT, STAGES>;
    static int occupancy() {
        static int occ = [] {
            auto k = spmv_merge_kernel<SR, Epi, kMergeBlock, IPT, STAGES>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            return blocks_per_sm(k, kMergeBlock, L::BYTES);
        }();
        return occ;
    }
    static uint32_t grid(const g1_graph* g, uint32_t n_tiles) {
        return std::max<uint32_t>(1, std::min<uint32_t>(n_tiles, (uint32_t)g->sm_count * occupancy()));
    }
};

template <class SR, class Epi>
uint32_t vector_grid(const g1_graph* g) {
    static int occ = blocks_per_sm(spmv_vector_kernel<SR, Epi, kVectorBlock, 32>, kVectorBlock, 0);
    const int tpr = vector_tpr(g);
    const uint64_t want = ceil_div((uint64_t)g->n * tpr, kVectorBlock);
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occ));
}

template <class SR>
MergeArgs<SR> merge_args(const g1_graph* g, int t, const MergePlan& p, const typename SR::x_t* x) {
    const Orientation& o = g->o[t];
    MergeArgs<SR> a;
    a.plan.n_rows = g->n;
    a.plan.nnz = g->m;
    a.plan.items = p.items;
    a.plan.n_tiles = p.n_tiles;
    a.plan.row_ptr = o.rp;
    a.plan.tile_row = p.tile_row.as<uint32_t>();
    a.plan.tile_nnz = p.tile_nnz.as<uint32_t>();
    a.col = o.col;
    a.val = static_cast<const typename SR::w_t*>(o.val);
    a.x = x;
    a.carry = p.carry.as<typename SR::value_t>();
    a.tail = p.tail.as<typename SR::value_t>();
    a.err = g->err_word;
    a.wait_limit = wait_polls(kWaitPolls);
    return a;
}

template <class SR>
NnzArgs<SR> nnz_args(const g1_graph* g, int t, const NnzPlan& p, const typename SR::x_t* x) {
    const Orientation& o = g->o[t];
    NnzArgs<SR> a;
    a.plan.n_rows = g->n;
    a.plan.nnz = g->m;
    a.plan.n_tiles = p.n_tiles;
    a.plan.n_nonempty = p.n_nonempty;
    a.plan.n_empty = p.n_empty;
    a.plan.tile_seg = p.tile_seg.as<uint32_t>();
    a.plan.sbits = p.sbits.as<uint32_t>();
    a.plan.nz_rows = p.rows.as<uint32_t>();
    a.plan.empty_rows = p.rows.as<uint32_t>() + p.n_nonempty;
    a.plan.row_ptr = o.rp;
    a.plan.n_fix = p.n_fix;
    a.plan.fix_tiles = p.fix_tiles.as<uint32_t>();
    a.plan.fix_info = p.fix_info.as<uint4>();
    a.plan.n_fix_short = p.n_fix_short;
    a.col = o.col;
    a.val = static_cast<const typename SR::w_t*>(o.val);
    a.x = x;
    a.carry = p.carry.as<typename SR::value_t>();
    a.tail = p.tail.as<typename SR::value_t>();
    a.err = g->err_word;
    a.wait_limit = wait_polls(kWaitPolls);
    return a;
}

template <class SR, class Epi, int WARPS, int HOT, int IPT, bool CONTIG = false>
g1_status launch_nnz2(g1_graph* g, int t, const typename SR::x_t* x, const Epi& main_epi,
                      const Epi& fix_epi, cudaStream_t s) {
    NnzPlan* p = nullptr;
    G1_TRY(ensure_nnz_plan(g, t, &p, 32u * IPT));
    using K = Nnz2Kernel<SR, Epi, WARPS, HOT, IPT, CONTIG>;
    const NnzArgs<SR> a = nnz_args<SR>(g, t, *p, x);
    if (((uintptr_t)a.col | (uintptr_t)a.val) & 31u)
        return fail(G1_ERR_UNSUPPORTED, "nnz SpMV: col/val not 32-byte aligned");
    auto mk = spmv_nnz2_kernel<SR, Epi, WARPS, HOT, IPT, CONTIG>;
    auto fk = spmv_nnz_fixup_kernel<SR, Epi, kMergeBlock>;
    if (profiling()) {
        prof_mark(s, true);
        mk<<<K::grid(g, p->n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
        prof_mark(s, false);
        fk<<<nnz_fix_grid<SR, Epi>(g, *p), kMergeBlock, 0, s>>>(a, fix_epi);
    } else {
        mk<<<K::grid(g, p->n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
        G1_CUDA(launch_pdl(fk, nnz_fix_grid<SR, Epi>(g, *p), kMergeBlock, 0, s, a, fix_epi));
    }
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

template <class SR, class Epi, int WARPS, int MINB, int HOT, bool HINTS = false, bool PIPE = false,
          bool PFL1 = false, int BULK = 0, int PFL2 = 0>
g1_status launch_nnz(g1_graph* g, int t, const NnzPlan& p, const typename SR::x_t* x,
                     const Epi& main_epi, const Epi& fix_epi, cudaStream_t s,
                     typename SR::value_t* carry = nullptr, typename SR::value_t* tail = nullptr) {
    using K = NnzKernel<SR, Epi, WARPS, MINB, HOT, HINTS, PIPE, PFL1, BULK, PFL2>;
    NnzArgs<SR> a = nnz_args<SR>(g, t, p, x);
    // a caller running concurrently with other SpMVs of the graph brings its
    // own per-tile partials (n_tiles each)
    if (carry) a.carry = carry;
    if (tail) a.tail = tail;
    // the tile kernel reads each lane's col/val with 32-byte loads
    if (((uintptr_t)a.col | (uintptr_t)a.val) & 31u)
        return fail(G1_ERR_UNSUPPORTED, "nnz SpMV: col/val not 32-byte aligned");
    const bool prof = profiling();
    // launched even without tiles: its blocks' epilogue partials are read.
    // Both kernels use programmatic dependent launch (the fixup's empty rows
    // overlap the main kernel's tail), except while the main kernel is being
    // timed: its bracketing events would sit between the two.
    auto mk = spmv_nnz_kernel<SR, Epi, WARPS, MINB, HOT, HINTS, PIPE, PFL1, BULK, PFL2>;
    auto fk = spmv_nnz_fixup_kernel<SR, Epi, kMergeBlock>;
    if (prof) {
        prof_mark(s, true);
        mk<<<K::grid(g, p.n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
        prof_mark(s, false);
        fk<<<nnz_fix_grid<SR, Epi>(g, p), kMergeBlock, 0, s>>>(a, fix_epi);
    } else {
        mk<<<K::grid(g, p.n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
        G1_CUDA(launch_pdl(fk, nnz_fix_grid<SR, Epi>(g, p), kMergeBlock, 0, s, a, fix_epi));
    }
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

// Grid sizes of the merge schedule (main, fixup) for the orientation's
// current tile size; builds the plan if needed.
template <class SR, class Epi>
g1_status merge_grids(g1_graph* g, int t, uint32_t* main_grid, uint32_t* fix_grid) {
    const int v = merge_variant(g, t);
    if (kMergeVariants[v].kind == 5) {
        NnzPlan* q = nullptr;
        G1_TRY(ensure_nnz_plan(g, t, &q, 32u * (uint32_t)kMergeVariants[v].ipt));
        switch (v) {
            case 32: *main_grid = Nnz2Kernel<SR, Epi, 32, 32768, 8>::grid(g, q->n_tiles); break;
            case 33: *main_grid = Nnz2Kernel<SR, Epi, 32, 32768, 16>::grid(g, q->n_tiles); break;
            case 34: *main_grid = Nnz2Kernel<SR, Epi, 32, 32768, 24>::grid(g, q->n_tiles); break;
            case 35: *main_grid = Nnz2Kernel<SR, Epi, 32, 16384, 16>::grid(g, q->n_tiles); break;
            case 36: *main_grid = Nnz2Kernel<SR, Epi, 32, 32768, 8, true>::grid(g, q->n_tiles); break;
            case 37: *main_grid = Nnz2Kernel<SR, Epi, 32, 24576, 8>::grid(g, q->n_tiles); break;
            case 38: *main_grid = Nnz2Kernel<SR, Epi, 32, 40960, 8>::grid(g, q->n_tiles); break;
            default: *main_grid = Nnz2Kernel<SR, Epi, 32, 24576, 8, true>::grid(g, q->n_tiles); break;
        }
        *fix_grid = nnz_fix_grid<SR, Epi>(g, *q);
        return G1_OK;
    }
    if (kMergeVariants[v].kind == 3) {
        NnzPlan* q = nullptr;
        G1_TRY(ensure_nnz_plan(g, t, &q));
        switch (v) {
            case 11: *main_grid = NnzKernel<SR, Epi, 16, 2, 16384>::grid(g, q->n_tiles); break;
            case 12: *main_grid = NnzKernel<SR, Epi, 32, 1, 0>::grid(g, q->n_tiles); break;
            case 13: *main_grid = NnzKernel<SR, Epi, 32, 1, 16384, true>::grid(g, q->n_tiles); break;
            case 14: *main_grid = NnzKernel<SR, Epi, 16, 2, 16384, true>::grid(g, q->n_tiles); break;
            case 15: *main_grid = NnzKernel<SR, Epi, 16, 3, 8192, true>::grid(g, q->n_tiles); break;
            case 16: *main_grid = NnzKernel<SR, Epi, 16, 3, 8192>::grid(g, q->n_tiles); break;
            case 17: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768>::grid(g, q->n_tiles); break;
            case 18: *main_grid = NnzKernel<SR, Epi, 32, 1, 49152>::grid(g, q->n_tiles); break;
            case 19: *main_grid = NnzKernel<SR, Epi, 24, 1, 32768, false, true>::grid(g, q->n_tiles); break;
            case 20: *main_grid = NnzKernel<SR, Epi, 16, 1, 32768, false, true>::grid(g, q->n_tiles); break;
            case 21: *main_grid = NnzKernel<SR, Epi, 24, 1, 32768, true, true>::grid(g, q->n_tiles); break;
            case 22: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, true>::grid(g, q->n_tiles); break;
            case 23: *main_grid = NnzKernel<SR, Epi, 32, 1, 16384, false, false, true>::grid(g, q->n_tiles); break;
            case 24: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, false, 1>::grid(g, q->n_tiles); break;
            case 25: *main_grid = NnzKernel<SR, Epi, 32, 1, 16384, false, false, false, 1>::grid(g, q->n_tiles); break;
            case 26: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, false, 2>::grid(g, q->n_tiles); break;
            case 27: *main_grid = NnzKernel<SR, Epi, 32, 1, 24576, false, false, false, 2>::grid(g, q->n_tiles); break;
            case 28: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, false, 0, 1>::grid(g, q->n_tiles); break;
            case 29: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, false, 0, 2>::grid(g, q->n_tiles); break;
            case 30: *main_grid = NnzKernel<SR, Epi, 32, 1, 32768, false, false, false, 0, 4>::grid(g, q->n_tiles); break;
            case 31: *main_grid = NnzKernel<SR, Epi, 24, 1, 32768, false, true, false, 0, 2>::grid(g, q->n_tiles); break;
            default: *main_grid = NnzKernel<SR, Epi, 32, 1, 16384>::grid(g, q->n_tiles); break;
        }
        *fix_grid = nnz_fix_grid<SR, Epi>(g, *q);
        return G1_OK;
    }
    MergePlan* p = nullptr;
    G1_TRY(ensure_plan(g, t, merge_items(v), &p));
    switch (v) {
        case 1: *main_grid = WarpMergeKernel<SR, Epi, 8, 7, 4, 0>::grid(g, p->n_tiles); break;
        case 2: *main_grid = WarpMergeKernel<SR, Epi, 32, 7, 1, 16384>::grid(g, p->n_tiles); break;
        case 3: *main_grid = MergeKernel<SR, Epi, 7, 2>::grid(g, p->n_tiles); break;
        case 4: *main_grid = MergeKernel<SR, Epi, 7, 1>::grid(g, p->n_tiles); break;
        case 5: *main_grid = WarpMergeKernel<SR, Epi, 32, 11, 1, 16384>::grid(g, p->n_tiles); break;
        case 6: *main_grid = WarpTmaKernel<SR, Epi, 24, 15, 16384>::grid(g, p->n_tiles); break;
        case 7: *main_grid = WarpTmaKernel<SR, Epi, 16, 31, 0>::grid(g, p->n_tiles); break;
        case 8: *main_grid = WarpTmaKernel<SR, Epi, 32, 15, 0>::grid(g, p->n_tiles); break;
        case 9: *main_grid = WarpTmaKernel<SR, Epi, 16, 23, 16384>::grid(g, p->n_tiles); break;
        default: *main_grid = WarpMergeKernel<SR, Epi, 8, 11, 3, 0>::grid(g, p->n_tiles); break;
    }
    *fix_grid = (uint32_t)std::max<uint64_t>(1, ceil_div(p->n_tiles, kMergeBlock));
    return G1_OK;
}

template <class SR, class Epi, int IPT, int STAGES>
g1_status launch_merge_v(g1_graph* g, int t, const MergePlan& p, const typename SR::x_t* x,
                         const Epi& main_epi, const Epi& fix_epi, cudaStream_t s) {
    using K = MergeKernel<SR, Epi, IPT, STAGES>;
    const MergeArgs<SR> a = merge_args<SR>(g, t, p, x);
    const bool prof = profiling();
    if (prof) prof_mark(s, true);
    spmv_merge_kernel<SR, Epi, kMergeBlock, IPT, STAGES>
        <<<K::grid(g, p.n_tiles), kMergeBlock, K::L::BYTES, s>>>(a, main_epi);
    if (prof) prof_mark(s, false);
    count_launches(2);
    spmv_fixup_kernel<SR, Epi, kMergeBlock>
        <<<(uint32_t)std::max<uint64_t>(1, ceil_div(p.n_tiles, kMergeBlock)), kMergeBlock, 0, s>>>(
            a, fix_epi);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

template <class SR, class Epi, int WARPS, int IPT, int MINB, int HOT>
g1_status launch_wmerge(g1_graph* g, int t, const MergePlan& p, const typename SR::x_t* x,
                        const Epi& main_epi, const Epi& fix_epi, cudaStream_t s) {
    using K = WarpMergeKernel<SR, Epi, WARPS, IPT, MINB, HOT>;
    const MergeArgs<SR> a = merge_args<SR>(g, t, p, x);
    const bool prof = profiling();
    if (prof) prof_mark(s, true);
    spmv_wmerge_kernel<SR, Epi, WARPS, IPT, MINB, HOT>
        <<<K::grid(g, p.n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
    if (prof) prof_mark(s, false);
    count_launches(2);
    spmv_fixup_kernel<SR, Epi, kMergeBlock>
        <<<(uint32_t)std::max<uint64_t>(1, ceil_div(p.n_tiles, kMergeBlock)), kMergeBlock, 0, s>>>(
            a, fix_epi);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

template <class SR, class Epi, int WARPS, int IPT, int HOT>
g1_status launch_wtma(g1_graph* g, int t, const MergePlan& p, const typename SR::x_t* x,
                      const Epi& main_epi, const Epi& fix_epi, cudaStream_t s) {
    using K = WarpTmaKernel<SR, Epi, WARPS, IPT, HOT>;
    const MergeArgs<SR> a = merge_args<SR>(g, t, p, x);
    const bool prof = profiling();
    if (prof) prof_mark(s, true);
    spmv_wtma_kernel<SR, Epi, WARPS, IPT, HOT>
        <<<K::grid(g, p.n_tiles), WARPS * 32, K::L::BYTES, s>>>(a, main_epi);
    if (prof) prof_mark(s, false);
    count_launches(2);
    spmv_fixup_kernel<SR, Epi, kMergeBlock>
        <<<(uint32_t)std::max<uint64_t>(1, ceil_div(p.n_tiles, kMergeBlock)), kMergeBlock, 0, s>>>(
            a, fix_epi);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

// Merge schedule: main kernel + fixup, with distinct epilogue instances.
template <class SR, class Epi>
g1_status launch_merge(g1_graph* g, int t, const typename SR::x_t* x, const Epi& main_epi,
                       const Epi& fix_epi, cudaStream_t s) {
    const int v = merge_variant(g, t);
    if (kMergeVariants[v].kind == 5) {
        switch (v) {
            case 32: return launch_nnz2<SR, Epi, 32, 32768, 8>(g, t, x, main_epi, fix_epi, s);
            case 33: return launch_nnz2<SR, Epi, 32, 32768, 16>(g, t, x, main_epi, fix_epi, s);
            case 34: return launch_nnz2<SR, Epi, 32, 32768, 24>(g, t, x, main_epi, fix_epi, s);
            case 35: return launch_nnz2<SR, Epi, 32, 16384, 16>(g, t, x, main_epi, fix_epi, s);
            case 36: return launch_nnz2<SR, Epi, 32, 32768, 8, true>(g, t, x, main_epi, fix_epi, s);
            case 37: return launch_nnz2<SR, Epi, 32, 24576, 8>(g, t, x, main_epi, fix_epi, s);
            case 38: return launch_nnz2<SR, Epi, 32, 40960, 8>(g, t, x, main_epi, fix_epi, s);
            default: return launch_nnz2<SR, Epi, 32, 24576, 8, true>(g, t, x, main_epi, fix_epi, s);
        }
    }
    if (kMergeVariants[v].kind == 3) {
        NnzPlan* q = nullptr;
        G1_TRY(ensure_nnz_plan(g, t, &q));
        switch (v) {
            case 11: return launch_nnz<SR, Epi, 16, 2, 16384>(g, t, *q, x, main_epi, fix_epi, s);
            case 12: return launch_nnz<SR, Epi, 32, 1, 0>(g, t, *q, x, main_epi, fix_epi, s);
            case 13: return launch_nnz<SR, Epi, 32, 1, 16384, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 14: return launch_nnz<SR, Epi, 16, 2, 16384, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 15: return launch_nnz<SR, Epi, 16, 3, 8192, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 16: return launch_nnz<SR, Epi, 16, 3, 8192>(g, t, *q, x, main_epi, fix_epi, s);
            case 17: return launch_nnz<SR, Epi, 32, 1, 32768>(g, t, *q, x, main_epi, fix_epi, s);
            case 18: return launch_nnz<SR, Epi, 32, 1, 49152>(g, t, *q, x, main_epi, fix_epi, s);
            case 19: return launch_nnz<SR, Epi, 24, 1, 32768, false, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 20: return launch_nnz<SR, Epi, 16, 1, 32768, false, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 21: return launch_nnz<SR, Epi, 24, 1, 32768, true, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 22: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 23: return launch_nnz<SR, Epi, 32, 1, 16384, false, false, true>(g, t, *q, x, main_epi, fix_epi, s);
            case 24: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, false, 1>(g, t, *q, x, main_epi, fix_epi, s);
            case 25: return launch_nnz<SR, Epi, 32, 1, 16384, false, false, false, 1>(g, t, *q, x, main_epi, fix_epi, s);
            case 26: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, false, 2>(g, t, *q, x, main_epi, fix_epi, s);
            case 27: return launch_nnz<SR, Epi, 32, 1, 24576, false, false, false, 2>(g, t, *q, x, main_epi, fix_epi, s);
            case 28: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, false, 0, 1>(g, t, *q, x, main_epi, fix_epi, s);
            case 29: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, false, 0, 2>(g, t, *q, x, main_epi, fix_epi, s);
            case 30: return launch_nnz<SR, Epi, 32, 1, 32768, false, false, false, 0, 4>(g, t, *q, x, main_epi, fix_epi, s);
            case 31: return launch_nnz<SR, Epi, 24, 1, 32768, false, true, false, 0, 2>(g, t, *q, x, main_epi, fix_epi, s);
            default: return launch_nnz<SR, Epi, 32, 1, 16384>(g, t, *q, x, main_epi, fix_epi, s);
        }
    }
    MergePlan* p = nullptr;
    G1_TRY(ensure_plan(g, t, merge_items(v), &p));
    if (p->n_tiles == 0) return G1_OK;
    switch (v) {
        case 1: return launch_wmerge<SR, Epi, 8, 7, 4, 0>(g, t, *p, x, main_epi, fix_epi, s);
        case 2: return launch_wmerge<SR, Epi, 32, 7, 1, 16384>(g, t, *p, x, main_epi, fix_epi, s);
        case 3: return launch_merge_v<SR, Epi, 7, 2>(g, t, *p, x, main_epi, fix_epi, s);
        case 4: return launch_merge_v<SR, Epi, 7, 1>(g, t, *p, x, main_epi, fix_epi, s);
        case 5: return launch_wmerge<SR, Epi, 32, 11, 1, 16384>(g, t, *p, x, main_epi, fix_epi, s);
        case 6: return launch_wtma<SR, Epi, 24, 15, 16384>(g, t, *p, x, main_epi, fix_epi, s);
        case 7: return launch_wtma<SR, Epi, 16, 31, 0>(g, t, *p, x, main_epi, fix_epi, s);
        case 8: return launch_wtma<SR, Epi, 32, 15, 0>(g, t, *p, x, main_epi, fix_epi, s);
        case 9: return launch_wtma<SR, Epi, 16, 23, 16384>(g, t, *p, x, main_epi, fix_epi, s);
        default: return launch_wmerge<SR, Epi, 8, 11, 3, 0>(g, t, *p, x, main_epi, fix_epi, s);
    }
}

template <class SR, class Epi>
g1_status launch_vector(g1_graph* g, int t, const typename SR::x_t* x, const Epi& epi,
                        cudaStream_t s) {
    const Orientation& o = g->o[t];
    if (g->n == 0) return G1_OK;
    const uint32_t grid = vector_grid<SR, Epi>(g);
    const auto* val = static_cast<const typename SR::w_t*>(o.val);
    const bool prof = profiling();
    if (prof) prof_mark(s, true);
    count_launches(1);
    switch (vector_tpr(g)) {
        case 1: spmv_vector_kernel<SR, Epi, kVectorBlock, 1><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
        case 2: spmv_vector_kernel<SR, Epi, kVectorBlock, 2><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
        case 4: spmv_vector_kernel<SR, Epi, kVectorBlock, 4><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
        case 8: spmv_vector_kernel<SR, Epi, kVectorBlock, 8><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
        case 16: spmv_vector_kernel<SR, Epi, kVectorBlock, 16><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
        default: spmv_vector_kernel<SR, Epi, kVectorBlock, 32><<<grid, kVectorBlock, 0, s>>>(g->n, o.rp, o.col, val, x, epi); break;
    }
    if (prof) prof_mark(s, false);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

// One SpMV with a single epilogue instance (no per-kernel epilogue state).
template <class SR, class Epi>
g1_status run_spmv(g1_graph* g, int t, g1_schedule sched, const typename SR::x_t* x,
                   const Epi& epi, cudaStream_t s) {
    if (resolve_schedule(g, t, sched) == G1_SCHED_VECTOR) return launch_vector<SR>(g, t, x, epi, s);
    return launch_merge<SR>(g, t, x, epi, epi, s);
}

}  // namespace g1
