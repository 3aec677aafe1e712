// Host-side launch of the SpMV schedules for the prebuilt semirings.
#pragma once

#include <algorithm>

#include "g1/spmv.cuh"
#include "internal.h"

namespace g1 {

constexpr int kMergeBlock = 256;
constexpr int kMergeIpt = 7;  // odd: consecutive threads' shared-memory reads fall in distinct banks
constexpr int kVectorBlock = 256;

template <class K>
int blocks_per_sm(K kernel, int block) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0) != cudaSuccess) {
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
    // Uniform small degrees: one short row per lane group, no merge bookkeeping.
    return (o.max_deg <= 64 && mean <= 16.0 && o.max_deg <= 8 * std::max(1.0, mean))
               ? G1_SCHED_VECTOR
               : G1_SCHED_MERGE;
}

template <class SR, class Epi>
uint32_t merge_main_grid(const g1_graph* g, int t) {
    static int occ = blocks_per_sm(spmv_merge_kernel<SR, Epi, kMergeBlock, kMergeIpt>, kMergeBlock);
    const uint32_t tiles = g->o[t].plan->n_tiles;
    return std::max<uint32_t>(1, std::min<uint32_t>(tiles, (uint32_t)g->sm_count * occ));
}

template <class SR, class Epi>
uint32_t merge_fixup_grid(const g1_graph* g, int t) {
    return (uint32_t)std::max<uint64_t>(1, ceil_div(g->o[t].plan->n_tiles, kMergeBlock));
}

template <class SR, class Epi>
uint32_t vector_grid(const g1_graph* g) {
    static int occ = blocks_per_sm(spmv_vector_kernel<SR, Epi, kVectorBlock, 32>, kVectorBlock);
    const int tpr = vector_tpr(g);
    const uint64_t want = ceil_div((uint64_t)g->n * tpr, kVectorBlock);
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->sm_count * occ));
}

template <class SR>
MergeArgs<SR> merge_args(const g1_graph* g, int t, const typename SR::x_t* x) {
    const Orientation& o = g->o[t];
    const MergePlan& p = *o.plan;
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
    return a;
}

// Merge schedule: main kernel + fixup, with distinct epilogue instances.
template <class SR, class Epi>
g1_status launch_merge(g1_graph* g, int t, const typename SR::x_t* x, const Epi& main_epi,
                       const Epi& fix_epi, cudaStream_t s) {
    G1_TRY(ensure_plan(g, t));
    if (g->o[t].plan->n_tiles == 0) return G1_OK;
    const MergeArgs<SR> a = merge_args<SR>(g, t, x);
    const bool prof = profiling();
    if (prof) prof_mark(s, true);
    spmv_merge_kernel<SR, Epi, kMergeBlock, kMergeIpt>
        <<<merge_main_grid<SR, Epi>(g, t), kMergeBlock, 0, s>>>(a, main_epi);
    if (prof) prof_mark(s, false);
    count_launches(2);
    spmv_fixup_kernel<SR, Epi, kMergeBlock>
        <<<merge_fixup_grid<SR, Epi>(g, t), kMergeBlock, 0, s>>>(a, fix_epi);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
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
