#pragma once
// The semiring SpMV operator of the GraphOne API (reference:
// archi/blas/spmv/def.hpp:8-76, cpu/cpu.hpp:8-33, cpu/naive.hpp:5-20,
// cuda/cuda.cuh:10-104):
//
//     y[r] = fold of functor_t::reduce over the nonzeros (r, c) of A of
//            functor_t::combine(A[r][c], x[c]), from functor_t::initialize()
//
//     auto spmv = blas::MakeCsrSpMV<arch, kind, functor_t>(
//         n_rows, n_cols, nnz, row_offsets, col_indices, values, x, y);
//     spmv();          // the CUDA kinds take spmv(bool sync = true)
//
// `kind` selects the schedule:
//   SpmvCpuNaive           the row loop on the host (host pointers);
//   SpmvCudaCsrVector      this library's CSR-vector kernel, 2/4/8/16 lanes
//                          per row by the mean row length (device pointers);
//   SpmvCudaCsrMergeBased  this library's warp-tile merge-path kernel and its
//                          carry fixup (device pointers).  The constructor
//                          partitions the merge path of row_offsets once and
//                          keeps the partition and the per-tile carries in
//                          device memory until destruction; each call runs
//                          the tile kernel and the fixup.
// The CUDA kinds run on the legacy default stream, read the arrays only
// within [0, n_rows] (offsets) and [0, nnz) (columns, values), so they need
// no padding or alignment beyond the element types', and take 4-byte
// unsigned index and offset types.  Integer folds equal the row loop's bit
// for bit; a floating-point fold associates differently (tiles, lanes), so
// its last bits may differ from the row loop's.
//
// Differences from the reference, result-neutral: the CUDA dispatchers own
// device memory and are move-only (the reference's merge dispatcher frees
// its buffer in the destructor of every copy); the CSR-vector dispatcher
// checks and synchronises on every call (the reference returns before both
// for rows of up to 8 nonzeros on average) and accepts n_rows == 0.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"

#ifdef __CUDACC__
#include <cuda_runtime.h>

#include "graphone_b200.h"
#include "g1/spmv.cuh"
#endif

namespace graph_one::blas {

template <typename index_t, typename offset_t, typename mat_value_t, typename vec_x_value_t,
          typename vec_y_value_t>
struct SpmvCsrParams {
    index_t n_rows;
    index_t n_cols;
    offset_t nnz;
    const offset_t* row_offsets;  // n_rows + 1
    const index_t* col_indices;   // nnz
    const mat_value_t* values;    // nnz
    const vec_x_value_t* vector_x;  // n_cols
    vec_y_value_t* vector_y;        // n_rows
};

// The reference's default operator: combine = min(a, x), reduce = +, from 0.
template <typename mat_value_t, typename vec_x_value_t, typename vec_y_value_t>
struct DefaultSpmvFunctor {
    __ONE_ARCH_INL__ static vec_y_value_t initialize() { return vec_y_value_t{0}; }
    __ONE_ARCH_INL__ static vec_y_value_t combine(const mat_value_t& a, const vec_x_value_t& x) {
        return (a < x) ? a : x;
    }
    __ONE_ARCH_INL__ static vec_y_value_t reduce(const vec_y_value_t& l, const vec_y_value_t& r) {
        return l + r;
    }
};

// The row loop (the name keeps the reference's spelling).
template <typename functor_t, typename index_t, typename offset_t, typename mat_value_t,
          typename vecx_value_t, typename vecy_value_t>
void SpMV_cpu_navie(index_t n_rows, const offset_t* Ap, const index_t* Aj, const mat_value_t* Ax,
                    const vecx_value_t* x, vecy_value_t* y) {
    for (index_t r = 0; r < n_rows; ++r) {
        vecy_value_t acc = functor_t::initialize();
        for (offset_t k = Ap[r]; k < Ap[r + 1]; ++k) acc = functor_t::reduce(acc, functor_t::combine(Ax[k], x[Aj[k]]));
        y[r] = acc;
    }
}

struct SpmvCpuNaive {
    constexpr static arch_t arch_type = arch_t::cpu;
};
struct SpmvCudaCsrVector {
    constexpr static arch_t arch_type = arch_t::cuda;
};
struct SpmvCudaCsrMergeBased {
    constexpr static arch_t arch_type = arch_t::cuda;
};

template <typename kind, typename functor_t, typename index_t, typename offset_t, typename mat_value_t,
          typename vec_x_value_t, typename vec_y_value_t>
struct SpmvDispatcher {};

template <typename functor_t, typename index_t, typename offset_t, typename mat_value_t,
          typename vec_x_value_t, typename vec_y_value_t>
struct SpmvDispatcher<SpmvCpuNaive, functor_t, index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t> {
    using spmv_params_t = SpmvCsrParams<index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t>;
    explicit SpmvDispatcher(const spmv_params_t& p) : params(p) {}
    void operator()() {
        SpMV_cpu_navie<functor_t>(params.n_rows, params.row_offsets, params.col_indices, params.values,
                                  params.vector_x, params.vector_y);
    }
    spmv_params_t params;
};

#ifdef __CUDACC__
namespace spmv_detail {

// The reference's SpMV functor (initialize / combine / reduce) as this
// library's semiring.
template <class F, class W, class X, class Y>
struct FunctorOps {
    using value_t = Y;
    using x_t = X;
    using w_t = W;
    __device__ static __forceinline__ Y identity() { return F::initialize(); }
    __device__ static __forceinline__ Y combine(const W& w, const X& x) { return F::combine(w, x); }
    __device__ static __forceinline__ Y reduce(const Y& a, const Y& b) { return F::reduce(a, b); }
};

template <class index_t, class offset_t>
constexpr bool kU32Indices = sizeof(index_t) == 4 && sizeof(offset_t) == 4 && std::is_unsigned_v<index_t> &&
                             std::is_unsigned_v<offset_t>;

// Tile t of the merge path starts at diagonal t * items: its (row, nonzero)
// coordinate by the merge-path search over the row ends row_ptr[1..n].
template <int kUnused = 0>
__global__ void merge_partition_kernel(const uint32_t* row_ptr, uint32_t n_rows, uint32_t nnz,
                                       uint32_t items, uint32_t n_tiles, uint32_t* tile_row,
                                       uint32_t* tile_nnz) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    const uint64_t total = (uint64_t)n_rows + nnz;
    const uint64_t d = (uint64_t)t * items < total ? (uint64_t)t * items : total;
    uint32_t i = 0, j = 0;
    g1::merge_path_search(d, row_ptr + 1, n_rows, nnz, &i, &j);
    tile_row[t] = i;
    tile_nnz[t] = j;
}

inline void check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    std::fprintf(stderr, "[ERROR] SpMV %s: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
}

inline void check(g1_status s, const char* what) {
    if (s == G1_OK) return;
    std::fprintf(stderr, "[ERROR] SpMV %s: %s (%s)\n", what, g1_status_string(s), g1_last_error());
    std::exit(1);
}

inline int sm_count() {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

}  // namespace spmv_detail

template <typename functor_t, typename index_t, typename offset_t, typename mat_value_t,
          typename vec_x_value_t, typename vec_y_value_t>
struct SpmvDispatcher<SpmvCudaCsrVector, functor_t, index_t, offset_t, mat_value_t, vec_x_value_t,
                      vec_y_value_t> {
    static_assert(spmv_detail::kU32Indices<index_t, offset_t>, "index and offset types must be 4-byte unsigned");
    using spmv_params_t = SpmvCsrParams<index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t>;
    using SR = spmv_detail::FunctorOps<functor_t, mat_value_t, vec_x_value_t, vec_y_value_t>;
    using Epi = g1::StoreEpilogue<vec_y_value_t>;
    static constexpr int kBlock = 256;

    explicit SpmvDispatcher(const spmv_params_t& p)
        : params(p), nnz_per_row(p.n_rows ? p.nnz / p.n_rows : 0) {}

    void operator()(bool sync = true) {
        if (params.n_rows == 0) return;
        if (nnz_per_row <= 2)
            launch<2>();
        else if (nnz_per_row <= 4)
            launch<4>();
        else if (nnz_per_row <= 8)
            launch<8>();
        else
            launch<16>();
        spmv_detail::check(cudaGetLastError(), "CSR-vector launch");
        g1_count_user_launches(1);
        if (sync) spmv_detail::check(cudaDeviceSynchronize(), "CSR-vector");
    }

    spmv_params_t params;
    offset_t nnz_per_row;

private:
    template <int TPR>
    void launch() {
        const uint64_t want = ((uint64_t)params.n_rows * TPR + kBlock - 1) / kBlock;
        const uint32_t grid =
            (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)spmv_detail::sm_count() * 8));
        g1::spmv_vector_kernel<SR, Epi, kBlock, TPR><<<grid, kBlock>>>(
            (uint32_t)params.n_rows, reinterpret_cast<const uint32_t*>(params.row_offsets),
            reinterpret_cast<const uint32_t*>(params.col_indices), params.values, params.vector_x,
            Epi{params.vector_y});
    }
};

template <typename functor_t, typename index_t, typename offset_t, typename mat_value_t,
          typename vec_x_value_t, typename vec_y_value_t>
struct SpmvDispatcher<SpmvCudaCsrMergeBased, functor_t, index_t, offset_t, mat_value_t, vec_x_value_t,
                      vec_y_value_t> {
    static_assert(spmv_detail::kU32Indices<index_t, offset_t>, "index and offset types must be 4-byte unsigned");
    using spmv_params_t = SpmvCsrParams<index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t>;
    using SR = spmv_detail::FunctorOps<functor_t, mat_value_t, vec_x_value_t, vec_y_value_t>;
    using Epi = g1::StoreEpilogue<vec_y_value_t>;
    // warp tiles of 32 x 7 merge items, 8 warps per block, no x cache
    static constexpr int kWarps = 8;
    static constexpr int kIpt = 7;
    static constexpr uint32_t kItems = 32 * kIpt;
    using Layout = g1::WarpMergeLayout<SR, kWarps, kIpt, 0>;

    explicit SpmvDispatcher(const spmv_params_t& p) : params(p) {
        n_tiles = (uint32_t)(((uint64_t)p.n_rows + p.nnz + kItems - 1) / kItems);
        const size_t entries = (size_t)n_tiles + 1;
        spmv_detail::check(g1_mem_alloc(&tile_row, entries * 4), "partition allocation");
        spmv_detail::check(g1_mem_alloc(&tile_nnz, entries * 4), "partition allocation");
        spmv_detail::check(g1_mem_alloc(&carry, entries * sizeof(vec_y_value_t)), "carry allocation");
        spmv_detail::check(g1_mem_alloc(&tail, entries * sizeof(vec_y_value_t)), "carry allocation");
        if (n_tiles == 0) return;
        spmv_detail::merge_partition_kernel<<<(unsigned)((entries + 255) / 256), 256>>>(
            reinterpret_cast<const uint32_t*>(p.row_offsets), (uint32_t)p.n_rows, (uint32_t)p.nnz, kItems,
            n_tiles, static_cast<uint32_t*>(tile_row), static_cast<uint32_t*>(tile_nnz));
        spmv_detail::check(cudaGetLastError(), "merge-path partition");
        g1_count_user_launches(1);
    }

    SpmvDispatcher(const SpmvDispatcher&) = delete;
    SpmvDispatcher& operator=(const SpmvDispatcher&) = delete;
    SpmvDispatcher(SpmvDispatcher&& o) noexcept
        : params(o.params), n_tiles(o.n_tiles), tile_row(std::exchange(o.tile_row, nullptr)),
          tile_nnz(std::exchange(o.tile_nnz, nullptr)), carry(std::exchange(o.carry, nullptr)),
          tail(std::exchange(o.tail, nullptr)) {}

    ~SpmvDispatcher() {
        // the kernels of earlier calls may still read these buffers
        if (tile_row || tile_nnz || carry || tail) cudaDeviceSynchronize();
        g1_mem_free(tile_row);
        g1_mem_free(tile_nnz);
        g1_mem_free(carry);
        g1_mem_free(tail);
    }

    void operator()(bool sync = true) {
        if (n_tiles == 0) return;
        static const bool attr_set = [] {
            if (Layout::BYTES > 48 * 1024)
                cudaFuncSetAttribute(g1::spmv_wmerge_kernel<SR, Epi, kWarps, kIpt, 3, 0, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Layout::BYTES);
            return true;
        }();
        (void)attr_set;
        g1::MergeArgs<SR> a{};
        a.plan.n_rows = (uint32_t)params.n_rows;
        a.plan.nnz = (uint32_t)params.nnz;
        a.plan.items = kItems;
        a.plan.n_tiles = n_tiles;
        a.plan.row_ptr = reinterpret_cast<const uint32_t*>(params.row_offsets);
        a.plan.tile_row = static_cast<const uint32_t*>(tile_row);
        a.plan.tile_nnz = static_cast<const uint32_t*>(tile_nnz);
        a.col = reinterpret_cast<const uint32_t*>(params.col_indices);
        a.val = params.values;
        a.x = params.vector_x;
        a.carry = static_cast<vec_y_value_t*>(carry);
        a.tail = static_cast<vec_y_value_t*>(tail);
        a.err = nullptr;
        const uint64_t want = (n_tiles + kWarps - 1) / kWarps;
        const uint32_t grid =
            (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)spmv_detail::sm_count() * 8));
        g1::spmv_wmerge_kernel<SR, Epi, kWarps, kIpt, 3, 0, true>
            <<<grid, kWarps * 32, Layout::BYTES>>>(a, Epi{params.vector_y});
        g1::spmv_fixup_kernel<SR, Epi, 256><<<(n_tiles + 255) / 256, 256>>>(a, Epi{params.vector_y});
        spmv_detail::check(cudaGetLastError(), "merge-path launch");
        g1_count_user_launches(2);
        if (sync) spmv_detail::check(cudaDeviceSynchronize(), "merge-path");
    }

    spmv_params_t params;
    uint32_t n_tiles = 0;

private:
    void* tile_row = nullptr;
    void* tile_nnz = nullptr;
    void* carry = nullptr;
    void* tail = nullptr;
};
#endif  // __CUDACC__

template <arch_t arch, typename kind, typename functor_t, typename index_t, typename offset_t,
          typename mat_value_t, typename vec_x_value_t, typename vec_y_value_t>
SpmvDispatcher<kind, functor_t, index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t> MakeCsrSpMV(
    index_t n_rows, index_t n_cols, offset_t nnz, const offset_t* row_offsets, const index_t* col_indices,
    const mat_value_t* values, const vec_x_value_t* vector_x, vec_y_value_t* vector_y) {
    static_assert(arch == kind::arch_type, "the schedule runs on another architecture");
    const SpmvCsrParams<index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t> p{
        n_rows, n_cols, nnz, row_offsets, col_indices, values, vector_x, vector_y};
    return SpmvDispatcher<kind, functor_t, index_t, offset_t, mat_value_t, vec_x_value_t, vec_y_value_t>(p);
}

}  // namespace graph_one::blas
