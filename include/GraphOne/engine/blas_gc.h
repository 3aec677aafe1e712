#pragma once
// The semiring SpMV ("BLAS") engine of the GraphOne API (reference:
// engine/blas_gc.h:21-474), with the user functor inlined into this
// library's merge-path SpMV (include/g1/spmv.cuh).
//
// One iteration of GraphOne's engine is Construct (x from the frontier via
// construct_each), Gather (y = A^T (+,x) x with gather_combine /
// gather_reduce, folded from default_result) and Apply (apply_each per
// vertex, frontier update).  Here Apply (and, for the dense and all-active
// frontiers, the next Construct, exactly as GraphOne's
// apply_construct_kernel pairs them) runs in the SpMV's epilogue for every
// completed row: y never reaches memory and there is no N-sized pass.  x is
// double-buffered across iterations where the epilogue writes the next x.
// For the sparse frontier x stays default_info between iterations; only the
// frontier's entries are set before and reset after the SpMV.
//
// Semantics kept from GraphOne: the same functor calls with the same
// arguments, the d_status copy of the launch, apply guarded by
// res != default_result() for the sparse and dense frontiers and unguarded
// for all-active; one host read-back of the new frontier size per
// iteration (the Run loop tests it).

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

#include "graphone_b200.h"
#include "g1/common.cuh"
#include "g1/semiring.cuh"
#include "g1/spmv.cuh"
#include "GraphOne/base/buffer.h"
#include "GraphOne/engine/base.h"
#include "GraphOne/frontier/frontier.h"
#include "GraphOne/graph/graph.h"
#include "GraphOne/macros.h"

namespace graph_one {
namespace engine {
namespace blas_detail {

template <class F, class D, class V>
struct SparseEpi {
    D ds;
    V* out;
    uint32_t* count;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t v, const typename F::gather_type& res) {
        if (res != F::default_result() && F::apply_each(V(v), res, ds)) g1::append(out, count, v);
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

template <class F, class D, class V>
struct DenseEpi {
    D ds;
    typename F::info_type* x_next;
    uint32_t* count;
    uint32_t local;
    __device__ __forceinline__ void begin() { local = 0; }
    __device__ __forceinline__ void emit(uint32_t v, const typename F::gather_type& res) {
        const bool pred = res != F::default_result() && F::apply_each(V(v), res, ds);
        x_next[v] = pred ? F::construct_each(V(v), ds) : F::default_info();
        local += pred ? 1u : 0u;
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char* smem) {
        const uint32_t s = g1::block_sum<uint32_t, BLOCK>(local, reinterpret_cast<uint32_t*>(smem));
        if (threadIdx.x == 0 && s) atomicAdd(count, s);
    }
};

template <class F, class D, class V>
struct AllActiveEpi {
    D ds;
    typename F::info_type* x_next;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ void emit(uint32_t v, const typename F::gather_type& res) {
        const bool pred = F::apply_each(V(v), res, ds);
        x_next[v] = pred ? F::construct_each(V(v), ds) : F::default_info();
    }
    template <int BLOCK>
    __device__ __forceinline__ void block_end(char*) {}
};

template <class F, class D, class V>
__global__ void construct_list_kernel(const V* list, uint32_t n, D ds, typename F::info_type* x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V v = list[i];
        x[v] = F::construct_each(v, ds);
    }
}

template <class V, class I>
__global__ void set_list_kernel(const V* list, uint32_t n, I value, I* x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[list[i]] = value;
}

template <class F, class D, class V>
__global__ void construct_all_kernel(uint32_t n, D ds, typename F::info_type* x) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        x[v] = F::construct_each(V(v), ds);
}

template <class I>
__global__ void fill_kernel(I* x, uint32_t n, I value) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        x[v] = value;
}

inline unsigned grid_for(uint32_t n) {
    const uint32_t want = (n + 255) / 256;
    return std::max(1u, std::min<uint32_t>(want, (uint32_t)detail::sm_count() * 8));
}

// Sparse steps of the sparse-frontier engine (BlasGcEngine<SPARSE_BASED>).
// Whether every edge's gather_combine with default_info gives default_result
// and default_result folds into itself: then a row without an in-neighbour on
// the frontier (x is default_info off the frontier) folds to default_result,
// which apply never sees.  *bad is set when not.
template <class F, class SR>
__global__ void sparse_check_kernel(const typename SR::w_t* val, uint32_t m, uint32_t* bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
        if (SR::combine(val[k], F::default_info()) != F::default_result()) atomicOr(bad, 1u);
    if (blockIdx.x == 0 && threadIdx.x == 0 &&
        SR::reduce(F::default_result(), F::default_result()) != F::default_result())
        atomicOr(bad, 1u);
}

// The frontier's out-neighbours (the rows it reaches), each listed once
// (its bit set first), and the sum of their in-degrees: cnt[0] rows,
// cnt[2..3] the sum (64-bit).  One warp per frontier vertex.
template <class V>
__global__ void sparse_expand_kernel(const V* in, uint32_t n_in, const uint32_t* out_rp, const uint32_t* out_col,
                                     const uint32_t* in_rp, uint32_t* bits, uint32_t* cand, uint32_t* cnt) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    unsigned long long* insum = reinterpret_cast<unsigned long long*>(cnt + 2);
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_in; i += warps) {
        const uint32_t u = (uint32_t)in[i];
        for (uint32_t k = out_rp[u] + lane; k < out_rp[u + 1]; k += 32) {
            const uint32_t v = out_col[k];
            const uint32_t bit = 1u << (v & 31u);
            if (atomicOr(&bits[v >> 5], bit) & bit) continue;  // listed already
            cand[atomicAdd(&cnt[0], 1u)] = v;
            atomicAdd(insum, (unsigned long long)(in_rp[v + 1] - in_rp[v]));
        }
    }
}

// The listed rows, one warp each: the row's fold over all its in-edges (the
// functor's gather_combine / gather_reduce, as the full pull folds it), then
// apply as SparseEpi does; the row's bit is cleared.
template <class F, class SR, class D, class V>
__global__ void sparse_rows_kernel(const uint32_t* cand, uint32_t nc, const uint32_t* in_rp, const uint32_t* in_col,
                                   const typename SR::w_t* in_val, const typename SR::x_t* x, D ds, V* out,
                                   uint32_t* count, uint32_t* bits) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += warps) {
        const uint32_t v = cand[i];
        typename SR::value_t acc = SR::identity();
        for (uint32_t k = in_rp[v] + lane; k < in_rp[v + 1]; k += 32)
            acc = SR::reduce(acc, SR::combine(in_val[k], x[in_col[k]]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = SR::reduce(acc, g1::shfl_down_any(0xffffffffu, acc, off));
        if (lane == 0) {
            atomicAnd(&bits[v >> 5], ~(1u << (v & 31u)));
            if (acc != F::default_result() && F::apply_each(V(v), acc, ds)) g1::append(out, count, v);
        }
    }
}

// Clears the bits of the listed rows (when the step pulls every row after all).
__global__ void sparse_clear_kernel(const uint32_t* cand, uint32_t nc, uint32_t* bits) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x)
        atomicAnd(&bits[cand[i] >> 5], ~(1u << (cand[i] & 31u)));
}

}  // namespace blas_detail

template <typename functor_t, typename comp_t, typename frontier_t>
class BlasGcEngineBase : public GcEngine<comp_t, frontier_t> {
public:
    using base_t = GcEngine<comp_t, frontier_t>;
    using graph_t = typename comp_t::graph_type;
    using dstatus_t = typename comp_t::dstatus_type;
    using vertex_t = typename graph_t::vertex_type;
    using edge_t = typename graph_t::edge_type;
    using weight_t = typename graph_t::weight_type;
    using info_t = typename functor_t::info_type;
    using gather_t = typename functor_t::gather_type;
    using SR = g1::FunctorSemiring<functor_t, weight_t>;

    // Warp tiles of 32 x 7 merge items, 32 warps per block, x[0, 16384)
    // cached in shared memory when x entries are 4 bytes.
    static constexpr int kWarps = 32;
    static constexpr int kIpt = 7;
    static constexpr int kHot = sizeof(info_t) <= 4 ? 16384 : 0;
    static constexpr uint32_t kItems = 32 * kIpt;
    // With 4-byte edge weights the library's default schedule instead: the
    // nnz-split tiles (256 nonzeros per warp tile, 32-byte col/val loads,
    // row starts from a bitmap; include/g1/spmv.cuh), x[0, 32768) cached.
    static constexpr bool kNnzOk = sizeof(weight_t) == 4 && sizeof(gather_t) <= 8;
    static constexpr int kNnzHot = sizeof(info_t) <= 4 ? 32768 : 0;

    BlasGcEngineBase(comp_t& comp, frontier_t& frontier)
        : base_t(comp, frontier), n_(comp.graph.num_vertices()),
          x_{DenseVec<arch_t::cuda, info_t>(std::max<vertex_t>(n_, 1)),
             DenseVec<arch_t::cuda, info_t>(std::max<vertex_t>(n_, 1))} {
        // a blocking stream: ordered with the legacy default stream the archi
        // primitives and the host hooks use
        detail::check_cuda(cudaStreamCreate(&stream_), "stream");
        g1_graph* h = comp.graph.handle();
        // the pull side: in-edges when the graph has them, else the main CSR
        // (GraphOne: engine/blas_gc.h:144-159)
        side_ = graph_t::has_transpose ? 1 : 0;
        const uint32_t *rp = nullptr, *ci = nullptr;
        const void* val = nullptr;
        detail::check_g1(g1_graph_arrays(h, side_, &rp, &ci, &val), "graph arrays");
        uint32_t tiles = 0;
        const uint32_t *tr = nullptr, *tn = nullptr;
        void *carry = nullptr, *tail = nullptr;
        detail::check_g1(g1_spmv_plan(h, side_, kItems, &tiles, &tr, &tn, &carry, &tail), "plan");
        args_.plan.n_rows = n_;
        args_.plan.nnz = comp.graph.num_edges();
        args_.plan.items = kItems;
        args_.plan.n_tiles = tiles;
        args_.plan.row_ptr = rp;
        args_.plan.tile_row = tr;
        args_.plan.tile_nnz = tn;
        args_.col = ci;
        args_.val = static_cast<const weight_t*>(val);
        args_.carry = static_cast<gather_t*>(carry);
        args_.tail = static_cast<gather_t*>(tail);
        args_.err = nullptr;
        if constexpr (kNnzOk) {
            g1_nnz_plan p{};
            // the tile kernel reads each lane's col/val with 32-byte loads
            if (!(((uintptr_t)ci | (uintptr_t)val) & 31u) &&
                g1_spmv_nnz_plan(h, side_, &p) == G1_OK) {
                nnz_ = true;
                nargs_.plan.n_rows = p.n_rows;
                nargs_.plan.nnz = p.nnz;
                nargs_.plan.n_tiles = p.n_tiles;
                nargs_.plan.n_nonempty = p.n_nonempty;
                nargs_.plan.n_empty = p.n_empty;
                nargs_.plan.tile_seg = p.tile_seg;
                nargs_.plan.sbits = p.sbits;
                nargs_.plan.nz_rows = p.rows;
                nargs_.plan.empty_rows = p.rows + p.n_nonempty;
                nargs_.plan.row_ptr = p.row_ptr;
                nargs_.plan.n_fix = p.n_fix;
                nargs_.plan.fix_tiles = p.fix_tiles;
                nargs_.plan.fix_info = static_cast<const uint4*>(p.fix_info);
                nargs_.plan.n_fix_short = p.n_fix_short;
                nargs_.col = ci;
                nargs_.val = static_cast<const weight_t*>(val);
                nargs_.carry = static_cast<gather_t*>(p.carry);
                nargs_.tail = static_cast<gather_t*>(p.tail);
                nargs_.err = nullptr;
            }
        }
    }

    ~BlasGcEngineBase() override {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }

protected:
    template <class Epi>
    void spmv(const info_t* x, const Epi& epi) {
        if constexpr (kNnzOk) {
            if (nnz_) {
                spmv_nnz(x, epi);
                return;
            }
        }
        using L = g1::WarpMergeLayout<SR, kWarps, kIpt, kHot>;
        auto kernel = g1::spmv_wmerge_kernel<SR, Epi, kWarps, kIpt, 1, kHot>;
        static const int occ = [&] {
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kWarps * 32, L::BYTES);
            return std::max(1, b);
        }();
        if (args_.plan.n_tiles == 0) return;
        g1::MergeArgs<SR> a = args_;
        a.x = x;
        const uint32_t grid = std::max<uint32_t>(
            1, std::min<uint32_t>((args_.plan.n_tiles + kWarps - 1) / kWarps,
                                  (uint32_t)detail::sm_count() * occ));
        kernel<<<grid, kWarps * 32, L::BYTES, stream_>>>(a, epi);
        g1::spmv_fixup_kernel<SR, Epi, 256>
            <<<(args_.plan.n_tiles + 255) / 256, 256, 0, stream_>>>(a, epi);
        detail::check_cuda(cudaGetLastError(), "merge SpMV launch");
        g1_count_user_launches(2);
    }

    // The nnz-split schedule: main kernel (one 1024-thread block per SM)
    // and the fixup of the rows that cross tiles and of the empty rows.
    template <class Epi>
    void spmv_nnz(const info_t* x, const Epi& epi) {
        using L = g1::NnzLayout<SR, 32, kNnzHot>;
        auto kernel = g1::spmv_nnz_kernel<SR, Epi, 32, 1, kNnzHot>;
        auto fixup = g1::spmv_nnz_fixup_kernel<SR, Epi, 256>;
        static const int occ = [&] {
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 32 * 32, L::BYTES);
            return std::max(1, b);
        }();
        static const int focc = [&] {
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fixup, 256, 0);
            return std::max(1, b);
        }();
        g1::NnzArgs<SR> a = nargs_;
        a.x = x;
        const uint32_t sms = (uint32_t)detail::sm_count();
        // launched even without tiles: its blocks' epilogue partials count
        const uint32_t grid = std::max<uint32_t>(
            1, std::min<uint32_t>((a.plan.n_tiles + 31) / 32, sms * occ));
        const uint32_t work = std::max(a.plan.n_fix, a.plan.n_empty);
        const uint32_t fgrid = std::max<uint32_t>(1, std::min<uint32_t>((work + 255) / 256, sms * focc));
        kernel<<<grid, 32 * 32, L::BYTES, stream_>>>(a, epi);
        fixup<<<fgrid, 256, 0, stream_>>>(a, epi);
        detail::check_cuda(cudaGetLastError(), "nnz SpMV launch");
        g1_count_user_launches(2);
    }

    void fill_x(int which, info_t value) {
        blas_detail::fill_kernel<<<blas_detail::grid_for(n_), 256, 0, stream_>>>(
            x_[which].data(), (uint32_t)n_, value);
        g1_count_user_launches(1);
    }

    vertex_t n_;
    int side_ = 1;
    cudaStream_t stream_{};
    DenseVec<arch_t::cuda, info_t> x_[2];
    g1::MergeArgs<SR> args_{};
    bool nnz_ = false;
    g1::NnzArgs<SR> nargs_{};
    detail::Counters counters_;
};

template <typename functor_t, typename comp_t, typename frontier_t, typename enable_t = void>
class BlasGcEngine;

// Sparse frontier (GraphOne: engine/blas_gc.h:171-247).
template <typename functor_t, typename comp_t, typename frontier_t>
class BlasGcEngine<functor_t, comp_t, frontier_t,
                   std::enable_if_t<frontier_t::kind == FrontierKind::SPARSE_BASED>>
    : public BlasGcEngineBase<functor_t, comp_t, frontier_t> {
    using B = BlasGcEngineBase<functor_t, comp_t, frontier_t>;

public:
    BlasGcEngine(comp_t& comp, frontier_t& frontier) : B(comp, frontier) {
        this->fill_x(0, functor_t::default_info());
        init_sparse(comp);
    }

    void Forward() override {
        using V = typename B::vertex_t;
        using D = typename B::dstatus_t;
        frontier_t& f = this->frontier_;
        const uint32_t n_in = f.input_size();
        typename B::info_t* x = this->x_[0].data();
        const D ds = this->d_status_;
        if (n_in)
            blas_detail::construct_list_kernel<functor_t, D, V>
                <<<blas_detail::grid_for(n_in), 256, 0, this->stream_>>>(f.input().data(), n_in, ds, x);
        f.reserve_output(this->n_);
        this->counters_.clear(this->stream_);
        if (!sparse_step(f, n_in, x, ds))
            this->spmv(x, blas_detail::SparseEpi<functor_t, D, V>{ds, f.output().data(),
                                                                  this->counters_.dev});
        if (n_in)
            blas_detail::set_list_kernel<<<blas_detail::grid_for(n_in), 256, 0, this->stream_>>>(
                f.input().data(), n_in, functor_t::default_info(), x);
        g1_count_user_launches(n_in ? 2 : 0);
        this->counters_.read(this->stream_);
        f.reset_output(this->counters_.count());
    }

private:
    // Sparse steps.  GraphOne pulls every row each iteration
    // (engine/blas_gc.h:199-245).  When a row without an in-neighbour on the
    // frontier folds to default_result (checked once on the device over the
    // graph's edge values, sparse_check_kernel), only the rows the frontier
    // reaches can be applied, so a step with a small frontier lists the
    // frontier's out-neighbours and folds just those rows, each over all its
    // in-edges as the full pull does: the same rows applied with the same
    // values.  Used on graphs of 2^20 edges or more (a full pull of a smaller
    // one costs a few microseconds) with both orientations, while the listed
    // rows hold fewer than m / 16 in-edges.
    static constexpr uint32_t kSparseMinEdges = 1u << 20;
    static constexpr uint32_t kSparseDiv = 16;

    void init_sparse(comp_t& comp) {
        const uint32_t m = this->args_.plan.nnz;
        if (this->side_ != 1 || m < kSparseMinEdges) return;
        const uint32_t* orp = nullptr;
        const uint32_t* oci = nullptr;
        const void* oval = nullptr;
        if (g1_graph_arrays(comp.graph.handle(), 0, &orp, &oci, &oval) != G1_OK || !orp) return;
        uint32_t* bad = this->counters_.dev + 15;
        detail::check_cuda(cudaMemsetAsync(bad, 0, 4, this->stream_), "sparse check");
        blas_detail::sparse_check_kernel<functor_t, typename B::SR>
            <<<blas_detail::grid_for(m), 256, 0, this->stream_>>>(this->args_.val, m, bad);
        g1_count_user_launches(1);
        this->counters_.read_set(this->stream_, 1);
        if (this->counters_.host[7] != 0u) return;
        out_rp_ = orp;
        out_col_ = oci;
        bits_ = DenseVec<arch_t::cuda, uint32_t>((this->n_ + 31) / 32 + 1);
        cand_ = DenseVec<arch_t::cuda, uint32_t>(std::max<typename B::vertex_t>(this->n_, 1));
        blas_detail::fill_kernel<<<blas_detail::grid_for((this->n_ + 31) / 32 + 1), 256, 0, this->stream_>>>(
            bits_.data(), (uint32_t)((this->n_ + 31) / 32 + 1), 0u);
        g1_count_user_launches(1);
    }

    template <class D>
    bool sparse_step(frontier_t& f, uint32_t n_in, const typename B::info_t* x, const D& ds) {
        using V = typename B::vertex_t;
        if (!out_rp_ || n_in == 0 || n_in > this->n_ / 32) return false;
        const uint32_t m = this->args_.plan.nnz;
        uint32_t* cnt = this->counters_.dev + 8;
        detail::check_cuda(cudaMemsetAsync(cnt, 0, 16, this->stream_), "sparse counters");
        blas_detail::sparse_expand_kernel<V><<<blas_detail::grid_for(n_in * 32), 256, 0, this->stream_>>>(
            f.input().data(), n_in, out_rp_, out_col_, this->args_.plan.row_ptr, bits_.data(), cand_.data(), cnt);
        g1_count_user_launches(1);
        this->counters_.read_set(this->stream_, 1);
        const uint32_t nc = this->counters_.host[0];
        const unsigned long long insum =
            (unsigned long long)this->counters_.host[2] | ((unsigned long long)this->counters_.host[3] << 32);
        if (insum >= m / kSparseDiv) {
            blas_detail::sparse_clear_kernel<<<blas_detail::grid_for(nc), 256, 0, this->stream_>>>(
                cand_.data(), nc, bits_.data());
            g1_count_user_launches(1);
            return false;
        }
        if (nc) {
            blas_detail::sparse_rows_kernel<functor_t, typename B::SR, D, V>
                <<<blas_detail::grid_for(nc * 32), 256, 0, this->stream_>>>(
                    cand_.data(), nc, this->args_.plan.row_ptr, this->args_.col, this->args_.val, x, ds,
                    f.output().data(), this->counters_.dev, bits_.data());
            g1_count_user_launches(1);
        }
        return true;
    }

    const uint32_t* out_rp_ = nullptr;
    const uint32_t* out_col_ = nullptr;
    DenseVec<arch_t::cuda, uint32_t> bits_;
    DenseVec<arch_t::cuda, uint32_t> cand_;
};

// Dense frontier: counts only (GraphOne: engine/blas_gc.h:250-351).
template <typename functor_t, typename comp_t, typename frontier_t>
class BlasGcEngine<functor_t, comp_t, frontier_t,
                   std::enable_if_t<frontier_t::kind == FrontierKind::DENSE_BASED>>
    : public BlasGcEngineBase<functor_t, comp_t, frontier_t> {
    using B = BlasGcEngineBase<functor_t, comp_t, frontier_t>;

public:
    BlasGcEngine(comp_t& comp, frontier_t& frontier) : B(comp, frontier) {}

    void Forward() override {
        using V = typename B::vertex_t;
        using D = typename B::dstatus_t;
        frontier_t& f = this->frontier_;
        const D ds = this->d_status_;
        auto& init = f.init_buf();
        if (!init.empty()) {
            this->fill_x(cur_, functor_t::default_info());
            blas_detail::construct_list_kernel<functor_t, D, V>
                <<<blas_detail::grid_for(init.size()), 256, 0, this->stream_>>>(
                    init.data(), init.size(), ds, this->x_[cur_].data());
            g1_count_user_launches(1);
            detail::check_cuda(cudaStreamSynchronize(this->stream_), "construct");
            init = std::remove_reference_t<decltype(init)>();
        }
        this->counters_.clear(this->stream_);
        this->spmv(this->x_[cur_].data(),
                   blas_detail::DenseEpi<functor_t, D, V>{ds, this->x_[cur_ ^ 1].data(),
                                                          this->counters_.dev, 0});
        cur_ ^= 1;
        this->counters_.read(this->stream_);
        f.output_size() = this->counters_.count();
    }

private:
    int cur_ = 0;
};

// All vertices active (GraphOne: engine/blas_gc.h:353-434).
template <typename functor_t, typename comp_t, typename frontier_t>
class BlasGcEngine<functor_t, comp_t, frontier_t,
                   std::enable_if_t<frontier_t::kind == FrontierKind::ALL_ACTIVE>>
    : public BlasGcEngineBase<functor_t, comp_t, frontier_t> {
    using B = BlasGcEngineBase<functor_t, comp_t, frontier_t>;

public:
    BlasGcEngine(comp_t& comp, frontier_t& frontier) : B(comp, frontier) {}

    void Forward() override {
        using V = typename B::vertex_t;
        using D = typename B::dstatus_t;
        const D ds = this->d_status_;
        if (first_) {
            first_ = false;
            blas_detail::construct_all_kernel<functor_t, D, V>
                <<<blas_detail::grid_for(this->n_), 256, 0, this->stream_>>>(
                    (uint32_t)this->n_, ds, this->x_[cur_].data());
            g1_count_user_launches(1);
        }
        this->spmv(this->x_[cur_].data(),
                   blas_detail::AllActiveEpi<functor_t, D, V>{ds, this->x_[cur_ ^ 1].data()});
        cur_ ^= 1;
        // the next host hook may read device state (d_status pointers)
        detail::check_cuda(cudaStreamSynchronize(this->stream_), "engine step");
    }

private:
    bool first_ = true;
    int cur_ = 0;
};

}  // namespace engine

constexpr graph_view_t BlasViews = graph_view_t::csr | graph_view_t::transpose;

// Base of user semiring functors (GraphOne: engine/blas_gc.h:440-474).
template <typename vertex_t, typename weight_t, typename dstatus_t, typename info_t,
          typename gather_t>
struct BlasFunctor {
    template <typename functor_t, typename comp_t, typename frontier_t>
    using engine_type = engine::BlasGcEngine<functor_t, comp_t, frontier_t>;
    using info_type = info_t;
    using gather_type = gather_t;

    __host__ __device__ __forceinline__ static info_t default_info() { return info_t{0}; }
    __host__ __device__ __forceinline__ static gather_t default_result() { return gather_t{0}; }
    __device__ __forceinline__ static info_t construct_each(const vertex_t&, const dstatus_t&) {
        return info_t{};
    }
    __device__ __forceinline__ static gather_t gather_combine(const weight_t&, const info_t&) {
        return gather_t{};
    }
    __device__ __forceinline__ static gather_t gather_reduce(const gather_t& lhs, const gather_t&) {
        return lhs;
    }
    /// true activates the vertex
    __device__ __forceinline__ static bool apply_each(const vertex_t&, const gather_t&, dstatus_t&) {
        return false;
    }
};

}  // namespace graph_one
