#pragma once
// The advance/filter engine of the GraphOne API (reference:
// engine/advance_gc.h:24-303), with the user functor inlined.
//
// GraphOne sizes an invalid-padded output by a degree-sum reduction, runs a
// block-scan load-balanced advance (functor::advance decides per edge
// whether dst is emitted), synchronises, then filters duplicates in a second
// pass (functor::filter, when the functor has one).  Here the advance
// appends emitted vertices compactly (warp-aggregated atomics) while
// accumulating their out-degrees, so the output's worst-case size for the
// next iteration is known without a separate reduction (with a filter step
// the filter does that accumulation instead).  Adjacency lists of 32 or more
// edges are walked by the whole warp (coalesced col/val reads); shorter ones
// by TPV lanes, TPV the power of two at or above the frontier's mean degree,
// so that a small frontier of low-degree vertices still gets about one
// thread per edge.  The filter step compacts the same way.  One read-back
// per step gives the host the new frontier size.

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

#include "graphone_b200.h"
#include "g1/common.cuh"
#include "GraphOne/engine/base.h"
#include "GraphOne/frontier/frontier.h"
#include "GraphOne/graph/graph.h"
#include "GraphOne/utils/limits.hpp"

namespace graph_one {
namespace engine {
namespace adv_detail {

// append with a capacity check (an overflow is recorded, never written);
// the appended vertices' out-degrees add to `deg_acc`, flushed once per warp
// at the end of the kernel (deg_flush) instead of one atomic per append
__device__ __forceinline__ void append_capped(uint32_t* out, uint32_t* ctr, uint32_t cap,
                                              uint32_t v, uint32_t deg, unsigned long long& deg_acc) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const uint32_t lane = g1::lane_id();
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(&ctr[0], (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
    if (slot < cap)
        out[slot] = v;
    else
        atomicExch(&ctr[1], 1u);
    deg_acc += deg;
}

// warp-wide sum of the lanes' degree accumulators into ctr[2..3] (u64)
__device__ __forceinline__ void deg_flush(uint32_t* ctr, unsigned long long deg_acc) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) deg_acc += __shfl_xor_sync(0xffffffffu, deg_acc, off);
    if (g1::lane_id() == 0 && deg_acc) atomicAdd(reinterpret_cast<unsigned long long*>(ctr + 2), deg_acc);
}

// DEG: accumulate the emitted vertices' out-degrees (not needed when a
// filter step follows: it accumulates those of its own output).
template <class F, bool DEG, class V, class E, class W, class D>
__device__ __forceinline__ void visit(V src, V dst, E e, W w, D& ds, const E* rp, uint32_t* out,
                                      uint32_t* ctr, uint32_t cap, unsigned long long& deg_acc) {
    if (F::advance(src, dst, e, w, ds))
        append_capped(out, ctr, cap, dst, DEG ? rp[dst + 1] - rp[dst] : 0u, deg_acc);
}

// TPV lanes per frontier vertex (1..32); vertices of 32 or more edges are
// walked by the whole warp.
// zero_next: the other counter set, zeroed for the next step (the host has
// read it back already).
template <class F, class V, class E, class W, class D, vstart_t VS, int TPV, bool DEG>
__global__ void __launch_bounds__(256)
advance_kernel(const E* rp, const V* col, const W* val, D ds, const V* in, uint32_t n_in,
               uint32_t* out, uint32_t* ctr, uint32_t cap, uint32_t* zero_next) {
    constexpr uint32_t VPW = 32 / TPV;  // vertices per warp and round
    if (blockIdx.x == 0 && threadIdx.x < 8) zero_next[threadIdx.x] = 0u;
    const uint32_t lane = g1::lane_id();
    const uint32_t sub = lane % TPV, grp = lane / TPV;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t rounds = (n_in + warps * VPW - 1) / (warps * VPW);
    D local = ds;  // functors may mutate their copy (reference: passed by value)
    unsigned long long deg_acc = 0;
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t i = (r * warps + wid) * VPW + grp;
        V u = utils::invalid_vertex<VS, V>();
        E b = 0, e = 0;
        if (i < n_in) {
            u = in[i];
            if (utils::is_vertex_valid<VS>(u)) {
                b = rp[u];
                e = rp[u + 1];
            }
        }
        unsigned big = __ballot_sync(0xffffffffu, sub == 0 && e - b >= 32);
        while (big) {
            const int src = __ffs(big) - 1;
            big &= big - 1;
            const V uu = __shfl_sync(0xffffffffu, u, src);
            const E bb = __shfl_sync(0xffffffffu, b, src);
            const E ee = __shfl_sync(0xffffffffu, e, src);
            for (E k = bb + lane; k < ee; k += 32)
                visit<F, DEG>(uu, col[k], k, val[k], local, rp, out, ctr, cap, deg_acc);
        }
        if (e - b < 32)
            for (E k = b + sub; k < e; k += TPV) visit<F, DEG>(u, col[k], k, val[k], local, rp, out, ctr, cap, deg_acc);
    }
    deg_flush(ctr, deg_acc);
}

// Lanes per vertex for a frontier of mean out-degree deg/n: the power of two
// at or above it (1..32).
inline int lanes_per_vertex(unsigned long long deg, uint32_t n) {
    const unsigned long long mean = n ? (deg + n - 1) / n : 1;
    int t = 1;
    while (t < 32 && (unsigned long long)t < mean) t <<= 1;
    return t;
}

// The filter reads the advance's output size from device memory (*n_dev),
// so advance and filter run back to back without a host round trip.
template <class F, class V, class E, class D, vstart_t VS>
__global__ void filter_kernel(const E* rp, D ds, const V* in, const uint32_t* n_dev, uint32_t* out,
                              uint32_t* ctr, uint32_t cap) {
    const uint32_t n = min(*n_dev, cap);
    unsigned long long deg_acc = 0;
    // warp-uniform rounds so that every lane reaches the final flush
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint32_t i = base + g1::lane_id();
        if (i >= n) continue;
        const V v = in[i];
        if (utils::is_vertex_valid<VS>(v) && !F::filter(v, ds))
            append_capped(out, ctr, cap, v, rp[v + 1] - rp[v], deg_acc);
    }
    deg_flush(ctr, deg_acc);
}

template <class V, class E, vstart_t VS>
__global__ void degree_sum_kernel(const E* rp, const V* in, uint32_t n, unsigned long long* sum) {
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V v = in[i];
        if (utils::is_vertex_valid<VS>(v)) s += rp[v + 1] - rp[v];
    }
    if (s) atomicAdd(sum, s);
}

inline unsigned grid_for(uint64_t n) {
    const uint64_t want = (n + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)detail::sm_count() * 8));
}

}  // namespace adv_detail

template <typename functor_t, typename comp_t, typename frontier_t>
class AdvanceGC : public GcEngine<comp_t, frontier_t> {
public:
    using base_t = GcEngine<comp_t, frontier_t>;
    using graph_t = typename comp_t::graph_type;
    using dstatus_t = typename comp_t::dstatus_type;
    using vertex_t = typename graph_t::vertex_type;
    using edge_t = typename graph_t::edge_type;
    using weight_t = typename graph_t::weight_type;
    constexpr static vstart_t VS = graph_t::vstart_value;
    static_assert(frontier_t::kind == SPARSE_BASED, "the advance engine needs a sparse frontier");
    static_assert(graph_t::has_normal, "the advance engine walks out-edges (normal view)");

    struct HasFilter {
        template <typename T>
        static std::true_type test(decltype(&T::filter));
        template <typename T>
        static std::false_type test(...);
        constexpr static bool value = decltype(test<functor_t>(0))::value;
    };

    AdvanceGC(comp_t& comp, frontier_t& frontier) : base_t(comp, frontier) {
        detail::check_cuda(cudaStreamCreate(&stream_), "stream");
        const uint32_t *rp = nullptr, *ci = nullptr;
        const void* val = nullptr;
        detail::check_g1(g1_graph_arrays(comp.graph.handle(), 0, &rp, &ci, &val), "graph arrays");
        rp_ = reinterpret_cast<const edge_t*>(rp);
        col_ = reinterpret_cast<const vertex_t*>(ci);
        val_ = static_cast<const weight_t*>(val);
        // An advance over a duplicate-free frontier emits at most one vertex
        // per edge: both lists get that room once, up front.
        const uint32_t room = std::max<uint32_t>(comp.graph.num_edges(), comp.graph.num_vertices()) + 1;
        frontier.reserve_output(room);
        frontier.swap_inout();
        frontier.reserve_output(room);
        frontier.swap_inout();
        check_cuda_alloc_ = true;
    }

    ~AdvanceGC() override {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }

    void Forward() override {
        frontier_t& f = this->frontier_;
        const dstatus_t ds = this->d_status_;
        const uint32_t n_in = f.input_size();
        if (!degree_known_) {  // first step: out-degree sum of the seeds
            counters_.clear(stream_);
            adv_detail::degree_sum_kernel<vertex_t, edge_t, VS>
                <<<adv_detail::grid_for(n_in), 256, 0, stream_>>>(rp_, f.input().data(), n_in,
                                                                 counters_.degree_sum_dev());
            g1_count_user_launches(1);
            counters_.read(stream_);
            next_degree_ = counters_.degree_sum();
            degree_known_ = true;
            // both counter sets start at zero; from here on each step's
            // advance zeroes the set of the step after it
            detail::check_cuda(cudaMemsetAsync(counters_.dev, 0, 64, stream_), "clear counters");
            set_ = 0;
        }
        // the advance emits at most one vertex per out-edge of the input
        const uint32_t cap = (uint32_t)std::min<unsigned long long>(next_degree_ + 1, 0xFFFFFFF0ull);
        f.reserve_output(cap);
        uint32_t* ctr = counters_.dev + 8 * set_;
        uint32_t* ctr_next = counters_.dev + 8 * (set_ ^ 1);
        constexpr bool kDeg = !HasFilter::value;
        const int tpv = adv_detail::lanes_per_vertex(next_degree_, n_in);
        const unsigned grid = adv_detail::grid_for((uint64_t)n_in * tpv);
#define G1_ADVANCE(T)                                                                                  \
    adv_detail::advance_kernel<functor_t, vertex_t, edge_t, weight_t, dstatus_t, VS, T, kDeg>          \
        <<<grid, 256, 0, stream_>>>(rp_, col_, val_, ds, f.input().data(), n_in, f.output().data(), \
                                    ctr, cap, ctr_next)
        switch (tpv) {
            case 1: G1_ADVANCE(1); break;
            case 2: G1_ADVANCE(2); break;
            case 4: G1_ADVANCE(4); break;
            case 8: G1_ADVANCE(8); break;
            case 16: G1_ADVANCE(16); break;
            default: G1_ADVANCE(32); break;
        }
#undef G1_ADVANCE
        g1_count_user_launches(1);
        if constexpr (HasFilter::value) {
            // filter the advance output (size on the device) into the input
            // list, which the advance no longer needs; counters at +4
            const uint32_t fcap = (uint32_t)std::min<uint64_t>(f.input().size(), 0xFFFFFFF0ull);
            adv_detail::filter_kernel<functor_t, vertex_t, edge_t, dstatus_t, VS>
                <<<adv_detail::grid_for(std::min<uint64_t>(cap, (uint64_t)detail::sm_count() * 2048)),
                   256, 0, stream_>>>(rp_, ds, f.output().data(), ctr, f.input().data(), ctr + 4, fcap);
            g1_count_user_launches(1);
            counters_.read_set(stream_, set_);
            if (counters_.overflow() || counters_.host[5]) LOG_ERROR("advance: frontier overflow");
            // GraphOne's Filter swaps in/out and fills the new output; the
            // Run loop's AfterEngine swaps again (engine/advance_gc.h:224-240)
            f.reset_output(counters_.count());
            f.swap_inout();
            f.reset_output(counters_.host[4]);
            next_degree_ = (unsigned long long)counters_.host[6] |
                           ((unsigned long long)counters_.host[7] << 32);
        } else {
            counters_.read_set(stream_, set_);
            if (counters_.overflow()) LOG_ERROR("advance: output frontier overflow");
            f.reset_output(counters_.count());
            next_degree_ = counters_.degree_sum();
        }
        set_ ^= 1;
    }

private:
    cudaStream_t stream_{};
    const edge_t* rp_ = nullptr;
    const vertex_t* col_ = nullptr;
    const weight_t* val_ = nullptr;
    detail::Counters counters_;
    bool degree_known_ = false;
    int set_ = 0;  // counter set of this step (dev + 8 * set_)
    bool check_cuda_alloc_ = false;
    unsigned long long next_degree_ = 0;
};

}  // namespace engine

constexpr graph_view_t AdvanceViews = graph_view_t::csr | graph_view_t::normal;

// Base of user advance functors (GraphOne: engine/advance_gc.h:289-303); a
// functor may add `static bool filter(const vertex_t&, const dstatus_t&)`.
template <typename vertex_t, typename edge_t, typename weight_t, typename dstatus_t,
          typename vprop_t = empty_t>
struct AdvanceFunctor {
    template <typename functor_t, typename comp_t, typename frontier_t>
    using engine_type = engine::AdvanceGC<functor_t, comp_t, frontier_t>;

    __device__ __forceinline__ static bool advance(const vertex_t&, const vertex_t&, const edge_t&,
                                                   const weight_t&, dstatus_t&) {
        return false;
    }
};

}  // namespace graph_one
