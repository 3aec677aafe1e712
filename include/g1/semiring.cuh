#pragma once
// Prebuilt semirings (the functors of GraphOne's apps, restated for the
// library's own instantiations) and the adapter that turns a GraphOne user
// functor into a semiring for the SpMV schedules.

#include <cfloat>
#include <type_traits>
#include "g1/common.cuh"

namespace g1 {

// min-plus over u32 with the sssp_blas functor's combine
// (apps/sssp_blas.cu:58-71 with dist_t = uint32_t): MAX is "unreached" and
// absorbs; sums wrap like the u32 arithmetic of the functor.
struct MinPlusU32 {
    using value_t = uint32_t;
    using x_t = uint32_t;
    using w_t = uint32_t;
    __host__ __device__ static __forceinline__ uint32_t identity() { return kU32Max; }
    __device__ static __forceinline__ uint32_t combine(const uint32_t& w, const uint32_t& x) {
        return x == kU32Max ? x : w + x;
    }
    __device__ static __forceinline__ uint32_t reduce(const uint32_t& a, const uint32_t& b) {
        return min(a, b);
    }
};

// Same over float distances, as the unchanged apps compute them
// (dist_t = float, kMaxDist = FLT_MAX; reduce = std::min(lhs, rhs)).
struct MinPlusF32 {
    using value_t = float;
    using x_t = float;
    using w_t = float;
    __host__ __device__ static __forceinline__ float identity() { return FLT_MAX; }
    __device__ static __forceinline__ float combine(const float& w, const float& x) {
        return x == FLT_MAX ? x : w + x;
    }
    __device__ static __forceinline__ float reduce(const float& a, const float& b) {
        return (b < a) ? b : a;
    }
};

// BFS: min-plus with every edge weight taken as 1 (the edge values are not
// read).
struct BfsU32 {
    static constexpr bool kReadsWeight = false;
    using value_t = uint32_t;
    using x_t = uint32_t;
    using w_t = uint32_t;
    __host__ __device__ static __forceinline__ uint32_t identity() { return kU32Max; }
    __device__ static __forceinline__ uint32_t combine(const uint32_t&, const uint32_t& x) {
        return x == kU32Max ? x : x + 1u;
    }
    __device__ static __forceinline__ uint32_t reduce(const uint32_t& a, const uint32_t& b) {
        return min(a, b);
    }
};

// plus-times over fp32 with fp32 accumulation (apps/pagerank_blas.cu:103-113).
struct PlusTimesF32 {
    using value_t = float;
    using x_t = float;
    using w_t = float;
    __host__ __device__ static __forceinline__ float identity() { return 0.0f; }
    __device__ static __forceinline__ float combine(const float& w, const float& x) {
        return x * w;
    }
    __device__ static __forceinline__ float reduce(const float& a, const float& b) {
        return a + b;
    }
};

// plus over fp32 with every edge weight taken as 1: y[v] = sum of x over
// v's in-neighbours (the transition of personalized PageRank, whose weights
// 1/out-degree are folded into x).  The edge values, of any 4-byte type, are
// not read.
struct PlusPatternF32 {
    static constexpr bool kReadsWeight = false;
    using value_t = float;
    using x_t = float;
    using w_t = uint32_t;
    __host__ __device__ static __forceinline__ float identity() { return 0.0f; }
    __device__ static __forceinline__ float combine(const uint32_t&, const float& x) { return x; }
    __device__ static __forceinline__ float reduce(const float& a, const float& b) {
        return a + b;
    }
};

// Whether a semiring's combine uses the edge value (kReadsWeight = false
// lets the schedules skip loading the values; semirings without the member,
// GraphOne's functors among them, read them).
template <class SR, class = void>
struct reads_weight : std::true_type {};
template <class SR>
struct reads_weight<SR, std::void_t<decltype(SR::kReadsWeight)>>
    : std::integral_constant<bool, SR::kReadsWeight> {};

// GraphOne user functor -> semiring, exactly as the reference's SpmvFunctor
// adapter (engine/blas_gc.h:113-128): initialize = default_result,
// combine = gather_combine, reduce = gather_reduce.
template <class F, class W>
struct FunctorSemiring {
    using value_t = typename F::gather_type;
    using x_t = typename F::info_type;
    using w_t = W;
    __device__ static __forceinline__ value_t identity() { return F::default_result(); }
    __device__ static __forceinline__ value_t combine(const w_t& w, const x_t& x) {
        return F::gather_combine(w, x);
    }
    __device__ static __forceinline__ value_t reduce(const value_t& a, const value_t& b) {
        return F::gather_reduce(a, b);
    }
};

}  // namespace g1
