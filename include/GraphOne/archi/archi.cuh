#pragma once
// Parallel primitives of the GraphOne API (reference: archi/thrust/
// functions.h:17-104 over Thrust, archi/only/cuda.cuh:37-99, archi/mem/
// def.hpp:9-43, archi/thrust/def.hpp:9-27).  The element-wise ones (fill,
// transform, for_each, transform_reduce) are this library's own grid-stride
// kernels on the default stream; iterators may be raw pointers or any
// random-access iterator usable in device code (thrust::counting_iterator
// included), and operators may be __device__ lambdas with or without a
// declared return type (the accumulator of transform_reduce is the type of
// `init`).  The multi-pass ones (copy_if, inclusive_scan, sort_by_key) and
// scatter, scatter_if and the vectorised lower_bound run on Thrust with the
// arch's execution policy, as in the reference.  Memory: memalloc / memfree
// / memset / memcpy<arch...> (device memory from libgraphone_b200).
// Launches: LaunchKernel / LaunchSync (GraphOne/archi/kernel/kernel.h);
// checks: checkCudaErrors / checkArchErrors (GraphOne/archi/check/check.h).

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/host_vector.h>
#include <thrust/scan.h>
#include <thrust/scatter.h>
#include <thrust/sort.h>

#include "graphone_b200.h"
#include "GraphOne/archi/check/check.h"
#include "GraphOne/archi/kernel/kernel.h"
#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"

namespace graph_one::archi {

namespace detail {

constexpr int kBlock = 256;

inline unsigned grid_for(size_t n) {
    static int sms = [] {
        int dev = 0, s = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
        return s;
    }();
    const size_t want = (n + kBlock - 1) / kBlock;
    return (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8));
}

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[ERROR] %s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

inline void check_launch(const char* what) { check(cudaGetLastError(), what); }

template <typename It, typename T>
__global__ void fill_kernel(It first, size_t n, T value) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        first[i] = value;
}

template <typename It, typename Out, typename Op>
__global__ void transform_kernel(It first, size_t n, Out out, Op op) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = op(first[i]);
}

template <typename It1, typename It2, typename Out, typename Op>
__global__ void transform2_kernel(It1 a, size_t n, It2 b, Out out, Op op) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = op(a[i], b[i]);
}

template <typename It, typename Op>
__global__ void for_each_kernel(It first, size_t n, Op op) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        op(first[i]);
}

// Per-block fold of op(first[i]) with bop; partial[b] holds the block's
// value and valid[b] whether the block saw any element.
template <typename It, typename Op, typename T, typename Bop>
__global__ void reduce_kernel(It first, size_t n, Op op, Bop bop, T* partial, int* valid) {
    __shared__ T s_val[kBlock];
    __shared__ int s_ok[kBlock];
    T acc{};
    int ok = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const T v = static_cast<T>(op(first[i]));
        acc = ok ? bop(acc, v) : v;
        ok = 1;
    }
    s_val[threadIdx.x] = acc;
    s_ok[threadIdx.x] = ok;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w && s_ok[threadIdx.x + w]) {
            s_val[threadIdx.x] = s_ok[threadIdx.x] ? bop(s_val[threadIdx.x], s_val[threadIdx.x + w])
                                                   : s_val[threadIdx.x + w];
            s_ok[threadIdx.x] = 1;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = s_val[0];
        valid[blockIdx.x] = s_ok[0];
    }
}

template <typename T>
struct Identity {
    __host__ __device__ T operator()(const T& v) const { return v; }
};

}  // namespace detail

template <arch_t arch, typename It, typename T>
void fill(It first, It last, const T& value) {
    const size_t n = (size_t)(last - first);
    if (n == 0) return;
    if constexpr (arch == arch_t::cpu) {
        std::fill(first, last, value);
    } else {
        using V = typename std::iterator_traits<It>::value_type;
        detail::fill_kernel<<<detail::grid_for(n), detail::kBlock>>>(first, n, V(value));
        detail::check_launch("archi::fill");
        g1_count_user_launches(1);
    }
}

template <arch_t arch, typename It, typename Out, typename Op>
Out transform(It first, It last, Out result, Op op) {
    const size_t n = (size_t)(last - first);
    if (n == 0) return result;
    if constexpr (arch == arch_t::cpu) {
        for (size_t i = 0; i < n; ++i) result[i] = op(first[i]);
    } else {
        detail::transform_kernel<<<detail::grid_for(n), detail::kBlock>>>(first, n, result, op);
        detail::check_launch("archi::transform");
        g1_count_user_launches(1);
    }
    return result + n;
}

template <arch_t arch, typename It1, typename It2, typename Out, typename Op>
Out transform(It1 first1, It1 last1, It2 first2, Out result, Op op) {
    const size_t n = (size_t)(last1 - first1);
    if (n == 0) return result;
    if constexpr (arch == arch_t::cpu) {
        for (size_t i = 0; i < n; ++i) result[i] = op(first1[i], first2[i]);
    } else {
        detail::transform2_kernel<<<detail::grid_for(n), detail::kBlock>>>(first1, n, first2,
                                                                           result, op);
        detail::check_launch("archi::transform");
        g1_count_user_launches(1);
    }
    return result + n;
}

template <arch_t arch, typename It, typename Op>
It for_each(It first, It last, Op op) {
    const size_t n = (size_t)(last - first);
    if (n == 0) return last;
    if constexpr (arch == arch_t::cpu) {
        for (size_t i = 0; i < n; ++i) op(first[i]);
    } else {
        detail::for_each_kernel<<<detail::grid_for(n), detail::kBlock>>>(first, n, op);
        detail::check_launch("archi::for_each");
        g1_count_user_launches(1);
    }
    return last;
}

template <arch_t arch, typename It, typename Op, typename T, typename Bop>
T transform_reduce(It first, It last, Op op, T init, Bop bop) {
    const size_t n = (size_t)(last - first);
    if (n == 0) return init;
    if constexpr (arch == arch_t::cpu) {
        T acc = init;
        for (size_t i = 0; i < n; ++i) acc = bop(acc, static_cast<T>(op(first[i])));
        return acc;
    } else {
        const unsigned grid = detail::grid_for(n);
        T* partial = nullptr;
        int* valid = nullptr;
        if (g1_mem_alloc(reinterpret_cast<void**>(&partial), sizeof(T) * grid) != G1_OK ||
            g1_mem_alloc(reinterpret_cast<void**>(&valid), sizeof(int) * grid) != G1_OK) {
            std::fprintf(stderr, "[ERROR] archi::transform_reduce: %s\n", g1_last_error());
            std::exit(1);
        }
        detail::reduce_kernel<<<grid, detail::kBlock>>>(first, n, op, bop, partial, valid);
        detail::check_launch("archi::transform_reduce");
        g1_count_user_launches(1);
        std::vector<T> hp(grid);
        std::vector<int> hv(grid);
        g1_mem_copy(hp.data(), partial, sizeof(T) * grid, 1, nullptr);
        g1_mem_copy(hv.data(), valid, sizeof(int) * grid, 1, nullptr);
        g1_mem_free(partial);
        g1_mem_free(valid);
        T acc = init;
        for (unsigned b = 0; b < grid; ++b)
            if (hv[b]) acc = bop(acc, hp[b]);
        return acc;
    }
}

// ------------------------------------------------ Thrust-backed primitives

template <arch_t arch>
struct ExecPolicy;
template <>
struct ExecPolicy<arch_t::cpu> {
    static constexpr decltype(thrust::host) value{};
};
template <>
struct ExecPolicy<arch_t::cuda> {
    static constexpr decltype(thrust::device) value{};
};
template <arch_t arch>
static const auto exec_policy = ExecPolicy<arch>::value;

template <arch_t arch>
struct ThrustVec;
template <>
struct ThrustVec<arch_t::cpu> {
    template <typename value_t>
    using type = thrust::host_vector<value_t>;
};
template <>
struct ThrustVec<arch_t::cuda> {
    template <typename value_t>
    using type = thrust::device_vector<value_t>;
};
template <arch_t arch, typename value_t>
using thrust_vec = typename ThrustVec<arch>::template type<value_t>;

namespace detail {
template <arch_t arch>
inline void check_thrust(const char* what) {
    if constexpr (arch == arch_t::cuda) check_launch(what);
}
}  // namespace detail

// Copies first[i] to the output where pred(stencil[i]); returns the end of the output.
template <arch_t arch, typename It1, typename It2, typename Out, typename Pred>
Out copy_if(It1 first, It1 last, It2 stencil, Out result, Pred pred) {
    Out end = thrust::copy_if(exec_policy<arch>, first, last, stencil, result, pred);
    detail::check_thrust<arch>("archi::copy_if");
    return end;
}

template <arch_t arch, typename It, typename Out, typename Op>
Out inclusive_scan(It first, It last, Out result, Op op) {
    Out end = thrust::inclusive_scan(exec_policy<arch>, first, last, result, op);
    detail::check_thrust<arch>("archi::inclusive_scan");
    return end;
}

// For each value, the first position in the sorted [first, last) not less than it.
template <arch_t arch, typename It, typename ValIt, typename Out>
Out lower_bound(It first, It last, ValIt values_first, ValIt values_last, Out output) {
    Out end = thrust::lower_bound(exec_policy<arch>, first, last, values_first, values_last, output);
    detail::check_thrust<arch>("archi::lower_bound");
    return end;
}

// result[map[i]] = first[i]
template <arch_t arch, typename It, typename MapIt, typename Out>
void scatter(It first, It last, MapIt map, Out result) {
    thrust::scatter(exec_policy<arch>, first, last, map, result);
    detail::check_thrust<arch>("archi::scatter");
}

// result[map[i]] = first[i] where stencil[i]
template <arch_t arch, typename It, typename MapIt, typename StIt, typename Out>
void scatter_if(It first, It last, MapIt map, StIt stencil, Out result) {
    thrust::scatter_if(exec_policy<arch>, first, last, map, stencil, result);
    detail::check_thrust<arch>("archi::scatter_if");
}

template <arch_t arch, typename KeyIt, typename ValIt>
void sort_by_key(KeyIt keys_first, KeyIt keys_last, ValIt values_first) {
    thrust::sort_by_key(exec_policy<arch>, keys_first, keys_last, values_first);
    detail::check_thrust<arch>("archi::sort_by_key");
}

// ---------------------------------------------------------------- memory

template <arch_t arch>
struct memalloc_t {
    template <typename T>
    static T* call(size_t size) {
        if constexpr (arch == arch_t::cpu) {
            return static_cast<T*>(std::calloc(size ? size : 1, sizeof(T)));
        } else {
            void* p = nullptr;
            if (g1_mem_alloc(&p, size * sizeof(T)) != G1_OK) {
                std::fprintf(stderr, "[ERROR] archi::memalloc: %s\n", g1_last_error());
                std::exit(1);
            }
            return static_cast<T*>(p);
        }
    }
};
template <arch_t arch>
struct memfree_t {
    template <typename T>
    static void call(T* ptr) {
        if constexpr (arch == arch_t::cpu)
            std::free(ptr);
        else
            g1_mem_free(ptr);
    }
};
template <arch_t arch>
struct memset_t {
    template <typename T>
    static void call(T* ptr, int value, size_t size) {
        if constexpr (arch == arch_t::cpu) {
            std::memset(ptr, value, size * sizeof(T));
        } else {
            detail::check(cudaMemset(ptr, value, size * sizeof(T)), "archi::memset");
        }
    }
};
template <arch_t dst_arch, arch_t src_arch>
struct memcpy_t {
    template <typename T>
    static void call(T* dst, const T* src, size_t size) {
        if (size == 0) return;
        if constexpr (dst_arch == arch_t::cpu && src_arch == arch_t::cpu) {
            std::memcpy(dst, src, size * sizeof(T));
        } else {
            const int kind = src_arch == arch_t::cpu ? 0 : (dst_arch == arch_t::cpu ? 1 : 2);
            if (g1_mem_copy(dst, src, size * sizeof(T), kind, nullptr) != G1_OK) {
                std::fprintf(stderr, "[ERROR] archi::memcpy: %s\n", g1_last_error());
                std::exit(1);
            }
            g1_stream_sync(nullptr);
        }
    }
};
template <arch_t arch, typename value_t>
constexpr auto memalloc = memalloc_t<arch>::template call<value_t>;
template <arch_t arch, typename value_t>
constexpr auto memfree = memfree_t<arch>::template call<value_t>;
template <arch_t arch, typename value_t>
constexpr auto memset = memset_t<arch>::template call<value_t>;
template <arch_t to_arch, arch_t from_arch, typename value_t>
constexpr auto memcpy = memcpy_t<to_arch, from_arch>::template call<value_t>;

namespace cuda {

// Atomic minimum returning the previous value (reference:
// archi/only/cuda.cuh:52-70).  Native for integers.  For floating point, one
// hardware integer atomic instead of a compare-and-swap loop: non-negative
// IEEE values order like their bit patterns as signed integers, negative ones
// reversed as unsigned integers, so a non-negative `value` is an integer
// atomicMin and a negative one an unsigned atomicMax on the same word (a
// stored negative value is never replaced by a non-negative one, and the
// reverse holds too).  NaN never replaces the stored value.
template <typename T>
__device__ __forceinline__ T AtomicMin(T* address, T value) {
    if constexpr (std::is_same_v<T, float>) {
        if (value != value) return *reinterpret_cast<volatile float*>(address);
        if (!signbit(value))
            return __int_as_float(::atomicMin(reinterpret_cast<int*>(address), __float_as_int(value)));
        return __uint_as_float(
            ::atomicMax(reinterpret_cast<unsigned int*>(address), __float_as_uint(value)));
    } else if constexpr (std::is_same_v<T, double>) {
        if (value != value) return *reinterpret_cast<volatile double*>(address);
        if (!signbit(value))
            return __longlong_as_double(::atomicMin(reinterpret_cast<long long*>(address),
                                                    __double_as_longlong(value)));
        return __longlong_as_double((long long)::atomicMax(
            reinterpret_cast<unsigned long long*>(address), (unsigned long long)__double_as_longlong(value)));
    } else {
        return ::atomicMin(address, value);
    }
}

}  // namespace cuda

}  // namespace graph_one::archi
