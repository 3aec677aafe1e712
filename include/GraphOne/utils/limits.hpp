#pragma once
// Invalid-value conventions of the GraphOne API (reference:
// utils/limits.hpp:10-73): UINT_MAX-style all-ones for unsigned ids, -1 for
// signed, NaN for floating point; vertex 0 is invalid when ids start at 1.

#include <limits>
#include <type_traits>

#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"

namespace graph_one::utils {

template <typename T, typename = void>
struct numeric_limits : std::numeric_limits<T> {};

template <typename T>
struct numeric_limits<T, std::enable_if_t<std::is_integral_v<T> && std::is_signed_v<T>>>
    : std::numeric_limits<T> {
    __host__ __device__ static constexpr T invalid() { return T(-1); }
};

template <typename T>
struct numeric_limits<T, std::enable_if_t<std::is_integral_v<T> && std::is_unsigned_v<T>>>
    : std::numeric_limits<T> {
    __host__ __device__ static constexpr T invalid() { return T(~T(0)); }
};

template <typename T>
struct numeric_limits<T, std::enable_if_t<std::is_floating_point_v<T>>> : std::numeric_limits<T> {
    __host__ __device__ static constexpr T invalid() { return std::numeric_limits<T>::quiet_NaN(); }
};

template <vstart_t v_start, typename vertex_t>
__host__ __device__ constexpr bool is_vertex_valid(vertex_t v) {
    static_assert(std::is_integral_v<vertex_t>, "vertex ids are integers");
    if constexpr (v_start == vstart_t::FROM_0_TO_0)
        return v != vertex_t(~vertex_t(0));
    else
        return v != 0;
}

template <vstart_t v_start, typename vertex_t>
__host__ __device__ constexpr vertex_t invalid_vertex() {
    if constexpr (v_start == vstart_t::FROM_0_TO_0)
        return vertex_t(~vertex_t(0));
    else
        return vertex_t(0);
}

}  // namespace graph_one::utils
