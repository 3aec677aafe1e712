#pragma once
// VecToString for thrust vectors (reference: utils/string_arch.h:8-31): the
// device vector is copied to the host first.

#include <string>

#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "GraphOne/utils/string.hpp"

namespace graph_one::utils {

template <typename T, typename F>
std::string VecToString(const thrust::host_vector<T>& vec, F str_func) {
    return VecToString(thrust::raw_pointer_cast(vec.data()), vec.size(), str_func);
}

template <typename T>
std::string VecToString(const thrust::host_vector<T>& vec) {
    return VecToString(thrust::raw_pointer_cast(vec.data()), vec.size());
}

template <typename T, typename F>
std::string VecToString(const thrust::device_vector<T>& vec, F str_func) {
    const thrust::host_vector<T> h = vec;
    return VecToString(h, str_func);
}

template <typename T>
std::string VecToString(const thrust::device_vector<T>& vec) {
    const thrust::host_vector<T> h = vec;
    return VecToString(h);
}

}  // namespace graph_one::utils
