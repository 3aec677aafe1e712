#pragma once
// Error checks of the GraphOne API (reference: archi/check/check.h:10-20,
// archi/check/cuda.cuh:7-19).  Here a failed CUDA call is always reported
// and ends the program (the reference stays silent unless DEBUG_CUDA is
// defined).

#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

#include "GraphOne/type.hpp"

namespace graph_one {

template <typename T>
void CheckCudaErr(T result, char const* const func, const char* const file, int const line) {
    if (result) {
        std::fprintf(stderr, "CUDA error at %s:%d code=%d(%s) \"%s\"\n", file, line,
                     static_cast<unsigned int>(result), cudaGetErrorName(static_cast<cudaError_t>(result)), func);
        std::exit(1);
    }
}

template <arch_t arch, typename T>
void checkArchErr(T val, char const* const func, const char* const file, int const line) {
    if constexpr (arch == arch_t::cuda) CheckCudaErr(val, func, file, line);
}

}  // namespace graph_one

#ifndef checkCudaErrors
#define checkCudaErrors(val) ::graph_one::CheckCudaErr((val), #val, __FILE__, __LINE__)
#endif
#define checkArchErrors(arch, val) ::graph_one::checkArchErr<arch>((val), #val, __FILE__, __LINE__)
