#pragma once
// Kernel launches of the GraphOne API (reference: archi/kernel/def.hpp:7-28,
// archi/kernel/cuda.cuh:11-99):
//
//   archi::LaunchKernel<arch, tparams>(LaunchParams<arch>(n), kernel, args...);
//   archi::LaunchSync<arch>();
//
// LaunchParams<cuda>(n, is_num_blocks = false, smem_bytes = 0, stream = 0):
// n threads (rounded up to blocks of tparams::block_size) or n blocks.
// tparams = empty_t selects LaunchTparams<arch>: 256 threads per block and
// the index helpers kernels use (global_tid, grid_threads, warp_id, ...).

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"

namespace graph_one::archi {

namespace cuda {
constexpr uint32_t kBlockSize = 256;
inline uint32_t GetNumBlock(int64_t n) {
    return (uint32_t)std::max<int64_t>(1, (n + kBlockSize - 1) / kBlockSize);
}
}  // namespace cuda

template <arch_t arch>
struct LaunchTparams {};
template <arch_t arch>
struct LaunchParams {};
template <arch_t arch>
struct Launcher {};

template <>
struct LaunchTparams<arch_t::cuda> {
    constexpr static uint32_t block_size = cuda::kBlockSize;
    constexpr static uint32_t warp_size = 32;
    __ONE_CUDA_INL__ static uint32_t grid_dim() { return gridDim.x; }
    __ONE_CUDA_INL__ static uint32_t block_id() { return blockIdx.x; }
    __ONE_CUDA_INL__ constexpr static uint32_t block_dim() { return block_size; }
    __ONE_CUDA_INL__ static uint32_t thread_id() { return threadIdx.x; }
    __ONE_CUDA_INL__ static uint32_t global_tid() { return block_id() * block_dim() + thread_id(); }
    __ONE_CUDA_INL__ static uint32_t grid_threads() { return grid_dim() * block_dim(); }
    __ONE_CUDA_INL__ static uint32_t warp_id() { return thread_id() >> 5; }
    __ONE_CUDA_INL__ static uint32_t lane_id() { return thread_id() & 31u; }
};

template <>
struct LaunchParams<arch_t::cuda> {
    LaunchParams(int64_t n, bool is_num_blocks = false, size_t smem = 0, cudaStream_t s = 0)
        : grid_dim(is_num_blocks ? (uint32_t)std::max<int64_t>(1, n) : cuda::GetNumBlock(n)),
          smem_bytes(smem), stream(s) {}
    dim3 grid_dim;
    size_t smem_bytes;
    cudaStream_t stream;
};

template <>
struct Launcher<arch_t::cuda> {
    constexpr static arch_t arch_value = arch_t::cuda;
    using err_t = cudaError_t;

    template <typename tparams, typename func_t, typename... args_t>
    static err_t launch(const LaunchParams<arch_value>& params, const func_t& func, args_t&&... args) {
        func<<<params.grid_dim, tparams::block_size, params.smem_bytes, params.stream>>>(
            std::forward<args_t>(args)...);
        return cudaGetLastError();
    }

    static err_t sync(cudaStream_t stream = 0) {
        return stream ? cudaStreamSynchronize(stream) : cudaDeviceSynchronize();
    }
};

template <arch_t arch, typename tparams, typename func_t, typename... args_t>
typename Launcher<arch>::err_t LaunchKernel(const LaunchParams<arch>& params, func_t& f, args_t&&... args) {
    using tp = std::conditional_t<std::is_same_v<tparams, empty_t>, LaunchTparams<arch>, tparams>;
    return Launcher<arch>::template launch<tp>(params, f, std::forward<args_t>(args)...);
}

template <arch_t arch, typename... args_t>
typename Launcher<arch>::err_t LaunchSync(args_t&&... args) {
    return Launcher<arch>::sync(std::forward<args_t>(args)...);
}

}  // namespace graph_one::archi
