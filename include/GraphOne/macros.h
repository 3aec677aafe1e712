#pragma once
// Function qualifiers of the GraphOne API (reference: archi/macro/macro.h,
// archi/macro/cuda.cuh).  User functors and lambdas are written with these.
// Without nvcc (host-only code such as the loader or the CPU SpMV built by a
// plain C++ compiler) they reduce to `inline` or to nothing.

#ifdef __CUDACC__
#define __ONE_CUDA_KERNEL__ __global__
#define __ONE_CUDA__ __device__
#define __ONE_CUDA_INL__ __device__ __forceinline__
#define __ONE_CPU_CUDA__ __host__ __device__
#define __ONE_CPU_CUDA_INL__ __host__ __device__ __forceinline__
#else
#define __ONE_CUDA_KERNEL__
#define __ONE_CUDA__
#define __ONE_CUDA_INL__ inline
#define __ONE_CPU_CUDA__
#define __ONE_CPU_CUDA_INL__ inline
#endif

#define __ONE_DEV__ __ONE_CUDA__
#define __ONE_DEV_INL__ __ONE_CUDA_INL__
#define __ONE_ARCH__ __ONE_CPU_CUDA__
#define __ONE_ARCH_INL__ __ONE_CPU_CUDA_INL__
