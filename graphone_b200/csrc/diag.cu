// Measurement support: the rate at which the SMs get random loads served.
// The pull SpMV's cold x gathers (those outside the shared-memory copy of x)
// are random 4-byte loads from an L2-resident x, one L2 request each; this
// rate, not HBM bandwidth, is the ceiling they run against.  The probe
// gathers from a buffer of the given footprint (resident in L1, L2 or HBM
// after the first pass, by its size) at hashed random positions, with 1024-
// thread blocks and a chosen number of independent loads per thread.
#include <algorithm>

#include <cooperative_groups.h>

#include "g1/common.cuh"
#include "internal.h"

namespace g1 {
namespace {

__device__ __forceinline__ uint32_t probe_hash(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (uint32_t)(z ^ (z >> 31));
}

// Each thread gathers `per_thread` items of T at hashed positions below
// `mask + 1` (a power of two inside the buffer), ILP independent loads in
// flight, and stores a fold of them.
template <class T, int ILP>
__global__ void __launch_bounds__(1024)
gather_probe_kernel(const T* __restrict__ buf, uint32_t mask, uint32_t per_thread, uint32_t* out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (uint32_t i = 0; i < per_thread; i += ILP) {
        T v[ILP];
#pragma unroll
        for (int k = 0; k < ILP; ++k) v[k] = __ldg(buf + (probe_hash(t * 1000003ull + i + k) & mask));
#pragma unroll
        for (int k = 0; k < ILP; ++k) {
            uint32_t w;
            memcpy(&w, &v[k], 4);
            acc ^= w;
        }
    }
    out[t] = acc;
}

template <class T, int ILP>
g1_status probe(int sms, uint32_t blocks_per_sm, uint64_t footprint, double* rate, cudaStream_t s) {
    DevBuf buf, out;
    const uint32_t grid = (uint32_t)sms * blocks_per_sm;
    G1_TRY(buf.ensure(footprint));
    G1_TRY(out.ensure((size_t)grid * 1024 * 4));
    G1_CUDA(cudaMemsetAsync(buf.p, 0, footprint, s));
    const uint32_t items = (uint32_t)(footprint / sizeof(T));
    const uint32_t per_thread = 512;  // a multiple of every ILP
    const uint64_t total = (uint64_t)grid * 1024 * per_thread;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    G1_CUDA(cudaEventCreate(&e0));
    G1_CUDA(cudaEventCreate(&e1));
    auto launch = [&] {
        gather_probe_kernel<T, ILP><<<grid, 1024, 0, s>>>(buf.as<T>(), items - 1, per_thread, out.as<uint32_t>());
    };
    launch();  // brings the buffer into the caches it fits
    cudaEventRecord(e0, s);
    const int reps = 4;
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, s);
    count_launches(reps + 1);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return fail_cuda(err, "gather probe");
    *rate = ms > 0.0f ? (double)total * reps / ((double)ms * 1e-3) : 0.0;
    return G1_OK;
}

template <class T>
g1_status probe_ilp(uint32_t in_flight, int sms, uint32_t bps, uint64_t fp, double* rate, cudaStream_t s) {
    switch (in_flight) {
        case 1: return probe<T, 1>(sms, bps, fp, rate, s);
        case 4: return probe<T, 4>(sms, bps, fp, rate, s);
        case 8: return probe<T, 8>(sms, bps, fp, rate, s);
        case 16: return probe<T, 16>(sms, bps, fp, rate, s);
        default: return probe<T, 32>(sms, bps, fp, rate, s);
    }
}

// Shared-memory gathers: each 1024-thread block (one per SM, 128 KB of
// shared memory) fills its words, then every thread gathers `iters` x 8
// words at hashed positions: from its own block's shared memory (REMOTE
// false) or from a random block of its thread-block cluster (distributed
// shared memory).  Cluster barriers before the gathers and before exit keep
// every block's memory alive while others read it.
constexpr uint32_t kSmemProbeWordsLog2 = 15;

__device__ __forceinline__ uint32_t probe_mix(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

template <bool REMOTE>
__global__ void __launch_bounds__(1024, 1) smem_gather_probe_kernel(uint32_t iters, uint32_t* out) {
    extern __shared__ uint32_t words[];
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    constexpr uint32_t kWords = 1u << kSmemProbeWordsLog2;
    for (uint32_t i = threadIdx.x; i < kWords; i += blockDim.x) words[i] = probe_mix(i + blockIdx.x);
    cl.sync();
    const uint32_t c = cl.num_blocks();
    uint32_t st = probe_mix(blockIdx.x * 1024u + threadIdx.x + 1u);
    uint32_t acc = 0;
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            st = probe_mix(st + (uint32_t)j + 0x9e3779b9u);
            const uint32_t* base = REMOTE ? cl.map_shared_rank(words, (st >> 24) % c) : words;
            v[j] = base[st & (kWords - 1)];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc ^= v[j];
    }
    cl.sync();
    out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <bool REMOTE>
g1_status smem_probe(uint32_t cluster, double* rate, uint32_t* blocks_out, cudaStream_t s) {
    auto k = smem_gather_probe_kernel<REMOTE>;
    const size_t smem = (size_t)4 << kSmemProbeWordsLog2;
    G1_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (cluster > 8) G1_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    G1_CUDA(cudaOccupancyMaxActiveClusters(&clusters, k, &cfg));
    if (clusters <= 0) return fail(G1_ERR_UNSUPPORTED, "g1_measure_smem_gather_rate: no cluster of that size fits");
    const uint32_t grid = (uint32_t)clusters * cluster;  // every cluster resident at once
    *blocks_out = grid;
    cfg.gridDim = dim3(grid);
    DevBuf out;
    G1_TRY(out.ensure((size_t)grid * 1024 * 4));
    const uint32_t iters = 256;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    G1_CUDA(cudaEventCreate(&e0));
    G1_CUDA(cudaEventCreate(&e1));
    const int reps = 4;
    cudaError_t err = cudaLaunchKernelEx(&cfg, k, iters, out.as<uint32_t>());
    if (err == cudaSuccess) err = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && err == cudaSuccess; ++r) err = cudaLaunchKernelEx(&cfg, k, iters, out.as<uint32_t>());
    if (err == cudaSuccess) err = cudaEventRecord(e1, s);
    count_launches(reps + 1);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return fail_cuda(err, "shared-memory gather probe");
    const double total = (double)grid * 1024 * iters * 8 * reps;
    *rate = ms > 0.0f ? total / ((double)ms * 1e-3) : 0.0;
    return G1_OK;
}

}  // namespace
}  // namespace g1

using namespace g1;

extern "C" g1_status g1_measure_smem_gather_rate(uint32_t cluster_size, int remote, double* gathers_per_s,
                                                 uint32_t* blocks, void* stream) {
    if (!gathers_per_s || (cluster_size != 1 && cluster_size != 2 && cluster_size != 4 && cluster_size != 8 &&
                           cluster_size != 16))
        return fail(G1_ERR_INVALID, "g1_measure_smem_gather_rate: cluster_size must be 1, 2, 4, 8 or 16");
    *gathers_per_s = 0.0;
    uint32_t b = 0;
    cudaStream_t s = as_stream(stream);
    const g1_status st = remote ? smem_probe<true>(cluster_size, gathers_per_s, &b, s)
                                : smem_probe<false>(cluster_size, gathers_per_s, &b, s);
    if (blocks) *blocks = b;
    return st;
}

extern "C" g1_status g1_measure_gather_rate(uint32_t item_bytes, uint32_t in_flight, uint32_t blocks_per_sm,
                                            uint64_t footprint_bytes, double* gathers_per_s, void* stream) {
    if (!gathers_per_s || (item_bytes != 4 && item_bytes != 16))
        return fail(G1_ERR_INVALID, "g1_measure_gather_rate: item_bytes must be 4 or 16");
    if (in_flight != 1 && in_flight != 4 && in_flight != 8 && in_flight != 16 && in_flight != 32)
        return fail(G1_ERR_INVALID, "g1_measure_gather_rate: in_flight must be 1, 4, 8, 16 or 32");
    if (blocks_per_sm < 1 || blocks_per_sm > 2)
        return fail(G1_ERR_INVALID, "g1_measure_gather_rate: blocks_per_sm must be 1 or 2");
    if (footprint_bytes < 65536 || footprint_bytes > (1ull << 32) || (footprint_bytes & (footprint_bytes - 1)))
        return fail(G1_ERR_INVALID, "g1_measure_gather_rate: footprint must be a power of two in [64 KiB, 4 GiB]");
    *gathers_per_s = 0.0;
    int dev = 0, sms = 0;
    G1_CUDA(cudaGetDevice(&dev));
    G1_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = as_stream(stream);
    return item_bytes == 4 ? probe_ilp<float>(in_flight, sms, blocks_per_sm, footprint_bytes, gathers_per_s, s)
                           : probe_ilp<uint4>(in_flight, sms, blocks_per_sm, footprint_bytes, gathers_per_s, s);
}
