#pragma once
// Device helpers shared by the prebuilt library (graphone_b200/csrc) and the
// functor-templated engines of the GraphOne-compatible headers.
//
// Everything here is sm_100a SIMT code: warp shuffles, warp-aggregated
// atomics and bounded spin-waits.  No tensor-core path exists for the graph
// semirings (min-plus and sparse plus-times are not dense contractions).

#include <cstdint>
#include <cstring>
#include <type_traits>
#include <cuda_runtime.h>

namespace g1 {

constexpr uint32_t kU32Max = 0xFFFFFFFFu;
constexpr int kWarp = 32;

// ---------------------------------------------------------------- shuffles
// Generic warp shuffles for any trivially copyable value of up to 16 bytes
// (the gather type of a user functor is an arbitrary scalar or small struct).
template <typename T>
__device__ __forceinline__ T shfl_up_any(unsigned mask, T v, int delta) {
    constexpr int W = (sizeof(T) + 3) / 4;
    static_assert(W <= 4, "gather values larger than 16 bytes are not supported");
    uint32_t w[W] = {};
    memcpy(w, &v, sizeof(T));
#pragma unroll
    for (int i = 0; i < W; ++i) w[i] = __shfl_up_sync(mask, w[i], delta);
    T out;
    memcpy(&out, w, sizeof(T));
    return out;
}

template <typename T>
__device__ __forceinline__ T shfl_any(unsigned mask, T v, int src) {
    constexpr int W = (sizeof(T) + 3) / 4;
    static_assert(W <= 4, "gather values larger than 16 bytes are not supported");
    uint32_t w[W] = {};
    memcpy(w, &v, sizeof(T));
#pragma unroll
    for (int i = 0; i < W; ++i) w[i] = __shfl_sync(mask, w[i], src);
    T out;
    memcpy(&out, w, sizeof(T));
    return out;
}

template <typename T>
__device__ __forceinline__ T shfl_down_any(unsigned mask, T v, int delta) {
    constexpr int W = (sizeof(T) + 3) / 4;
    uint32_t w[W] = {};
    memcpy(w, &v, sizeof(T));
#pragma unroll
    for (int i = 0; i < W; ++i) w[i] = __shfl_down_sync(mask, w[i], delta);
    T out;
    memcpy(&out, w, sizeof(T));
    return out;
}

// Read-only (non-coherent, L1-cached) load for values the kernel never
// writes; plain load for types __ldg does not cover.
template <typename T>
__device__ __forceinline__ T ldg_any(const T* p) {
    if constexpr (sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) == 16) {
        if constexpr (std::is_arithmetic<T>::value) return __ldg(p);
        else return *p;
    } else {
        return *p;
    }
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// ------------------------------------------------- warp-aggregated append
// Appends v to out[] (counter *count): one atomic per group of converged
// lanes, each lane writes its own slot.  Callers guarantee capacity.
__device__ __forceinline__ void append(uint32_t* out, uint32_t* count, uint32_t v) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const uint32_t lane = lane_id();
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    out[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// append() that also adds `d` (e.g. the vertex's out-degree) to *sum, with
// one atomic per converged group for each counter.
__device__ __forceinline__ void append_sum(uint32_t* out, uint32_t* count,
                                           unsigned long long* sum, uint32_t v, uint32_t d) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const uint32_t lane = lane_id();
    const uint32_t tot = __reduce_add_sync(mask, d);
    uint32_t base = 0;
    if ((int)lane == leader) {
        base = atomicAdd(count, (uint32_t)__popc(mask));
        atomicAdd(sum, (unsigned long long)tot);
    }
    base = __shfl_sync(mask, base, leader);
    out[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// ------------------------------------------------------- block reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += shfl_down_any(0xffffffffu, v, d);
    return v;
}

// Sum over the block; the result is valid in thread 0.  `scratch` holds one
// T per warp.  Contains __syncthreads(): call from every thread.
template <typename T, int BLOCK>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if (lane_id() == 0) scratch[w] = v;
    __syncthreads();
    T r = T(0);
    if (threadIdx.x < 32) {
        r = (threadIdx.x < BLOCK / 32) ? scratch[threadIdx.x] : T(0);
        r = warp_sum(r);
    }
    return r;
}

// Fills the shared-memory x cache with x[0, hot): 16-byte loads, eight in
// flight per thread before their stores (one L2 round trip instead of one
// per element), when x is 16-byte aligned; element loads otherwise.
template <int THREADS, class X>
__device__ __forceinline__ void fill_x_cache(X* xc, const X* x, uint32_t hot) {
    uint32_t done = 0;
    if constexpr (sizeof(X) == 4) {
        if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0) {
            const uint32_t nv = hot / 4;
            const uint4* src = reinterpret_cast<const uint4*>(x);
            uint4* dst = reinterpret_cast<uint4*>(xc);
            for (uint32_t base = 0; base < nv; base += 8 * THREADS) {
                uint4 r[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint32_t i = base + q * THREADS + threadIdx.x;
                    if (i < nv) r[q] = __ldg(src + i);
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint32_t i = base + q * THREADS + threadIdx.x;
                    if (i < nv) dst[i] = r[q];
                }
            }
            done = nv * 4;
        }
    }
    for (uint32_t i = done + threadIdx.x; i < hot; i += THREADS) xc[i] = ldg_any(x + i);
}

// ------------------------------------------- TMA bulk copies + mbarriers
// 1-D bulk copies global -> shared (cp.async.bulk) completing on an
// mbarrier transaction count.  Source, destination and size must be
// multiples of 16 bytes; callers pad and align their ranges.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Default poll limit of the waits on bulk copies: a few seconds, far longer
// than any copy that is not stuck.
constexpr uint32_t kWaitPolls = 1u << 22;
// Waits for phase `parity` of the barrier, giving up after `limit` polls
// (each poll suspends the thread for a bounded hardware interval).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint32_t limit = kWaitPolls) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ------------------------------------------ programmatic dependent launch
// For kernels launched with the programmatic stream serialization
// attribute: grid_dependency_wait() returns once the preceding grid in the
// stream has completed and its writes are visible; grid_launch_dependents()
// lets the next grid start launching once every block of this grid has
// issued it (or exited).  Both are no-ops for ordinary launches.
__device__ __forceinline__ void grid_dependency_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------------- ceil division
// ------------------------------------------ L2 cache policies and hints

// Access policies for ld ...L2::cache_hint: streamed data is evicted first,
// gathered data that is reused (x vectors) last.
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// 16-byte read-only load with an L2 policy.
__device__ __forceinline__ uint4 ldg_v4_policy(const void* ptr, uint64_t pol) {
    uint4 r;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(ptr), "l"(pol));
    return r;
}
// 32-byte read-only load (sm_100 256-bit vector load); `ptr` must be
// 32-byte aligned.
__device__ __forceinline__ void ldg_v8(const void* ptr, uint4& lo, uint4& hi) {
    asm("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(lo.x), "=r"(lo.y), "=r"(lo.z), "=r"(lo.w), "=r"(hi.x), "=r"(hi.y), "=r"(hi.z), "=r"(hi.w)
        : "l"(ptr));
}
// The same for data read once (a stream): the lines are not kept in L1, so
// L1 stays with the data that is read again.
__device__ __forceinline__ void ldg_v8_stream(const void* ptr, uint4& lo, uint4& hi) {
    asm("ld.global.nc.L1::no_allocate.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(lo.x), "=r"(lo.y), "=r"(lo.z), "=r"(lo.w), "=r"(hi.x), "=r"(hi.y), "=r"(hi.z), "=r"(hi.w)
        : "l"(ptr));
}
// 4-byte read-only load with an L2 policy.
__device__ __forceinline__ uint32_t ldg_u32_policy(const void* ptr, uint64_t pol) {
    uint32_t r;
    asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(ptr), "l"(pol));
    return r;
}
// 4-byte load through a generic address: one instruction whether `p` points
// into this block's shared memory or into global memory.
__device__ __forceinline__ uint32_t ld_generic_u32(const void* p) {
    uint32_t v;
    asm volatile("ld.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Brings the line holding `p` into L2 ahead of use.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// Brings [p, p + bytes) into L2 ahead of use with one bulk prefetch (the
// TMA engine: no registers, nothing to wait for).  `p` must be 16-byte
// aligned and `bytes` a multiple of 16; the range must lie inside one
// allocation.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
// Brings the line holding `p` into this SM's L1 ahead of use.
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__host__ __device__ __forceinline__ uint64_t ceil_div(uint64_t a, uint64_t b) {
    return (a + b - 1) / b;
}

// ---------------------------------------------- device-side error status
// Kernels that can fail (bounded waits, capacity checks) record a code here
// instead of trapping; the host reads it after the launch sequence.
enum DeviceError : uint32_t {
    kDevOk = 0,
    kDevTimeout = 1,      // a bounded spin-wait ran out
    kDevOverflow = 2,     // a frontier/queue would have exceeded its capacity
    kDevInvalid = 3,      // a caller-supplied vertex id was out of range (skipped)
};

__device__ __forceinline__ void set_error(uint32_t* flag, uint32_t code) {
    if (flag) atomicCAS(flag, 0u, code);
}

}  // namespace g1
