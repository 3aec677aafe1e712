#pragma once
// Engine bases of the GraphOne API (reference: engine/base.h:5-51) and the
// host-side plumbing the functor-templated engines share: one CUDA stream
// per engine, a pinned read-back area and the launch configuration of the
// library's kernel templates instantiated with the user's functor.

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

#include "graphone_b200.h"
#include "g1/common.cuh"
#include "GraphOne/utils/log.hpp"
#include "GraphOne/utils/pinned.h"

namespace graph_one::engine {

template <typename comp_t>
class BaseEngine {
protected:
    using graph_type = typename comp_t::graph_type;
    using hstatus_type = typename comp_t::hstatus_type;
    using dstatus_type = typename comp_t::dstatus_type;
    const graph_type& graph_;
    hstatus_type& h_status_;
    dstatus_type& d_status_;

public:
    explicit BaseEngine(comp_t& comp)
        : graph_(comp.graph), h_status_(comp.h_status), d_status_(comp.d_status) {}
    virtual ~BaseEngine() = default;
    virtual void Forward() = 0;
};

template <typename comp_t, typename frontier_t>
class GcEngine : public BaseEngine<comp_t> {
protected:
    frontier_t& frontier_;

public:
    GcEngine(comp_t& comp, frontier_t& frontier) : BaseEngine<comp_t>(comp), frontier_(frontier) {}
};

namespace detail {

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) LOG_ERROR(what, ": ", cudaGetErrorString(e));
}

inline void check_g1(g1_status s, const char* what) {
    if (s != G1_OK) LOG_ERROR(what, ": ", g1_status_string(s), ": ", g1_last_error());
}

inline int sm_count() {
    static int n = [] {
        int dev = 0, s = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
        return s;
    }();
    return n;
}

// Device counters and a host mirror for the one read-back per iteration:
// [0] appended vertices, [1] overflow flag, [2..3] out-degree sum (u64);
// [4..7] the same for a second compaction in the same step.  The mirror is
// a slot of the process's pinned block (ordinary memory if none is left).
struct Counters {
    uint32_t* dev = nullptr;
    uint32_t* host = nullptr;
    uint32_t own_[16] = {};
    Counters() {
        check_g1(g1_mem_alloc(reinterpret_cast<void**>(&dev), 64), "counters");
        host = ::graph_one::detail::PinnedSlots::get().take();
        if (!host) host = own_;
    }
    ~Counters() {
        g1_mem_free(dev);
        if (host != own_) ::graph_one::detail::PinnedSlots::get().give(host);
    }
    Counters(const Counters&) = delete;
    Counters& operator=(const Counters&) = delete;
    void clear(cudaStream_t s) { check_cuda(cudaMemsetAsync(dev, 0, 32, s), "clear counters"); }
    void read(cudaStream_t s) { read_set(s, 0); }
    // The 8 words of set `set` (0 or 1: dev + 8 * set) into host[0..7].
    void read_set(cudaStream_t s, int set) {
        check_cuda(cudaMemcpyAsync(host, dev + 8 * set, 32, cudaMemcpyDeviceToHost, s), "read counters");
        check_cuda(cudaStreamSynchronize(s), "engine step");
    }
    uint32_t count() const { return host[0]; }
    bool overflow() const { return host[1] != 0; }
    unsigned long long degree_sum() const {
        return (unsigned long long)host[2] | ((unsigned long long)host[3] << 32);
    }
    unsigned long long* degree_sum_dev() { return reinterpret_cast<unsigned long long*>(dev + 2); }
};

}  // namespace detail
}  // namespace graph_one::engine
