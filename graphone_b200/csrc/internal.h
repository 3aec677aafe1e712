// Internal state of libgraphone_b200.so (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "graphone_b200.h"

namespace g1 {

class SlotEngine;

// Records the failure message for g1_last_error() and returns the status.
g1_status fail(g1_status s, const std::string& msg);
g1_status fail_cuda(cudaError_t e, const char* what);

#define G1_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return ::g1::fail_cuda(e_, #call); \
    } while (0)

#define G1_TRY(call)                     \
    do {                                 \
        g1_status s_ = (call);           \
        if (s_ != G1_OK) return s_;      \
    } while (0)

// Owning device buffer; capacity grows, never shrinks.
// Device memory of the library.  Freed blocks go to a per-device cache and
// are reused by later requests of about their size (a new graph of the same
// shape allocates and frees nothing); a block is reused only after a device
// synchronisation that follows its release, so no queued kernel can still
// touch it.  The cache holds at most a quarter of the device's memory and
// is emptied when an allocation fails.
void dev_block_release(int dev, void* p, size_t bytes);
g1_status dev_block_get(size_t want, void** p, size_t* got, int* dev);
// Bytes the cache holds on `dev` (reusable without the driver).
size_t dev_block_cached(int dev);
// Frees the cached blocks of `dev` (the current device); returns their bytes.
size_t dev_block_drain(int dev);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int dev = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) dev_block_release(dev, p, bytes);
        p = nullptr;
        bytes = 0;
    }
    g1_status ensure(size_t want);
    // Exchanges the blocks (and their devices) of two buffers.
    void swap(DevBuf& o) {
        std::swap(p, o.p);
        std::swap(bytes, o.bytes);
        std::swap(dev, o.dev);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Pinned host scratch for small read-backs (sizes, counters).
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    g1_status ensure(size_t want);
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Merge-path plan of one orientation.
struct MergePlan {
    uint32_t items = 0;
    uint32_t n_tiles = 0;
    DevBuf tile_row, tile_nnz, carry, tail;
};

// nnz-split plan of one orientation (tiles of 256 nonzeros): rank of the
// row holding each tile's first nonzero, the row-start bitmap over the
// nonzeros, the non-empty rows in order followed by the empty rows.
struct NnzPlan {
    uint32_t tile = 0;  // nonzeros per tile
    uint32_t n_tiles = 0, n_nonempty = 0, n_empty = 0, n_fix = 0;
    uint32_t n_fix_short = 0;  // fix entries [0, n_fix_short) end in the tile after their first
    DevBuf tile_seg, sbits, rows, carry, tail;
    DevBuf fix_tiles;  // tiles in which a row begun in an earlier tile ends
    DevBuf fix_info;   // per such tile: {tile, row, first tile of the row, 0}; rows that
                       // span one boundary first, then longer chains, each in tile order
};

struct Orientation {
    bool present = false;
    uint32_t* rp = nullptr;
    uint32_t* col = nullptr;
    void* val = nullptr;
    DevBuf b_rp, b_col, b_val;  // storage unless shared with the other side
    uint32_t max_deg = 0;
    std::map<uint32_t, std::unique_ptr<MergePlan>> plans;  // by items per tile
    int tuned_sched = 0;  // 0 = not tuned, else g1_schedule
    int tuned_variant = -1;  // merge kernel variant chosen by g1_autotune (-1 = default)
    std::map<uint32_t, std::unique_ptr<NnzPlan>> nnz_plans;  // by nonzeros per tile
};

// Captured CUDA graphs of the device-driven traversal engines (traverse.cu):
// per mode (engine x {SSSP, BFS}) a graph of 2^i pairs of steps for each
// i < kSizes, valid for the state store they were captured on (`key`).
struct AdvGraphs {
    static constexpr int kSizes = 8;
    static constexpr int kModes = 4;  // {advance, BLAS pull} x {SSSP, BFS}
    cudaGraphExec_t exec[kModes][kSizes] = {};
    const void* key[kModes] = {};
    unsigned long long param[kModes] = {};  // a launch argument the graphs hold (the sparse-pull limit)
    cudaStream_t capture = nullptr;
    AdvGraphs() = default;
    AdvGraphs(const AdvGraphs&) = delete;
    AdvGraphs& operator=(const AdvGraphs&) = delete;
    void reset(int mode) {
        for (auto& x : exec[mode])
            if (x) {
                cudaGraphExecDestroy(x);
                x = nullptr;
            }
        key[mode] = nullptr;
        param[mode] = 0;
    }
    ~AdvGraphs() {
        for (int m = 0; m < kModes; ++m) reset(m);
        if (capture) cudaStreamDestroy(capture);
    }
};

// Named, growable workspaces of one graph.
struct Workspace {
    std::map<std::string, std::unique_ptr<DevBuf>> bufs;
    PinnedBuf pinned;
    template <class T>
    g1_status get(const std::string& name, size_t count, T** out) {
        auto& b = bufs[name];
        if (!b) b.reset(new DevBuf());
        G1_TRY(b->ensure(count * sizeof(T) + 64));
        *out = b->as<T>();
        return G1_OK;
    }
    size_t bytes() const {
        size_t s = 0;
        for (auto& kv : bufs) s += kv.second ? kv.second->bytes : 0;
        return s;
    }
};

}  // namespace g1

struct g1_graph {
    int device = 0;
    uint32_t n = 0;
    uint32_t m = 0;
    g1_dtype vtype = G1_U32;
    bool symmetric = false;
    // 0 = out-edges (normal), 1 = in-edges (transpose), 2 = PageRank's
    // hot-column copy of 1 on graphs kept in the caller's order (its own
    // column array; rows, values and plans are 1's)
    g1::Orientation o[3];
    g1::Workspace ws;
    std::mutex mu;
    int sm_count = 148;
    // Per-vertex sum of out-edge weights (PageRank's iweights denominator),
    // derived once per graph like the merge-path plans.
    bool outw_ready = false;
    // PageRank: empty in-edge rows with out-weight (workspace "pr_empty_active")
    // and the count of isolated vertices, for the nnz schedule
    bool pr_empty_ready = false;
    uint32_t pr_active_empty = 0, pr_isolated = 0;
    // Row pieces of the in-edge CSR for the multi-source pull kernels, the
    // rows with more than one piece (hubs) and the out-degrees (PPR).
    bool pieces_ready = false;
    uint32_t n_pieces = 0;
    bool hubs_ready = false;
    uint32_t n_hubs = 0, n_hub_pieces = 0;
    bool outdeg_ready = false;
    // Mean u32 edge weight (bucket width of the near-far engine), -1 until known.
    double mean_weight = -1.0;
    // Push/pull switches (g1_autotune_traversal may change them): the
    // single-source AUTO engine pushes while the frontier's out-degree sum is
    // below m / push_div; the slot engines list the next iteration's row
    // pieces while the changed vertices' out-edges are below (m + n) / slot_div.
    uint32_t push_div = 16;
    uint32_t slot_div = 8;
    // Slot engines of the batched BFS / SSSP / PPR entry points (by kind),
    // kept between calls.
    std::shared_ptr<g1::SlotEngine> slot_cache[3];
    // CUDA graphs of the device-driven advance engine.
    std::unique_ptr<g1::AdvGraphs> adv_graphs;
    // Degree-ordered relabelling (G1_GRAPH_RELABEL): perm maps a caller's
    // vertex id to the internal id, iperm the reverse.
    bool relabeled = false;
    g1::DevBuf perm, iperm;
    // PageRank's hot-column layout (orientation 2): a g1_hot_columns mode
    int hot_mode = 0;
    // Device error word written by kernels (bounded waits that ran out).
    g1::DevBuf err_buf;
    uint32_t* err_word = nullptr;
};

namespace g1 {

// Makes `dev` current for the scope.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

bool is_device_ptr(const void* p);
// Copies n bytes to a device or host destination from device memory.
g1_status copy_out(void* dst, const void* dev_src, size_t bytes, cudaStream_t s);

g1_status ensure_plan(g1_graph* g, int t, uint32_t items, MergePlan** out);
// The nnz-split plan for tiles of `tile` nonzeros (a multiple of 32; 256 is
// the default schedule's).
g1_status ensure_nnz_plan(g1_graph* g, int t, NnzPlan** out, uint32_t tile = 256);
// Graph creation of a large in-edge CSR with f32 values from host memory:
// uploads its columns and values on s while a second stream sums the
// arrived chunks' out-weights for PageRank (pagerank.cu).
g1_status upload_transpose_with_outw(g1_graph* g, const uint32_t* col, const void* val, cudaStream_t s);
// Per-vertex out-degrees (edge count, n words in the graph's workspace),
// derived once per graph; the caller holds g->mu.
g1_status out_degrees(g1_graph* g, uint32_t** deg, cudaStream_t s);
// Single-source personalized PageRank on the SpMV schedules (pagerank.cu).
// A run's state lives in caller-owned device memory (`words` 4-byte words,
// 256-byte aligned), so runs on different streams share no scratch.
// ppr_prepare derives the graph's out-degrees and nnz plan (the caller holds
// g->mu); ppr_enqueue then reads only the graph's fixed arrays and enqueues
// the run on `s`: src is a caller id when perm (the graph's relabelling) is
// given; *rank_out points into the store (internal vertex order).
struct PprPlan {
    const uint32_t* deg = nullptr;
    const NnzPlan* plan = nullptr;  // null: the CSR-vector schedule
    size_t words = 0;
    // sparse steps (0: none): the out-edge CSR and the limit on the in-edges
    // of the rows a step reaches
    const uint32_t* out_rp = nullptr;
    const uint32_t* out_col = nullptr;
    unsigned long long sparse_limit = 0;
    uint32_t sparse_steps = 0;  // the steps that may be sparse (the first ones)
    // the in-edge CSR the SpMV runs on: 1, or its hot-column copy 2 with x
    // stored by hot id (xperm: vertex -> hot id)
    int t = 1;
    const uint32_t* xperm = nullptr;
};
size_t ppr_state_words(uint32_t n, const NnzPlan* plan);
g1_status ppr_prepare(g1_graph* g, cudaStream_t s, PprPlan* out);
g1_status ppr_enqueue(g1_graph* g, const PprPlan& pl, uint32_t* store, uint32_t src, float alpha,
                      uint32_t iters, const uint32_t* perm, cudaStream_t s, const float** rank_out);
// g1_ppr with the graph's workspace as the store (caller vertex src, ranks
// in caller order into rank_out, host or device); the caller holds g->mu.
g1_status ppr_locked(g1_graph* g, uint32_t src, float alpha, uint32_t iters, float* rank_out,
                     cudaStream_t s);
// Near-far SSSP (unit = BFS) from internal vertex src in one persistent
// launch; *dist_out points to the graph's workspace distances.  frontier:
// no distance buckets (threshold infinite), so every round relaxes the
// out-edges of all vertices the previous round improved -- the advance /
// filter frontier algorithm, in one launch (for BFS the same rounds as the
// near-far engine's levels).
g1_status nearfar_traverse(g1_graph* g, uint32_t src, bool unit, uint32_t** dist_out, uint32_t* rounds,
                           cudaStream_t s, bool frontier = false);
// The same in caller-owned buffers, enqueued only: buffers laid out in one
// store of nearfar_words(n) words (256-byte aligned), the bucket width (mean weight based; the caller holds
// g->mu the first time), the launch, and the outcome from a host copy of the
// control block (nearfar_ctl_bytes() bytes at NfBuffers::ctl).
struct NfBuffers {
    unsigned long long* key;  // per vertex: distance << 32 | tag of its last improvement
    uint32_t *dist, *near[2], *far[2], *ctl;
};
size_t nearfar_words(uint32_t n);  // 4-byte words of one store
void nearfar_layout(uint32_t n, uint32_t* store, NfBuffers* b);
g1_status nearfar_delta(g1_graph* g, bool unit, cudaStream_t s, uint32_t* out);
// src: internal id, or a caller id when perm (the graph's relabelling) is given
g1_status nearfar_launch(const g1_graph* g, uint32_t src, bool unit, uint32_t delta, const NfBuffers& b,
                         cudaStream_t s, const uint32_t* perm = nullptr);
g1_status nearfar_result(const uint32_t* host_ctl, uint32_t* rounds);
uint32_t nearfar_ctl_bytes();
// Graphs of small uniform degree (grids, meshes), where the near-far engine
// beats frontier engines and batches.
inline bool nearfar_suits(const g1_graph* g) {
    return g->o[0].present && g->o[0].max_deg <= 16 && (uint64_t)g->m <= 8ull * g->n;
}
// Vertex-order conversions of a relabelled graph (4-byte values).
g1_status to_caller_order(g1_graph* g, uint32_t* dev_out, const uint32_t* internal, cudaStream_t s);
g1_status to_internal_order(g1_graph* g, uint32_t* dev_out, const uint32_t* caller, cudaStream_t s);
g1_status internal_vertex(g1_graph* g, uint32_t v, uint32_t* out, cudaStream_t s);
// copy_out of an n-vector of 4-byte values in internal order to the caller.
g1_status copy_out_vertices(g1_graph* g, void* dst, const void* internal, cudaStream_t s);
g1_status spmv_dispatch(g1_graph* g, int transpose, g1_semiring sr, g1_schedule sched,
                        const void* x, void* y, cudaStream_t s);
// Single-source SSSP (unit: BFS) from caller vertex `src` on `engine`;
// the caller holds g->mu.
g1_status traverse_locked(g1_graph* g, uint32_t src, g1_engine engine, bool unit, uint32_t* out,
                          uint32_t* iters_out, cudaStream_t s);
// Reads and clears the graph's device error word (synchronises `s`).
g1_status check_device_error(g1_graph* g, cudaStream_t s);

// While alive, the calling thread is capturing a CUDA graph: the SpMV timer
// (profiling) records nothing.
struct CaptureScope {
    CaptureScope();
    ~CaptureScope();
};

// Poll limit of the bounded device waits: `dflt` unless a test lowered it
// with g1_test_set_wait_polls.
uint32_t wait_polls(uint32_t dflt);

// Kernel launch accounting (g1_kernel_launches) and the SpMV kernel timer
// (g1_profile_begin/end).
void count_launches(uint64_t n);
bool profiling();
void prof_mark(cudaStream_t s, bool start);
inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// Orientation the pull (gather) engines read: in-edges.
inline int pull_side(const g1_graph* g) { return g->o[1].present ? 1 : 0; }
// Orientation the push (advance) engines read: out-edges.
inline int push_side(const g1_graph* g) { return g->o[0].present ? 0 : 1; }

}  // namespace g1
