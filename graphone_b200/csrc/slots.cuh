// Multi-source traversal state with per-source slots (internal).
//
// A SlotEngine holds K <= 256 query slots over one graph: BFS levels, SSSP
// distances or personalized-PageRank ranks of K sources, stored vertex-major
// (one vertex's values for all slots are one contiguous row of K words) so
// that every pull step reads and writes whole rows.  Slots are independent:
// a source can be admitted into a free slot between any two iterations and
// a slot is retired as soon as its own query is complete, while the other
// slots keep iterating.  The batched entry points (g1_bfs_batch,
// g1_sssp_batch, g1_ppr_batch) and the serving loop (g1_server_*) both run
// on it.
//
// Per-slot arithmetic never depends on the other slots, the slot index or K:
//   BFS / SSSP: the fixpoint of a min-plus relaxation (order-free);
//   PPR: each lane accumulates its own column over a row's in-edges in CSR
//        order, hub rows are summed from fixed row pieces in piece order and
//        the dangling mass from fixed per-warp partials in warp order,
// so a query's result is bit-identical alone, in a batch, or admitted into a
// running batch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "internal.h"

namespace g1 {

enum SlotKind : int { kSlotBfs = 0, kSlotSssp = 1, kSlotPpr = 2 };
constexpr uint32_t kMaxSlots = 256;
// Row pieces: a vertex's in-edge range is cut into pieces of at most this
// many edges, one warp each, so hub rows spread over many warps.
constexpr uint32_t kPieceEdges = 1024;

struct Frontier;  // frontier state of one iteration (slots.cu)

// Up to 256 bits by value (kernel argument).
struct Bits256 {
    uint32_t w[8];
};

// Read-only per-graph arrays the slot kernels use, built once per graph
// (under the graph's lock) and never reallocated afterwards.
struct SlotGraph {
    const uint32_t* rp = nullptr;   // in-edge CSR
    const uint32_t* col = nullptr;
    const uint32_t* val = nullptr;  // u32 weights (SSSP)
    const uint32_t* piece_v = nullptr;
    const uint32_t* piece_e = nullptr;
    const uint32_t* piece_off = nullptr;  // first piece of each vertex (n + 1)
    const uint32_t* out_rp = nullptr;     // out-edge CSR (frontier marking), or null
    const uint32_t* out_col = nullptr;
    const uint32_t* piece_hp = nullptr;  // hub-piece index of a piece (or ~0u)
    const uint32_t* hub_v = nullptr;     // hub rows (more than one piece)
    const uint32_t* hub_hp = nullptr;    // first hub-piece index of each hub row
    const uint32_t* out_deg = nullptr;   // out-degree (PPR transition weights)
    const uint32_t* perm = nullptr;      // caller id -> internal id, or null
    uint32_t n = 0, m = 0, n_pieces = 0, n_hubs = 0, n_hub_pieces = 0;
    int sm_count = 148;
    // the next iteration's row pieces are listed while the changed vertices'
    // out-edges are below (m + n) / sparse_div
    uint32_t sparse_div = 8;
};

// Builds (once per graph) the arrays `kind` needs and fills `out`.  The
// caller holds g->mu.
g1_status slot_graph(g1_graph* g, int kind, cudaStream_t s, SlotGraph* out);

class SlotEngine {
   public:
    SlotEngine() = default;
    SlotEngine(const SlotEngine&) = delete;
    SlotEngine& operator=(const SlotEngine&) = delete;
    ~SlotEngine() { release(); }

    // Device bytes an engine of K slots needs on `g`.
    static size_t bytes(const SlotGraph& sg, int kind, uint32_t K);
    // Allocates the state for K slots (K rounded up to a multiple of 32).
    g1_status init(const SlotGraph& sg, int kind, uint32_t K, float alpha, uint32_t ppr_iters,
                   cudaStream_t s);
    void release();
    // PPR: damping and iteration count of the queries admitted from now on
    // (the damping may change only while no slot is occupied).
    g1_status set_alpha(float alpha, uint32_t ppr_iters, cudaStream_t s);
    bool ready() const { return rows_.p != nullptr; }
    int kind() const { return kind_; }
    uint32_t capacity() const { return K_; }
    uint32_t occupied() const { return n_used_; }
    uint32_t iterations() const { return it_; }
    size_t device_bytes() const;

    // Lowest free slot, or -1.
    int take_slot();
    // Enqueues the admission of cnt sources (caller vertex ids, already
    // checked < n) into the given slots (from take_slot).
    g1_status admit(const uint32_t* slots, const uint32_t* srcs, uint32_t cnt, cudaStream_t s);
    // How many iterations the next step may run (PPR: the fewest remaining
    // iterations over the occupied slots; BFS/SSSP: `want`).
    uint32_t max_step(uint32_t want) const;
    // Enqueues `iters` iterations and the read-back of the slots that
    // changed in the last one.  The caller waits for the stream before
    // finished().
    g1_status step(uint32_t iters, cudaStream_t s);
    // Slots whose query completed with the last step (host, after the wait).
    void finished(std::vector<uint32_t>* out) const;
    // Iterations the slot's query has run.
    uint32_t slot_iterations(uint32_t slot) const { return it_ - start_[slot]; }
    // Enqueues copies of cnt slots' results (caller vertex order, n 4-byte
    // values each) into device buffers outs[i].
    g1_status extract(const uint32_t* slots, uint32_t cnt, void* const* outs, cudaStream_t s);
    void free_slot(uint32_t slot);

   private:
    Frontier frontier(uint32_t it);
    Bits256 occupied_bits() const;
    // Enqueues n iterations on s, then the advance of the device iteration
    // counter: the body of a captured step.  The buffers rotate with the
    // iteration (period 6); `phase` is the completed iterations mod 6 when
    // the step runs, and each iteration reads its number from the counter.
    g1_status enqueue_iterations(uint32_t n, uint32_t phase, cudaStream_t s);
    // The executable graph of 2^i iterations starting at rotation `phase`,
    // captured on first use.
    g1_status step_graph(int i, uint32_t phase, cudaGraphExec_t* out);
    void drop_graphs();

    SlotGraph sg_;
    int kind_ = 0;
    uint32_t K_ = 0, W_ = 0, WP_ = 1;
    uint32_t it_ = 0;  // iterations run
    float alpha_ = 0.85f;
    uint32_t ppr_iters_ = 0;
    uint32_t n_used_ = 0;
    std::vector<uint8_t> used_;
    std::vector<uint32_t> start_;  // it_ when the slot was admitted
    uint32_t pull_grid_ = 1;       // blocks of 256 threads of the pull kernels
    DevBuf rows_;      // n*K: BFS levels, SSSP distances, PPR rank (buffer 0)
    DevBuf rows2_;     // PPR rank buffer 1
    DevBuf bits_[3];   // n*W: BFS frontier / SSSP changed rows, triple-buffered
    DevBuf seen_;      // n*W: BFS visited rows
    DevBuf iw_;        // n: PPR alpha / out-degree
    DevBuf hub_part_;  // n_hub_pieces*K: PPR partial sums of hub row pieces
    DevBuf dang_part_; // warps*K floats: PPR dangling partial sums per warp
    DevBuf slot_dev_;  // admission / extraction lists, slot sources, start iterations
    DevBuf chw_;       // 2 x 8 words: slots changed in the last iteration
    // Frontier-driven iterations (BFS / SSSP): a sparse iteration pulls only
    // the row pieces of vertices with a changed in-neighbour.
    DevBuf mark_;      // n: iteration a vertex was listed for
    DevBuf plist_[2];  // row pieces to pull, written one iteration ahead
    DevBuf clist_[3];  // vertices changed per iteration (their bit rows are cleared two later)
    DevBuf ctr_;       // 4 x 4 words per iteration: list size, list valid, changed count
    DevBuf ptrs_;      // K output pointers for extract
    PinnedBuf host_;   // pinned mirror of chw and staging of small uploads
    // Steps run as CUDA graphs of 2^i iterations (i < kStepGraphs) per
    // rotation phase, captured once on a private stream and replayed on the
    // caller's.
    static constexpr int kStepGraphs = 8;
    static constexpr uint32_t kPhases = 6;
    cudaGraphExec_t graphs_[kStepGraphs][kPhases] = {};
    cudaStream_t capture_ = nullptr;
    Bits256 occ_dev_{};  // occupied slots as last written to the device
    bool occ_dev_valid_ = false;
};

}  // namespace g1
