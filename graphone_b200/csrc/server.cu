// Serving loop: continuous batching of BFS / SSSP / personalized-PageRank
// queries over resident graphs.
//
// One host thread runs the loop.  Each (graph, query kind) pair has an
// executor: a slot engine (slots.cuh) on its own non-blocking stream, a
// queue of waiting queries and the queries in its slots.  A loop turn, per
// executor whose previous step has completed (event query, no blocking):
//   1. the queries whose results were enqueued last turn are complete;
//   2. slots whose query finished in the last step are extracted into the
//      queries' outputs and freed;
//   3. waiting queries take free slots (the engine's state is allocated on
//      first use, sized by free device memory);
//   4. the next step (a few iterations, sized so a step takes ~0.3 ms) is
//      launched and an event recorded behind it.
// Executors never wait for one another, so work on different graphs and
// kinds overlaps on the device, and a query joins a running batch at the
// next step boundary instead of waiting for the batch to drain.
//
// Batches pay only when many queries share a step: a step of one 32-slot
// word costs about what a full word's does, and up to a few dozen queries
// the single-source engines finish them sooner one by one.  So the server
// also has solo lanes: worker threads that each run one query at a time,
// never two of one graph at once, the next one chosen by lane_stretch (see
// dispatch_lanes: shortest expected first, with waiting time counted in), on the
// single-source engines (the calls a plain per-request user makes:
// traverse.cu's AUTO engine, which picks the near-far engine on grids, and
// pagerank.cu's SpMV PPR), each on its own stream.
//   - SSSP and BFS on graphs of small uniform degree (grids) always take a
//     lane: batched Bellman-Ford relaxes such graphs' vertices many times
//     over, and batched BFS steps through thousands of levels;
//   - the other executors are hybrid: with their slots empty and fewer than
//     a word of queries waiting (or a queue that one-by-one runs clear
//     within solo_queue_ms) their queries take the lanes; beyond that they
//     are batched on the slot engine, concurrently with the lanes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <pthread.h>

#include "internal.h"
#include "slots.cuh"

namespace g1 {
namespace {

using Clock = std::chrono::steady_clock;

constexpr double kStepTargetUs = 300.0;
constexpr uint32_t kMaxGroup = 64;

struct Request {
    uint64_t id = 0;
    uint32_t graph = 0;
    int kind = 0;
    uint32_t src = 0;
    void* out = nullptr;
    void* out_dev = nullptr;  // device-accessible address of out, or null (pageable)
    Clock::time_point t_sub, t_done;
    g1_status st = G1_OK;
    bool done = false;
};

struct Exec {
    g1_graph* g = nullptr;
    int kind = 0;
    SlotGraph sg;
    bool usable = false;  // the graph supports this kind
    SlotEngine eng;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    bool inflight = false;
    bool stepped = false;  // the in-flight work includes a step
    uint32_t step_iters = 0;
    Clock::time_point t_launch, last_busy;
    uint32_t group = 1;
    std::deque<Request*> pending;
    std::vector<Request*> slot_req;  // query of each slot
    std::vector<Request*> retiring;  // results enqueued before ev
    DevBuf staging;                  // pageable outputs
    // Where the executor's queries run (init_exec):
    //  - lane_only: SSSP and BFS on graphs of small uniform degree (grids)
    //    always run one at a time on the server's solo lanes, where the AUTO
    //    engine picks the near-far engine (batched Bellman-Ford relaxes such
    //    graphs' vertices many times over; batched BFS steps through
    //    thousands of levels);
    //  - hybrid: while its slots are empty and the queue is short
    //    (lane_mode), the executor's queries go to the solo lane too (SSSP /
    //    BFS: traverse.cu's AUTO engine; PPR: pagerank.cu's SpMV schedules,
    //    4 bytes per edge and iteration where a slot step reads a 128-byte
    //    rank row per edge); beyond that they are batched on the slot engine;
    //  - neither: always batched (solo_queue_ms < 0, or SSSP / BFS without
    //    the out-edge CSR the AUTO engine pushes over).
    bool lane_only = false;
    bool hybrid = false;
    std::atomic<bool> on_lane{false};  // one of its queries runs on a lane
    std::atomic<double> solo_ms{0.0};  // moving average of its lane query time (0: none yet)
    std::atomic<uint32_t> solo_runs{0};  // lane queries run
};

// A hybrid executor batches on its slot engine once at least kSlotMinQueue
// queries (one 32-slot word) wait and running them one by one would take
// longer than the server's solo_queue_ms (default kSoloQueueMs).  Below a
// word of queries a slot step costs about as much as a full word's, which
// single-source runs beat.
constexpr double kSoloQueueMs = 20.0;
constexpr double kLaneStretch = 2.0;
constexpr size_t kSlotMinQueue = 32;
// One lane by default: with two, the concurrent queries slowed each other
// (p99 of the bench's mixed stream 1-10% above one lane's at every load; the
// near-far kernel, a cooperative launch over every SM, waits for the other
// lane's kernels to drain).
constexpr uint32_t kDefaultLanes = 1;

struct Lane {
    std::thread th;
    std::mutex mu;  // req, exec, stop
    std::condition_variable cv;
    Request* req = nullptr;
    Exec* exec = nullptr;
    bool stop = false;
    std::atomic<bool> busy{false};
    std::atomic<const g1_graph*> graph{nullptr};  // the graph of its query, while busy
};

}  // namespace
}  // namespace g1

using namespace g1;

struct g1_server {
    int device = 0;
    uint32_t max_batch = 256;
    uint64_t reserve = 0, limit = 0;
    float alpha = 0.85f;
    uint32_t ppr_iters = 20;
    uint32_t idle_ms = 0;  // 0: engine state is kept until memory is needed
    double solo_queue_ms = kSoloQueueMs;  // negative: never solo
    double lane_stretch = kLaneStretch;   // <= 0: the lanes take the oldest query first
    std::vector<std::unique_ptr<Exec>> execs;  // graph * 3 + kind
    std::mutex mu;                             // everything below
    std::condition_variable cv_in, cv_done;
    std::deque<Request*> inbox;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread th;
    std::vector<double> lat;
    uint64_t submitted = 0, completed = 0, failed = 0, steps = 0;
    uint32_t max_occ = 0;
    bool have_first = false;
    Clock::time_point t_first, t_last;
    std::atomic<uint64_t> dev_bytes{0};
    std::atomic<uint32_t> engines{0};
    std::mutex graphs_mu;  // add_graph vs the loop's view of execs
    std::atomic<size_t> n_execs{0};
    // The solo lanes: worker threads each running one query at a time on
    // the single-source engines (the engines of plain per-request calls),
    // never two of one graph.
    std::vector<std::unique_ptr<g1::Lane>> lanes;
};

namespace g1 {
namespace {

void complete(g1_server* S, std::vector<Request*>& rs, g1_status st) {
    if (rs.empty()) return;
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (Request* r : rs) {
            r->st = st;
            r->t_done = now;
            r->done = true;
            if (st == G1_OK) {
                ++S->completed;
                S->lat.push_back(std::chrono::duration<double, std::milli>(now - r->t_sub).count());
            } else {
                ++S->failed;
            }
            S->t_last = now;
        }
    }
    rs.clear();
    S->cv_done.notify_all();
}

void complete_one(g1_server* S, Request* r, g1_status st) {
    std::vector<Request*> v{r};
    complete(S, v, st);
}

bool holds_memory(const Exec& E) { return E.eng.ready(); }

void release_engine(g1_server* S, Exec& E) {
    if (!holds_memory(E)) return;
    S->dev_bytes -= E.eng.device_bytes();
    S->engines -= 1;
    E.eng.release();
    E.staging.release();
}

bool idle(const Exec& E) {
    return holds_memory(E) && E.eng.occupied() == 0 && !E.inflight && E.pending.empty() &&
           E.retiring.empty() && !E.on_lane.load();
}

// Frees the state of one idle engine other than `self`.
bool release_one_idle(g1_server* S, const Exec* self) {
    const size_t ne = S->n_execs.load();
    for (size_t i = 0; i < ne; ++i) {
        Exec& E = *S->execs[i];
        if (&E != self && idle(E)) {
            release_engine(S, E);
            return true;
        }
    }
    return false;
}

bool others_hold_memory(g1_server* S, const Exec* self) {
    const size_t ne = S->n_execs.load();
    for (size_t i = 0; i < ne; ++i) {
        const Exec& E = *S->execs[i];
        if (&E != self && holds_memory(E)) return true;
    }
    return false;
}

// Free device memory on the current device, counting the library's cache of
// released blocks (reusable, or freed when an allocation needs the room).
size_t device_free_bytes() {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return free_b;
    }
    return free_b + dev_block_cached(dev);
}

// Allocates the executor's engine: the largest slot count (halving from
// max_batch down to 32) whose state fits the free device memory minus the
// reserve and the server's limit.
bool allocate(g1_server* S, Exec& E) {
    for (uint32_t K = (S->max_batch + 31) / 32 * 32;;) {
        const size_t need = SlotEngine::bytes(E.sg, E.kind, K);
        const size_t free_b = device_free_bytes();
        const bool fits = need + S->reserve <= free_b && (!S->limit || S->dev_bytes + need <= S->limit);
        if (!fits && release_one_idle(S, &E)) continue;
        if (fits) {
            if (E.eng.init(E.sg, E.kind, K, S->alpha, S->ppr_iters, E.s) == G1_OK) {
                S->dev_bytes += E.eng.device_bytes();
                S->engines += 1;
                E.slot_req.assign(E.eng.capacity(), nullptr);
                E.group = 1;
                return true;
            }
            E.eng.release();
            cudaGetLastError();
        }
        if (K <= 32) return false;
        K = std::max<uint32_t>(32, K / 2);
    }
}

void fail_exec(g1_server* S, Exec& E, g1_status st) {
    std::vector<Request*> rs;
    for (auto& r : E.slot_req)
        if (r) {
            rs.push_back(r);
            r = nullptr;
        }
    rs.insert(rs.end(), E.retiring.begin(), E.retiring.end());
    E.retiring.clear();
    complete(S, rs, st);
    E.inflight = false;
    release_engine(S, E);
}

// Extracts the finished slots' results (enqueued on E.s).
g1_status retire(g1_server* S, Exec& E, const std::vector<uint32_t>& fin) {
    if (fin.empty()) return G1_OK;
    const size_t row = (size_t)E.g->n * 4;
    std::vector<uint32_t> ext_s;
    std::vector<void*> ext_o;
    std::vector<std::pair<Request*, size_t>> host;
    for (uint32_t sl : fin) {
        Request* r = E.slot_req[sl];
        if (!r) continue;
        ext_s.push_back(sl);
        if (r->out_dev) {
            ext_o.push_back(r->out_dev);
        } else {
            host.emplace_back(r, host.size());
            ext_o.push_back(nullptr);
        }
    }
    if (!host.empty()) {
        G1_TRY(E.staging.ensure(host.size() * row + 16));
        size_t h = 0;
        for (size_t i = 0; i < ext_o.size(); ++i)
            if (!ext_o[i]) ext_o[i] = E.staging.as<char>() + (h++) * row;
    }
    G1_TRY(E.eng.extract(ext_s.data(), (uint32_t)ext_s.size(), ext_o.data(), E.s));
    for (auto& hr : host)
        G1_CUDA(cudaMemcpyAsync(hr.first->out, E.staging.as<char>() + hr.second * row, row,
                                cudaMemcpyDeviceToHost, E.s));
    for (uint32_t sl : fin) {
        if (E.slot_req[sl]) E.retiring.push_back(E.slot_req[sl]);
        E.slot_req[sl] = nullptr;
        E.eng.free_slot(sl);
    }
    return G1_OK;
}

// A solo lane's thread: runs the query handed to it on the single-source
// engines (the calls of g1_sssp / g1_bfs with G1_ENGINE_AUTO and of g1_ppr),
// on its own stream, then completes it.
void lane_worker(g1_server* S, Lane* L) {
    pthread_setname_np(pthread_self(), "g1-lane");
    cudaSetDevice(S->device);
    cudaStream_t ls = nullptr;
    const bool have_stream = cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking) == cudaSuccess;
    if (!have_stream) cudaGetLastError();
    for (;;) {
        Request* r = nullptr;
        Exec* E = nullptr;
        {
            std::unique_lock<std::mutex> lk(L->mu);
            L->cv.wait(lk, [&] { return L->req != nullptr || L->stop; });
            if (!L->req) break;
            r = L->req;
            E = L->exec;
        }
        g1_status st = G1_ERR_DEVICE;
        const auto t0 = Clock::now();
        if (have_stream) {
            std::lock_guard<std::mutex> lk(E->g->mu);
            if (E->kind == kSlotPpr)
                st = ppr_locked(E->g, r->src, S->alpha, S->ppr_iters, static_cast<float*>(r->out), ls);
            else
                st = traverse_locked(E->g, r->src, G1_ENGINE_AUTO, E->kind == kSlotBfs,
                                     static_cast<uint32_t*>(r->out), nullptr, ls);
        }
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        // the first lane query of an executor also pays one-time costs
        // (engine state, plans, captured CUDA graphs): it sets no estimate
        if (E->solo_runs.fetch_add(1) > 0) {
            const double prev = E->solo_ms.load();
            E->solo_ms.store(prev == 0.0 ? ms : 0.75 * prev + 0.25 * ms);
        }
        complete_one(S, r, st);
        {
            std::lock_guard<std::mutex> lk(L->mu);
            L->req = nullptr;
            L->exec = nullptr;
        }
        E->on_lane.store(false);
        L->graph.store(nullptr);
        L->busy.store(false);
    }
    if (have_stream) cudaStreamDestroy(ls);
}

bool lanes_busy(const g1_server* S) {
    for (const auto& L : S->lanes)
        if (L->busy.load()) return true;
    return false;
}

// Whether the executor's waiting queries go to the solo lane: always for
// lane_only executors; for hybrid ones while their slots are empty, the
// last step's results are completed and the queue is short.
bool lane_mode(const g1_server* S, const Exec& E) {
    if (E.lane_only) return true;
    if (!E.hybrid || S->solo_queue_ms < 0.0) return false;
    if (E.eng.occupied() > 0 || E.inflight || !E.retiring.empty()) return false;
    const double solo = E.solo_ms.load();
    return !(E.pending.size() >= kSlotMinQueue && solo > 0.0 &&
             (double)E.pending.size() * solo > S->solo_queue_ms);
}

// Hands each free lane the oldest waiting query of the executors in lane
// mode whose graph no other lane is working on (the calls of one graph
// would only wait for each other's lock).
// Which waiting query a free lane takes: the head of the executor with the
// lowest score, expected_ms - waited_ms / lane_stretch (expected_ms: the
// executor's moving average of its lane queries, 0 until one has run).
// Short queries go first, so a burst of them does not queue behind a long
// traversal, while a query's own wait keeps lowering its score: a query
// expected to take T ms longer than the others waits at most about
// lane_stretch * T before it is next.  lane_stretch <= 0: oldest first.
bool dispatch_lanes(g1_server* S, bool stopping) {
    if (stopping) return false;
    bool any = false;
    const auto now = Clock::now();
    for (auto& Lp : S->lanes) {
        Lane* L = Lp.get();
        if (L->busy.load()) continue;
        Exec* best = nullptr;
        double best_score = 0.0;
        const size_t ne = S->n_execs.load();
        for (size_t i = 0; i < ne; ++i) {
            Exec& E = *S->execs[i];
            if (E.pending.empty() || !lane_mode(S, E)) continue;
            bool graph_busy = false;
            for (const auto& O : S->lanes) graph_busy |= O->busy.load() && O->graph.load() == E.g;
            if (graph_busy) continue;
            const double waited = std::chrono::duration<double, std::milli>(now - E.pending.front()->t_sub).count();
            const double score =
                S->lane_stretch > 0.0 ? E.solo_ms.load() - waited / S->lane_stretch : -waited;
            if (!best || score < best_score) {
                best = &E;
                best_score = score;
            }
        }
        if (!best) break;  // no other lane would find one either
        Request* r = best->pending.front();
        best->pending.pop_front();
        best->on_lane.store(true);
        L->graph.store(best->g);
        L->busy.store(true);
        {
            std::lock_guard<std::mutex> lk(L->mu);
            L->req = r;
            L->exec = best;
        }
        if (!L->th.joinable()) L->th = std::thread(lane_worker, S, L);
        L->cv.notify_one();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            ++S->steps;
            S->max_occ = std::max(S->max_occ, 1u);
        }
        best->last_busy = Clock::now();
        any = true;
    }
    return any;
}

// One turn of one executor; true if anything happened.
bool service(g1_server* S, Exec& E, bool stopping, std::vector<uint32_t>& fin) {
    if (E.lane_only) return false;  // the lane runs its queries
    bool progress = false;
    if (E.inflight) {
        const cudaError_t q = cudaEventQuery(E.ev);
        if (q == cudaErrorNotReady) return false;
        progress = true;
        E.inflight = false;
        if (q != cudaSuccess) {
            cudaGetLastError();
            fail_exec(S, E, G1_ERR_DEVICE);
            return true;
        }
        complete(S, E.retiring, G1_OK);
        if (E.stepped) {
            const double us = std::chrono::duration<double, std::micro>(Clock::now() - E.t_launch).count();
            const double per_it = us / std::max<uint32_t>(1, E.step_iters);
            E.group = (uint32_t)std::min<double>(kMaxGroup, std::max(1.0, kStepTargetUs / std::max(per_it, 1.0)));
            E.eng.finished(&fin);
            if (retire(S, E, fin) != G1_OK) {
                fail_exec(S, E, G1_ERR_DEVICE);
                return true;
            }
            // a traversal that ran longer than any shortest path can
            for (uint32_t i = 0; i < E.eng.capacity() && E.kind != kSlotPpr; ++i)
                if (E.slot_req[i] && E.eng.slot_iterations(i) > E.g->n + 2) {
                    complete_one(S, E.slot_req[i], G1_ERR_TIMEOUT);
                    E.slot_req[i] = nullptr;
                    E.eng.free_slot(i);
                }
        }
    }
    if (lane_mode(S, E)) return progress;  // its queries wait for the lane
    // admission
    if (!stopping && !E.pending.empty()) {
        if (!E.eng.ready() && !allocate(S, E) && !others_hold_memory(S, &E)) {
            std::vector<Request*> rs(E.pending.begin(), E.pending.end());
            E.pending.clear();
            complete(S, rs, G1_ERR_OOM);
            progress = true;
        }
        if (E.eng.ready()) {
            std::vector<uint32_t> adm_s, adm_v;
            while (!E.pending.empty()) {
                const int sl = E.eng.take_slot();
                if (sl < 0) break;
                Request* r = E.pending.front();
                E.pending.pop_front();
                E.slot_req[sl] = r;
                adm_s.push_back((uint32_t)sl);
                adm_v.push_back(r->src);
            }
            if (!adm_s.empty()) {
                progress = true;
                if (E.eng.admit(adm_s.data(), adm_v.data(), (uint32_t)adm_s.size(), E.s) != G1_OK) {
                    fail_exec(S, E, G1_ERR_DEVICE);
                    return true;
                }
            }
        }
    }
    E.stepped = false;
    if (E.eng.ready() && E.eng.occupied() > 0) {
        E.step_iters = E.eng.max_step(E.group);
        if (E.eng.step(E.step_iters, E.s) != G1_OK) {
            fail_exec(S, E, G1_ERR_DEVICE);
            return true;
        }
        E.stepped = true;
        E.t_launch = Clock::now();
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->steps;
        S->max_occ = std::max(S->max_occ, E.eng.occupied());
    }
    if (E.stepped || !E.retiring.empty()) {
        if (cudaEventRecord(E.ev, E.s) != cudaSuccess) {
            cudaGetLastError();
            fail_exec(S, E, G1_ERR_DEVICE);
            return true;
        }
        E.inflight = true;
        E.last_busy = Clock::now();
        progress = true;
    }
    return progress;
}

bool busy(const Exec& E) {
    return E.inflight || E.eng.occupied() > 0 || !E.pending.empty() || E.on_lane.load();
}

void loop(g1_server* S) {
    pthread_setname_np(pthread_self(), "g1-serve");
    cudaSetDevice(S->device);
    std::vector<Request*> fresh;
    std::vector<uint32_t> fin;
    for (;;) {
        bool stopping = false;
        bool any_busy = false;
        const size_t ne = S->n_execs.load();
        for (size_t i = 0; i < ne; ++i) any_busy |= busy(*S->execs[i]);
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->inbox.empty() && !any_busy && !S->stop)
                S->cv_in.wait_for(lk, std::chrono::milliseconds(20));
            fresh.assign(S->inbox.begin(), S->inbox.end());
            S->inbox.clear();
            stopping = S->stop;
        }
        for (Request* r : fresh) S->execs[(size_t)r->graph * 3 + r->kind]->pending.push_back(r);
        if (stopping) {
            std::vector<Request*> rs;
            for (size_t i = 0; i < ne; ++i) {
                Exec& E = *S->execs[i];
                rs.insert(rs.end(), E.pending.begin(), E.pending.end());
                E.pending.clear();
            }
            complete(S, rs, G1_ERR_INVALID);
        }
        bool progress = false;
        for (size_t i = 0; i < ne; ++i) progress |= service(S, *S->execs[i], stopping, fin);
        progress |= dispatch_lanes(S, stopping);
        const auto now = Clock::now();
        bool still = lanes_busy(S);
        for (size_t i = 0; i < ne; ++i) {
            Exec& E = *S->execs[i];
            still |= busy(E) || !E.retiring.empty();
            if (S->idle_ms && idle(E) &&
                std::chrono::duration<double, std::milli>(now - E.last_busy).count() > S->idle_ms)
                release_engine(S, E);
        }
        if (stopping && !still) break;
        if (!progress && still) std::this_thread::sleep_for(std::chrono::microseconds(10));
    }
    for (size_t i = 0; i < S->n_execs.load(); ++i) release_engine(S, *S->execs[i]);
}

g1_status server_status_of(const Request& r) { return r.st; }

}  // namespace
}  // namespace g1

extern "C" g1_status g1_server_create(int device, const g1_server_config* cfg, g1_server** out) {
    if (!out) return fail(G1_ERR_INVALID, "g1_server_create: null output");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return fail(G1_ERR_INVALID, "g1_server_create: no such device");
    }
    std::unique_ptr<g1_server> S(new g1_server());
    S->device = device;
    if (cfg) {
        if (cfg->max_batch > kMaxSlots) return fail(G1_ERR_INVALID, "max_batch above 256");
        if (cfg->max_batch) S->max_batch = cfg->max_batch;
        S->reserve = cfg->reserve_bytes;
        S->limit = cfg->memory_limit;
        if (cfg->ppr_alpha != 0.0f) {
            if (!(cfg->ppr_alpha > 0.0f && cfg->ppr_alpha < 1.0f))
                return fail(G1_ERR_INVALID, "ppr_alpha must be in (0, 1)");
            S->alpha = cfg->ppr_alpha;
        }
        if (cfg->ppr_iters) S->ppr_iters = cfg->ppr_iters;
        if (cfg->idle_release_ms) S->idle_ms = cfg->idle_release_ms;
        if (cfg->solo_queue_ms) S->solo_queue_ms = cfg->solo_queue_ms;
        if (cfg->solo_lanes > 16) return fail(G1_ERR_INVALID, "solo_lanes above 16");
        if (cfg->lane_stretch != 0.0f) S->lane_stretch = cfg->lane_stretch;
    }
    // executors for up to 4096 graphs; the vector never reallocates
    S->execs.reserve(3 * 4096);
    const uint32_t nl = cfg && cfg->solo_lanes ? cfg->solo_lanes : kDefaultLanes;
    for (uint32_t i = 0; i < nl; ++i) S->lanes.emplace_back(new Lane());
    S->th = std::thread(loop, S.get());
    *out = S.release();
    return G1_OK;
}

namespace g1 {
namespace {

// The executor of one (graph, query kind): its stream and event, and the
// slot view of the graph when the graph supports the kind.
g1_status init_exec(g1_graph* g, int kind, Exec& E) {
    E.g = g;
    E.kind = kind;
    G1_CUDA(cudaStreamCreateWithFlags(&E.s, cudaStreamNonBlocking));
    G1_CUDA(cudaEventCreateWithFlags(&E.ev, cudaEventDisableTiming));
    E.last_busy = Clock::now();
    if (kind == kSlotSssp && g->vtype != G1_U32) return G1_OK;
    std::lock_guard<std::mutex> lk(g->mu);
    G1_TRY(slot_graph(g, kind, E.s, &E.sg));
    if ((kind == kSlotSssp || kind == kSlotBfs) && nearfar_suits(g)) {
        E.lane_only = true;
        uint32_t delta = 0;  // derived once per graph, ahead of the first query
        G1_TRY(nearfar_delta(g, kind == kSlotBfs, E.s, &delta));
    }
    E.hybrid = !E.lane_only && (kind == kSlotPpr || g->o[0].present);
    E.usable = true;
    return G1_OK;
}

}  // namespace
}  // namespace g1

extern "C" g1_status g1_server_add_graph(g1_server* S, g1_graph* g, uint32_t* graph_id) {
    if (!S || !g || !graph_id) return fail(G1_ERR_INVALID, "g1_server_add_graph: null argument");
    if (g->device != S->device) return fail(G1_ERR_INVALID, "graph lives on another device");
    if (!g->o[1].present)
        return fail(G1_ERR_UNSUPPORTED, "serving needs the in-edge CSR (G1_GRAPH_BUILD_OTHER)");
    std::lock_guard<std::mutex> add_lk(S->graphs_mu);
    const size_t ne = S->n_execs.load();
    if (ne + 3 > S->execs.capacity()) return fail(G1_ERR_INVALID, "too many graphs");
    DeviceGuard dg(g->device);
    std::unique_ptr<Exec> ex[3];
    for (int kind = 0; kind < 3; ++kind) {
        ex[kind].reset(new Exec());
        const g1_status st = init_exec(g, kind, *ex[kind]);
        if (st != G1_OK) {
            // nothing of this graph is visible to the loop yet
            for (auto& e : ex) {
                if (!e) continue;
                if (e->ev) cudaEventDestroy(e->ev);
                if (e->s) cudaStreamDestroy(e->s);
            }
            return st;
        }
    }
    // the loop only reads execs[0, n_execs)
    for (auto& e : ex) S->execs.push_back(std::move(e));
    *graph_id = (uint32_t)(ne / 3);
    S->n_execs.store(ne + 3);
    return G1_OK;
}

extern "C" g1_status g1_server_submit(g1_server* S, uint32_t graph_id, g1_query_kind kind, uint32_t src,
                                      void* out, uint64_t* ticket) {
    if (!S || !out || !ticket) return fail(G1_ERR_INVALID, "g1_server_submit: null argument");
    if ((size_t)graph_id * 3 + 3 > S->n_execs.load()) return fail(G1_ERR_INVALID, "unknown graph id");
    if (kind < G1_QUERY_BFS || kind > G1_QUERY_PPR) return fail(G1_ERR_INVALID, "unknown query kind");
    Exec& E = *S->execs[(size_t)graph_id * 3 + kind];
    if (!E.usable) return fail(G1_ERR_INVALID, "SSSP needs u32 edge weights");
    if (src >= E.g->n) return fail(G1_ERR_INVALID, "source vertex out of range");
    std::unique_ptr<Request> r(new Request());
    r->graph = graph_id;
    r->kind = kind;
    r->src = src;
    r->out = out;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, out) == cudaSuccess) {
        if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)
            r->out_dev = out;
        else if (a.type == cudaMemoryTypeHost && a.devicePointer)
            r->out_dev = a.devicePointer;
    } else {
        cudaGetLastError();
    }
    r->t_sub = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stop) return fail(G1_ERR_INVALID, "server is stopping");
        r->id = S->next_id++;
        *ticket = r->id;
        S->inbox.push_back(r.get());
        if (!S->have_first) {
            S->have_first = true;
            S->t_first = r->t_sub;
        }
        ++S->submitted;
        S->reqs.emplace(r->id, std::move(r));
    }
    S->cv_in.notify_one();
    return G1_OK;
}

static g1_status take_result(g1_server* S, uint64_t ticket, double* latency_ms) {
    auto it = S->reqs.find(ticket);
    const Request& r = *it->second;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_sub).count();
    const g1_status st = server_status_of(r);
    S->reqs.erase(it);
    if (st != G1_OK) return fail(st, "query failed in the serving loop");
    return G1_OK;
}

extern "C" g1_status g1_server_poll(g1_server* S, uint64_t ticket, int* done, double* latency_ms) {
    if (!S || !done) return fail(G1_ERR_INVALID, "g1_server_poll: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(G1_ERR_INVALID, "unknown ticket");
    *done = it->second->done ? 1 : 0;
    if (!*done) return G1_OK;
    return take_result(S, ticket, latency_ms);
}

extern "C" g1_status g1_server_wait(g1_server* S, uint64_t ticket, uint32_t timeout_ms, double* latency_ms) {
    if (!S) return fail(G1_ERR_INVALID, "g1_server_wait: null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(G1_ERR_INVALID, "unknown ticket");
    Request* r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_ms) {
        if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return fail(G1_ERR_TIMEOUT, "query not done within the timeout");
    } else {
        S->cv_done.wait(lk, ready);
    }
    return take_result(S, ticket, latency_ms);
}

extern "C" g1_status g1_server_stats(g1_server* S, int reset, g1_server_metrics* out) {
    if (!S || !out) return fail(G1_ERR_INVALID, "g1_server_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    std::vector<double> lat;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        lat = S->lat;
        out->submitted = S->submitted;
        out->completed = S->completed;
        out->failed = S->failed;
        out->steps = S->steps;
        out->max_occupancy = S->max_occ;
        if (S->have_first && S->completed) {
            const double s = std::chrono::duration<double>(S->t_last - S->t_first).count();
            out->queries_per_s = s > 0 ? (double)S->completed / s : 0.0;
        }
        if (reset) {
            S->lat.clear();
            S->submitted = S->completed = S->failed = S->steps = 0;
            S->max_occ = 0;
            S->have_first = false;
        }
    }
    out->engines = S->engines.load();
    out->device_bytes = S->dev_bytes.load();
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double q) {
            const double pos = q * (double)(lat.size() - 1);
            const size_t i = (size_t)pos;
            const double f = pos - (double)i;
            return i + 1 < lat.size() ? lat[i] * (1.0 - f) + lat[i + 1] * f : lat[i];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        double sum = 0;
        for (double x : lat) sum += x;
        out->mean_ms = sum / (double)lat.size();
        out->max_ms = lat.back();
    }
    return G1_OK;
}

extern "C" g1_status g1_server_destroy(g1_server* S) {
    if (!S) return G1_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_in.notify_all();
    if (S->th.joinable()) S->th.join();
    // the loop ended only after the lanes' last queries completed
    for (auto& L : S->lanes) {
        {
            std::lock_guard<std::mutex> lk(L->mu);
            L->stop = true;
        }
        L->cv.notify_all();
        if (L->th.joinable()) L->th.join();
    }
    {
        DeviceGuard dg(S->device);
        for (auto& e : S->execs) {
            if (e->s) cudaStreamSynchronize(e->s);
            if (e->ev) cudaEventDestroy(e->ev);
            if (e->s) cudaStreamDestroy(e->s);
        }
    }
    delete S;
    return G1_OK;
}
