// Batched multi-source entry points: k BFS, SSSP or personalized-PageRank
// queries on one graph run through the graph's slot engine, at most 256 at
// a time; a slot whose query finished is refilled with the next source
// while the others keep iterating.  Results are source-major (out[i*n + v]),
// the layout of k single-source calls, and bit-identical to them.
#include <algorithm>
#include <chrono>
#include <memory>
#include <vector>

#include "g1/common.cuh"
#include "internal.h"
#include "slots.cuh"

namespace g1 {
namespace {

// Iterations per step grow while a step is shorter than this (host round
// trips dominate) and shrink while it is longer than the upper bound.
constexpr double kStepLowUs = 200.0, kStepHighUs = 2000.0;
constexpr uint32_t kMaxGroup = 64;

g1_status run_queries(g1_graph* g, int kind, const uint32_t* srcs_in, uint32_t k, void* out,
                      uint32_t* iters_out, float alpha, uint32_t ppr_iters, uint32_t cap,
                      cudaStream_t s) {
    const uint32_t n = g->n;
    if (iters_out) *iters_out = 0;
    if (k == 0) return G1_OK;
    std::vector<uint32_t> src(k);
    if (is_device_ptr(srcs_in)) {
        G1_CUDA(cudaMemcpyAsync(src.data(), srcs_in, (size_t)k * 4, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
    } else {
        std::copy(srcs_in, srcs_in + k, src.begin());
    }
    for (uint32_t v : src)
        if (v >= n) return fail(G1_ERR_INVALID, "source vertex out of range");
    SlotGraph sg;
    G1_TRY(slot_graph(g, kind, s, &sg));
    auto& eng = g->slot_cache[kind];
    const uint32_t K = std::min<uint32_t>(cap, (std::min<uint32_t>(k, cap) + 31) / 32 * 32);
    if (!eng) eng = std::make_shared<SlotEngine>();
    if (!eng->ready() || eng->capacity() != K)
        G1_TRY(eng->init(sg, kind, K, alpha, ppr_iters, s));
    else
        G1_TRY(eng->set_alpha(alpha, ppr_iters, s));

    const bool dev_out = is_device_ptr(out);
    char* out_b = static_cast<char*>(out);
    const size_t row_bytes = (size_t)n * 4;
    const uint32_t chunk = dev_out ? kMaxSlots : 32;
    DevBuf staging;
    if (!dev_out) G1_TRY(staging.ensure(std::min<uint32_t>(chunk, K) * row_bytes + 16));

    std::vector<int64_t> slot_q(eng->capacity(), -1);
    std::vector<uint32_t> adm_s, adm_v, fin, ext_s;
    std::vector<void*> ext_o;
    uint32_t next = 0, done = 0, group = 1, max_it = 0;
    const bool no_steps = kind == kSlotPpr && ppr_iters == 0;
    while (done < k) {
        adm_s.clear();
        adm_v.clear();
        while (next < k) {
            const int sl = eng->take_slot();
            if (sl < 0) break;
            slot_q[sl] = next;
            adm_s.push_back((uint32_t)sl);
            adm_v.push_back(src[next]);
            ++next;
        }
        G1_TRY(eng->admit(adm_s.data(), adm_v.data(), (uint32_t)adm_s.size(), s));
        const auto t0 = std::chrono::steady_clock::now();
        if (!no_steps) G1_TRY(eng->step(eng->max_step(group), s));
        G1_CUDA(cudaStreamSynchronize(s));
        const double us =
            std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
        if (kind != kSlotPpr) {
            if (us < kStepLowUs) group = std::min(kMaxGroup, group * 2);
            if (us > kStepHighUs) group = std::max(1u, group / 2);
        }
        eng->finished(&fin);
        for (size_t c0 = 0; c0 < fin.size(); c0 += chunk) {
            const size_t c1 = std::min(fin.size(), c0 + chunk);
            ext_s.assign(fin.begin() + c0, fin.begin() + c1);
            ext_o.clear();
            for (size_t c = c0; c < c1; ++c) {
                const size_t q = (size_t)slot_q[fin[c]];
                ext_o.push_back(dev_out ? (void*)(out_b + q * row_bytes)
                                        : (void*)(staging.as<char>() + (c - c0) * row_bytes));
            }
            G1_TRY(eng->extract(ext_s.data(), (uint32_t)ext_s.size(), ext_o.data(), s));
            if (!dev_out) {
                for (size_t c = c0; c < c1; ++c) {
                    const size_t q = (size_t)slot_q[fin[c]];
                    G1_CUDA(cudaMemcpyAsync(out_b + q * row_bytes, ext_o[c - c0], row_bytes,
                                            cudaMemcpyDeviceToHost, s));
                }
            }
            G1_CUDA(cudaStreamSynchronize(s));  // extraction staging is reused
        }
        for (uint32_t sl : fin) {
            max_it = std::max(max_it, eng->slot_iterations(sl));
            slot_q[sl] = -1;
            eng->free_slot(sl);
            ++done;
        }
        if (!fin.empty() || done == k || kind == kSlotPpr) continue;
        for (uint32_t i = 0; i < eng->capacity(); ++i)
            if (slot_q[i] >= 0 && eng->slot_iterations(i) > n + 2)
                return fail(G1_ERR_TIMEOUT, "multi-source traversal did not converge");
    }
    if (iters_out) *iters_out = max_it;
    return G1_OK;
}

g1_status entry(g1_graph* g, int kind, const uint32_t* srcs, uint32_t k, void* out, uint32_t* iters_out,
                float alpha, uint32_t ppr_iters, uint32_t cap, void* stream) {
    if (!g || (k && (!srcs || !out))) return fail(G1_ERR_INVALID, "multi-source query: bad argument");
    if (kind == kSlotPpr && !(alpha > 0.0f && alpha < 1.0f))
        return fail(G1_ERR_INVALID, "personalized PageRank: damping must be in (0, 1)");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    return run_queries(g, kind, srcs, k, out, iters_out, alpha, ppr_iters, cap, as_stream(stream));
}

// Caller ids of up to k vertices with out-edges, evenly spread over the
// internal order (the push side's CSR).
g1_status tune_sources(g1_graph* g, uint32_t k, cudaStream_t s, std::vector<uint32_t>* out) {
    const int t = push_side(g);
    std::vector<uint32_t> rp((size_t)g->n + 1);
    G1_CUDA(cudaMemcpyAsync(rp.data(), g->o[t].rp, rp.size() * 4, cudaMemcpyDeviceToHost, s));
    std::vector<uint32_t> iperm;
    if (g->relabeled) {
        iperm.resize(g->n);
        G1_CUDA(cudaMemcpyAsync(iperm.data(), g->iperm.p, (size_t)g->n * 4, cudaMemcpyDeviceToHost, s));
    }
    G1_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> cand;
    for (uint32_t v = 0; v < g->n; ++v)
        if (rp[v + 1] > rp[v]) cand.push_back(v);
    out->clear();
    if (cand.empty()) return G1_OK;
    for (uint32_t i = 0; i < k && i < cand.size(); ++i) {
        const uint32_t v = cand[(size_t)i * cand.size() / std::min<size_t>(k, cand.size())];
        out->push_back(g->relabeled ? iperm[v] : v);
    }
    return G1_OK;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace g1

using namespace g1;

// Times SSSP from `n_sources` spread sources under each candidate push/pull
// threshold and keeps the fastest: the single-source AUTO engine's
// (m / push_div, push while the frontier's out-degree sum is below it) and
// the slot engines' ((m + n) / slot_div, sparse iterations while the changed
// vertices' out-edges are below it).
extern "C" g1_status g1_autotune_traversal(g1_graph* g, uint32_t n_sources, uint32_t* push_div,
                                           uint32_t* slot_div, void* stream) {
    if (!g) return fail(G1_ERR_INVALID, "g1_autotune_traversal: null graph");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStream_t s = as_stream(stream);
    const uint32_t k = std::min<uint32_t>(64, n_sources ? n_sources : 16);
    std::vector<uint32_t> src;
    G1_TRY(tune_sources(g, k, s, &src));
    if (!src.empty() && g->vtype == G1_U32) {
        uint32_t* out = nullptr;
        G1_TRY(g->ws.get("tune_dist", g->n, &out));
        // single-source AUTO: push/pull applies unless the near-far engine runs
        if (g->o[0].present && g->o[1].present && !nearfar_suits(g)) {
            const uint32_t cands[] = {4, 8, 16, 32, 64, 128};
            double best = 1e300;
            uint32_t best_div = g->push_div;
            for (uint32_t d : cands) {
                g->push_div = d;
                G1_TRY(traverse_locked(g, src[0], G1_ENGINE_AUTO, false, out, nullptr, s));
                const auto t0 = std::chrono::steady_clock::now();
                for (uint32_t v : src) G1_TRY(traverse_locked(g, v, G1_ENGINE_AUTO, false, out, nullptr, s));
                G1_CUDA(cudaStreamSynchronize(s));
                const double t = seconds_since(t0);
                if (t < best) {
                    best = t;
                    best_div = d;
                }
            }
            g->push_div = best_div;
        }
        // slot engines: batched SSSP over the same sources
        if (g->o[1].present) {
            const uint32_t kb = std::min<uint32_t>((uint32_t)src.size(), 32);
            uint32_t* bout = nullptr;
            G1_TRY(g->ws.get("tune_batch", (size_t)kb * g->n, &bout));
            const uint32_t cands[] = {2, 4, 8, 16, 32};
            double best = 1e300;
            uint32_t best_div = g->slot_div;
            for (uint32_t d : cands) {
                g->slot_div = d;
                g->slot_cache[kSlotSssp].reset();  // its captured steps hold the threshold
                G1_TRY(run_queries(g, kSlotSssp, src.data(), kb, bout, nullptr, 0.85f, 0, kMaxSlots, s));
                const auto t0 = std::chrono::steady_clock::now();
                G1_TRY(run_queries(g, kSlotSssp, src.data(), kb, bout, nullptr, 0.85f, 0, kMaxSlots, s));
                G1_CUDA(cudaStreamSynchronize(s));
                const double t = seconds_since(t0);
                if (t < best) {
                    best = t;
                    best_div = d;
                }
            }
            g->slot_div = best_div;
            for (auto& e : g->slot_cache) e.reset();
        }
    }
    if (push_div) *push_div = g->push_div;
    if (slot_div) *slot_div = g->slot_div;
    return G1_OK;
}

extern "C" g1_status g1_set_traversal_thresholds(g1_graph* g, uint32_t push_div, uint32_t slot_div) {
    if (!g) return fail(G1_ERR_INVALID, "g1_set_traversal_thresholds: null graph");
    std::lock_guard<std::mutex> lk(g->mu);
    if (push_div) g->push_div = push_div;
    if (slot_div && slot_div != g->slot_div) {
        g->slot_div = slot_div;
        for (auto& e : g->slot_cache) e.reset();  // their captured steps hold the threshold
    }
    return G1_OK;
}

extern "C" g1_status g1_bfs_batch(g1_graph* g, const uint32_t* srcs, uint32_t k,
                                  uint32_t* levels_out, uint32_t* iters_out, void* stream) {
    return entry(g, kSlotBfs, srcs, k, levels_out, iters_out, 0.85f, 0, kMaxSlots, stream);
}

extern "C" g1_status g1_sssp_batch(g1_graph* g, const uint32_t* srcs, uint32_t k,
                                   uint32_t* dist_out, uint32_t* iters_out, void* stream) {
    return entry(g, kSlotSssp, srcs, k, dist_out, iters_out, 0.85f, 0, kMaxSlots, stream);
}

extern "C" g1_status g1_ppr_batch(g1_graph* g, const uint32_t* srcs, uint32_t k, float alpha,
                                  uint32_t iters, float* rank_out, void* stream) {
    return entry(g, kSlotPpr, srcs, k, rank_out, nullptr, alpha, iters, kMaxSlots, stream);
}
