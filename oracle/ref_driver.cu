// Reference CPU driver -- test and CPU-baseline infrastructure only.
//
// Compiled by oracle/Makefile against GraphOne's own headers (the reference
// source tree, include path given on the command line) into
// oracle/_ref/libgraphone_ref.so.  It runs the reference's own host code for
// the hot path:
//   * GraphLoader::LoadEdgesFromTxt + EdgeCache::ToCsr
//     (loader/graph_loader.h:32-122, loader/edge_cache.h:50-105), and
//   * blas::SpMV_cpu_navie (archi/blas/spmv/cpu/naive.hpp:8-20),
// The engines have no host path in the reference (engine/blas_gc.h:130-132
// hard-wires the CUDA SpMV), so the engine loops around SpMV_cpu_navie below
// restate Construct/Apply from engine/blas_gc.h:199-245 (sparse frontier) and
// :388-428 (all-active) with the app functors of apps/sssp_blas.cu:48-84 and
// apps/pagerank_blas.cu:86-123.  Threads split SpMV_cpu_navie by row range.
//
// Nothing in the product links this file; bench.py's reference arm and the
// tests load it through ctypes.

#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <thread>
#include <vector>
#include <algorithm>

#include "GraphOne/loader/graph_loader.h"
#include "GraphOne/archi/blas/spmv/cpu/naive.hpp"

using namespace graph_one;

namespace {

constexpr uint32_t kU32Max = std::numeric_limits<uint32_t>::max();

// min-plus functor of apps/sssp_blas.cu:58-71 in the SpMV adapter form of
// engine/blas_gc.h:113-128, over u32 distances.
struct MinPlusU32 {
    static uint32_t initialize() { return kU32Max; }
    static uint32_t combine(const uint32_t& w, const uint32_t& info) {
        return (info == kU32Max) ? info : w + info;
    }
    static uint32_t reduce(const uint32_t& a, const uint32_t& b) { return std::min(a, b); }
};

// plus-times functor of apps/pagerank_blas.cu:103-113.
struct PlusTimesF32 {
    static float initialize() { return 0.0f; }
    static float combine(const float& w, const float& info) { return info * w; }
    static float reduce(const float& a, const float& b) { return a + b; }
};

template <typename F, typename V, typename X, typename Y>
void spmv_threads(uint32_t n, const uint32_t* rp, const uint32_t* ci, const V* v,
                  const X* x, Y* y, int threads) {
    if (threads <= 1 || n < 4096) {
        blas::SpMV_cpu_navie<F>(n, rp, ci, v, x, y);
        return;
    }
    // Balance by nonzeros: each thread takes a contiguous row range.
    std::vector<std::thread> pool;
    const uint64_t m = rp[n];
    uint32_t r0 = 0;
    for (int t = 0; t < threads; ++t) {
        uint64_t target = m * (uint64_t)(t + 1) / (uint64_t)threads;
        uint32_t r1 = (t == threads - 1)
                          ? n
                          : (uint32_t)(std::upper_bound(rp, rp + n + 1, (uint32_t)target) - rp - 1);
        if (r1 < r0) r1 = r0;
        if (r1 > r0) {
            pool.emplace_back([=] {
                blas::SpMV_cpu_navie<F>(r1 - r0, rp + r0, ci, v, x, y + r0);
            });
        }
        r0 = r1;
    }
    for (auto& th : pool) th.join();
}

struct Loaded {
    EdgeCache<vstart_t::FROM_0_TO_0, uint32_t, vid_t, eid_t> cache;
};
std::unique_ptr<Loaded> g_loaded;

}  // namespace

extern "C" {

// Loads a GraphOne ".adj" edge list with the reference loader (u32 edge data,
// default options except `directed`).  Returns 0 on success.
int ref_load_adj(const char* path, int directed, uint32_t* n_out, uint64_t* m_out) {
    LoadEdgeOpts opts;
    opts.is_directed = directed != 0;
    GraphLoader<vstart_t::FROM_0_TO_0> loader;
    g_loaded.reset(new Loaded{loader.LoadEdgesFromTxt<uint32_t>(path, opts)});
    *n_out = g_loaded->cache.num_vertices();
    *m_out = g_loaded->cache.num_edges();
    return 0;
}

// The same with the loader's other switches: first-seen vertex renumbering
// (GraphLoader(reorder_vid)), self loops and duplicate edges kept.
int ref_load_adj_opts(const char* path, int directed, int reorder, int keep_self, int keep_dup,
                      uint32_t* n_out, uint64_t* m_out) {
    LoadEdgeOpts opts;
    opts.is_directed = directed != 0;
    opts.keep_self_loop = keep_self != 0;
    opts.keep_duplicate_edges = keep_dup != 0;
    GraphLoader<vstart_t::FROM_0_TO_0> loader(reorder != 0);
    g_loaded.reset(new Loaded{loader.LoadEdgesFromTxt<uint32_t>(path, opts)});
    *n_out = g_loaded->cache.num_vertices();
    *m_out = g_loaded->cache.num_edges();
    return 0;
}

// EdgeCache::ToCsr<cpu, transpose> of the last loaded graph.
int ref_to_csr(int transpose, uint32_t* row_ptr, uint32_t* col, uint32_t* val) {
    if (!g_loaded) return 1;
    auto fill = [&](auto&& csr) {
        std::memcpy(row_ptr, csr.row_offsets.data(), sizeof(uint32_t) * (csr.n_rows + 1));
        std::memcpy(col, csr.col_indices.data(), sizeof(uint32_t) * csr.nnz);
        std::memcpy(val, csr.values.data(), sizeof(uint32_t) * csr.nnz);
    };
    if (transpose)
        fill(g_loaded->cache.ToCsr<arch_t::cpu, true>());
    else
        fill(g_loaded->cache.ToCsr<arch_t::cpu, false>());
    return 0;
}

void ref_spmv_minplus_u32(uint32_t n, const uint32_t* rp, const uint32_t* ci,
                          const uint32_t* v, const uint32_t* x, uint32_t* y, int threads) {
    spmv_threads<MinPlusU32>(n, rp, ci, v, x, y, threads);
}

void ref_spmv_plustimes_f32(uint32_t n, const uint32_t* rp, const uint32_t* ci,
                            const float* v, const float* x, float* y, int threads) {
    spmv_threads<PlusTimesF32>(n, rp, ci, v, x, y, threads);
}

// SSSP on the sparse-frontier BLAS engine around SpMV_cpu_navie; returns the
// iteration count.  max_iters bounds a time-limited sample (0 = no bound).
int ref_sssp_blas_u32(uint32_t n, const uint32_t* trp, const uint32_t* tci,
                      const uint32_t* tv, uint32_t src, uint32_t* dist, int threads,
                      int max_iters) {
    std::vector<uint32_t> x(n), y(n), fin{src}, fout;
    std::fill(dist, dist + n, kU32Max);
    dist[src] = 0;
    int it = 0;
    while (!fin.empty() && (max_iters <= 0 || it < max_iters)) {
        ++it;
        std::fill(x.begin(), x.end(), kU32Max);
        for (uint32_t f : fin) x[f] = dist[f];
        spmv_threads<MinPlusU32>(n, trp, tci, tv, x.data(), y.data(), threads);
        fout.clear();
        for (uint32_t v = 0; v < n; ++v)
            if (y[v] != kU32Max && y[v] < dist[v]) {
                dist[v] = y[v];
                fout.push_back(v);
            }
        fin.swap(fout);
    }
    return it;
}

// PageRank on the all-active BLAS engine around SpMV_cpu_navie, fp32, fixed
// iteration count.  mode 0: reference formula; mode 1: dangling mass
// redistributed uniformly.  iweights from the out-degree weights (the caller
// passes out_w = per-vertex sum of out-edge weights).
void ref_pagerank_f32(uint32_t n, const uint32_t* trp, const uint32_t* tci, const float* tv,
                      const float* out_w, float alpha, int iters, int mode, float* rank,
                      int threads) {
    std::vector<float> iw(n), x(n), y(n);
    for (uint32_t u = 0; u < n; ++u) iw[u] = out_w[u] != 0 ? alpha / out_w[u] : 0;
    const float base0 = (1.0 - alpha) / n;
    for (uint32_t u = 0; u < n; ++u) rank[u] = 1.0 / n;
    for (int it = 0; it < iters; ++it) {
        double dang = 0.0;
        for (uint32_t u = 0; u < n; ++u) {
            x[u] = rank[u] * iw[u];
            if (out_w[u] == 0) dang += rank[u];
        }
        spmv_threads<PlusTimesF32>(n, trp, tci, tv, x.data(), y.data(), threads);
        const float base = mode == 1 ? (float)(base0 + alpha * dang / n) : base0;
        for (uint32_t v = 0; v < n; ++v) rank[v] = base + y[v];
    }
}

}  // extern "C"
