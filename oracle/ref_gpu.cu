// Reference GPU engines on caller CSR arrays -- baseline and checker
// infrastructure only (never linked by the product).
//
// Compiled by oracle/Makefile against GraphOne's own headers (the reference
// source tree, include path given on the command line, the same three include
// shims as ref_driver.cu) into oracle/_ref/libgraphone_refgpu.so for sm_100a.
// It drives GraphOne's own GPU code for the hot path, unchanged:
//   * Run<F>(comp, frontier) (base/run.h:8-39) over
//   * BlasGcEngine<ALL_ACTIVE> / <SPARSE_BASED> (engine/blas_gc.h:171-434),
//     whose Gather is SpmvDispatcher<SpmvCudaCsrMergeBased> -- the merge-based
//     SpMV (archi/blas/spmv/cuda/cuda.cuh:64-114,
//     merge_based/merge_based_spmv.cuh) -- and whose Apply is
//     apply_construct_kernel (engine/blas_gc.h:27-76);
//   * AdvanceGC (engine/advance_gc.h:162-283).
// The components and functors below are written here against GraphOne's
// public API, the way an application would (GraphOne's pagerank_blas app does
// not compile with CUDA 12.9: apps/pagerank_blas.cu:67-74 has a device lambda
// without a return type).  They follow the semantics of apps/pagerank_blas.cu
// (reference PageRank formula, iweights = alpha / out-weight), and of
// apps/sssp_blas.cu / apps/sssp_adv.cu with uint32 distances (UINT32_MAX =
// unreachable) instead of float.  PageRank runs a fixed iteration count
// instead of the app's max-difference test.
//
// Timing: CUDA events on the default stream (GraphOne's engines launch there
// and synchronise the host inside their steps), around Run<> only: the graph
// is already on the device, as in the app's own timer (sssp_blas.cu:112-117).

#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <cuda_runtime.h>

#include "GraphOne/graph_one.h"

using namespace graph_one;

namespace refgpu {

constexpr arch_t kArch = arch_t::cuda;
constexpr uint32_t kInf = std::numeric_limits<uint32_t>::max();

template <typename W>
using DevCsr = CsrMat<kArch, W, vid_t, eid_t, vstart_t::FROM_0_TO_0>;

template <graph_view_t views, typename W>
using DevGraph = Graph<kArch, views, vstart_t::FROM_0_TO_0, empty_t, vid_t, eid_t, W>;

// A device CSR holding copies of the caller's host arrays.
template <typename W>
DevCsr<W> upload(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci, const W* v) {
    Buffer<kArch, eid_t, vid_t> r(n + 1);
    Buffer<kArch, vid_t, eid_t> c(m);
    Buffer<kArch, W, eid_t> w(m);
    cudaMemcpy(r.data(), rp, sizeof(eid_t) * (n + 1), cudaMemcpyHostToDevice);
    if (m) {
        cudaMemcpy(c.data(), ci, sizeof(vid_t) * m, cudaMemcpyHostToDevice);
        cudaMemcpy(w.data(), v, sizeof(W) * m, cudaMemcpyHostToDevice);
    }
    return DevCsr<W>(n, n, m, std::move(r), std::move(c), std::move(w));
}

struct Timer {
    cudaEvent_t a, b;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void start() { cudaEventRecord(a, 0); }
    double stop() {
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

// ------------------------------------------------------------- PageRank

struct PrHost {
    float alpha;
    int iters;
    int done;
    DenseVec<kArch, float>& iweights;
    DenseVec<kArch, float>& rank_a;
    DenseVec<kArch, float>& rank_b;
};

struct PrDev {
    float* iweights;
    float* ranks[2];
    int cur = 0;
    float base = 0.f;
};

template <typename graph_t>
struct FixedPageRank : ComponentX<graph_t, PrHost, PrDev> {
    using base_t = ComponentX<graph_t, PrHost, PrDev>;
    using base_t::ComponentX;

    void Init() override {
        auto g = this->graph.ToArch();
        const float alpha = this->h_status.alpha;
        archi::transform<kArch>(
            thrust::make_counting_iterator<vid_t>(0),
            thrust::make_counting_iterator<vid_t>(g.num_vertices), this->h_status.iweights.begin(),
            [g, alpha] __device__(const vid_t& u) -> float {
                float s = 0;
                const eid_t e0 = g.get_starting_out_edge(u);
                const eid_t e1 = e0 + g.get_out_degree(u);
                for (eid_t e = e0; e < e1; ++e) s += g.get_out_edge_weight(e);
                return s != 0 ? alpha / s : 0;
            });
        this->d_status.base = (1.0 - alpha) / g.num_vertices;
        this->d_status.cur = 0;
        archi::fill<kArch>(this->h_status.rank_a.begin(), this->h_status.rank_a.end(),
                           1.0f / g.num_vertices);
        archi::fill<kArch>(this->h_status.rank_b.begin(), this->h_status.rank_b.end(), 0.f);
        this->h_status.done = 0;
    }
    bool IsConvergent() override { return this->h_status.done >= this->h_status.iters; }
    void AfterEngine() override {
        this->d_status.cur ^= 1;
        ++this->h_status.done;
    }
};

struct PrFunctor : BlasFunctor<vid_t, float, PrDev, float, float> {
    __ONE_ARCH_INL__ static float default_info() { return 0.f; }
    __ONE_ARCH_INL__ static float default_result() { return 0.f; }
    __ONE_DEV_INL__ static float construct_each(const vid_t& u, const PrDev& d) {
        return d.ranks[d.cur][u] * d.iweights[u];
    }
    __ONE_DEV_INL__ static float gather_combine(const float& w, const float& x) { return x * w; }
    __ONE_DEV_INL__ static float gather_reduce(const float& a, const float& b) { return a + b; }
    __ONE_DEV_INL__ static bool apply_each(const vid_t& v, const float& y, PrDev& d) {
        d.ranks[d.cur][v] = d.base + y;
        return true;
    }
};

// The SpMV adapter the BLAS engine builds around a functor
// (engine/blas_gc.h:113-128), for timing the dispatcher alone.
struct PlusTimes {
    __ONE_DEV_INL__ static float initialize() { return 0.f; }
    __ONE_DEV_INL__ static float combine(const float& w, const float& x) { return x * w; }
    __ONE_DEV_INL__ static float reduce(const float& a, const float& b) { return a + b; }
};

// ------------------------------------------------------------- SSSP (BLAS)

struct SsspHost {
    vid_t src;
    DenseVec<kArch, uint32_t>& dist;
    DenseVec<kArch, uint32_t>& visited;
    int iters;
};

struct SsspDev {
    uint32_t iter;
    uint32_t* dist;
    uint32_t* visited;
};

template <typename graph_t>
struct SsspComp : ComponentX<graph_t, SsspHost, SsspDev> {
    using base_t = ComponentX<graph_t, SsspHost, SsspDev>;
    using base_t::ComponentX;
    void Init() override {
        archi::fill<kArch>(this->h_status.dist.begin(), this->h_status.dist.end(), kInf);
        this->h_status.dist.set(this->h_status.src, 0u);
        archi::fill<kArch>(this->h_status.visited.begin(), this->h_status.visited.end(), 0u);
        this->d_status.iter = 0;
        this->h_status.iters = 0;
    }
    void BeforeEngine() override {
        ++this->d_status.iter;
        ++this->h_status.iters;
    }
};

struct SsspBlasFunctor : BlasFunctor<vid_t, uint32_t, SsspDev, uint32_t, uint32_t> {
    __ONE_ARCH_INL__ static uint32_t default_info() { return kInf; }
    __ONE_ARCH_INL__ static uint32_t default_result() { return kInf; }
    __ONE_DEV_INL__ static uint32_t construct_each(const vid_t& u, const SsspDev& d) {
        return d.dist[u];
    }
    __ONE_DEV_INL__ static uint32_t gather_combine(const uint32_t& w, const uint32_t& x) {
        return x == kInf ? x : w + x;
    }
    __ONE_DEV_INL__ static uint32_t gather_reduce(const uint32_t& a, const uint32_t& b) {
        return a < b ? a : b;
    }
    __ONE_DEV_INL__ static bool apply_each(const vid_t& v, const uint32_t& y, SsspDev& d) {
        if (y < d.dist[v]) {
            d.dist[v] = y;
            return true;
        }
        return false;
    }
};

// ------------------------------------------------------------- SSSP (advance)

struct SsspAdvFunctor : AdvanceFunctor<vid_t, eid_t, uint32_t, SsspDev> {
    __ONE_DEV_INL__ static bool advance(const vid_t& u, const vid_t& v, const eid_t&,
                                        const uint32_t& w, SsspDev& d) {
        const uint32_t cand = d.dist[u] + w;
        return cand < archi::cuda::AtomicMin(&d.dist[v], cand);
    }
    __ONE_DEV_INL__ static bool filter(const vid_t& v, const SsspDev& d) {
        if (d.visited[v] == d.iter) return true;
        d.visited[v] = d.iter;
        return false;
    }
};

template <typename F, typename G>
int run_sssp(G& g, uint32_t n, const uint32_t* srcs, int nsrc, uint32_t* dist_out,
             double* ms_out, int* iters_out) {
    DenseVec<kArch, uint32_t> dist(n);
    DenseVec<kArch, uint32_t> visited(n);
    Timer t;
    for (int i = 0; i < nsrc; ++i) {
        SsspHost h{srcs[i], dist, visited, 0};
        SsspDev d{0, dist.data(), visited.data()};
        SpDblFrontier<kArch, vid_t> frontier(n, {srcs[i]});
        SsspComp<G> comp(g, h, d);
        t.start();
        Run<F>(comp, frontier);
        ms_out[i] = t.stop();
        if (iters_out) iters_out[i] = h.iters;
        if (i == 0 && dist_out)
            cudaMemcpy(dist_out, dist.data(), sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

}  // namespace refgpu

using namespace refgpu;

extern "C" {

// PageRank on GraphOne's all-active BLAS engine: `reps` runs of Run<> with
// `iters` iterations each (ms_runs[r] per run), the reference formula
// rank' = (1 - alpha)/N + A^T (rank * iweights).  rank_out gets the last
// run's ranks.  Then `spmv_reps` calls of the engine's merge-based SpMV
// dispatcher alone on the same in-edge CSR (ms_spmv[i] per call).
// Out-edge CSR (rp, ci, v) gives the iweights, in-edge CSR (trp, tci, tv)
// the SpMV, both fp32 values.  Returns 0 on success.
int refgpu_pagerank(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci, const float* v,
                    const uint32_t* trp, const uint32_t* tci, const float* tv, float alpha,
                    int iters, int reps, float* rank_out, double* ms_runs, int spmv_reps,
                    double* ms_spmv) {
    using G = DevGraph<BlasViews | graph_view_t::normal, float>;
    G g(upload<float>(n, m, rp, ci, v), upload<float>(n, m, trp, tci, tv), empty_t{});
    DenseVec<kArch, float> iw(n), ra(n), rb(n);
    PrHost h{alpha, iters, 0, iw, ra, rb};
    PrDev d{iw.data(), {ra.data(), rb.data()}};
    AllActiveFrontier<kArch, vid_t> frontier(n, {});
    Timer t;
    for (int r = 0; r < reps; ++r) {
        FixedPageRank<G> comp(g, h, d);
        t.start();
        Run<PrFunctor>(comp, frontier);
        ms_runs[r] = t.stop();
    }
    // the last iteration wrote ranks[cur] before AfterEngine flipped cur
    const float* last = iters > 0 ? d.ranks[d.cur ^ 1] : d.ranks[d.cur];
    cudaMemcpy(rank_out, last, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (spmv_reps > 0) {
        auto ref = g.ToArch();
        auto spmv = blas::MakeCsrSpMV<kArch, blas::SpmvCudaCsrMergeBased, PlusTimes>(
            ref.num_vertices, ref.num_vertices, ref.num_edges, ref.trans_row_offsets,
            ref.trans_col_indices, ref.trans_values, iw.data(), ra.data());
        spmv(true);
        for (int i = 0; i < spmv_reps; ++i) {
            t.start();
            spmv(false);
            ms_spmv[i] = t.stop();
        }
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// SSSP on GraphOne's sparse-frontier BLAS engine (min-plus SpMV over the
// in-edge CSR), one Run<> per source; ms_out[i] and iters_out[i] per source,
// dist_out the first source's distances.
int refgpu_sssp_blas_u32(uint32_t n, uint32_t m, const uint32_t* trp, const uint32_t* tci,
                         const uint32_t* tv, const uint32_t* srcs, int nsrc, uint32_t* dist_out,
                         double* ms_out, int* iters_out) {
    using G = DevGraph<BlasViews, uint32_t>;
    G g(upload<uint32_t>(n, m, trp, tci, tv), empty_t{});
    return run_sssp<SsspBlasFunctor>(g, n, srcs, nsrc, dist_out, ms_out, iters_out);
}

// SSSP on GraphOne's advance/filter engine (push over the out-edge CSR,
// atomicMin relax, visited-iteration filter), one Run<> per source.
int refgpu_sssp_adv_u32(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci,
                        const uint32_t* v, const uint32_t* srcs, int nsrc, uint32_t* dist_out,
                        double* ms_out, int* iters_out) {
    using G = DevGraph<AdvanceViews, uint32_t>;
    G g(upload<uint32_t>(n, m, rp, ci, v), empty_t{});
    return run_sssp<SsspAdvFunctor>(g, n, srcs, nsrc, dist_out, ms_out, iters_out);
}

}  // extern "C"
