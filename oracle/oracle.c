/*
 * GraphOne oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the algorithms that GraphOne's
 * hot path computes (the semiring SpMV engine and the advance/filter engine,
 * plus the three apps that drive them).  It exists to CHECK the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * may load it.  Nothing in graphone_b200/ links or calls this file.
 *
 * Reference citations are paths inside the GraphOne source tree.
 *
 * Parity pinning: GraphOne ships no golden vectors for this path (its tests
 * are print-only and read a dataset that is not in the tree).  This file is
 * pinned instead against the reference's own code: oracle/ref_driver.cpp
 * compiles GraphOne's GraphLoader / EdgeCache::ToCsr and SpMV_cpu_navie from
 * the reference sources into oracle/_ref/, and tests/test_oracle.py checks the
 * two against each other on generated graphs (see tests/golden/ for the
 * committed fixtures made that way).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_U32_MAX 0xFFFFFFFFu
#define ORC_GOLDEN 0x9E3779B97F4A7C15ULL

/* ------------------------------------------------------------------ */
/* Seeded counter-based generator (the synthetic-input specification). */
/* ------------------------------------------------------------------ */

/* splitmix64 finaliser (Steele, Lea, Flood 2014). */
uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* ctr-th output of a splitmix64 stream started at `seed`. */
uint64_t orc_rng(uint64_t seed, uint64_t ctr) {
    return orc_mix64(seed + (ctr + 1) * ORC_GOLDEN);
}

/*
 * Raw RMAT samples (Chakrabarti et al. 2004): sample i descends `scale`
 * levels; level l draws r = rng(seed, i*scale + l) >> 11 (53 bits) and picks
 * quadrant (0,0) if r < tA, (0,1) if r < tAB, (1,0) if r < tABC, else (1,1).
 * The thresholds are floor(p * 2^53) of the cumulative probabilities.
 */
void orc_rmat_samples(int scale, uint64_t n_samples, uint64_t tA, uint64_t tAB,
                      uint64_t tABC, uint64_t seed, uint32_t *src, uint32_t *dst) {
    for (uint64_t i = 0; i < n_samples; ++i) {
        uint32_t s = 0, d = 0;
        for (int l = 0; l < scale; ++l) {
            uint64_t r = orc_rng(seed, i * (uint64_t)scale + (uint64_t)l) >> 11;
            uint32_t rb, cb;
            if (r < tA) { rb = 0; cb = 0; }
            else if (r < tAB) { rb = 0; cb = 1; }
            else if (r < tABC) { rb = 1; cb = 0; }
            else { rb = 1; cb = 1; }
            s = (s << 1) | rb;
            d = (d << 1) | cb;
        }
        src[i] = s;
        dst[i] = d;
    }
}

/* Weight of edge key (lo*n+hi for an undirected pair): uniform in [wlo, whi]. */
uint32_t orc_edge_weight(uint64_t wseed, uint64_t key, uint32_t wlo, uint32_t whi) {
    uint64_t r = orc_rng(wseed, key) >> 11;
    return wlo + (uint32_t)(r % (uint64_t)(whi - wlo + 1));
}

/* ------------------------------------------------------------------ */
/* CSR build: restates EdgeCache::ToCsr (loader/edge_cache.h:50-105).  */
/* ------------------------------------------------------------------ */
/*
 * Counting sort by row (src, or dst when `transpose`), stable in the input
 * order.  GraphLoader sorts and dedups edges by (src,dst) first
 * (loader/graph_loader.h:290-296), so rows come out with increasing columns.
 * row_ptr has n+1 entries.
 */
void orc_csr_build(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                   const uint32_t *w, int transpose, uint32_t *row_ptr,
                   uint32_t *col, uint32_t *val) {
    memset(row_ptr, 0, sizeof(uint32_t) * ((size_t)n + 1));
    const uint32_t *rows = transpose ? dst : src;
    const uint32_t *cols = transpose ? src : dst;
    for (uint64_t i = 0; i < m; ++i) row_ptr[rows[i] + 1]++;
    for (uint32_t r = 0; r < n; ++r) row_ptr[r + 1] += row_ptr[r];
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n + 1));
    memcpy(cur, row_ptr, sizeof(uint32_t) * ((size_t)n + 1));
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t p = cur[rows[i]]++;
        col[p] = cols[i];
        if (val && w) val[p] = w[i];
    }
    free(cur);
}

/* ------------------------------------------------------------------ */
/* Semiring SpMV: restates blas::SpMV_cpu_navie                         */
/* (archi/blas/spmv/cpu/naive.hpp:8-20) with the engine's functor       */
/* adapter (engine/blas_gc.h:113-128).                                  */
/* ------------------------------------------------------------------ */

/* min-plus with the sssp_blas functor (apps/sssp_blas.cu:58-71):
 * combine(w, info) = info==MAX ? MAX : w+info (u32, wrapping), reduce = min,
 * initialize = default_result = MAX. */
void orc_spmv_minplus_u32(uint32_t n_rows, const uint32_t *rp, const uint32_t *ci,
                          const uint32_t *v, const uint32_t *x, uint32_t *y) {
    for (uint32_t r = 0; r < n_rows; ++r) {
        uint32_t acc = ORC_U32_MAX;
        for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) {
            uint32_t info = x[ci[k]];
            uint32_t c = (info == ORC_U32_MAX) ? info : v[k] + info;
            acc = c < acc ? c : acc;
        }
        y[r] = acc;
    }
}

/* plus-times in fp32 with sequential fp32 accumulation
 * (apps/pagerank_blas.cu:103-113). */
void orc_spmv_plustimes_f32(uint32_t n_rows, const uint32_t *rp, const uint32_t *ci,
                            const float *v, const float *x, float *y) {
    for (uint32_t r = 0; r < n_rows; ++r) {
        float acc = 0.0f;
        for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) acc = acc + x[ci[k]] * v[k];
        y[r] = acc;
    }
}

/* plus-times in fp64 (the FP64 oracle of the fp32 kernels). */
void orc_spmv_plustimes_f64(uint32_t n_rows, const uint32_t *rp, const uint32_t *ci,
                            const double *v, const double *x, double *y) {
    for (uint32_t r = 0; r < n_rows; ++r) {
        double acc = 0.0;
        for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) acc += x[ci[k]] * v[k];
        y[r] = acc;
    }
}

/* ------------------------------------------------------------------ */
/* SSSP on the BLAS engine with a sparse frontier.                      */
/* Restates Run (base/run.h:8-39) driving                               */
/* BlasGcEngine<SPARSE_BASED>::Forward (engine/blas_gc.h:193-245) with  */
/* the sssp_blas component and functor (apps/sssp_blas.cu:29-84), u32.  */
/* Returns the number of engine iterations.                              */
/* ------------------------------------------------------------------ */
int orc_sssp_blas_u32(uint32_t n, const uint32_t *trp, const uint32_t *tci,
                      const uint32_t *tv, uint32_t src, uint32_t *dist) {
    uint32_t *x = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *y = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *fin = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *fout = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    /* SSSPComp::Init: fill MAX, dists[src] = 0 (sssp_blas.cu:35-41). */
    for (uint32_t v = 0; v < n; ++v) dist[v] = ORC_U32_MAX;
    dist[src] = 0;
    uint32_t fin_n = 1;
    fin[0] = src;
    int iters = 0;
    while (fin_n > 0) { /* SpDblFrontier::IsConvergent (frontier/sparse_dbl.h:144-146) */
        ++iters;
        /* Construct (blas_gc.h:199-217): x = default_info; x[f] = construct_each(f). */
        for (uint32_t v = 0; v < n; ++v) x[v] = ORC_U32_MAX;
        for (uint32_t i = 0; i < fin_n; ++i) x[fin[i]] = dist[fin[i]];
        /* Gather (blas_gc.h:219-222): y = A^T (min,+) x. */
        orc_spmv_minplus_u32(n, trp, tci, tv, x, y);
        /* Apply (blas_gc.h:224-245): pred = res != default_result && apply_each;
         * copy_if keeps vertex-id order. */
        uint32_t out_n = 0;
        for (uint32_t v = 0; v < n; ++v) {
            if (y[v] != ORC_U32_MAX && y[v] < dist[v]) {
                dist[v] = y[v];
                fout[out_n++] = v;
            }
        }
        /* AfterEngine swaps in/out (sparse_dbl.h:140-142). */
        uint32_t *t = fin; fin = fout; fout = t;
        fin_n = out_n;
    }
    free(x); free(y); free(fin); free(fout);
    return iters;
}

/* Same engine with float distances, exactly as the unchanged app computes
 * them (dist_t = float, kMaxDist = FLT_MAX; apps/sssp_blas.cu:12-14). */
int orc_sssp_blas_f32(uint32_t n, const uint32_t *trp, const uint32_t *tci,
                      const float *tv, uint32_t src, float *dist) {
    const float kmax = 3.40282346638528859812e+38F;
    float *x = (float *)malloc(sizeof(float) * (n ? n : 1));
    float *y = (float *)malloc(sizeof(float) * (n ? n : 1));
    uint32_t *fin = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *fout = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t v = 0; v < n; ++v) dist[v] = kmax;
    dist[src] = 0.0f;
    uint32_t fin_n = 1;
    fin[0] = src;
    int iters = 0;
    while (fin_n > 0) {
        ++iters;
        for (uint32_t v = 0; v < n; ++v) x[v] = kmax;
        for (uint32_t i = 0; i < fin_n; ++i) x[fin[i]] = dist[fin[i]];
        for (uint32_t r = 0; r < n; ++r) {
            float acc = kmax;
            for (uint32_t k = trp[r]; k < trp[r + 1]; ++k) {
                float info = x[tci[k]];
                float c = (info == kmax) ? info : tv[k] + info;
                acc = c < acc ? c : acc;
            }
            y[r] = acc;
        }
        uint32_t out_n = 0;
        for (uint32_t v = 0; v < n; ++v) {
            if (y[v] != kmax && y[v] < dist[v]) {
                dist[v] = y[v];
                fout[out_n++] = v;
            }
        }
        uint32_t *t = fin; fin = fout; fout = t;
        fin_n = out_n;
    }
    free(x); free(y); free(fin); free(fout);
    return iters;
}

/* ------------------------------------------------------------------ */
/* SSSP on the advance/filter engine.                                   */
/* Restates AdvanceGC::Forward (engine/advance_gc.h:180-244) with the   */
/* sssp_adv functor (apps/sssp_adv.cu:48-72), u32, sequential order.    */
/* The reference pads the advance output with invalid vertices          */
/* (advance_gc.h:153-156); padding carries no result, so this version   */
/* keeps the emitted vertices only.  Final distances are the unique     */
/* shortest-path distances, independent of relaxation order.           */
/* ------------------------------------------------------------------ */
int orc_sssp_advance_u32(uint32_t n, const uint32_t *rp, const uint32_t *ci,
                         const uint32_t *v, uint32_t src, uint32_t *dist) {
    uint32_t *visited = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    uint64_t cap = 1024;
    uint32_t *fin = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    uint32_t *fout = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    for (uint32_t u = 0; u < n; ++u) dist[u] = ORC_U32_MAX;
    dist[src] = 0;
    uint64_t fin_n = 1;
    fin[0] = src;
    uint32_t iter = 0;
    int iters = 0;
    while (fin_n > 0) {
        ++iter; /* SSSPComp::BeforeEngine (sssp_adv.cu:43-45) */
        ++iters;
        uint64_t need = 0;
        for (uint64_t i = 0; i < fin_n; ++i) need += rp[fin[i] + 1] - rp[fin[i]];
        if (need > cap) { /* both buffers always hold `cap` entries */
            cap = need;
            fout = (uint32_t *)realloc(fout, sizeof(uint32_t) * cap);
            fin = (uint32_t *)realloc(fin, sizeof(uint32_t) * cap);
        }
        uint64_t out_n = 0;
        /* advance: dists[dst] = min(dists[dst], dists[src]+w); emit when improved */
        for (uint64_t i = 0; i < fin_n; ++i) {
            uint32_t s = fin[i];
            for (uint32_t e = rp[s]; e < rp[s + 1]; ++e) {
                uint32_t d = ci[e];
                uint32_t cand = dist[s] + v[e];
                uint32_t old = dist[d];
                if (cand < old) {
                    dist[d] = cand;
                    fout[out_n++] = d;
                }
            }
        }
        /* filter: drop v when visited[v]==iter, else mark (sssp_adv.cu:62-71) */
        uint64_t kept = 0;
        for (uint64_t i = 0; i < out_n; ++i) {
            uint32_t d = fout[i];
            if (visited[d] == iter) continue;
            visited[d] = iter;
            fout[kept++] = d;
        }
        uint32_t *t = fin; fin = fout; fout = t;
        fin_n = kept;
    }
    free(visited); free(fin); free(fout);
    return iters;
}

/* BFS levels (no reference app): hop distance from src, MAX if unreachable.
 * Equal to orc_sssp_blas_u32 with every weight 1. */
int orc_bfs(uint32_t n, const uint32_t *rp, const uint32_t *ci, uint32_t src,
            uint32_t *level) {
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t u = 0; u < n; ++u) level[u] = ORC_U32_MAX;
    level[src] = 0;
    uint32_t head = 0, tail = 0;
    q[tail++] = src;
    uint32_t depth = 0;
    while (head < tail) {
        uint32_t u = q[head++];
        if (level[u] > depth) depth = level[u];
        for (uint32_t e = rp[u]; e < rp[u + 1]; ++e) {
            uint32_t d = ci[e];
            if (level[d] == ORC_U32_MAX) {
                level[d] = level[u] + 1;
                q[tail++] = d;
            }
        }
    }
    free(q);
    return (int)depth;
}

/* Dijkstra (binary heap): an independent check of the two SSSP restatements. */
static void heap_push(uint64_t *h, uint64_t *hn, uint64_t key) {
    uint64_t i = (*hn)++;
    h[i] = key;
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (h[p] <= h[i]) break;
        uint64_t t = h[p]; h[p] = h[i]; h[i] = t;
        i = p;
    }
}
static uint64_t heap_pop(uint64_t *h, uint64_t *hn) {
    uint64_t top = h[0];
    h[0] = h[--(*hn)];
    uint64_t i = 0;
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < *hn && h[l] < h[m]) m = l;
        if (r < *hn && h[r] < h[m]) m = r;
        if (m == i) break;
        uint64_t t = h[m]; h[m] = h[i]; h[i] = t;
        i = m;
    }
    return top;
}
void orc_dijkstra_u32(uint32_t n, const uint32_t *rp, const uint32_t *ci,
                      const uint32_t *v, uint32_t src, uint32_t *dist) {
    uint64_t m = rp[n];
    uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (m + 2));
    uint64_t hn = 0;
    for (uint32_t u = 0; u < n; ++u) dist[u] = ORC_U32_MAX;
    dist[src] = 0;
    heap_push(h, &hn, (uint64_t)src);
    while (hn) {
        uint64_t k = heap_pop(h, &hn);
        uint32_t u = (uint32_t)(k & 0xFFFFFFFFu);
        uint32_t du = (uint32_t)(k >> 32);
        if (du != dist[u]) continue;
        for (uint32_t e = rp[u]; e < rp[u + 1]; ++e) {
            uint32_t d = ci[e];
            uint32_t c = du + v[e];
            if (c < dist[d]) {
                dist[d] = c;
                heap_push(h, &hn, ((uint64_t)c << 32) | d);
            }
        }
    }
    free(h);
}

/* ------------------------------------------------------------------ */
/* PageRank, FP64.                                                      */
/* Restates the pagerank_blas component and functor                     */
/* (apps/pagerank_blas.cu:36-123) on BlasGcEngine<ALL_ACTIVE>           */
/* (engine/blas_gc.h:377-428), for a fixed iteration count:             */
/*   iweights[u] = alpha / sum_w_out(u), 0 if sum is 0   (:41-53)       */
/*   x[u]        = rank[u] * iweights[u]                  (:95-101)      */
/*   y[v]        = sum over in-edges (u,v) of x[u]*w      (:103-113)     */
/*   rank'[v]    = (1-alpha)/N + y[v]                     (:115-121)     */
/* mode 0 = the reference formula above (dangling mass dropped);        */
/* mode 1 = dangling mass alpha*sum(rank[dangling])/N added to every v.  */
/* Inputs are the transpose CSR (row v lists the sources u).            */
/* ------------------------------------------------------------------ */
void orc_pagerank_f64(uint32_t n, const uint32_t *trp, const uint32_t *tci,
                      const float *tv, double alpha, int iters, int mode,
                      double *rank_out) {
    double *outw = (double *)calloc(n ? n : 1, sizeof(double));
    double *iw = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *x = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *r = rank_out;
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t k = trp[v]; k < trp[v + 1]; ++k) outw[tci[k]] += (double)tv[k];
    for (uint32_t u = 0; u < n; ++u) iw[u] = outw[u] != 0.0 ? alpha / outw[u] : 0.0;
    for (uint32_t u = 0; u < n; ++u) r[u] = 1.0 / (double)n;
    for (int it = 0; it < iters; ++it) {
        double dang = 0.0;
        for (uint32_t u = 0; u < n; ++u) {
            x[u] = r[u] * iw[u];
            if (outw[u] == 0.0) dang += r[u];
        }
        double base = (1.0 - alpha) / (double)n;
        if (mode == 1) base += alpha * dang / (double)n;
        for (uint32_t v = 0; v < n; ++v) {
            double acc = 0.0;
            for (uint32_t k = trp[v]; k < trp[v + 1]; ++k) acc += x[tci[k]] * (double)tv[k];
            r[v] = base + acc; /* r is overwritten only after x was fully built */
        }
    }
    free(outw); free(iw); free(x);
}

/* Personalized PageRank (no reference app): the pagerank_blas iteration
 * with the teleport (1-alpha) and the dangling mass alpha*sum(rank[dangling])
 * both sent to the source vertex only.  rank starts as the indicator of src. */
void orc_ppr_f64(uint32_t n, const uint32_t *trp, const uint32_t *tci, const float *tv,
                 double alpha, int iters, uint32_t src, double *rank_out) {
    double *outw = (double *)calloc(n ? n : 1, sizeof(double));
    double *x = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *r = rank_out;
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t k = trp[v]; k < trp[v + 1]; ++k) outw[tci[k]] += (double)tv[k];
    for (uint32_t u = 0; u < n; ++u) r[u] = (u == src) ? 1.0 : 0.0;
    for (int it = 0; it < iters; ++it) {
        double dang = 0.0;
        for (uint32_t u = 0; u < n; ++u) {
            x[u] = outw[u] != 0.0 ? r[u] * (alpha / outw[u]) : 0.0;
            if (outw[u] == 0.0) dang += r[u];
        }
        for (uint32_t v = 0; v < n; ++v) {
            double acc = 0.0;
            for (uint32_t k = trp[v]; k < trp[v + 1]; ++k) acc += x[tci[k]] * (double)tv[k];
            r[v] = acc + ((v == src) ? (1.0 - alpha) + alpha * dang : 0.0);
        }
    }
    free(outw); free(x);
}
