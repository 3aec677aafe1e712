// Near-far single-source shortest paths / BFS in one persistent launch.
//
// For graphs of small uniform degree and large diameter (grids, meshes,
// road-like graphs) the frontier engines are bound by per-iteration host
// round trips (thousands of iterations) and, for SSSP, by Bellman-Ford's
// repeated relaxations of the same vertices.  This engine keeps the whole
// traversal on the device and orders the work by distance:
//   * vertices whose tentative distance is below the threshold T form the
//     near queue; a relax round pushes every near vertex's out-edges
//     (atomicMin); improved vertices below T join the next near queue,
//     the others the far pile (each vertex at most once per queue and per
//     bucket, by the tag kept beside its distance);
//   * when the near queue runs dry, T moves to (smallest pending distance)
//     + delta and the far pile is split into the new near queue and the
//     rest; entries below the old T are stale and dropped.
// This is the near-far variant of delta-stepping (Davidson, Baxter, Garland
// and Owens, IPDPS 2014).  Steps are separated by one grid barrier of the
// cooperative launch (one 1024-thread block per SM); every barrier wait is
// bounded and reports a timeout through the control block instead of
// hanging.  Final distances are the
// unique shortest-path distances, bit-identical to the other engines.
#include <algorithm>
#include <cstdlib>

#include "g1/common.cuh"
#include "internal.h"

namespace g1 {

// Control block.  The traversal is a sequence of steps separated by one
// grid barrier each; values a step reads are never written during that step:
// per-step values rotate through three slots (step s reads slot s % 3,
// fills slot (s+1) % 3 and resets slot (s+2) % 3).
struct NfCtl {
    unsigned long long bar;  // grid barrier: block arrivals so far (never reset)
    uint32_t qn[3];      // near-queue size
    uint32_t kind[3];    // 1: the step is a threshold move (after a minimum step)
    uint32_t thresh[3];  // T
    uint32_t minfar[3];  // smallest pending far distance
    uint32_t fn[2];      // far-pile sizes (double-buffered piles)
    uint32_t err;        // 1 = a barrier wait ran out
    uint32_t rounds;     // relax rounds
};

// Per vertex one 64-bit key: the tentative distance in the high half, in the
// low half the tag of its last improvement, 2 * round + (1 if it went to the
// far pile).  One atomicMin on the key both improves the distance and
// returns whether the vertex was already queued this round (same round, near
// tag) or is already on the current far pile (a tag from this bucket): no
// second, dependent atomic on a separate stamp array.
__device__ __forceinline__ unsigned long long nf_key(uint32_t d, uint32_t tag) {
    return ((unsigned long long)d << 32) | tag;
}

struct NfArgs {
    const uint32_t* rp;
    const uint32_t* col;
    const uint32_t* val;
    uint32_t n;
    uint32_t delta;
    unsigned long long* key;  // distance << 32 | tag
    uint32_t* dist;           // the distances, written at the end
    uint32_t* near[2];
    uint32_t* far[2];
    NfCtl* ctl;
    uint32_t spin_limit;  // polls before a barrier wait gives up
};

// About 2-3 s of waiting before a barrier gives up.
constexpr uint32_t kNfSpinLimit = 1u << 23;

__device__ __forceinline__ uint32_t ld_vol(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ uint32_t ld_dist(const unsigned long long* key) {
    return (uint32_t)(*(const volatile unsigned long long*)key >> 32);
}

__device__ __forceinline__ void red_add_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long r;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(r) : "l"(p) : "memory");
    return r;
}

// Counting grid barrier over a monotonic arrival count: barrier k (k = 1,
// 2, ...) is passed once k * nblocks blocks have arrived.  The block's
// writes are released by its thread 0's arrival (a fire-and-forget add,
// after bar.sync) and the other blocks' writes acquired by the load that
// sees the count; one word, no reset and no generation word, so a wait is
// one polling round trip after the last arrival.  false if the wait ran
// out (the kernel then returns: the host reports G1_ERR_TIMEOUT).
// The control words a step reads, copied into shared memory by thread 0 of
// each block after the barrier (one read per block instead of one per warp
// of the same few words).
struct NfStepCtl {
    uint32_t qn, thresh, kind, fn, minfar, err;
};

__device__ __forceinline__ void nf_read_ctl(const NfCtl* c, uint32_t st, uint32_t fp, NfStepCtl* sc) {
    const uint32_t cur = st % 3;
    sc->qn = ld_vol(&c->qn[cur]);
    sc->thresh = ld_vol(&c->thresh[cur]);
    sc->kind = ld_vol(&c->kind[cur]);
    sc->fn = ld_vol(&c->fn[fp]);
    sc->minfar = ld_vol(&c->minfar[cur]);
    sc->err = ld_vol(&c->err);
}

// Also loads the control words of step `st_next` (far pile `fp`) into sc.
__device__ bool nf_barrier(NfCtl* c, uint32_t nblocks, uint32_t st_next, uint32_t fp, NfStepCtl* sc,
                           uint32_t spin_limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long target = (unsigned long long)st_next * nblocks;
        red_add_release_u64(&c->bar, 1ull);
        uint32_t spins = 0;
        while (ld_acquire_u64(&c->bar) < target) {
            if (++spins > spin_limit) {
                atomicOr(&c->err, 1u);
                break;
            }
        }
        nf_read_ctl(c, st_next, fp, sc);
    }
    __syncthreads();
    return (sc->err & 1u) == 0u;
}

// src is an internal vertex id, or a caller id mapped through perm.
__global__ void nf_init_kernel(uint32_t n, uint32_t src, const uint32_t* perm, uint32_t t0,
                               unsigned long long* key, uint32_t* near0, NfCtl* ctl) {
    if (perm) src = perm[src];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        key[v] = nf_key(v == src ? 0u : kU32Max, 0u);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        near0[0] = src;
        NfCtl c{};
        c.qn[0] = 1u;
        c.thresh[0] = t0;
        c.minfar[0] = c.minfar[1] = c.minfar[2] = kU32Max;
        *ctl = c;
    }
}

// Position for one entry in a queue, one atomic per group of converged
// lanes (the lanes executing this call together share a single atomicAdd).
__device__ __forceinline__ uint32_t agg_slot(uint32_t* ctr) {
    const unsigned mask = __activemask();
    const uint32_t lane = lane_id();
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// TPV lanes per near-queue item (1..32, the power of two at or above the
// graph's mean degree): a step's edges then run about one per thread, where
// one lane per item would chain its items' edges (each an atomicMin and an
// append) one after another.  Lists of 32 or more edges are pushed by
// the whole warp.
template <bool UNIT, int TPV>
__global__ void __launch_bounds__(1024, 1) nf_kernel(NfArgs a) {
    const uint32_t nb = gridDim.x;
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gs = gridDim.x * blockDim.x;
    NfCtl* c = a.ctl;
    uint32_t par = 0, fp = 0;
    uint32_t gen = 1;      // round number (every step counts one)
    uint32_t bucket = 1;   // tags from here on belong to the current far pile's bucket
    __shared__ NfStepCtl sc;
    if (threadIdx.x == 0) nf_read_ctl(c, 0, 0, &sc);
    __syncthreads();
    for (uint32_t st = 0;; ++st) {
        const uint32_t cur = st % 3, nxt = (st + 1) % 3, old = (st + 2) % 3;
        const uint32_t qn = sc.qn;
        const uint32_t T = sc.thresh;
        const bool move = sc.kind != 0u;
        const uint32_t fn = sc.fn;
        // 0 = relax round, 1 = smallest far distance, 2 = threshold move
        const int step = move ? 2 : qn > 0 ? 0 : (fn == 0 ? -1 : (UNIT ? 2 : 1));
        if (step < 0) return;
        if (gt == 0) {
            c->qn[old] = 0u;
            c->kind[old] = 0u;
            c->minfar[old] = kU32Max;
            if (step != 2) {
                c->fn[fp ^ 1] = 0u;  // the other pile is empty until the next move
                c->thresh[nxt] = T;
            }
            if (step == 0) c->rounds += 1u;
            if (step == 1) c->kind[nxt] = 1u;
        }
        if (step == 0) {
            ++gen;
            const uint32_t* in = a.near[par];
            uint32_t* outq = a.near[par ^ 1];
            uint32_t* farq = a.far[fp];
            const uint32_t near_tag = 2u * gen;
            auto relax = [&](uint32_t du, uint32_t e) {
                const uint32_t v = a.col[e];
                const uint32_t nd = du + (UNIT ? 1u : a.val[e]);
                // no plain pre-check: one dependent memory access fewer on the
                // critical path of a step
                const bool is_near = nd < T;
                const unsigned long long old = atomicMin(a.key + v, nf_key(nd, near_tag + (is_near ? 0u : 1u)));
                if (nd >= (uint32_t)(old >> 32)) return;
                const uint32_t tag = (uint32_t)old;
                if (is_near) {
                    // queued once per round (BFS: every improvement in a round
                    // sets the same level, so only the first one succeeds); a
                    // vertex that went to the far pile earlier in the round
                    // still joins the near queue
                    if (UNIT || tag != near_tag) outq[agg_slot(&c->qn[nxt])] = v;
                } else if (tag < 2u * bucket) {
                    // not on the current far pile yet
                    farq[agg_slot(&c->fn[fp])] = v;
                }
            };
            const uint32_t lane = lane_id();
            constexpr uint32_t VPW = 32 / TPV;  // items per warp and round
            const uint32_t sub = lane % TPV, grp = lane / TPV;
            const uint32_t gw = gt >> 5, nw = gs >> 5;
            // warp-uniform rounds: lists of 32 or more edges are pushed by the
            // whole warp, shorter ones by the item's TPV lanes
            for (uint32_t base = gw * VPW; base < qn; base += nw * VPW) {
                const uint32_t i = base + grp;
                uint32_t du = 0, b = 0, e1 = 0;
                if (i < qn) {
                    const uint32_t u = in[i];
                    du = ld_dist(a.key + u);
                    b = a.rp[u];
                    e1 = a.rp[u + 1];
                }
                unsigned big = __ballot_sync(0xffffffffu, sub == 0 && e1 - b >= 32);
                while (big) {
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const uint32_t bb = __shfl_sync(0xffffffffu, b, src);
                    const uint32_t ee = __shfl_sync(0xffffffffu, e1, src);
                    const uint32_t dd = __shfl_sync(0xffffffffu, du, src);
                    for (uint32_t e = bb + lane; e < ee; e += 32) relax(dd, e);
                }
                if (e1 - b < 32)
                    for (uint32_t e = b + sub; e < e1; e += TPV) relax(du, e);
            }
            par ^= 1;
        } else if (step == 1) {
            uint32_t mn = kU32Max;
            const uint32_t* fin = a.far[fp];
            for (uint32_t i = gt; i < fn; i += gs) {
                const uint32_t d = ld_dist(a.key + fin[i]);
                if (d >= T) mn = min(mn, d);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, off));
            if (lane_id() == 0 && mn != kU32Max) atomicMin(&c->minfar[nxt], mn);
        } else {
            // move the threshold: the far pile splits into the next near
            // queue and the remaining pile; entries below T are stale
            uint32_t tn;
            if (UNIT) {
                tn = T + 1u;
            } else {
                const uint32_t mf = sc.minfar;
                const uint64_t base = (mf != kU32Max && mf > T) ? mf : T;
                const uint64_t t64 = base + a.delta;
                tn = t64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)t64;
            }
            if (gt == 0) c->thresh[nxt] = tn;
            ++gen;
            // the new bucket's far pile starts here: a vertex carried over is
            // tagged into it, so the next rounds do not add it again
            bucket = gen;
            const uint32_t* fin = a.far[fp];
            uint32_t* fout = a.far[fp ^ 1];
            uint32_t* outq = a.near[par ^ 1];
            // every vertex is on the pile at most once and no relaxation runs
            // in this step: plain loads and stores of the keys
            for (uint32_t i = gt; i < fn; i += gs) {
                const uint32_t v = fin[i];
                const uint32_t d = ld_dist(a.key + v);
                if (d < T) continue;
                if (d < tn) {
                    outq[agg_slot(&c->qn[nxt])] = v;
                } else {
                    a.key[v] = nf_key(d, 2u * bucket + 1u);
                    fout[agg_slot(&c->fn[fp ^ 1])] = v;
                }
            }
            par ^= 1;
            fp ^= 1;
        }
        if (!nf_barrier(c, nb, st + 1, fp, &sc, a.spin_limit)) return;
    }
}

namespace {

// Reads the control block back through the graph's pinned scratch and
// reports its outcome.
g1_status ws_pinned_ctl(g1_graph* g, const uint32_t* ctl, cudaStream_t s, uint32_t* rounds) {
    G1_TRY(g->ws.pinned.ensure(sizeof(NfCtl) + 64));
    G1_CUDA(cudaMemcpyAsync(g->ws.pinned.p, ctl, sizeof(NfCtl), cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    return nearfar_result(g->ws.pinned.as<uint32_t>(), rounds);
}

__global__ void weight_sum_kernel(const uint32_t* val, uint32_t m, unsigned long long* sum) {
    unsigned long long s = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) s += val[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane_id() == 0 && s) atomicAdd(sum, s);
}

}  // namespace

// Bucket width: a multiple of the mean edge weight (G1_NEARFAR_DELTA_SCALE,
// default 32); BFS needs no buckets.
g1_status nearfar_delta(g1_graph* g, bool unit, cudaStream_t s, uint32_t* out) {
    if (unit) {
        *out = 1u;
        return G1_OK;
    }
    if (g->mean_weight < 0.0) {
        const Orientation& o = g->o[0];
        unsigned long long* sum = nullptr;
        G1_TRY(g->ws.get("nf_wsum", 2, &sum));
        G1_CUDA(cudaMemsetAsync(sum, 0, 8, s));
        const uint32_t grid = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(ceil_div(g->m, 256), (uint64_t)g->sm_count * 8));
        if (g->m) weight_sum_kernel<<<grid, 256, 0, s>>>(static_cast<const uint32_t*>(o.val), g->m, sum);
        count_launches(1);
        unsigned long long h = 0;
        G1_CUDA(cudaMemcpyAsync(&h, sum, 8, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        g->mean_weight = g->m ? (double)h / (double)g->m : 1.0;
    }
    double scale = 32.0;
    if (const char* e = std::getenv("G1_NEARFAR_DELTA_SCALE")) scale = std::max(0.01, std::atof(e));
    *out = (uint32_t)std::max(1.0, std::min(2.0e9, g->mean_weight * scale));
    return G1_OK;
}

// The distances out of the keys.
__global__ void nf_dist_kernel(const unsigned long long* key, uint32_t n, uint32_t* dist) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        dist[v] = (uint32_t)(key[v] >> 32);
}

size_t nearfar_words(uint32_t n) {
    // keys (8 bytes each), distances; two near queues and two far piles
    // (each vertex at most once in each); the control block (16-byte aligned)
    return 3 * (size_t)n + 4 * ((size_t)n + 1) + sizeof(NfCtl) / 4 + 8;
}

void nearfar_layout(uint32_t n, uint32_t* p, NfBuffers* b) {
    b->key = reinterpret_cast<unsigned long long*>(p);  // the store is 256-byte aligned
    b->dist = p + 2 * (size_t)n;
    uint32_t* q = p + 3 * (size_t)n;
    b->near[0] = q;
    b->near[1] = q + (n + 1);
    b->far[0] = q + 2 * (size_t)(n + 1);
    b->far[1] = q + 3 * (size_t)(n + 1);
    uintptr_t c = reinterpret_cast<uintptr_t>(q + 4 * (size_t)(n + 1));
    c = (c + 15) & ~uintptr_t(15);
    b->ctl = reinterpret_cast<uint32_t*>(c);
}

g1_status nearfar_launch(const g1_graph* g, uint32_t src, bool unit, uint32_t delta, const NfBuffers& b,
                         cudaStream_t s, const uint32_t* perm) {
    if (!g->o[0].present) return fail(G1_ERR_UNSUPPORTED, "near-far engine needs the out-edge CSR");
    const uint32_t n = g->n;
    NfArgs a;
    const Orientation& o = g->o[0];
    a.rp = o.rp;
    a.col = o.col;
    a.val = static_cast<const uint32_t*>(o.val);
    a.n = n;
    a.delta = delta;
    a.key = b.key;
    a.dist = b.dist;
    a.near[0] = b.near[0];
    a.near[1] = b.near[1];
    a.far[0] = b.far[0];
    a.far[1] = b.far[1];
    a.ctl = reinterpret_cast<NfCtl*>(b.ctl);
    a.spin_limit = wait_polls(kNfSpinLimit);
    const uint32_t gi = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n, 256), (uint64_t)g->sm_count * 8));
    // BFS: a threshold above every level -- each step is one level and the
    // far pile stays empty
    nf_init_kernel<<<gi, 256, 0, s>>>(n, src, perm, unit ? kU32Max : a.delta, a.key, a.near[0], a.ctl);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    // every block of a cooperative launch is resident, so the grid barrier
    // only ever waits for running blocks; one 1024-thread block per SM keeps
    // the barrier's arrivals few
    int tpv = 1;
    const uint64_t mean = g->n ? ceil_div(g->m, g->n) : 1;
    while (tpv < 32 && (uint64_t)tpv < mean) tpv <<= 1;
    const void* fn = nullptr;
#define G1_NF_FN(T) fn = unit ? (const void*)nf_kernel<true, T> : (const void*)nf_kernel<false, T>
    switch (tpv) {
        case 1: G1_NF_FN(1); break;
        case 2: G1_NF_FN(2); break;
        case 4: G1_NF_FN(4); break;
        case 8: G1_NF_FN(8); break;
        case 16: G1_NF_FN(16); break;
        default: G1_NF_FN(32); break;
    }
#undef G1_NF_FN
    int per_sm = 0;
    G1_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 1024, 0));
    if (per_sm < 1) return fail(G1_ERR_UNSUPPORTED, "near-far engine: kernel does not fit an SM");
    void* params[] = {&a};
    G1_CUDA(cudaLaunchCooperativeKernel(fn, dim3((uint32_t)g->sm_count), dim3(1024), params, 0, s));
    nf_dist_kernel<<<gi, 256, 0, s>>>(a.key, n, a.dist);
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status nearfar_result(const uint32_t* host_ctl, uint32_t* rounds) {
    NfCtl h;
    memcpy(&h, host_ctl, sizeof(h));
    if (h.err & 1u) return fail(G1_ERR_TIMEOUT, "near-far engine: a grid barrier wait ran out");
    if (rounds) *rounds = h.rounds;
    return G1_OK;
}

uint32_t nearfar_ctl_bytes() { return (uint32_t)sizeof(NfCtl); }

g1_status nearfar_traverse(g1_graph* g, uint32_t src, bool unit, uint32_t** dist_out, uint32_t* rounds,
                           cudaStream_t s, bool frontier) {
    uint32_t delta = kU32Max;  // frontier: the first threshold is already infinite
    if (!frontier) G1_TRY(nearfar_delta(g, unit, s, &delta));
    uint32_t* store = nullptr;
    G1_TRY(g->ws.get("nf_store", nearfar_words(g->n), &store));
    NfBuffers b;
    nearfar_layout(g->n, store, &b);
    G1_TRY(nearfar_launch(g, src, unit, delta, b, s));
    G1_TRY(ws_pinned_ctl(g, b.ctl, s, rounds));
    *dist_out = b.dist;
    return G1_OK;
}

}  // namespace g1
