// libgraphone_b200: status, memory, graph residency, merge-path plans and the
// prebuilt SpMV entry points.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <vector>
#include <cstdio>
#include <cstring>
#include <string>

#include "g1/semiring.cuh"
#include "g1/spmv.cuh"
#include "internal.h"
#include "spmv_launch.cuh"

namespace g1 {

namespace {
thread_local std::string t_last_error;
std::atomic<uint64_t> g_launches{0};
// Poll limit of the bounded device waits set by g1_test_set_wait_polls
// (negative: each wait's default).
std::atomic<int64_t> g_wait_polls{-1};

struct Profiler {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> pool;  // reused events
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> marks;
    cudaEvent_t pending = nullptr;
    size_t used = 0;
    cudaEvent_t next() {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
};
Profiler& prof() {
    static Profiler p;
    return p;
}
}  // namespace

uint32_t wait_polls(uint32_t dflt) {
    const int64_t p = g_wait_polls.load();
    return p < 0 ? dflt : (uint32_t)p;
}

namespace {
thread_local int t_capturing = 0;
}

// Kernels enqueued while this thread captures a CUDA graph are counted when
// the graph is launched, by the caller.
void count_launches(uint64_t n) {
    if (t_capturing == 0) g_launches.fetch_add(n, std::memory_order_relaxed);
}
CaptureScope::CaptureScope() { ++t_capturing; }
CaptureScope::~CaptureScope() { --t_capturing; }

bool profiling() { return prof().on && t_capturing == 0; }

void prof_mark(cudaStream_t s, bool start) {
    Profiler& p = prof();
    std::lock_guard<std::mutex> lk(p.mu);
    if (!p.on) return;
    cudaEvent_t e = p.next();
    cudaEventRecord(e, s);
    if (start) {
        p.pending = e;
    } else if (p.pending) {
        p.marks.emplace_back(p.pending, e);
        p.pending = nullptr;
    }
}

g1_status fail(g1_status s, const std::string& msg) {
    t_last_error = msg;
    return s;
}

g1_status fail_cuda(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();  // clear a non-sticky error
    return fail(e == cudaErrorMemoryAllocation ? G1_ERR_OOM : G1_ERR_DEVICE, m);
}

namespace {

struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, void*> ready;             // idle: reusable now
    std::vector<std::pair<size_t, void*>> pending;  // released since the last device sync
    size_t cached = 0;                              // bytes in both
    size_t cap = 0;                                 // 0 until the device's size is known
};
constexpr int kCacheDevices = 64;
BlockCache g_cache[kCacheDevices];

// Frees every cached block of `dev` (current device); the caller holds c.mu.
void cache_drain_locked(BlockCache& c) {
    if (!c.pending.empty()) cudaDeviceSynchronize();
    for (auto& kv : c.ready) cudaFree(kv.second);
    for (auto& pr : c.pending) cudaFree(pr.second);
    c.ready.clear();
    c.pending.clear();
    c.cached = 0;
}

// The smallest ready block of at least `want` bytes and at most about twice
// that (1 MiB of slack for small requests); the caller holds c.mu.
bool cache_take_locked(BlockCache& c, size_t want, void** p, size_t* got) {
    auto it = c.ready.lower_bound(want);
    if (it == c.ready.end() || it->first > std::max(2 * want, want + (size_t(1) << 20))) return false;
    *p = it->second;
    *got = it->first;
    c.cached -= it->first;
    c.ready.erase(it);
    return true;
}

}  // namespace

void dev_block_release(int dev, void* p, size_t bytes) {
    if (!p) return;
    if (dev < 0 || dev >= kCacheDevices) {
        cudaFree(p);
        return;
    }
    BlockCache& c = g_cache[dev];
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.cap == 0 || c.cached + bytes > c.cap) {
        cudaFree(p);  // over the cap: back to the driver (cudaFree synchronises the device)
        return;
    }
    c.pending.emplace_back(bytes, p);
    c.cached += bytes;
}

size_t dev_block_drain(int dev) {
    if (dev < 0 || dev >= kCacheDevices) return 0;
    BlockCache& c = g_cache[dev];
    std::lock_guard<std::mutex> lk(c.mu);
    const size_t b = c.cached;
    cache_drain_locked(c);
    return b;
}

size_t dev_block_cached(int dev) {
    if (dev < 0 || dev >= kCacheDevices) return 0;
    BlockCache& c = g_cache[dev];
    std::lock_guard<std::mutex> lk(c.mu);
    return c.cached;
}

g1_status dev_block_get(size_t want, void** p, size_t* got, int* dev_out) {
    int dev = 0;
    G1_CUDA(cudaGetDevice(&dev));
    *dev_out = dev;
    const size_t b = (want + 255) & ~size_t(255);
    if (dev < kCacheDevices) {
        BlockCache& c = g_cache[dev];
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.cap == 0) {
            size_t fr = 0, total = 0;
            if (cudaMemGetInfo(&fr, &total) == cudaSuccess) c.cap = total / 4;
            else cudaGetLastError();
        }
        if (cache_take_locked(c, b, p, got)) return G1_OK;
        if (!c.pending.empty()) {
            // released blocks become reusable once the device has drained
            G1_CUDA(cudaDeviceSynchronize());
            for (auto& pr : c.pending) c.ready.emplace(pr.first, pr.second);
            c.pending.clear();
            if (cache_take_locked(c, b, p, got)) return G1_OK;
        }
        cudaError_t e = cudaMalloc(p, b);
        if (e == cudaErrorMemoryAllocation && c.cached > 0) {
            cudaGetLastError();
            cache_drain_locked(c);
            e = cudaMalloc(p, b);
        }
        if (e != cudaSuccess) {
            *p = nullptr;
            return fail_cuda(e, "cudaMalloc(workspace)");
        }
        *got = b;
        return G1_OK;
    }
    cudaError_t e = cudaMalloc(p, b);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail_cuda(e, "cudaMalloc(workspace)");
    }
    *got = b;
    return G1_OK;
}

g1_status DevBuf::ensure(size_t want) {
    if (want <= bytes) return G1_OK;
    release();
    void* q = nullptr;
    size_t got = 0;
    int d = 0;
    G1_TRY(dev_block_get(want, &q, &got, &d));
    p = q;
    bytes = got;
    dev = d;
    return G1_OK;
}

g1_status PinnedBuf::ensure(size_t want) {
    if (want <= bytes) return G1_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    G1_CUDA(cudaHostAlloc(&p, want, cudaHostAllocDefault));
    bytes = want;
    return G1_OK;
}

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

g1_status copy_out(void* dst, const void* dev_src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return G1_OK;
    const bool dev = is_device_ptr(dst);
    G1_CUDA(cudaMemcpyAsync(dst, dev_src, bytes,
                            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    if (!dev) G1_CUDA(cudaStreamSynchronize(s));
    return G1_OK;
}

// ------------------------------------------------------------ kernels

__global__ void merge_partition_kernel(const uint32_t* row_ptr, uint32_t n_rows, uint32_t nnz,
                                       uint32_t items, uint32_t n_tiles, uint32_t* tile_row,
                                       uint32_t* tile_nnz) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    const uint64_t total = (uint64_t)n_rows + nnz;
    uint64_t d = (uint64_t)t * items;
    if (d > total) d = total;
    uint32_t i, j;
    merge_path_search(d, row_ptr + 1, n_rows, nnz, &i, &j);
    tile_row[t] = i;
    tile_nnz[t] = j;
}

// Checks row_ptr[0]==0, row_ptr[n]==m, monotone rows, col < n; records the
// first violation class in *bad (1 = offsets, 2 = column out of range).
__global__ void validate_csr_kernel(const uint32_t* rp, const uint32_t* col, uint32_t n,
                                    uint32_t m, uint32_t* bad, uint32_t* max_deg) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = tid; r < n; r += stride) {
        const uint32_t a = rp[r], b = rp[r + 1];
        if (b < a || b > m) atomicCAS(bad, 0u, 1u);
        else atomicMax(max_deg, b - a);
    }
    if (tid == 0 && (rp[0] != 0 || rp[n] != m)) atomicCAS(bad, 0u, 1u);
    for (uint64_t k = tid; k < m; k += stride)
        if (col[k] >= n) atomicCAS(bad, 0u, 2u);
}

__global__ void max_degree_kernel(const uint32_t* rp, uint32_t n, uint32_t* max_deg) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t mx = 0;
    for (uint64_t r = tid; r < n; r += stride) mx = max(mx, rp[r + 1] - rp[r]);
    atomicMax(max_deg, mx);
}

// Sort keys of a CSR rebuild: for every nonzero (row, col) the new
// (row', col') = swap ? (map(col), map(row)) : (map(row), map(col)) packed
// as (row' << 32) | col'; row found by binary search; map may be null.
__global__ void rebuild_keys_kernel(const uint32_t* rp, const uint32_t* col, uint32_t n,
                                    uint32_t m, const uint32_t* map, int swap, uint64_t* keys,
                                    uint32_t* idx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
        uint32_t lo = 0, hi = n;  // last row r with rp[r] <= k
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (rp[mid] <= k) lo = mid; else hi = mid - 1;
        }
        uint32_t r = lo, c = col[k];
        if (map) {
            r = map[r];
            c = map[c];
        }
        keys[k] = swap ? (((uint64_t)c << 32) | r) : (((uint64_t)r << 32) | c);
        idx[k] = (uint32_t)k;
    }
}

__global__ void degree_kernel(const uint32_t* rp, uint32_t n, uint32_t* deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        deg[v] = rp[v + 1] - rp[v];
}

__global__ void histogram_kernel(const uint32_t* col, uint32_t m, uint32_t* deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride)
        atomicAdd(&deg[col[k]], 1u);
}

__global__ void iota_kernel(uint32_t* p, uint32_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        p[v] = (uint32_t)v;
}

// perm[iperm[k]] = k
__global__ void invert_perm_kernel(const uint32_t* iperm, uint32_t n, uint32_t* perm) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        perm[iperm[k]] = (uint32_t)k;
}

// out[v] = in[perm[v]]: internal (relabelled) order -> caller's order
__global__ void gather_perm_kernel(uint32_t* out, const uint32_t* in, const uint32_t* perm,
                                   uint32_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        out[v] = in[perm[v]];
}

// out[perm[v]] = in[v]: caller's order -> internal order
__global__ void scatter_perm_kernel(uint32_t* out, const uint32_t* in, const uint32_t* perm,
                                    uint32_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        out[perm[v]] = in[v];
}

__global__ void transpose_scatter_kernel(const uint64_t* keys, const uint32_t* idx,
                                         const uint32_t* val_in, uint32_t m, uint32_t* col_out,
                                         uint32_t* val_out, uint32_t* counts) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
        const uint64_t key = keys[k];
        col_out[k] = (uint32_t)(key & 0xffffffffu);
        val_out[k] = val_in[idx[k]];
        atomicAdd(&counts[key >> 32], 1u);
    }
}

__global__ void fill_u32_kernel(uint32_t* p, uint32_t v, size_t n) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

// ------------------------------------------------------------ helpers

namespace {

uint32_t grid_for(uint64_t n, int block, int sm_count, int per_sm = 8) {
    uint64_t g = ceil_div(n ? n : 1, (uint64_t)block);
    uint64_t cap = (uint64_t)sm_count * per_sm;
    return (uint32_t)std::max<uint64_t>(1, std::min(g, cap));
}

// Allocates an orientation's arrays.  The padding past row_ptr[n] and past
// the last nonzero is zero-filled: bulk copies and warp tiles read whole
// aligned ranges without bounds checks (a padding column 0 is a valid index).
// Arrays of n + 1 row offsets and m columns and values, each followed by a
// zeroed pad (the tile kernels' 32-byte loads may run past the last
// nonzero); the caller writes [0, n + 1) and [0, m) on stream s.
g1_status alloc_orientation(Orientation& o, uint32_t n, uint32_t m, cudaStream_t s) {
    const size_t rp_bytes = ((size_t)n + 1 + 64) * 4;
    const size_t nz_bytes = ((size_t)m + kWarpTilePad + 64) * 4;
    G1_TRY(o.b_rp.ensure(rp_bytes));
    G1_TRY(o.b_col.ensure(nz_bytes));
    G1_TRY(o.b_val.ensure(nz_bytes));
    const size_t rp_used = ((size_t)n + 1) * 4, nz_used = (size_t)m * 4;
    G1_CUDA(cudaMemsetAsync(static_cast<char*>(o.b_rp.p) + rp_used, 0, o.b_rp.bytes - rp_used, s));
    G1_CUDA(cudaMemsetAsync(static_cast<char*>(o.b_col.p) + nz_used, 0, o.b_col.bytes - nz_used, s));
    G1_CUDA(cudaMemsetAsync(static_cast<char*>(o.b_val.p) + nz_used, 0, o.b_val.bytes - nz_used, s));
    o.rp = o.b_rp.as<uint32_t>();
    o.col = o.b_col.as<uint32_t>();
    o.val = o.b_val.p;
    o.present = true;
    return G1_OK;
}

g1_status upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return G1_OK;
    const bool dev = is_device_ptr(src);
    G1_CUDA(cudaMemcpyAsync(dst, src, bytes, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    return G1_OK;
}

// Builds `dst` from `src` on the device: the transpose when `swap`, with
// vertex ids renamed through `map` when given.  Stable: rows of the result
// list their columns in increasing order (like EdgeCache::ToCsr on a sorted
// edge cache).
g1_status rebuild_csr(g1_graph* g, const Orientation& src, Orientation& dst, bool swap,
                      const uint32_t* map, cudaStream_t s) {
    const uint32_t n = g->n, m = g->m;
    G1_TRY(alloc_orientation(dst, n, m, s));
    G1_CUDA(cudaMemsetAsync(dst.rp, 0, ((size_t)n + 1) * 4, s));
    if (m == 0) return G1_OK;
    DevBuf keys, keys2, idx, idx2, counts, temp;
    G1_TRY(keys.ensure((size_t)m * 8));
    G1_TRY(keys2.ensure((size_t)m * 8));
    G1_TRY(idx.ensure((size_t)m * 4));
    G1_TRY(idx2.ensure((size_t)m * 4));
    G1_TRY(counts.ensure(((size_t)n + 1) * 4));
    G1_CUDA(cudaMemsetAsync(counts.p, 0, ((size_t)n + 1) * 4, s));
    const uint32_t grid = grid_for(m, 256, g->sm_count);
    rebuild_keys_kernel<<<grid, 256, 0, s>>>(src.rp, src.col, n, m, map, swap ? 1 : 0,
                                             keys.as<uint64_t>(), idx.as<uint32_t>());
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    int row_bits = 1;
    while (row_bits < 32 && (1ull << row_bits) < n) ++row_bits;
    const int end_bit = 32 + row_bits;
    size_t tb = 0;
    G1_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                            idx.as<uint32_t>(), idx2.as<uint32_t>(), (int)m, 0,
                                            end_bit, s));
    G1_TRY(temp.ensure(tb));
    G1_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                            idx.as<uint32_t>(), idx2.as<uint32_t>(), (int)m, 0,
                                            end_bit, s));
    transpose_scatter_kernel<<<grid, 256, 0, s>>>(keys2.as<uint64_t>(), idx2.as<uint32_t>(),
                                                  static_cast<const uint32_t*>(src.val), m, dst.col,
                                                  static_cast<uint32_t*>(dst.val),
                                                  counts.as<uint32_t>());
    G1_CUDA(cudaGetLastError());
    size_t tb2 = 0;
    G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, counts.as<uint32_t>(), dst.rp, (int)n + 1, s));
    DevBuf temp2;
    G1_TRY(temp2.ensure(tb2));
    G1_CUDA(cub::DeviceScan::ExclusiveSum(temp2.p, tb2, counts.as<uint32_t>(), dst.rp, (int)n + 1, s));
    G1_CUDA(cudaStreamSynchronize(s));  // temporaries die here
    return G1_OK;
}

// Moves the arrays of `fresh` into `o` (old arrays are freed).
void adopt(Orientation& o, Orientation& fresh) {
    o.b_rp.swap(fresh.b_rp);
    o.b_col.swap(fresh.b_col);
    o.b_val.swap(fresh.b_val);
    o.rp = o.b_rp.as<uint32_t>();
    o.col = o.b_col.as<uint32_t>();
    o.val = o.b_val.p;
    o.present = true;
    o.plans.clear();
}

// Degree-ordered relabelling: internal id k is the k-th vertex by
// decreasing out-degree (ties by id).  The hottest x entries of the pull
// SpMV become a contiguous prefix that the warp-tile kernel caches in
// shared memory.
g1_status relabel_by_degree(g1_graph* g, cudaStream_t s) {
    const uint32_t n = g->n;
    DevBuf deg, deg2, ids, temp;
    G1_TRY(deg.ensure((size_t)n * 4 + 16));
    G1_TRY(deg2.ensure((size_t)n * 4 + 16));
    G1_TRY(ids.ensure((size_t)n * 4 + 16));
    G1_TRY(g->iperm.ensure((size_t)n * 4 + 16));
    G1_TRY(g->perm.ensure((size_t)n * 4 + 16));
    const uint32_t grid = grid_for(std::max(n, g->m), 256, g->sm_count);
    if (g->o[0].present) {
        degree_kernel<<<grid, 256, 0, s>>>(g->o[0].rp, n, deg.as<uint32_t>());
    } else {
        G1_CUDA(cudaMemsetAsync(deg.p, 0, (size_t)n * 4, s));
        histogram_kernel<<<grid, 256, 0, s>>>(g->o[1].col, g->m, deg.as<uint32_t>());
    }
    iota_kernel<<<grid, 256, 0, s>>>(ids.as<uint32_t>(), n);
    count_launches(2);
    G1_CUDA(cudaGetLastError());
    size_t tb = 0;
    G1_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, deg.as<uint32_t>(),
                                                      deg2.as<uint32_t>(), ids.as<uint32_t>(),
                                                      g->iperm.as<uint32_t>(), (int)n, 0, 32, s));
    G1_TRY(temp.ensure(tb));
    G1_CUDA(cub::DeviceRadixSort::SortPairsDescending(temp.p, tb, deg.as<uint32_t>(),
                                                      deg2.as<uint32_t>(), ids.as<uint32_t>(),
                                                      g->iperm.as<uint32_t>(), (int)n, 0, 32, s));
    invert_perm_kernel<<<grid, 256, 0, s>>>(g->iperm.as<uint32_t>(), n, g->perm.as<uint32_t>());
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    const uint32_t* map = g->perm.as<uint32_t>();
    for (int t = 0; t < 2; ++t) {
        Orientation& o = g->o[t];
        if (!o.present || !o.b_rp.p) continue;  // shared arrays are renamed once
        Orientation fresh;
        G1_TRY(rebuild_csr(g, o, fresh, false, map, s));
        adopt(o, fresh);
    }
    if (g->symmetric) {
        const int own = g->o[0].b_rp.p ? 0 : 1;
        Orientation& o = g->o[own];
        Orientation& other = g->o[own ^ 1];
        other.rp = o.rp;
        other.col = o.col;
        other.val = o.val;
        other.plans.clear();
    }
    g->relabeled = true;
    g->outw_ready = false;  // per-vertex data derived before are in the old ids
    g->outdeg_ready = false;
    G1_CUDA(cudaStreamSynchronize(s));
    return G1_OK;
}

}  // namespace

// The orientation whose plans serve t: symmetric graphs share one CSR and
// its plans; the hot-column copy (2) has the in-edge CSR's rows.
static Orientation& plan_owner(g1_graph* g, int t) {
    const int u = t == 2 ? 1 : t;
    return (u == 1 && g->symmetric && g->o[0].present) ? g->o[0] : g->o[u];
}

g1_status ensure_plan(g1_graph* g, int t, uint32_t items, MergePlan** out) {
    Orientation& o = g->o[t];
    if (!o.present) return fail(G1_ERR_UNSUPPORTED, "orientation not built");
    Orientation& owner = plan_owner(g, t);
    auto it = owner.plans.find(items);
    if (it != owner.plans.end()) {
        *out = it->second.get();
        return G1_OK;
    }
    std::unique_ptr<MergePlan> p(new MergePlan());
    p->items = items;
    const uint64_t total = (uint64_t)g->n + g->m;
    p->n_tiles = (uint32_t)ceil_div(total, p->items);
    G1_TRY(p->tile_row.ensure(((size_t)p->n_tiles + 1) * 4));
    G1_TRY(p->tile_nnz.ensure(((size_t)p->n_tiles + 1) * 4));
    G1_TRY(p->carry.ensure(((size_t)p->n_tiles + 1) * 16));
    G1_TRY(p->tail.ensure(((size_t)p->n_tiles + 1) * 16));
    const uint32_t blocks = (uint32_t)ceil_div((uint64_t)p->n_tiles + 1, 256);
    merge_partition_kernel<<<blocks, 256>>>(o.rp, g->n, g->m, p->items, p->n_tiles,
                                            p->tile_row.as<uint32_t>(), p->tile_nnz.as<uint32_t>());
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    G1_CUDA(cudaDeviceSynchronize());
    *out = p.get();
    owner.plans[items] = std::move(p);
    return G1_OK;
}

// ------------------------------------------------------------- nnz plan

__global__ void nnz_flag_kernel(const uint32_t* rp, uint32_t n, uint32_t* flag) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        flag[r] = rp[r + 1] > rp[r] ? 1u : 0u;
}

// Non-empty rows to rows[rank], empty rows after them; start bits of the
// non-empty rows' first nonzeros.
__global__ void nnz_place_kernel(const uint32_t* rp, uint32_t n, const uint32_t* rank,
                                 uint32_t n_nonempty, uint32_t* rows, uint32_t* sbits) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const uint32_t k = rank[r];
        if (rp[r + 1] > rp[r]) {
            rows[k] = (uint32_t)r;
            atomicOr(&sbits[rp[r] >> 5], 1u << (rp[r] & 31));
        } else {
            rows[n_nonempty + ((uint32_t)r - k)] = (uint32_t)r;
        }
    }
}

// tile_seg[t] = rank of the row holding nonzero t*tile (the last row r with
// rp[r] <= t*tile; it is non-empty); n_nonempty past the last nonzero.
__global__ void nnz_tile_seg_kernel(const uint32_t* rp, uint32_t n, uint32_t nnz, const uint32_t* rank,
                                    uint32_t n_nonempty, uint32_t n_tiles, uint32_t tile,
                                    uint32_t* tile_seg) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    const uint64_t k = (uint64_t)t * tile;
    if (k >= nnz) {
        tile_seg[t] = n_nonempty;
        return;
    }
    uint32_t lo = 0, hi = n;  // last r in [0, n) with rp[r] <= k
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (rp[mid] <= k) lo = mid; else hi = mid - 1;
    }
    tile_seg[t] = rank[lo];
}

// Tiles t >= 1 whose first nonzero continues a row begun earlier and in
// which that row ends (another row starts inside, or the next tile starts
// with a row, or the matrix ends).
__global__ void nnz_fix_flag_kernel(const uint32_t* sbits, uint32_t n_tiles, uint32_t nnz, uint32_t tile,
                                    uint32_t* flag) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n_tiles) return;
    uint32_t f = 0;
    if (t > 0 && t < n_tiles) {
        const uint32_t w0 = t * (tile / 32);
        if (!(sbits[w0] & 1u)) {
            uint32_t any = 0;
            for (uint32_t q = 0; q < tile / 32; ++q) any |= sbits[w0 + q];
            const bool end_start = (uint64_t)(t + 1) * tile >= nnz || (sbits[w0 + tile / 32] & 1u);
            f = (any != 0u || end_start) ? 1u : 0u;
        }
    }
    flag[t] = f;
}

__global__ void nnz_fix_place_kernel(const uint32_t* flag, const uint32_t* pos, uint32_t n_tiles,
                                     uint32_t* fix_tiles) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_tiles && flag[t]) fix_tiles[pos[t]] = t;
}

// is_long[i]: fix entry i's row spans more than one tile boundary (its
// first nonzero lies before tile t-1).
__global__ void nnz_fix_long_kernel(const uint32_t* fix_tiles, uint32_t n_fix, const uint32_t* tile_seg,
                                    const uint32_t* nz_rows, const uint32_t* rp, uint32_t tile,
                                    uint32_t* is_long) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n_fix) return;
    if (i == n_fix) {
        is_long[i] = 0;
        return;
    }
    const uint32_t t = fix_tiles[i];
    const uint32_t row = nz_rows[tile_seg[t]];
    is_long[i] = rp[row] / tile + 1 < t ? 1u : 0u;
}

// The fixup's per-entry facts {tile, row, first tile of the row}, resolved
// once per graph instead of through tile_seg -> rows -> row_ptr on every
// launch: entries of rows that cross one boundary first, then the longer
// chains, each in tile order (lpos: exclusive scan of is_long).
__global__ void nnz_fix_info_kernel(const uint32_t* fix_tiles, uint32_t n_fix, const uint32_t* tile_seg,
                                    const uint32_t* nz_rows, const uint32_t* rp, uint32_t tile,
                                    const uint32_t* lpos, uint32_t n_short, uint4* info) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_fix) return;
    const uint32_t t = fix_tiles[i];
    const uint32_t row = nz_rows[tile_seg[t]];
    const uint32_t first = rp[row] / tile;
    info[first + 1 < t ? n_short + lpos[i] : i - lpos[i]] = make_uint4(t, row, first, 0u);
}

g1_status ensure_nnz_plan(g1_graph* g, int t, NnzPlan** out, uint32_t tile) {
    Orientation& o = g->o[t];
    if (!o.present) return fail(G1_ERR_UNSUPPORTED, "orientation not built");
    if (tile == 0 || tile % 32 != 0) return fail(G1_ERR_INVALID, "nnz plan: tile not a multiple of 32");
    Orientation& owner = plan_owner(g, t);
    auto& slot = owner.nnz_plans[tile];
    if (slot) {
        *out = slot.get();
        return G1_OK;
    }
    const uint32_t n = g->n, m = g->m;
    std::unique_ptr<NnzPlan> p(new NnzPlan());
    p->tile = tile;
    p->n_tiles = (uint32_t)ceil_div(m, tile);
    const size_t words = (size_t)p->n_tiles * (tile / 32) + 2 + 16;
    G1_TRY(p->tile_seg.ensure(((size_t)p->n_tiles + 1) * 4 + 16));
    G1_TRY(p->sbits.ensure(words * 4));
    G1_TRY(p->rows.ensure(((size_t)n + 1) * 4));
    G1_TRY(p->carry.ensure(((size_t)p->n_tiles + 1) * 16));
    G1_TRY(p->tail.ensure(((size_t)p->n_tiles + 1) * 16));
    // scratch shared by every phase below (vertices, tiles, fix entries)
    DevBuf flag, rank, temp;
    const size_t scratch = ((size_t)std::max(n, p->n_tiles) + 1) * 4;
    G1_TRY(flag.ensure(scratch));
    G1_TRY(rank.ensure(scratch));
    const uint32_t grid = grid_for(n, 256, g->sm_count);
    G1_CUDA(cudaMemset(p->sbits.p, 0, words * 4));
    G1_CUDA(cudaMemset(flag.p, 0, ((size_t)n + 1) * 4));
    nnz_flag_kernel<<<grid, 256>>>(o.rp, n, flag.as<uint32_t>());
    size_t tb = 0;
    G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.as<uint32_t>(), rank.as<uint32_t>(), (int)n + 1));
    G1_TRY(temp.ensure(tb + 16));
    G1_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, flag.as<uint32_t>(), rank.as<uint32_t>(), (int)n + 1));
    uint32_t nne = 0;
    G1_CUDA(cudaMemcpy(&nne, rank.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost));
    p->n_nonempty = nne;
    p->n_empty = n - nne;
    nnz_place_kernel<<<grid, 256>>>(o.rp, n, rank.as<uint32_t>(), nne, p->rows.as<uint32_t>(),
                                    p->sbits.as<uint32_t>());
    nnz_tile_seg_kernel<<<(uint32_t)ceil_div((uint64_t)p->n_tiles + 1, 256), 256>>>(
        o.rp, n, m, rank.as<uint32_t>(), nne, p->n_tiles, tile, p->tile_seg.as<uint32_t>());
    // tiles the fixup visits, in tile order (a deterministic compaction)
    {
        uint32_t* fflag = flag.as<uint32_t>();
        uint32_t* fpos = rank.as<uint32_t>();
        const uint32_t tb = (uint32_t)ceil_div((uint64_t)p->n_tiles + 1, 256);
        nnz_fix_flag_kernel<<<tb, 256>>>(p->sbits.as<uint32_t>(), p->n_tiles, m, tile, fflag);
        size_t sb = 0;
        G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, fflag, fpos, (int)p->n_tiles + 1));
        G1_TRY(temp.ensure(sb + 16));
        G1_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, sb, fflag, fpos, (int)p->n_tiles + 1));
        uint32_t nfix = 0;
        G1_CUDA(cudaMemcpy(&nfix, fpos + p->n_tiles, 4, cudaMemcpyDeviceToHost));
        p->n_fix = nfix;
        G1_TRY(p->fix_tiles.ensure(((size_t)nfix + 1) * 4));
        nnz_fix_place_kernel<<<tb, 256>>>(fflag, fpos, p->n_tiles, p->fix_tiles.as<uint32_t>());
        G1_TRY(p->fix_info.ensure(((size_t)nfix + 1) * 16));
        p->n_fix_short = 0;
        if (nfix > 0) {
            // fix entries by kind (flag, rank reused: nfix <= n_tiles)
            uint32_t* lflag = flag.as<uint32_t>();
            uint32_t* lpos = rank.as<uint32_t>();
            const uint32_t fb = (uint32_t)ceil_div((uint64_t)nfix + 1, 256);
            nnz_fix_long_kernel<<<fb, 256>>>(p->fix_tiles.as<uint32_t>(), nfix, p->tile_seg.as<uint32_t>(),
                                             p->rows.as<uint32_t>(), o.rp, tile, lflag);
            size_t lb = 0;
            G1_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, lb, lflag, lpos, (int)nfix + 1));
            G1_TRY(temp.ensure(lb + 16));
            G1_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, lb, lflag, lpos, (int)nfix + 1));
            uint32_t nlong = 0;
            G1_CUDA(cudaMemcpy(&nlong, lpos + nfix, 4, cudaMemcpyDeviceToHost));
            p->n_fix_short = nfix - nlong;
            nnz_fix_info_kernel<<<fb, 256>>>(p->fix_tiles.as<uint32_t>(), nfix, p->tile_seg.as<uint32_t>(),
                                             p->rows.as<uint32_t>(), o.rp, tile, lpos, p->n_fix_short,
                                             p->fix_info.as<uint4>());
        }
    }
    count_launches(p->n_fix > 0 ? 7 : 5);
    G1_CUDA(cudaGetLastError());
    G1_CUDA(cudaDeviceSynchronize());
    *out = p.get();
    slot = std::move(p);
    return G1_OK;
}

g1_status to_caller_order(g1_graph* g, uint32_t* dev_out, const uint32_t* internal,
                          cudaStream_t s) {
    gather_perm_kernel<<<grid_for(g->n, 256, g->sm_count), 256, 0, s>>>(
        dev_out, internal, g->perm.as<uint32_t>(), g->n);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status to_internal_order(g1_graph* g, uint32_t* dev_out, const uint32_t* caller,
                            cudaStream_t s) {
    scatter_perm_kernel<<<grid_for(g->n, 256, g->sm_count), 256, 0, s>>>(
        dev_out, caller, g->perm.as<uint32_t>(), g->n);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status internal_vertex(g1_graph* g, uint32_t v, uint32_t* out, cudaStream_t s) {
    if (!g->relabeled) {
        *out = v;
        return G1_OK;
    }
    G1_CUDA(cudaMemcpyAsync(out, g->perm.as<uint32_t>() + v, 4, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    return G1_OK;
}

g1_status copy_out_vertices(g1_graph* g, void* dst, const void* internal, cudaStream_t s) {
    if (!g->relabeled) return copy_out(dst, internal, (size_t)g->n * 4, s);
    uint32_t* tmp = nullptr;
    G1_TRY(g->ws.get("perm_out", g->n, &tmp));
    G1_TRY(to_caller_order(g, tmp, static_cast<const uint32_t*>(internal), s));
    return copy_out(dst, tmp, (size_t)g->n * 4, s);
}

g1_status check_device_error(g1_graph* g, cudaStream_t s) {
    uint32_t h = 0;
    G1_CUDA(cudaMemcpyAsync(&h, g->err_word, 4, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    if (h == 0) return G1_OK;
    G1_CUDA(cudaMemsetAsync(g->err_word, 0, 4, s));
    if (h == kDevTimeout) return fail(G1_ERR_TIMEOUT, "a bounded device wait ran out");
    if (h == kDevOverflow) return fail(G1_ERR_OVERFLOW, "a device queue overflowed");
    if (h == kDevInvalid) return fail(G1_ERR_INVALID, "a vertex id in the input was out of range");
    return fail(G1_ERR_DEVICE, "device error word " + std::to_string(h));
}

}  // namespace g1

using namespace g1;

extern "C" {

const char* g1_status_string(g1_status s) {
    switch (s) {
        case G1_OK: return "ok";
        case G1_ERR_INVALID: return "invalid argument";
        case G1_ERR_OOM: return "out of device memory";
        case G1_ERR_DEVICE: return "CUDA error";
        case G1_ERR_TIMEOUT: return "device wait timed out";
        case G1_ERR_UNSUPPORTED: return "unsupported";
        case G1_ERR_OVERFLOW: return "device queue overflow";
    }
    return "unknown status";
}

const char* g1_last_error(void) { return t_last_error.c_str(); }

const char* g1_version(void) { return "graphone_b200 0.1 sm_100a"; }

uint64_t g1_kernel_launches(void) { return g_launches.load(); }

g1_status g1_test_set_wait_polls(int64_t polls) {
    g_wait_polls.store(polls < 0 ? -1 : std::min<int64_t>(polls, 0xFFFFFFFFll));
    return G1_OK;
}

void g1_count_user_launches(uint64_t n) { count_launches(n); }

g1_status g1_profile_begin(void) {
    Profiler& p = prof();
    std::lock_guard<std::mutex> lk(p.mu);
    p.marks.clear();
    p.used = 0;
    p.pending = nullptr;
    p.on = true;
    return G1_OK;
}

g1_status g1_profile_end(double* spmv_ms, uint64_t* spmv_launches) {
    Profiler& p = prof();
    std::lock_guard<std::mutex> lk(p.mu);
    p.on = false;
    double total = 0.0;
    for (auto& m : p.marks) {
        G1_CUDA(cudaEventSynchronize(m.second));
        float ms = 0.0f;
        G1_CUDA(cudaEventElapsedTime(&ms, m.first, m.second));
        total += ms;
    }
    if (spmv_ms) *spmv_ms = total;
    if (spmv_launches) *spmv_launches = p.marks.size();
    p.marks.clear();
    p.used = 0;
    return G1_OK;
}

g1_status g1_mem_alloc(void** ptr, size_t bytes) {
    if (!ptr) return fail(G1_ERR_INVALID, "g1_mem_alloc: null out pointer");
    *ptr = nullptr;
    const size_t b = ((bytes ? bytes : 1) + 255) & ~size_t(255);
    G1_CUDA(cudaMalloc(ptr, b));
    G1_CUDA(cudaMemset(*ptr, 0, b));
    return G1_OK;
}

g1_status g1_mem_free(void* ptr) {
    if (ptr) G1_CUDA(cudaFree(ptr));
    return G1_OK;
}

g1_status g1_release_cached_memory(size_t* released_bytes) {
    int dev = 0;
    G1_CUDA(cudaGetDevice(&dev));
    const size_t b = dev_block_drain(dev);
    if (released_bytes) *released_bytes = b;
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status g1_mem_copy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
    if (bytes == 0) return G1_OK;
    if (!dst || !src) return fail(G1_ERR_INVALID, "g1_mem_copy: null pointer");
    cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                       : kind == 1 ? cudaMemcpyDeviceToHost
                                   : cudaMemcpyDeviceToDevice;
    G1_CUDA(cudaMemcpyAsync(dst, src, bytes, k, as_stream(stream)));
    if (kind == 1) G1_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return G1_OK;
}

g1_status g1_mem_fill_u32(void* dst, uint32_t value, size_t count, void* stream) {
    if (count == 0) return G1_OK;
    if (!dst) return fail(G1_ERR_INVALID, "g1_mem_fill_u32: null pointer");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    fill_u32_kernel<<<grid_for(count, 256, sms), 256, 0, as_stream(stream)>>>(
        static_cast<uint32_t*>(dst), value, count);
    count_launches(1);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

g1_status g1_stream_sync(void* stream) {
    G1_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return G1_OK;
}

// Edges from which graph creation sums a directed in-edge CSR's out-weights
// during its upload.
constexpr uint32_t kEagerOutwMinEdges = 1u << 22;

g1_status g1_graph_create(const uint32_t* row_ptr, const uint32_t* col, const void* val,
                          g1_dtype vtype, uint32_t n, uint32_t m, uint32_t flags, void* stream,
                          g1_graph** out) {
    if (!out) return fail(G1_ERR_INVALID, "g1_graph_create: null out pointer");
    *out = nullptr;
    if (!row_ptr || (m > 0 && (!col || !val)))
        return fail(G1_ERR_INVALID, "g1_graph_create: null CSR array");
    if (vtype != G1_U32 && vtype != G1_F32)
        return fail(G1_ERR_INVALID, "g1_graph_create: unknown value type");
    if ((uint64_t)n + m >= 0xFFFFFFFFull || n == 0xFFFFFFFFu)
        return fail(G1_ERR_INVALID, "g1_graph_create: n + m must stay below 2^32 - 1");
    cudaStream_t s = as_stream(stream);
    std::unique_ptr<g1_graph> g(new g1_graph());
    G1_CUDA(cudaGetDevice(&g->device));
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, g->device);
    G1_TRY(g->err_buf.ensure(16));
    g->err_word = g->err_buf.as<uint32_t>();
    G1_CUDA(cudaMemsetAsync(g->err_word, 0, 16, s));
    g->n = n;
    g->m = m;
    g->vtype = vtype;
    g->symmetric = (flags & G1_GRAPH_SYMMETRIC) != 0;
    const int side = (flags & G1_GRAPH_INPUT_TRANSPOSE) ? 1 : 0;
    Orientation& o = g->o[side];
    G1_TRY(alloc_orientation(o, n, m, s));
    G1_TRY(upload(o.rp, row_ptr, ((size_t)n + 1) * 4, s));
    // A large directed in-edge CSR with f32 values (a PageRank input) from
    // host memory, kept as it is (no out-edge CSR built, not relabelled):
    // its out-weights are summed while the copy is in flight.
    if (side == 1 && !g->symmetric && vtype == G1_F32 && m >= kEagerOutwMinEdges &&
        !(flags & (G1_GRAPH_BUILD_OTHER | G1_GRAPH_RELABEL)) && !is_device_ptr(col) &&
        !is_device_ptr(val)) {
        G1_TRY(upload_transpose_with_outw(g.get(), col, val, s));
    } else {
        G1_TRY(upload(o.col, col, (size_t)m * 4, s));
        G1_TRY(upload(o.val, val, (size_t)m * 4, s));
    }

    DevBuf chk;
    G1_TRY(chk.ensure(16));
    G1_CUDA(cudaMemsetAsync(chk.p, 0, 16, s));
    uint32_t* d_bad = chk.as<uint32_t>();
    uint32_t* d_maxdeg = d_bad + 1;
    const uint32_t grid = grid_for((uint64_t)std::max(n, m), 256, g->sm_count);
    count_launches(1);
    if (!(flags & G1_GRAPH_NO_VALIDATE)) {
        validate_csr_kernel<<<grid, 256, 0, s>>>(o.rp, o.col, n, m, d_bad, d_maxdeg);
    } else {
        max_degree_kernel<<<grid, 256, 0, s>>>(o.rp, n, d_maxdeg);
    }
    G1_CUDA(cudaGetLastError());
    uint32_t h[2] = {0, 0};
    G1_CUDA(cudaMemcpyAsync(h, chk.p, 8, cudaMemcpyDeviceToHost, s));
    G1_CUDA(cudaStreamSynchronize(s));
    if (h[0] == 1) return fail(G1_ERR_INVALID, "g1_graph_create: malformed row offsets");
    if (h[0] == 2) return fail(G1_ERR_INVALID, "g1_graph_create: column index out of range");
    o.max_deg = h[1];

    Orientation& other = g->o[side ^ 1];
    if (g->symmetric) {
        other.present = true;
        other.rp = o.rp;
        other.col = o.col;
        other.val = o.val;
        other.max_deg = o.max_deg;
    } else if (flags & G1_GRAPH_BUILD_OTHER) {
        G1_TRY(rebuild_csr(g.get(), o, other, true, nullptr, s));
        G1_CUDA(cudaMemsetAsync(chk.p, 0, 16, s));
        max_degree_kernel<<<grid, 256, 0, s>>>(other.rp, n, d_maxdeg);
        count_launches(1);
        G1_CUDA(cudaMemcpyAsync(h, chk.p, 8, cudaMemcpyDeviceToHost, s));
        G1_CUDA(cudaStreamSynchronize(s));
        other.max_deg = h[1];
    }
    if (flags & G1_GRAPH_RELABEL) G1_TRY(relabel_by_degree(g.get(), s));
    *out = g.release();
    return G1_OK;
}

g1_status g1_graph_destroy(g1_graph* g) {
    if (!g) return G1_OK;
    DeviceGuard dg(g->device);
    cudaDeviceSynchronize();
    delete g;
    return G1_OK;
}

g1_status g1_graph_info(const g1_graph* g, uint32_t* n, uint32_t* m, int* has_normal,
                        int* has_transpose) {
    if (!g) return fail(G1_ERR_INVALID, "g1_graph_info: null graph");
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (has_normal) *has_normal = g->o[0].present;
    if (has_transpose) *has_transpose = g->o[1].present;
    return G1_OK;
}

g1_status g1_graph_arrays(const g1_graph* g, int transpose, const uint32_t** row_ptr,
                          const uint32_t** col, const void** val) {
    if (!g || transpose < 0 || transpose > 1) return fail(G1_ERR_INVALID, "g1_graph_arrays");
    const Orientation& o = g->o[transpose];
    if (!o.present) return fail(G1_ERR_UNSUPPORTED, "g1_graph_arrays: orientation not built");
    if (row_ptr) *row_ptr = o.rp;
    if (col) *col = o.col;
    if (val) *val = o.val;
    return G1_OK;
}

size_t g1_graph_device_bytes(const g1_graph* g) {
    if (!g) return 0;
    size_t s = g->ws.bytes();
    for (int t = 0; t < 3; ++t) {
        const Orientation& o = g->o[t];
        s += o.b_rp.bytes + o.b_col.bytes + o.b_val.bytes;
        for (auto& kv : o.plans)
            s += kv.second->tile_row.bytes + kv.second->tile_nnz.bytes + kv.second->carry.bytes +
                 kv.second->tail.bytes;
    }
    return s;
}

g1_status g1_spmv_plan(g1_graph* g, int transpose, uint32_t items_per_tile, uint32_t* n_tiles,
                       const uint32_t** tile_row, const uint32_t** tile_nnz, void** carry,
                       void** tail) {
    if (!g || transpose < 0 || transpose > 1) return fail(G1_ERR_INVALID, "g1_spmv_plan");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    MergePlan* pp = nullptr;
    const uint32_t items =
        items_per_tile ? items_per_tile : merge_items(merge_variant(g, transpose));
    G1_TRY(ensure_plan(g, transpose, items, &pp));
    const MergePlan& p = *pp;
    if (n_tiles) *n_tiles = p.n_tiles;
    if (tile_row) *tile_row = p.tile_row.as<uint32_t>();
    if (tile_nnz) *tile_nnz = p.tile_nnz.as<uint32_t>();
    if (carry) *carry = p.carry.p;
    if (tail) *tail = p.tail.p;
    return G1_OK;
}

g1_status g1_spmv_nnz_plan(g1_graph* g, int transpose, g1_nnz_plan* out) {
    if (!g || transpose < 0 || transpose > 1 || !out) return fail(G1_ERR_INVALID, "g1_spmv_nnz_plan");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    NnzPlan* pp = nullptr;
    G1_TRY(ensure_nnz_plan(g, transpose, &pp));
    const NnzPlan& p = *pp;
    out->n_rows = g->n;
    out->nnz = g->m;
    out->n_tiles = p.n_tiles;
    out->n_nonempty = p.n_nonempty;
    out->n_empty = p.n_empty;
    out->n_fix = p.n_fix;
    out->n_fix_short = p.n_fix_short;
    out->tile_seg = p.tile_seg.as<uint32_t>();
    out->sbits = p.sbits.as<uint32_t>();
    out->rows = p.rows.as<uint32_t>();
    out->row_ptr = g->o[transpose].rp;
    out->fix_tiles = p.fix_tiles.as<uint32_t>();
    out->fix_info = p.fix_info.p;
    out->carry = p.carry.p;
    out->tail = p.tail.p;
    return G1_OK;
}

g1_status g1_spmv(g1_graph* g, int transpose, g1_semiring sr, g1_schedule sched, const void* x,
                  void* y, void* stream) {
    if (!g || transpose < 0 || transpose > 1 || !x || !y)
        return fail(G1_ERR_INVALID, "g1_spmv: bad argument");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    if (!g->o[transpose].present) return fail(G1_ERR_UNSUPPORTED, "g1_spmv: orientation not built");
    const bool fval = sr == G1_SR_MINPLUS_F32 || sr == G1_SR_PLUSTIMES_F32;
    if (sr != G1_SR_BFS_U32 && fval != (g->vtype == G1_F32))
        return fail(G1_ERR_INVALID, "g1_spmv: semiring value type does not match the graph");
    cudaStream_t s = as_stream(stream);
    if (g->relabeled) {
        // x and y are in the caller's vertex order
        uint32_t *xi = nullptr, *yi = nullptr;
        G1_TRY(g->ws.get("spmv_xi", g->n, &xi));
        G1_TRY(g->ws.get("spmv_yi", g->n, &yi));
        G1_TRY(to_internal_order(g, xi, static_cast<const uint32_t*>(x), s));
        G1_TRY(spmv_dispatch(g, transpose, sr, sched, xi, yi, s));
        return to_caller_order(g, static_cast<uint32_t*>(y), yi, s);
    }
    return spmv_dispatch(g, transpose, sr, sched, x, y, s);
}

}  // extern "C"

namespace g1 {
g1_status spmv_dispatch(g1_graph* g, int transpose, g1_semiring sr, g1_schedule sched,
                        const void* x, void* y, cudaStream_t s) {
    switch (sr) {
        case G1_SR_MINPLUS_U32:
            return run_spmv<MinPlusU32>(g, transpose, sched, static_cast<const uint32_t*>(x),
                                        StoreEpilogue<uint32_t>{static_cast<uint32_t*>(y)}, s);
        case G1_SR_MINPLUS_F32:
            return run_spmv<MinPlusF32>(g, transpose, sched, static_cast<const float*>(x),
                                        StoreEpilogue<float>{static_cast<float*>(y)}, s);
        case G1_SR_PLUSTIMES_F32:
            return run_spmv<PlusTimesF32>(g, transpose, sched, static_cast<const float*>(x),
                                          StoreEpilogue<float>{static_cast<float*>(y)}, s);
        case G1_SR_BFS_U32:
            return run_spmv<BfsU32>(g, transpose, sched, static_cast<const uint32_t*>(x),
                                    StoreEpilogue<uint32_t>{static_cast<uint32_t*>(y)}, s);
    }
    return fail(G1_ERR_INVALID, "g1_spmv: unknown semiring");
}
}  // namespace g1

extern "C" {

g1_status g1_graph_set_schedule(g1_graph* g, int transpose, g1_schedule sched, int variant) {
    if (!g || transpose < 0 || transpose > 1) return fail(G1_ERR_INVALID, "g1_graph_set_schedule");
    if (sched == G1_SCHED_MERGE && (variant < 0 || variant >= kNumMergeVariants))
        return fail(G1_ERR_INVALID, "g1_graph_set_schedule: merge variant out of range");
    std::lock_guard<std::mutex> lk(g->mu);
    for (int t = 0; t < 2; ++t) {
        if (t != transpose && !(g->o[t].present && g->o[t].rp == g->o[transpose].rp)) continue;
        g->o[t].tuned_sched = sched == G1_SCHED_AUTO ? 0 : sched;
        g->o[t].tuned_variant = sched == G1_SCHED_MERGE ? variant : -1;
    }
    return G1_OK;
}

g1_status g1_autotune(g1_graph* g, float* merge_ms, float* vector_ms, int* merge_variant,
                      void* stream) {
    if (!g) return fail(G1_ERR_INVALID, "g1_autotune: null graph");
    DeviceGuard dg(g->device);
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStream_t s = as_stream(stream);
    const int t = pull_side(g);
    if (!g->o[t].present) return fail(G1_ERR_UNSUPPORTED, "g1_autotune: no CSR");
    uint32_t *x = nullptr, *y = nullptr;
    G1_TRY(g->ws.get("tune_x", g->n, &x));
    G1_TRY(g->ws.get("tune_y", g->n, &y));
    G1_CUDA(cudaMemsetAsync(x, 0, (size_t)g->n * 4, s));
    cudaEvent_t e0, e1;
    G1_CUDA(cudaEventCreate(&e0));
    G1_CUDA(cudaEventCreate(&e1));
    // candidates: every merge variant, and CSR-vector
    float best_merge = 1e30f, vec = 1e30f;
    int best_variant = kDefaultVariant;
    Orientation& o = g->o[t];
    auto time_it = [&](g1_schedule sc, float* out) -> g1_status {
        for (int rep = 0; rep < 2; ++rep)
            G1_TRY((run_spmv<BfsU32>(g, t, sc, x, StoreEpilogue<uint32_t>{y}, s)));
        cudaEventRecord(e0, s);
        for (int rep = 0; rep < 5; ++rep)
            G1_TRY((run_spmv<BfsU32>(g, t, sc, x, StoreEpilogue<uint32_t>{y}, s)));
        cudaEventRecord(e1, s);
        G1_CUDA(cudaEventSynchronize(e1));
        cudaEventElapsedTime(out, e0, e1);
        *out /= 5;
        return G1_OK;
    };
    for (int c = 0; c < kNumMergeVariants; ++c) {
        o.tuned_variant = c;
        float ms = 0;
        G1_TRY(time_it(G1_SCHED_MERGE, &ms));
        if (ms < best_merge) {
            best_merge = ms;
            best_variant = c;
        }
    }
    G1_TRY(time_it(G1_SCHED_VECTOR, &vec));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    o.tuned_variant = best_variant;
    o.tuned_sched = best_merge <= vec ? G1_SCHED_MERGE : G1_SCHED_VECTOR;
    Orientation& other = g->o[t ^ 1];
    if (other.present && other.rp == o.rp) {
        other.tuned_sched = o.tuned_sched;
        other.tuned_variant = o.tuned_variant;
    }
    if (merge_ms) *merge_ms = best_merge;
    if (vector_ms) *vector_ms = vec;
    if (merge_variant) *merge_variant = best_variant;
    return check_device_error(g, s);
}

}  // extern "C"
