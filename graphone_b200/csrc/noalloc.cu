// g1_spmv_noalloc: the merge-path SpMV for callers that cannot allocate.
//
// Some callers of this library may not call cudaMalloc at all: a host
// process that hands out device memory only through its own arena or caching
// pool (a driver allocation outside it would break its accounting and
// fragment the pool), a plugin loaded into such a host, or a
// latency-critical loop where cudaMalloc's implicit device-wide
// synchronisation is unacceptable.  g1_spmv (the
// regular entry point) keeps its merge-path partition and per-tile carries in
// memory owned by a g1_graph, created with cudaMalloc.  This entry point
// instead uses one file-scope device array as its scratch: the caller passes
// its own device CSR, x and y, and nothing is allocated.
//
// The scratch array holds the partition of (n + m) merge items into tiles of
// kNoAllocItems items plus one carry and one tail value per tile, for at most
// kNoAllocMaxTiles tiles (4 MiB).  Every GPU that loads the library holds
// this array until the process exits.  All calls on a device share it, and it
// keeps the last call's contents: calls whose work overlaps on the GPU race on
// it (serialise them, e.g. on one stream).  Nothing in it needs to start at
// zero: each call writes every element it later reads (the partition kernel
// writes tile_row/tile_nnz, the tile kernel writes carry/tail of every tile)
// before reading it, so stale contents from an earlier call are never used.
//
// Every call looks up the array's device address with cudaGetSymbolAddress,
// with the calling device current, and passes that address to the kernels.
// The address is not cached: after cudaDeviceReset (or any other teardown of
// the primary context) the module is loaded again and the array may move.
// The library is compiled without relocatable device code and CUDA loads
// modules lazily by default, so the first call on a device (in a context)
// loads this file's module: the driver then allocates the 4 MiB array and
// the module's code on that device.  Make that first call at set-up time,
// before any stream capture, or set CUDA_MODULE_LOADING=EAGER to load the
// module when the library's CUDA context starts.
#include <cuda_runtime.h>

#include "g1/semiring.cuh"
#include "g1/spmv.cuh"
#include "internal.h"

namespace g1 {

__global__ void merge_partition_kernel(const uint32_t* row_ptr, uint32_t n_rows, uint32_t nnz,
                                       uint32_t items, uint32_t n_tiles, uint32_t* tile_row,
                                       uint32_t* tile_nnz);

namespace {

constexpr int kNoAllocWarps = 8;
constexpr int kNoAllocIpt = 7;
constexpr uint32_t kNoAllocItems = 32 * kNoAllocIpt;  // merge items per warp tile
constexpr uint32_t kNoAllocMaxTiles = 1u << 18;       // (n + m) <= 58,720,256
// tile_row, tile_nnz: max_tiles + 1 each; carry, tail: max_tiles + 1 4-byte values each
constexpr size_t kNoAllocWords = 4 * ((size_t)kNoAllocMaxTiles + 1);

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// Device address of the scratch array on the current device, looked up on
// every call.  In host code g_noalloc_scratch names a host-side stand-in,
// never a device address: only the looked-up pointer is passed to kernels.
g1_status scratch_for_current_device(uint32_t** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(scratch)");
    *out = static_cast<uint32_t*>(p);
    return G1_OK;
}

template <class SR>
g1_status run_noalloc(const uint32_t* row_ptr, const uint32_t* col, const void* val, uint32_t n,
                      uint32_t m, const void* x, void* y, uint32_t* scratch, cudaStream_t s) {
    using Epi = StoreEpilogue<typename SR::value_t>;
    const uint32_t n_tiles = (uint32_t)ceil_div((uint64_t)n + m, kNoAllocItems);
    const size_t stride = (size_t)kNoAllocMaxTiles + 1;
    MergeArgs<SR> a;
    a.plan.n_rows = n;
    a.plan.nnz = m;
    a.plan.items = kNoAllocItems;
    a.plan.n_tiles = n_tiles;
    a.plan.row_ptr = row_ptr;
    a.plan.tile_row = scratch;
    a.plan.tile_nnz = scratch + stride;
    a.col = col;
    a.val = static_cast<const typename SR::w_t*>(val);
    a.x = static_cast<const typename SR::x_t*>(x);
    a.carry = reinterpret_cast<typename SR::value_t*>(scratch + 2 * stride);
    a.tail = reinterpret_cast<typename SR::value_t*>(scratch + 3 * stride);
    a.err = nullptr;
    int sms = 0, dev = 0;
    G1_CUDA(cudaGetDevice(&dev));
    G1_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    merge_partition_kernel<<<(unsigned)ceil_div((uint64_t)n_tiles + 1, 256), 256, 0, s>>>(
        row_ptr, n, m, kNoAllocItems, n_tiles, scratch, scratch + stride);
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(ceil_div(n_tiles, kNoAllocWarps), (uint64_t)sms * 8));
    using L = WarpMergeLayout<SR, kNoAllocWarps, kNoAllocIpt, 0>;
    spmv_wmerge_kernel<SR, Epi, kNoAllocWarps, kNoAllocIpt, 3, 0, true>
        <<<grid, kNoAllocWarps * 32, L::BYTES, s>>>(a, Epi{static_cast<typename SR::value_t*>(y)});
    spmv_fixup_kernel<SR, Epi, 256><<<(unsigned)std::max<uint64_t>(1, ceil_div(n_tiles, 256)), 256, 0, s>>>(
        a, Epi{static_cast<typename SR::value_t*>(y)});
    count_launches(3);
    G1_CUDA(cudaGetLastError());
    return G1_OK;
}

}  // namespace
}  // namespace g1

using namespace g1;

extern "C" g1_status g1_spmv_noalloc(const uint32_t* row_ptr, const uint32_t* col, const void* val,
                                     uint32_t n, uint32_t m, g1_semiring sr, const void* x,
                                     void* y, void* stream) {
    if (!row_ptr || !x || !y || (m > 0 && (!col || !val)))
        return fail(G1_ERR_INVALID, "g1_spmv_noalloc: null pointer");
    if (n == 0) return G1_OK;
    const uint64_t tiles = ceil_div((uint64_t)n + m, kNoAllocItems);
    if (tiles > kNoAllocMaxTiles)
        return fail(G1_ERR_INVALID,
                    "g1_spmv_noalloc: n + m above the scratch limit of 58,720,256 merge items");
    uint32_t* scratch = nullptr;
    G1_TRY(scratch_for_current_device(&scratch));
    cudaStream_t s = as_stream(stream);
    switch (sr) {
        case G1_SR_MINPLUS_U32: return run_noalloc<MinPlusU32>(row_ptr, col, val, n, m, x, y, scratch, s);
        case G1_SR_MINPLUS_F32: return run_noalloc<MinPlusF32>(row_ptr, col, val, n, m, x, y, scratch, s);
        case G1_SR_PLUSTIMES_F32: return run_noalloc<PlusTimesF32>(row_ptr, col, val, n, m, x, y, scratch, s);
        case G1_SR_BFS_U32: return run_noalloc<BfsU32>(row_ptr, col, val, n, m, x, y, scratch, s);
    }
    return fail(G1_ERR_INVALID, "g1_spmv_noalloc: unknown semiring");
}
