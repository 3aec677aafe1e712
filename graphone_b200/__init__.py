"""Python view of libgraphone_b200.so (the C ABI in include/graphone_b200.h).

The library is the product: this module only loads it with ctypes and turns
g1_status codes into exceptions.  There is no CPU fallback: importing works
without a GPU (the library loads; no kernel runs), and every compute call
fails with G1Error when no CUDA device is present.

    import graphone_b200 as g1
    g = g1.Graph.from_csr(row_ptr, col, val, symmetric=True)
    dist = g.sssp(0)                  # numpy uint32, UINT32_MAX = unreachable
    rank = g.pagerank(0.85, 30)       # numpy float32
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgraphone_b200.so")
U32_MAX = 0xFFFFFFFF

G1_U32, G1_F32 = 0, 1
SR_MINPLUS_U32, SR_MINPLUS_F32, SR_PLUSTIMES_F32, SR_BFS_U32 = 0, 1, 2, 3
SCHED_AUTO, SCHED_MERGE, SCHED_VECTOR = 0, 1, 2
ENGINE_BLAS, ENGINE_ADVANCE, ENGINE_AUTO, ENGINE_NEARFAR = 0, 1, 2, 3
PR_REFERENCE, PR_DANGLING = 0, 1
HOT_COLUMNS_AUTO, HOT_COLUMNS_OFF, HOT_COLUMNS_ON = 0, 1, 2
# Kernel family of each merge-schedule variant, indexed like kMergeVariants
# in csrc/spmv_launch.cuh: "warp" = spmv_wmerge_kernel (warp tiles, plain
# loads), "cta_tma" = spmv_merge_kernel (CTA tiles staged by bulk copies),
# "warp_tma" = spmv_wtma_kernel (warp tiles staged by bulk copies), "nnz" =
# spmv_nnz_kernel (nnz-split warp tiles, 16-byte loads, row-start bitmap),
# "nnz2" = spmv_nnz2_kernel (nnz-split tiles of 32 x 8, 16 or 24 nonzeros).
MERGE_VARIANTS = ("warp", "warp", "warp", "cta_tma", "cta_tma", "warp",
                  "warp_tma", "warp_tma", "warp_tma", "warp_tma", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz",
                  "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz", "nnz",
                  "nnz2", "nnz2", "nnz2", "nnz2", "nnz2", "nnz2", "nnz2", "nnz2")
DEFAULT_MERGE_VARIANT = 17
GRAPH_SYMMETRIC, GRAPH_INPUT_TRANSPOSE, GRAPH_BUILD_OTHER, GRAPH_NO_VALIDATE = 1, 2, 4, 8
GRAPH_RELABEL = 16

STATUS = {0: "G1_OK", 1: "G1_ERR_INVALID", 2: "G1_ERR_OOM", 3: "G1_ERR_DEVICE",
          4: "G1_ERR_TIMEOUT", 5: "G1_ERR_UNSUPPORTED", 6: "G1_ERR_OVERFLOW"}


class G1Error(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None
P = C.c_void_p


def _declare(L):
    s = C.c_int
    L.g1_status_string.restype = C.c_char_p
    L.g1_status_string.argtypes = [s]
    L.g1_last_error.restype = C.c_char_p
    L.g1_version.restype = C.c_char_p
    L.g1_mem_alloc.argtypes = [C.POINTER(P), C.c_size_t]
    L.g1_mem_free.argtypes = [P]
    L.g1_mem_copy.argtypes = [P, P, C.c_size_t, C.c_int, P]
    L.g1_release_cached_memory.argtypes = [C.POINTER(C.c_size_t)]
    L.g1_mem_fill_u32.argtypes = [P, C.c_uint32, C.c_size_t, P]
    L.g1_stream_sync.argtypes = [P]
    L.g1_kernel_launches.restype = C.c_uint64
    L.g1_count_user_launches.argtypes = [C.c_uint64]
    L.g1_test_set_wait_polls.argtypes = [C.c_int64]
    L.g1_set_traversal_thresholds.argtypes = [P, C.c_uint32, C.c_uint32]
    L.g1_graph_set_hot_columns.argtypes = [P, C.c_int]
    L.g1_measure_smem_gather_rate.argtypes = [C.c_uint32, C.c_int, C.POINTER(C.c_double),
                                              C.POINTER(C.c_uint32), P]
    L.g1_measure_gather_rate.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                         C.POINTER(C.c_double), P]
    L.g1_profile_begin.argtypes = []
    L.g1_profile_end.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    L.g1_graph_create.argtypes = [P, P, P, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, P,
                                  C.POINTER(P)]
    L.g1_graph_destroy.argtypes = [P]
    L.g1_graph_info.argtypes = [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.g1_graph_arrays.argtypes = [P, C.c_int, C.POINTER(P), C.POINTER(P), C.POINTER(P)]
    L.g1_graph_device_bytes.restype = C.c_size_t
    L.g1_graph_device_bytes.argtypes = [P]
    L.g1_spmv_plan.argtypes = [P, C.c_int, C.c_uint32, C.POINTER(C.c_uint32),
                               C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P)]
    L.g1_spmv.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P, P]
    L.g1_spmv_nnz_plan.argtypes = [P, C.c_int, P]
    L.g1_spmv_noalloc.argtypes = [P, P, P, C.c_uint32, C.c_uint32, C.c_int, P, P, P]
    L.g1_graph_set_schedule.argtypes = [P, C.c_int, C.c_int, C.c_int]
    L.g1_autotune.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int), P]
    L.g1_autotune_traversal.argtypes = [P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), P]
    L.g1_pagerank.argtypes = [P, C.c_float, C.c_int, C.c_int, P, P]
    L.g1_sssp.argtypes = [P, C.c_uint32, C.c_int, P, C.POINTER(C.c_uint32), P]
    L.g1_bfs.argtypes = [P, C.c_uint32, C.c_int, P, C.POINTER(C.c_uint32), P]
    L.g1_advance_run.argtypes = [P, C.c_int, P, C.c_uint32, P, P, C.c_uint32, P, C.POINTER(C.c_uint32), P]
    L.g1_bfs_batch.argtypes = [P, P, C.c_uint32, P, C.POINTER(C.c_uint32), P]
    L.g1_sssp_batch.argtypes = [P, P, C.c_uint32, P, C.POINTER(C.c_uint32), P]
    L.g1_ppr.argtypes = [P, C.c_uint32, C.c_float, C.c_uint32, P, P]
    L.g1_ppr_batch.argtypes = [P, P, C.c_uint32, C.c_float, C.c_uint32, P, P]
    L.g1_server_create.argtypes = [C.c_int, C.POINTER(ServerConfig), C.POINTER(P)]
    L.g1_server_add_graph.argtypes = [P, P, C.POINTER(C.c_uint32)]
    L.g1_server_submit.argtypes = [P, C.c_uint32, C.c_int, C.c_uint32, P, C.POINTER(C.c_uint64)]
    L.g1_server_poll.argtypes = [P, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.g1_server_wait.argtypes = [P, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]
    L.g1_server_stats.argtypes = [P, C.c_int, C.POINTER(ServerStats)]
    L.g1_server_destroy.argtypes = [P]
    return L


def lib():
    """The loaded library; raises if it was not built (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m graphone_b200.build`")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


# Every symbol include/graphone_b200.h declares (checked by the CPU tests).
EXPORTS = (
    "g1_status_string", "g1_last_error", "g1_version", "g1_mem_alloc", "g1_mem_free",
    "g1_mem_copy", "g1_release_cached_memory", "g1_mem_fill_u32", "g1_stream_sync", "g1_kernel_launches",
    "g1_count_user_launches", "g1_test_set_wait_polls", "g1_measure_gather_rate",
    "g1_measure_smem_gather_rate",
    "g1_profile_begin", "g1_profile_end", "g1_graph_create",
    "g1_graph_destroy", "g1_graph_info", "g1_graph_arrays", "g1_graph_device_bytes",
    "g1_spmv_plan", "g1_spmv_nnz_plan", "g1_spmv", "g1_spmv_noalloc", "g1_graph_set_schedule", "g1_autotune", "g1_autotune_traversal", "g1_set_traversal_thresholds", "g1_graph_set_hot_columns", "g1_pagerank", "g1_sssp", "g1_bfs", "g1_advance_run",
    "g1_bfs_batch", "g1_sssp_batch", "g1_ppr", "g1_ppr_batch",
    "g1_server_create", "g1_server_add_graph", "g1_server_submit", "g1_server_poll",
    "g1_server_wait", "g1_server_stats", "g1_server_destroy",
)


def check(status: int) -> None:
    if status != 0:
        msg = lib().g1_last_error().decode(errors="replace")
        raise G1Error(status, msg)


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def kernel_launches() -> int:
    return int(lib().g1_kernel_launches())


def release_cached_memory() -> int:
    """Returns the device blocks the library keeps for reuse (from closed
    graphs, plans and engines) on the current device to the driver; the
    number of bytes released."""
    b = C.c_size_t()
    check(lib().g1_release_cached_memory(C.byref(b)))
    return b.value


def test_set_wait_polls(polls: int) -> None:
    """Lowers the poll limit of every bounded device wait (negative: the
    defaults), so that tests can make the waits run out."""
    check(lib().g1_test_set_wait_polls(polls))


def measure_smem_gather_rate(cluster_size: int = 1, remote: bool = False, stream=None):
    """(random 4-byte shared-memory loads per second, blocks that ran): from a
    block's own shared memory, or from random blocks of its thread-block
    cluster (remote); see g1_measure_smem_gather_rate."""
    r, b = C.c_double(), C.c_uint32()
    check(lib().g1_measure_smem_gather_rate(cluster_size, 1 if remote else 0, C.byref(r), C.byref(b),
                                            _stream(stream)))
    return r.value, b.value


def measure_gather_rate(item_bytes: int = 4, in_flight: int = 8, blocks_per_sm: int = 1,
                        footprint: int = 1 << 24, stream=None) -> float:
    """Random loads per second served to the SMs of the current device
    (g1_measure_gather_rate); the default (4-byte loads from a 16 MiB,
    L2-resident buffer) is the ceiling of the SpMV's cold x gathers."""
    r = C.c_double()
    check(lib().g1_measure_gather_rate(item_bytes, in_flight, blocks_per_sm, footprint, C.byref(r),
                                       _stream(stream)))
    return r.value


def profile_begin() -> None:
    check(lib().g1_profile_begin())


def profile_end():
    """(summed ms, launch count) of the SpMV main kernels since profile_begin()."""
    ms, n = C.c_double(), C.c_uint64()
    check(lib().g1_profile_end(C.byref(ms), C.byref(n)))
    return ms.value, n.value


class Graph:
    """A device-resident graph (owns a g1_graph handle)."""

    def __init__(self, handle: int, n: int, m: int):
        self._h = C.c_void_p(handle)
        self.n = n
        self.m = m

    @classmethod
    def from_csr(cls, row_ptr, col, val, *, symmetric=False, input_transpose=False,
                 build_other=True, validate=True, relabel=False, stream=None) -> "Graph":
        """CSR arrays: numpy (host) or torch tensors (host or device)."""
        if isinstance(row_ptr, np.ndarray):
            row_ptr = np.ascontiguousarray(row_ptr, np.uint32)
            col = np.ascontiguousarray(col, np.uint32)
            if val.dtype.kind == "f":
                val = np.ascontiguousarray(val, np.float32)
            else:
                val = np.ascontiguousarray(val, np.uint32)
            vtype = G1_F32 if val.dtype == np.float32 else G1_U32
        else:
            vtype = G1_F32 if val.dtype.is_floating_point else G1_U32
        n = len(row_ptr) - 1
        m = len(col)
        flags = ((GRAPH_SYMMETRIC if symmetric else 0)
                 | (GRAPH_INPUT_TRANSPOSE if input_transpose else 0)
                 | (GRAPH_BUILD_OTHER if build_other and not symmetric else 0)
                 | (0 if validate else GRAPH_NO_VALIDATE)
                 | (GRAPH_RELABEL if relabel else 0))
        out = C.c_void_p()
        check(lib().g1_graph_create(_ptr(row_ptr), _ptr(col) if m else None,
                                    _ptr(val) if m else None, vtype, n, m, flags,
                                    _stream(stream), C.byref(out)))
        return cls(out.value, n, m)

    @classmethod
    def from_gen(cls, g, *, relabel=False, stream=None) -> "Graph":
        """From a graphone_b200.gen.CsrGraph (out-edge CSR; transpose built on the GPU)."""
        rp, ci, v = g.np("n")
        return cls.from_csr(rp, ci, v, symmetric=g.symmetric, relabel=relabel, stream=stream)

    def close(self):
        if self._h:
            lib().g1_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def device_bytes(self) -> int:
        return lib().g1_graph_device_bytes(self._h)

    def info(self):
        n, m, hn, ht = C.c_uint32(), C.c_uint32(), C.c_int(), C.c_int()
        check(lib().g1_graph_info(self._h, C.byref(n), C.byref(m), C.byref(hn), C.byref(ht)))
        return n.value, m.value, bool(hn.value), bool(ht.value)

    def plan(self, transpose: int = 1, items_per_tile: int = 0):
        tiles = C.c_uint32()
        tr, tn, ca, ta = P(), P(), P(), P()
        check(lib().g1_spmv_plan(self._h, transpose, items_per_tile, C.byref(tiles), C.byref(tr),
                                 C.byref(tn), C.byref(ca), C.byref(ta)))
        return tiles.value, tr.value, tn.value

    def spmv(self, x, y, semiring: int, transpose: int = 1, schedule: int = SCHED_AUTO,
             stream=None):
        """y = A (semiring) x on device buffers (torch tensors)."""
        check(lib().g1_spmv(self._h, transpose, semiring, schedule, _ptr(x), _ptr(y),
                            _stream(stream)))

    def set_schedule(self, schedule: int, variant: int = 0, transpose: int = 1):
        check(lib().g1_graph_set_schedule(self._h, transpose, schedule, variant))

    def autotune(self, stream=None):
        """(best merge ms, vector ms, winning merge variant); the faster
        schedule becomes the graph's G1_SCHED_AUTO choice."""
        a, b, v = C.c_float(), C.c_float(), C.c_int()
        check(lib().g1_autotune(self._h, C.byref(a), C.byref(b), C.byref(v), _stream(stream)))
        return a.value, b.value, v.value

    def set_traversal_thresholds(self, push_div=0, slot_div=0):
        """Sets the push/pull divisors by hand (0 keeps one): see
        g1_set_traversal_thresholds."""
        check(lib().g1_set_traversal_thresholds(self._h, push_div, slot_div))

    def set_hot_columns(self, mode: int = HOT_COLUMNS_AUTO):
        """PageRank's column layout on this graph: see g1_graph_set_hot_columns."""
        check(lib().g1_graph_set_hot_columns(self._h, mode))

    def autotune_traversal(self, n_sources=16, stream=None):
        """(push_div, slot_div): the push/pull thresholds g1_autotune_traversal
        picked for this graph by timing SSSP from n_sources sources."""
        a, b = C.c_uint32(), C.c_uint32()
        check(lib().g1_autotune_traversal(self._h, n_sources, C.byref(a), C.byref(b), _stream(stream)))
        return a.value, b.value

    def pagerank(self, alpha=0.85, iters=30, mode=PR_DANGLING, out=None, stream=None):
        if out is None:
            out = np.empty(self.n, np.float32)
        check(lib().g1_pagerank(self._h, alpha, iters, mode, _ptr(out), _stream(stream)))
        return out

    def sssp(self, src, engine=ENGINE_AUTO, out=None, stream=None, return_iters=False):
        if out is None:
            out = np.empty(self.n, np.uint32)
        it = C.c_uint32()
        check(lib().g1_sssp(self._h, src, engine, _ptr(out), C.byref(it), _stream(stream)))
        return (out, it.value) if return_iters else out

    def advance_run(self, frontier, n_frontier, dist, visited, it, out_frontier, unit=False, stream=None):
        """One push relax step (g1_advance_run) over device tensors: returns
        the length of the new frontier written to out_frontier."""
        n_out = C.c_uint32()
        check(lib().g1_advance_run(self._h, int(bool(unit)), _ptr(frontier), n_frontier, _ptr(dist),
                                   _ptr(visited), it, _ptr(out_frontier), C.byref(n_out), _stream(stream)))
        return n_out.value

    def _batch(self, fn, srcs, out, stream, return_iters):
        if isinstance(srcs, np.ndarray) or isinstance(srcs, (list, tuple)):
            srcs = np.ascontiguousarray(np.asarray(srcs, dtype=np.uint32))
        k = len(srcs)
        if out is None:
            out = np.empty((k, self.n), np.uint32)
        it = C.c_uint32()
        check(fn(self._h, _ptr(srcs), k, _ptr(out), C.byref(it), _stream(stream)))
        return (out, it.value) if return_iters else out

    def bfs_batch(self, srcs, out=None, stream=None, return_iters=False):
        """Levels of k sources, shape (k, n), one multi-source pass."""
        return self._batch(lib().g1_bfs_batch, srcs, out, stream, return_iters)

    def sssp_batch(self, srcs, out=None, stream=None, return_iters=False):
        """Distances of k sources, shape (k, n), one multi-source pass."""
        return self._batch(lib().g1_sssp_batch, srcs, out, stream, return_iters)

    def ppr(self, src, alpha=0.85, iters=20, out=None, stream=None):
        """Personalized PageRank of one source (numpy float32 when out is None)."""
        if out is None:
            out = np.empty(self.n, np.float32)
        check(lib().g1_ppr(self._h, src, alpha, iters, _ptr(out), _stream(stream)))
        return out

    def ppr_batch(self, srcs, alpha=0.85, iters=20, out=None, stream=None):
        """Personalized PageRanks of k sources, shape (k, n) float32."""
        srcs = np.ascontiguousarray(np.asarray(srcs, dtype=np.uint32))
        k = len(srcs)
        if out is None:
            out = np.empty((k, self.n), np.float32)
        check(lib().g1_ppr_batch(self._h, _ptr(srcs), k, alpha, iters, _ptr(out), _stream(stream)))
        return out

    def bfs(self, src, engine=ENGINE_AUTO, out=None, stream=None, return_iters=False):
        if out is None:
            out = np.empty(self.n, np.uint32)
        it = C.c_uint32()
        check(lib().g1_bfs(self._h, src, engine, _ptr(out), C.byref(it), _stream(stream)))
        return (out, it.value) if return_iters else out


QUERY_BFS, QUERY_SSSP, QUERY_PPR = 0, 1, 2


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("reserve_bytes", C.c_uint64),
                ("memory_limit", C.c_uint64), ("ppr_alpha", C.c_float),
                ("ppr_iters", C.c_uint32), ("idle_release_ms", C.c_uint32),
                ("solo_queue_ms", C.c_int32), ("solo_lanes", C.c_uint32),
                ("lane_stretch", C.c_float)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("queries_per_s", C.c_double), ("steps", C.c_uint64),
                ("max_occupancy", C.c_uint32), ("engines", C.c_uint32),
                ("device_bytes", C.c_uint64)]


class Server:
    """The serving loop (g1_server_*): continuous batching over resident graphs.

        srv = g1.Server(max_batch=256)
        gid = srv.add_graph(G)                      # a Graph with the in-edge CSR
        t = srv.submit(gid, g1.QUERY_SSSP, src, out)  # out: device tensor / host array
        srv.wait(t)                                 # latency in ms
    """

    def __init__(self, device=0, max_batch=0, reserve_bytes=0, memory_limit=0,
                 ppr_alpha=0.0, ppr_iters=0, idle_release_ms=0, solo_queue_ms=0, solo_lanes=0,
                 lane_stretch=0.0):
        cfg = ServerConfig(max_batch, reserve_bytes, memory_limit, ppr_alpha, ppr_iters,
                           idle_release_ms, solo_queue_ms, solo_lanes, lane_stretch)
        h = C.c_void_p()
        check(lib().g1_server_create(device, C.byref(cfg), C.byref(h)))
        self._h = h.value
        self._graphs = []  # keep the Graph objects alive while registered
        self._outs = {}    # each query's output buffer, alive until it is done

    def add_graph(self, graph) -> int:
        gid = C.c_uint32()
        check(lib().g1_server_add_graph(self._h, graph.handle, C.byref(gid)))
        self._graphs.append(graph)
        return gid.value

    def submit(self, graph_id, kind, src, out) -> int:
        """Queues one query; `out` is kept alive until wait or poll reports
        the query done (the library writes into it until then)."""
        t = C.c_uint64()
        check(lib().g1_server_submit(self._h, graph_id, kind, src, _ptr(out), C.byref(t)))
        self._outs[t.value] = out
        return t.value

    def poll(self, ticket):
        """None while running, else the latency in ms (raises if the query failed)."""
        done, lat = C.c_int(), C.c_double()
        st = lib().g1_server_poll(self._h, ticket, C.byref(done), C.byref(lat))
        if done.value or st != 0:
            self._outs.pop(ticket, None)
        check(st)
        return lat.value if done.value else None

    def wait(self, ticket, timeout_ms=0) -> float:
        lat = C.c_double()
        st = lib().g1_server_wait(self._h, ticket, timeout_ms, C.byref(lat))
        if st != 4:  # anything but a timeout: the query is done and forgotten
            self._outs.pop(ticket, None)
        check(st)
        return lat.value

    def stats(self, reset=False) -> dict:
        st = ServerStats()
        check(lib().g1_server_stats(self._h, 1 if reset else 0, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            check(lib().g1_server_destroy(self._h))
            self._h = None
            self._outs = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
