"""ctypes view of the oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline, parity and
reference legs may import this module, as checkers and baselines.  ``lib()``
is the plain-C restatement (oracle/oracle.c); ``ref()`` is GraphOne's own
host code compiled from the reference sources (oracle/ref_driver.cu ->
oracle/_ref/libgraphone_ref.so), or None when that library was not built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
U32_MAX = 0xFFFFFFFF

_lib = None
_ref = None
_ref_tried = False

P = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def build(ref: bool = False) -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-j4", "-C", HERE, "ref", "dropin", "reftests"], check=True)


def app(name: str):
    """Path of a GraphOne app built unchanged against this repository's
    headers (oracle/_ref/apps_g1), or None when it was not built."""
    p = os.path.join(HERE, "_ref", "apps_g1", name)
    return p if os.path.exists(p) else None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_mix64.restype = C.c_uint64
        L.orc_mix64.argtypes = [C.c_uint64]
        L.orc_rng.restype = C.c_uint64
        L.orc_rng.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_rmat_samples.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                       C.c_uint64, C.c_uint64, P, P]
        L.orc_edge_weight.restype = C.c_uint32
        L.orc_edge_weight.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32]
        L.orc_csr_build.argtypes = [C.c_uint32, C.c_uint64, P, P, P, C.c_int, P, P, P]
        for f in ("orc_spmv_minplus_u32", "orc_spmv_plustimes_f32", "orc_spmv_plustimes_f64"):
            getattr(L, f).argtypes = [C.c_uint32, P, P, P, P, P]
        for f in ("orc_sssp_blas_u32", "orc_sssp_blas_f32", "orc_sssp_advance_u32"):
            getattr(L, f).restype = C.c_int
            getattr(L, f).argtypes = [C.c_uint32, P, P, P, C.c_uint32, P]
        L.orc_bfs.restype = C.c_int
        L.orc_bfs.argtypes = [C.c_uint32, P, P, C.c_uint32, P]
        L.orc_dijkstra_u32.argtypes = [C.c_uint32, P, P, P, C.c_uint32, P]
        L.orc_pagerank_f64.argtypes = [C.c_uint32, P, P, P, C.c_double, C.c_int, C.c_int, P]
        L.orc_ppr_f64.argtypes = [C.c_uint32, P, P, P, C.c_double, C.c_int, C.c_uint32, P]
        _lib = L
    return _lib


def ref():
    """GraphOne's own host code, or None if oracle/_ref was not built."""
    global _ref, _ref_tried
    if not _ref_tried:
        _ref_tried = True
        path = os.path.join(HERE, "_ref", "libgraphone_ref.so")
        if os.path.exists(path):
            R = C.CDLL(path)
            R.ref_load_adj.restype = C.c_int
            R.ref_load_adj.argtypes = [C.c_char_p, C.c_int, P, P]
            R.ref_load_adj_opts.restype = C.c_int
            R.ref_load_adj_opts.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, P, P]
            R.ref_to_csr.restype = C.c_int
            R.ref_to_csr.argtypes = [C.c_int, P, P, P]
            R.ref_spmv_minplus_u32.argtypes = [C.c_uint32, P, P, P, P, P, C.c_int]
            R.ref_spmv_plustimes_f32.argtypes = [C.c_uint32, P, P, P, P, P, C.c_int]
            R.ref_sssp_blas_u32.restype = C.c_int
            R.ref_sssp_blas_u32.argtypes = [C.c_uint32, P, P, P, C.c_uint32, P, C.c_int, C.c_int]
            R.ref_pagerank_f32.argtypes = [C.c_uint32, P, P, P, P, C.c_float, C.c_int,
                                           C.c_int, P, C.c_int]
            _ref = R
    return _ref


# ---------------------------------------------------------------- wrappers

def u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def rmat_samples(scale, n_samples, thresholds, seed):
    s = np.empty(n_samples, np.uint32)
    d = np.empty(n_samples, np.uint32)
    tA, tAB, tABC = thresholds
    lib().orc_rmat_samples(scale, n_samples, tA, tAB, tABC, seed, _ptr(s), _ptr(d))
    return s, d


def csr_build(n, src, dst, w, transpose):
    src, dst = u32(src), u32(dst)
    w = u32(w) if w is not None else np.zeros(len(src), np.uint32)
    rp = np.empty(n + 1, np.uint32)
    ci = np.empty(len(src), np.uint32)
    v = np.empty(len(src), np.uint32)
    lib().orc_csr_build(n, len(src), _ptr(src), _ptr(dst), _ptr(w), int(transpose),
                        _ptr(rp), _ptr(ci), _ptr(v))
    return rp, ci, v


def spmv_minplus_u32(rp, ci, v, x):
    rp, ci, v, x = u32(rp), u32(ci), u32(v), u32(x)
    y = np.empty(len(rp) - 1, np.uint32)
    lib().orc_spmv_minplus_u32(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), _ptr(y))
    return y


def spmv_plustimes_f32(rp, ci, v, x):
    rp, ci = u32(rp), u32(ci)
    v = np.ascontiguousarray(v, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty(len(rp) - 1, np.float32)
    lib().orc_spmv_plustimes_f32(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), _ptr(y))
    return y


def spmv_plustimes_f64(rp, ci, v, x):
    rp, ci = u32(rp), u32(ci)
    v = np.ascontiguousarray(v, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(len(rp) - 1, np.float64)
    lib().orc_spmv_plustimes_f64(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), _ptr(y))
    return y


def sssp_blas_u32(trp, tci, tv, src):
    trp, tci, tv = u32(trp), u32(tci), u32(tv)
    n = len(trp) - 1
    d = np.empty(n, np.uint32)
    it = lib().orc_sssp_blas_u32(n, _ptr(trp), _ptr(tci), _ptr(tv), src, _ptr(d))
    return d, it


def sssp_blas_f32(trp, tci, tv, src):
    trp, tci = u32(trp), u32(tci)
    tv = np.ascontiguousarray(tv, np.float32)
    n = len(trp) - 1
    d = np.empty(n, np.float32)
    it = lib().orc_sssp_blas_f32(n, _ptr(trp), _ptr(tci), _ptr(tv), src, _ptr(d))
    return d, it


def sssp_advance_u32(rp, ci, v, src):
    rp, ci, v = u32(rp), u32(ci), u32(v)
    n = len(rp) - 1
    d = np.empty(n, np.uint32)
    it = lib().orc_sssp_advance_u32(n, _ptr(rp), _ptr(ci), _ptr(v), src, _ptr(d))
    return d, it


def dijkstra_u32(rp, ci, v, src):
    rp, ci, v = u32(rp), u32(ci), u32(v)
    n = len(rp) - 1
    d = np.empty(n, np.uint32)
    lib().orc_dijkstra_u32(n, _ptr(rp), _ptr(ci), _ptr(v), src, _ptr(d))
    return d


def bfs(rp, ci, src):
    rp, ci = u32(rp), u32(ci)
    n = len(rp) - 1
    lv = np.empty(n, np.uint32)
    lib().orc_bfs(n, _ptr(rp), _ptr(ci), src, _ptr(lv))
    return lv


def pagerank_f64(trp, tci, tv, alpha=0.85, iters=30, mode=1):
    trp, tci = u32(trp), u32(tci)
    tv = np.ascontiguousarray(tv, np.float32)
    n = len(trp) - 1
    r = np.empty(n, np.float64)
    lib().orc_pagerank_f64(n, _ptr(trp), _ptr(tci), _ptr(tv), alpha, iters, mode, _ptr(r))
    return r


def ppr_f64(trp, tci, tv, src, alpha=0.85, iters=20):
    trp, tci = u32(trp), u32(tci)
    tv = np.ascontiguousarray(tv, np.float32)
    n = len(trp) - 1
    r = np.empty(n, np.float64)
    lib().orc_ppr_f64(n, _ptr(trp), _ptr(tci), _ptr(tv), alpha, iters, src, _ptr(r))
    return r


def rel_l1(a, ref_):
    a = np.asarray(a, np.float64)
    ref_ = np.asarray(ref_, np.float64)
    return float(np.abs(a - ref_).sum() / max(np.abs(ref_).sum(), 1e-300))
