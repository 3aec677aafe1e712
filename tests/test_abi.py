"""The C ABI library loads and exports every entry point the header declares.
CPU only: no kernel runs."""
import ctypes as C
import os
import re

import graphone_b200 as g1

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "graphone_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(g1_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = g1.lib()
    decl = header_functions()
    assert len(decl) >= 15
    missing = [f for f in decl if not hasattr(L, f)]
    assert not missing, missing
    assert sorted(g1.EXPORTS) == decl


def test_library_reports_sm100a():
    assert b"sm_100a" in g1.lib().g1_version()


def test_status_strings_and_argument_errors_without_gpu():
    L = g1.lib()
    assert L.g1_status_string(0) == b"ok"
    assert L.g1_status_string(1) == b"invalid argument"
    out = C.c_void_p()
    st = L.g1_graph_create(None, None, None, 0, 4, 4, 0, None, C.byref(out))
    assert st == 1 and out.value is None
    assert b"null" in L.g1_last_error()
    st = L.g1_graph_create(None, None, None, 0, 0, 0, 0, None, None)
    assert st == 1
    assert L.g1_sssp(None, 0, 0, None, None, None) == 1
    assert L.g1_pagerank(None, C.c_float(0.85), 30, 1, None, None) == 1


# Entry points for which null arguments are valid (a no-op, optional outputs,
# the default stream) or that take no pointer at all.
NULL_OK = {"g1_graph_destroy", "g1_mem_free", "g1_server_destroy", "g1_profile_begin",
           "g1_profile_end", "g1_release_cached_memory", "g1_stream_sync",
           "g1_graph_device_bytes", "g1_kernel_launches", "g1_count_user_launches",
           "g1_status_string", "g1_last_error", "g1_version", "g1_test_set_wait_polls"}


def test_every_entry_point_rejects_null_arguments_before_any_device_work():
    """Every other entry point, called with null pointers and sizes of 1,
    returns G1_ERR_INVALID from its argument checks (it reaches no CUDA
    call, which would answer G1_ERR_DEVICE on a machine without a GPU)."""
    L = g1.lib()
    checked = []
    for name in sorted(g1.EXPORTS):
        if name in NULL_OK:
            continue
        f = getattr(L, name)
        args = []
        for t in f.argtypes or []:
            if t in (C.c_float, C.c_double):
                args.append(0.5)
            elif t in (C.c_int, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int64):
                args.append(1)
            else:
                args.append(None)
        st = f(*args)
        assert st == 1, (name, st, L.g1_last_error())
        checked.append(name)
    assert len(checked) >= 20


def test_python_variant_table_matches_the_launcher():
    src = open(os.path.join(ROOT, "graphone_b200", "csrc", "spmv_launch.cuh")).read()
    n = int(re.search(r"kNumMergeVariants\s*=\s*(\d+)", src).group(1))
    d = int(re.search(r"kDefaultVariant\s*=\s*(\d+)", src).group(1))
    table = re.search(r"kMergeVariants\[\]\s*=\s*\{(.*?)\};", src, re.S).group(1)
    kinds = [int(k) for k in re.findall(r"\{\s*(\d+)\s*,", table)]
    names = {0: "warp", 1: "cta_tma", 2: "warp_tma", 3: "nnz", 5: "nnz2"}
    assert len(g1.MERGE_VARIANTS) == n == len(kinds)
    assert tuple(names[k] for k in kinds) == g1.MERGE_VARIANTS
    assert g1.DEFAULT_MERGE_VARIANT == d


def test_size_and_argument_limits_are_refused_before_any_device_work():
    """n + m at or above 2^32 - 1 (the u32 ids and offsets), an unknown
    hot-column mode, and probe arguments out of range: each is refused with
    G1_ERR_INVALID by the argument checks, before any CUDA call."""
    import numpy as np
    L = g1.lib()
    rp = np.zeros(2, np.uint32)
    ci = np.zeros(1, np.uint32)
    val = np.zeros(1, np.uint32)
    out = C.c_void_p()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    st = L.g1_graph_create(p(rp), p(ci), p(val), 0, 0xFFFFFFFF - 5, 5, 0, None, C.byref(out))
    assert st == 1 and out.value is None
    assert b"2^32" in L.g1_last_error()
    st = L.g1_graph_create(p(rp), p(ci), p(val), 7, 1, 1, 0, None, C.byref(out))
    assert st == 1 and b"value type" in L.g1_last_error()
    fake = C.c_void_p(16)  # never dereferenced: the mode check comes first
    assert L.g1_graph_set_hot_columns(fake, 3) == 1
    assert L.g1_graph_set_hot_columns(None, 0) == 1
    r, b = C.c_double(), C.c_uint32()
    for cl in (0, 3, 32):
        assert L.g1_measure_smem_gather_rate(cl, 1, C.byref(r), C.byref(b), None) == 1
    assert L.g1_measure_gather_rate(8, 8, 1, 1 << 24, C.byref(r), None) == 1
    assert L.g1_measure_gather_rate(4, 8, 1, 1000, C.byref(r), None) == 1
