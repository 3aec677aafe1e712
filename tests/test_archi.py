"""GraphOne's archi:: primitives (include/GraphOne/archi/archi.cuh: copy_if,
inclusive_scan, lower_bound, scatter, scatter_if, sort_by_key, fill,
transform, transform_reduce, for_each, the memalloc / memcpy / memset /
memfree functors and, on the GPU, LaunchKernel / LaunchSync) with arch_t::cpu against numpy.  The driver
(tests/archi_driver.cu) is built with nvcc; its cuda mode runs under
`-m gpu` (tests/test_zzz_spmv_api_gpu.py).  CPU only."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                                reason="nvcc not available")


@pytest.fixture(scope="module")
def archi_driver(tmp_path_factory):
    lib = os.path.join(ROOT, "graphone_b200")
    exe = tmp_path_factory.mktemp("archi") / "archi_driver"
    r = subprocess.run([shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2",
                        "--extended-lambda", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "archi_driver.cu"),
                        "-o", str(exe), "-L", lib, "-lgraphone_b200", "-Xlinker", f"-rpath={lib}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    keys = rng.permutation(4 * n)[:n].astype(np.uint32)
    vals = rng.integers(0, 1 << 20, n).astype(np.uint32)
    flags = (rng.random(n) < 0.4).astype(np.uint32)
    perm = rng.permutation(n).astype(np.uint32)
    srt = np.sort(rng.integers(0, 3 * n, n)).astype(np.uint32)
    queries = rng.integers(0, 3 * n + 5, n).astype(np.uint32)
    return [keys, vals, flags, perm, srt, queries]


def run_archi(exe, tmp_path, kind, arrs):
    n = len(arrs[0])
    inp, out = tmp_path / f"a_{kind}.bin", tmp_path / f"o_{kind}.bin"
    with open(inp, "wb") as f:
        np.array([n], np.uint32).tofile(f)
        for a in arrs:
            a.tofile(f)
    r = subprocess.run([exe, kind, str(inp), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    raw = open(out, "rb").read()
    count = int(np.frombuffer(raw[:4], np.uint32)[0])
    body = np.frombuffer(raw[4:4 + 4 * 10 * n], np.uint32).reshape(10, n)
    sq, each = np.frombuffer(raw[4 + 4 * 10 * n:], np.uint64)
    return count, body, int(sq), int(each)


def check_archi(arrs, count, body, sq, each):
    keys, vals, flags, perm, srt, queries = arrs
    n = len(keys)
    sel = vals[flags != 0]
    assert count == len(sel) and np.array_equal(body[0][:count], sel)
    assert np.array_equal(body[1], np.maximum.accumulate(vals))
    assert np.array_equal(body[2], np.searchsorted(srt, queries, side="left").astype(np.uint32))
    sc = np.zeros(n, np.uint32)
    sc[perm] = vals
    assert np.array_equal(body[3], sc)
    sci = np.zeros(n, np.uint32)
    sci[perm[flags != 0]] = vals[flags != 0]
    assert np.array_equal(body[4], sci)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(body[5], keys[order]) and np.array_equal(body[6], vals[order])
    assert np.all(body[7] == 7)
    assert np.array_equal(body[8], (3 * vals.astype(np.uint64) + 1).astype(np.uint32))
    assert np.array_equal(body[9], (2 * vals.astype(np.uint64) + 5).astype(np.uint32))
    assert sq == int((vals.astype(np.uint64) ** 2).sum())
    assert each == int(vals.astype(np.uint64).sum())


@pytest.mark.parametrize("n", [1, 257, 5000])
def test_archi_primitives_on_the_host(archi_driver, tmp_path, n):
    arrs = inputs(n, n)
    check_archi(arrs, *run_archi(archi_driver, tmp_path, "cpu", arrs))
