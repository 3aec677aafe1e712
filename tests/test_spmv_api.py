"""GraphOne's SpMV operator API (include/GraphOne/archi/blas/spmv/spmv.h:
blas::MakeCsrSpMV / SpmvDispatcher / SpMV_cpu_navie / DefaultSpmvFunctor)
with the SpmvCpuNaive schedule against the oracle and, when oracle/_ref is
built, GraphOne's own SpMV_cpu_navie.  The driver (tests/spmv_api_driver.cu)
is built with nvcc; the CUDA schedules are compiled into it here and run
only under `-m gpu`.  CPU only."""
import ctypes as C
import os
import shutil
import subprocess
import zlib

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INT_MAX = np.iinfo(np.int32).max

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                                reason="nvcc not available")


def nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    from graphone_b200 import build as B
    lib = os.path.join(ROOT, "graphone_b200")
    if not os.path.exists(os.path.join(lib, "libgraphone_b200.so")):
        B.build()
    exe = tmp_path_factory.mktemp("spmv_api") / "spmv_api_driver"
    r = subprocess.run([nvcc(), "-std=c++17", "-O2", "--extended-lambda", "--expt-relaxed-constexpr",
                        "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "spmv_api_driver.cu"), "-o", str(exe),
                        "-L", lib, "-lgraphone_b200", "-Xlinker", f"-rpath={lib}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


def make_csr(rng, n, deg, hub=False, empty_frac=0.3):
    lens = rng.poisson(deg, n).astype(np.int64)
    lens[rng.random(n) < empty_frac] = 0
    if hub and n > 1:
        lens[n // 2] = 40 * (deg + 1) + 700  # one row across many merge tiles
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(lens)
    m = int(rp[-1])
    ci = np.sort(rng.integers(0, n, m)).astype(np.uint32) if m else np.zeros(0, np.uint32)
    for r in range(n):  # sorted columns per row
        ci[rp[r]:rp[r + 1]] = np.sort(ci[rp[r]:rp[r + 1]])
    wi = rng.integers(1, 65, m).astype(np.int32)
    wf = rng.random(m).astype(np.float32)
    xi = rng.integers(0, 1000, n).astype(np.int32)
    xi[rng.random(n) < 0.4] = INT_MAX
    xf = rng.random(n).astype(np.float32)
    return rp, ci, wi, wf, xi, xf


def run(driver, tmp_path, kind, csr):
    rp, ci, wi, wf, xi, xf = csr
    n, m = len(rp) - 1, len(ci)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([n, m], np.uint32).tofile(f)
        for a in (rp, ci, wi, wf, xi, xf):
            a.tofile(f)
    r = subprocess.run([driver, kind, str(inp), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    raw = np.fromfile(out, np.uint32)
    assert raw.size == 3 * n
    return raw[:n].view(np.int32), raw[n:2 * n].view(np.float32), raw[2 * n:].view(np.int32)


def expected_int(csr):
    """Row folds restated: the INT_MAX-guarded min-plus of GraphOne's
    test/spmv_test.cu and DefaultSpmvFunctor's sum of min(a, x)
    (archi/blas/spmv/def.hpp:27-45)."""
    rp, ci, wi, _, xi, _ = csr
    n = len(rp) - 1
    y1 = np.full(n, INT_MAX, np.int64)
    y3 = np.zeros(n, np.int64)
    for r in range(n):
        s, e = int(rp[r]), int(rp[r + 1])
        if e > s:
            xs = xi[ci[s:e]].astype(np.int64)
            ws = wi[s:e].astype(np.int64)
            y1[r] = np.where(xs == INT_MAX, INT_MAX, ws + xs).min()
            y3[r] = np.minimum(ws, xs).sum()
    return y1.astype(np.int32), y3.astype(np.int32)


CASES = {
    "random": dict(n=3000, deg=6.0),
    "hub": dict(n=2000, deg=3.0, hub=True),
    "dense_rows": dict(n=500, deg=40.0, empty_frac=0.0),
    "all_empty": dict(n=300, deg=0.0),
    "single": dict(n=1, deg=0.0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_cpu_schedule_matches_oracle_and_graphone(driver, tmp_path, case):
    csr = make_csr(np.random.default_rng(zlib.crc32(case.encode())), **CASES[case])
    y1, y2, y3 = run(driver, tmp_path, "cpu", csr)
    e1, e3 = expected_int(csr)
    assert np.array_equal(y1, e1)
    assert np.array_equal(y3, e3)
    rp, ci, _, wf, _, xf = csr
    # the oracle's fp32 row loop folds in the same order: the same bits
    assert np.array_equal(y2.view(np.uint32), O.spmv_plustimes_f32(rp, ci, wf, xf).view(np.uint32))
    R = O.ref()
    if R is not None:
        yr = np.zeros(len(rp) - 1, np.float32)
        R.ref_spmv_plustimes_f32(len(rp) - 1, O._ptr(rp), O._ptr(ci), O._ptr(wf), O._ptr(xf), O._ptr(yr), 1)
        assert np.array_equal(y2.view(np.uint32), yr.view(np.uint32))
