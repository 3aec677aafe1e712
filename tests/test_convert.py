"""GraphOne's sparse-format conversions (include/GraphOne/mat/convert.h:
mat::ToCsc, mat::OffsetsToIndices) on host matrices against the oracle's
counting-sort transpose: column offsets, rows ascending within each column,
values carried along.  The driver (tests/convert_driver.cu) is built with
nvcc.  CPU only."""
import os
import shutil
import subprocess
import zlib

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                                reason="nvcc not available")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    lib = os.path.join(ROOT, "graphone_b200")
    exe = tmp_path_factory.mktemp("convert") / "convert_driver"
    r = subprocess.run([shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2",
                        "--extended-lambda", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "convert_driver.cu"),
                        "-o", str(exe), "-L", lib, "-lgraphone_b200", "-Xlinker", f"-rpath={lib}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


CASES = {"random": (2000, 8.0), "sparse": (5000, 0.5), "empty": (50, 0.0), "single": (1, 0.0), "dense": (60, 50.0)}


@pytest.mark.parametrize("case", sorted(CASES))
def test_to_csc_matches_oracle_transpose(driver, tmp_path, case):
    n, deg = CASES[case]
    rng = np.random.default_rng(zlib.crc32(case.encode()))
    lens = rng.poisson(deg, n)
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(lens)
    m = int(rp[-1])
    ci = rng.integers(0, n, m).astype(np.uint32)
    for r in range(n):
        ci[rp[r]:rp[r + 1]] = np.sort(ci[rp[r]:rp[r + 1]])
    v = rng.integers(0, 1 << 30, m).astype(np.uint32)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([n, m], np.uint32).tofile(f)
        for a in (rp, ci, v):
            a.tofile(f)
    r = subprocess.run([driver, str(inp), str(out)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr[-2000:]
    raw = np.fromfile(out, np.uint32)
    co, ri, vv, rows = raw[:n + 1], raw[n + 1:n + 1 + m], raw[n + 1 + m:n + 1 + 2 * m], raw[n + 1 + 2 * m:]
    src = np.repeat(np.arange(n, dtype=np.uint32), lens)
    assert np.array_equal(rows, src)
    trp, tci, tv = O.csr_build(n, src, ci, v, transpose=True)
    assert np.array_equal(co, trp) and np.array_equal(ri, tci) and np.array_equal(vv, tv)
