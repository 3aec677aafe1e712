"""GraphOne's Graph accessors on a graph from graph::build (both views):
get_out_degree / get_in_degree per vertex and graph_mat() /
graph_transpose_mat() against the loader's CSR restated (tests/test_loader.py)
and the oracle's counting sort.

Collected last (file name) so that a failure here cannot hide the others."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_loader import CASES, parse

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph_driver(tmp_path_factory):
    lib = os.path.join(ROOT, "graphone_b200")
    exe = tmp_path_factory.mktemp("graph_api") / "graph_api_driver"
    r = subprocess.run([shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2",
                        "--extended-lambda", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "graph_api_driver.cu"),
                        "-o", str(exe), "-L", lib, "-lgraphone_b200", "-Xlinker", f"-rpath={lib}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


@pytest.mark.parametrize("case", ["tricky", "random"])
def test_graph_accessors(graph_driver, tmp_path, case):
    text = CASES[case]()
    path = tmp_path / f"{case}.adj"
    path.write_text(text)
    out = tmp_path / "out.bin"
    r = subprocess.run([graph_driver, str(path), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    raw = np.fromfile(out, np.uint32)
    n, m = int(raw[0]), int(raw[1])
    en, src, dst, w = parse(text, True)
    assert (n, m) == (en, len(src))
    od, idg = raw[2:2 + n], raw[2 + n:2 + 2 * n]
    rest = raw[2 + 2 * n:]
    mats = [rest[:n + 1 + 2 * m], rest[n + 1 + 2 * m:]]
    for t, got in enumerate(mats):
        erp, eci, ev = O.csr_build(n, src, dst, w, transpose=bool(t))
        assert np.array_equal(got[:n + 1], erp)
        assert np.array_equal(got[n + 1:n + 1 + m], eci)
        assert np.array_equal(got[n + 1 + m:], ev)
        assert np.array_equal(od if t == 0 else idg, np.diff(erp.astype(np.int64)).astype(np.uint32))
