"""GraphOne's own test programs for the hot path, built unchanged against
this repository's headers (oracle/_ref/tests_g1), run on the GPU on a sample
file, their printed results checked:
  spmv_test        y = A (min, +) x with x = INT_MAX but x[1] = 0 through
                   blas::MakeCsrSpMV<cuda, SpmvCudaCsrMergeBased>;
  mat_builder_test the CSR of the undirected sample and its mat::ToCsc;
  buffer_test      host and device Buffer round trips.

Collected last (file name) so that a failure here cannot hide the others."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_loader import parse

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G1 = os.path.join(ROOT, "oracle", "_ref", "tests_g1")
INT_MAX = np.iinfo(np.int32).max

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.isdir(G1), reason="oracle/_ref/tests_g1 not built")]

SAMPLE = "% sample\n0 1 5\n1 2 3\n2 0 7\n5 3 2\n3 5 2\n0 1 5\n4 1 9\n7\t6\n2 3 4\n6 1 1\n"


def run_program(tmp_path, name):
    d = tmp_path / "datasets" / "sample"
    d.mkdir(parents=True, exist_ok=True)
    (d / "sample.adj").write_text(SAMPLE)
    run = tmp_path / "run"
    run.mkdir(exist_ok=True)
    r = subprocess.run([os.path.join(G1, name)], cwd=run, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def buffer_field(text, label):
    m = re.search(re.escape(label) + r"Buffer\{ size_:(\d+), data_:\[([^\]]*)\] \}", text)
    assert m, (label, text[:2000])
    vals = [int(v) for v in m.group(2).split(",") if v != ""]
    assert len(vals) == int(m.group(1))
    return np.array(vals, np.int64)


def test_spmv_test(tmp_path):
    out = run_program(tmp_path, "spmv_test")
    n, src, dst, w = parse(SAMPLE, True)
    rp, ci, v = O.csr_build(n, src, dst, w, transpose=False)
    x = np.full(n, INT_MAX, np.int64)
    x[1] = 0
    y = np.full(n, INT_MAX, np.int64)
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            if x[ci[k]] != INT_MAX:
                y[r] = min(y[r], int(v[k]) + x[ci[k]])
    assert np.array_equal(buffer_field(out, "y: "), y)


def test_mat_builder_test(tmp_path):
    out = run_program(tmp_path, "mat_builder_test")
    n, src, dst, w = parse(SAMPLE, False)
    rp, ci, v = O.csr_build(n, src, dst, w, transpose=False)
    trp, tci, tv = O.csr_build(n, src, dst, w, transpose=True)
    csr, csc = out.split("CscMat{")
    assert np.array_equal(buffer_field(csr, "row_offsets:"), rp)
    assert np.array_equal(buffer_field(csr, "col_indices:"), ci)
    assert np.array_equal(buffer_field(csc, "col_offsets:"), trp)
    assert np.array_equal(buffer_field(csc, "row_indices:"), tci)
    assert np.array_equal(buffer_field(csc, "values:"), tv)


def test_buffer_test(tmp_path):
    out = run_program(tmp_path, "buffer_test")
    lines = out.splitlines()
    assert lines[:10] == [str(i) for i in range(10)]
    dev = [ln for ln in lines if re.fullmatch(r"\d+ - \d+", ln)]
    assert dev == [f"{i} - {9 - i}" for i in range(10)]
    assert out.count("Buffer{ size_:0, data_:[] }") == 4
