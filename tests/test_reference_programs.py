"""GraphOne's own test programs for the hot path (test/loader_test.cpp,
buffer_test.cu, spmv_test.cu, mat_builder_test.cu), unchanged, compiled
against this repository's include/ (oracle/_ref/tests_g1, built by
`make -C oracle reftests` when the reference tree is present).
loader_test is host-only: built against both header trees, it prints the
same bytes on the same sample file (its edge list with first-seen
renumbering, the CSR and the transposed CSR).  CPU only."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G1 = os.path.join(ROOT, "oracle", "_ref", "tests_g1")
REF = os.path.join(ROOT, "oracle", "_ref", "tests_ref")

pytestmark = pytest.mark.skipif(not os.path.isdir(G1), reason="oracle/_ref/tests_g1 not built")


def test_graphone_test_programs_build_unchanged_against_these_headers():
    for t in ("loader_test", "buffer_test", "spmv_test", "mat_builder_test"):
        assert os.access(os.path.join(G1, t), os.X_OK), t


def sample_files():
    rng = np.random.default_rng(11)
    a, b = rng.integers(0, 400, 3000), rng.integers(0, 400, 3000)
    w = (np.minimum(a, b) * 31 + np.maximum(a, b)) % 50 + 1
    rand = "\n".join(f"{x} {y} {z}" for x, y, z in zip(a, b, w)) + "\n"
    return {
        "small": "% sample\n0 1 5\n1 2 3\n2 0 7\n5 3 2\n3 5 2\n0 1 5\n4 4 1\n7\t6\n2 3 4\n",
        "sparse_ids": "% ids far apart: renumbering compacts them\n100 7 1\n7 3000 2\n3000 100 3\n42 42 9\n",
        "random": rand,
    }


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "loader_test")), reason="reference loader_test not built")
@pytest.mark.parametrize("name", sorted(sample_files()))
def test_loader_test_prints_the_same_bytes_on_both_header_trees(tmp_path, name):
    # the program reads ../datasets/sample/sample.adj
    d = tmp_path / "datasets" / "sample"
    d.mkdir(parents=True)
    (d / "sample.adj").write_text(sample_files()[name])
    run = tmp_path / "run"
    run.mkdir()
    outs = []
    for exe in (os.path.join(G1, "loader_test"), os.path.join(REF, "loader_test")):
        r = subprocess.run([exe], cwd=run, capture_output=True, timeout=60)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(r.stdout)
    assert outs[0] == outs[1]
    assert b"edge_cache:[" in outs[0] and b"A^T:CsrMat{" in outs[0]
