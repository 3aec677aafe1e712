"""The apps' result files (GraphOne's "Elapsed time" line then "<vid>-<%f>"
per vertex, apps/sssp_blas.cu:123-134) and the comparator
(graphone_b200.results): written, read back and compared on the CPU against
the oracle's results, with the CLI's exit codes."""
import os
import subprocess
import sys

import numpy as np

from graphone_b200 import gen, results
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def cli(*args):
    return subprocess.run([sys.executable, "-m", "graphone_b200.results", *args],
                          capture_output=True, text=True, cwd=ROOT)


def test_sssp_result_round_trip_and_compare(tmp_path):
    g = gen.rmat(10, 8, False, (1, 64))  # directed: some vertices unreachable
    rp, ci, v = g.np("n")
    d = O.dijkstra_u32(rp, ci, v, 0)
    assert (d == O.U32_MAX).any()
    a = str(tmp_path / "a.txt")
    results.write_result(a, d, 12.0)
    lines = open(a).read().splitlines()
    assert lines[0] == "Elapsed time: 12 ms"
    assert lines[1] == "0-0.000000"
    # unreachable prints as the apps print FLT_MAX with "%f"
    u = int(np.nonzero(d == O.U32_MAX)[0][0])
    assert lines[1 + u] == f"{u}-340282346638528859811704183484516925440.000000"
    r = results.read_result(a)
    assert r.elapsed_ms == 12.0 and len(r.values) == g.n
    assert results.compare(r, d).same
    # the same distances from the oracle's BLAS-engine loop compare equal too
    trp, tci, tv = g.np("t")
    d2, _ = O.sssp_blas_u32(trp, tci, tv, 0)
    b = str(tmp_path / "b.txt")
    results.write_result(b, d2, 3.0)
    assert cli("compare", a, b).returncode == 0
    # one distance off by one: different, reported
    d3 = d.copy()
    k = int(np.nonzero(d3 != O.U32_MAX)[0][5])
    d3[k] += 1
    c = str(tmp_path / "c.txt")
    results.write_result(c, d3)
    r3 = cli("compare", a, c)
    assert r3.returncode == 1 and f"vertex {k}:" in r3.stdout and "DIFFERENT" in r3.stdout
    cmp = results.compare(results.read_result(c), d)
    assert not cmp.same and cmp.n_different == 1


def test_pagerank_results_compare_within_tolerance(tmp_path):
    g = gen.rmat(10, 16, False, float_values=True)
    trp, tci, tv = g.np("t")
    r64 = O.pagerank_f64(trp, tci, tv, 0.85, 30, 1)
    a = str(tmp_path / "pr64.txt")
    b = str(tmp_path / "pr32.txt")
    results.write_result(a, r64)
    results.write_result(b, r64 * (1 + 1e-7))
    assert cli("compare", a, b, "--kind", "pagerank").returncode == 0
    results.write_result(b, r64 * (1 + 1e-4))
    assert cli("compare", a, b, "--kind", "pagerank").returncode == 1
    # "%f" keeps six decimals: exact comparison of ranks fails, tolerance passes
    assert cli("compare", a, b, "--kind", "pagerank", "--tol", "1e-3").returncode == 0


def test_sizes_limit_and_unreadable_files(tmp_path):
    a = str(tmp_path / "a.txt")
    b = str(tmp_path / "b.txt")
    results.write_result(a, np.arange(10, dtype=np.uint32))
    results.write_result(b, np.arange(8, dtype=np.uint32))
    assert cli("compare", a, b).returncode == 1  # sizes differ
    # GraphOne's loader drops trailing isolated vertices: compare a prefix
    assert cli("compare", a, b, "--limit", "8").returncode == 0
    bad = tmp_path / "bad.txt"
    bad.write_text("Elapsed time: 1 ms\nnot a line\n")
    assert cli("compare", a, str(bad)).returncode == 2
    assert cli("compare", a, str(tmp_path / "missing.txt")).returncode == 2
    # ids out of order are read by id
    c = tmp_path / "c.txt"
    c.write_text("Elapsed time: 0 ms\n2-2.000000\n0-0.000000\n1-1.000000\n")
    assert np.array_equal(results.read_result(str(c)).values, [0.0, 1.0, 2.0])
