"""GraphOne's own apps, unchanged, built against this repository's headers
(oracle/_ref/apps_g1, made by `make -C oracle dropin` from the reference
sources) and run on the GPU: their printed results must match the oracle."""
import os
import subprocess

import numpy as np
import pytest

from graphone_b200 import gen, results
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FLT_MAX = np.float32(3.4028234663852886e38)


def run_app(path, args, tmp_path, name="out.txt"):
    out = os.path.join(str(tmp_path), name)
    r = subprocess.run([path, *args, "-o", out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = results.read_result(out)
    assert res.elapsed_ms is not None and not np.isnan(res.values).any()
    return res.values, int(res.elapsed_ms)


def sssp_expected(g, src, n_out):
    rp, ci, v = g.np("n")
    d = O.dijkstra_u32(rp, ci, v, src)[:n_out]
    return np.where(d == O.U32_MAX, FLT_MAX, d.astype(np.float32)).astype(np.float32)


GRAPHS = {
    "rmat11": lambda: gen.rmat(11, 8, True, (1, 64)),
    "grid48": lambda: gen.grid2d(48, 48, (1, 100)),
    # 2^20 edges or more: sssp_blas's engine takes its sparse steps (small
    # frontiers fold only the rows they reach)
    "rmat17": lambda: gen.rmat(17, 8, True, (1, 64)),
}


@pytest.mark.parametrize("name", sorted(GRAPHS))
@pytest.mark.parametrize("app", ["sssp_blas", "sssp_blas2", "sssp_adv"])
def test_sssp_app_on_graphone_b200(cuda, app, name, tmp_path):
    path = O.app(app)
    if path is None:
        pytest.skip("apps_g1 not built (needs the reference sources at build time)")
    g = GRAPHS[name]()
    adj = os.path.join(str(tmp_path), "g.adj")
    gen.write_adj(g, adj, directed=False)
    src = int(np.argmax(np.diff(g.np("n")[0].astype(np.int64)) > 0))
    vals, _ = run_app(path, ["-i", adj, "--src", str(src)], tmp_path)
    assert np.array_equal(vals.astype(np.float32), sssp_expected(g, src, len(vals)))


def pagerank_app_expected(g, n, alpha=0.85, tol=1e-6):
    """The pagerank_blas loop in FP64: stop when max|r_k - r_{k-1}| <= tol
    (checked before every iteration, the first time against the zero array)
    and report r_{k-1} (the array opt_idx points at after the final flip)."""
    trp, tci, tv = g.np("t")
    trp = trp[: n + 1]
    outw = np.bincount(tci, weights=tv.astype(np.float64), minlength=n)[:n]
    iw = np.where(outw != 0, alpha / np.where(outw != 0, outw, 1), 0.0)
    hist = [np.zeros(n), np.full(n, 1.0 / n)]
    rows = np.repeat(np.arange(n), np.diff(trp.astype(np.int64)))
    while np.max(np.abs(hist[-1] - hist[-2])) > tol and len(hist) < 500:
        x = hist[-1] * iw
        y = np.bincount(rows, weights=x[tci] * tv, minlength=n)
        hist.append((1 - alpha) / n + y)
    return hist


def test_pagerank_app_on_graphone_b200(cuda, tmp_path):
    path = O.app("pagerank_blas")
    if path is None:
        pytest.skip("apps_g1 not built (needs the reference sources at build time)")
    g = gen.rmat(11, 8, False, float_values=True)
    adj = os.path.join(str(tmp_path), "g.adj")
    gen.write_adj(g, adj, directed=True)
    vals, _ = run_app(path, ["-i", adj, "-d"], tmp_path)
    hist = pagerank_app_expected(g, len(vals))
    # The app prints "%f" (six decimals, absolute error <= 5e-7); fp32 vs
    # fp64 may stop one iteration apart (consecutive iterates differ by at
    # most the 1e-6 convergence threshold).  The report is the second-to-last
    # array of the run.
    errs = [float(np.max(np.abs(vals - h))) for h in hist[-3:-1]]
    assert min(errs) < 2e-6, errs


@pytest.mark.parametrize("app", ["sssp_blas", "sssp_adv", "sssp_blas2"])
def test_app_output_compares_equal_to_the_oracle_with_the_cli(cuda, app, tmp_path):
    """The comparator CLI (python -m graphone_b200.results compare) on a
    result file of an unchanged app and one written from the oracle's
    Dijkstra in the apps' format: same; with one distance changed: not."""
    path = O.app(app)
    if path is None:
        pytest.skip("apps_g1 not built (needs the reference sources at build time)")
    g = gen.rmat(12, 8, True, (1, 64))
    adj = os.path.join(str(tmp_path), "g.adj")
    gen.write_adj(g, adj, directed=False)
    vals, _ = run_app(path, ["-i", adj, "--src", "0"], tmp_path, "app.txt")
    rp, ci, v = g.np("n")
    d = O.dijkstra_u32(rp, ci, v, 0)[: len(vals)]
    ref = os.path.join(str(tmp_path), "oracle.txt")
    results.write_result(ref, d)
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "-m", "graphone_b200.results", "compare", os.path.join(str(tmp_path), "app.txt"), ref]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=root)
    assert r.returncode == 0, r.stdout + r.stderr
    k = int(np.nonzero(d != O.U32_MAX)[0][-1])
    d[k] += 1
    results.write_result(ref, d)
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=root)
    assert r.returncode == 1 and f"vertex {k}:" in r.stdout
