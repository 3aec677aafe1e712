"""The oracle against GraphOne's own code (golden fixtures) and against
independent algorithms.  CPU only."""
import glob
import os

import numpy as np
import pytest
import torch

from graphone_b200 import gen
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


GRAPHS = {
    "rmat8_sym": lambda: gen.rmat(8, 16, True, (1, 64)),
    "rmat9_dir": lambda: gen.rmat(9, 16, False, (1, 64)),
    "grid16": lambda: gen.grid2d(16, 16, (1, 100)),
    "rmat8_pr": lambda: gen.rmat(8, 16, False, float_values=True),
}


def test_generator_matches_c_restatement():
    tA, tAB, tABC = gen.rmat_thresholds(0.57, 0.19, 0.19)
    s, d = gen.rmat_samples(11, 8, seed=99)
    s2, d2 = O.rmat_samples(11, 8 << 11, (tA, tAB, tABC), 99)
    assert np.array_equal(s.numpy(), s2) and np.array_equal(d.numpy(), d2)
    keys = torch.arange(0, 5000, dtype=torch.int64) * 7919
    w = (gen._lsr(gen.rng(1234, keys), 11) % 64 + 1).numpy()
    w2 = np.array([O.lib().orc_edge_weight(1234, int(k), 1, 64) for k in keys.tolist()])
    assert np.array_equal(w, w2)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_csr_matches_reference_loader(name):
    """gen's CSR == GraphLoader + EdgeCache::ToCsr on the same edges; so does
    the oracle's restated counting sort."""
    gold = load(name)
    g = GRAPHS[name]()
    n_ref = int(gold["n"])
    assert int(gold["m"]) == g.m
    for tag, which in (("n", "n"), ("t", "t")):
        rp, ci, v = g.np(which)
        assert np.array_equal(rp[: n_ref + 1], gold[f"{tag}_rp"])
        assert np.all(rp[n_ref:] == g.m)  # trailing isolated vertices only
        assert np.array_equal(ci, gold[f"{tag}_col"])
        if v.dtype == np.uint32:
            assert np.array_equal(v, gold[f"{tag}_val"])
    # oracle counting sort from the (src, dst)-sorted edge list
    rp, ci, v = g.np("n")
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
    vv = v if v.dtype == np.uint32 else v.astype(np.uint32)
    trp, tci, tv = O.csr_build(g.n, src, ci, vv, transpose=True)
    assert np.array_equal(trp[: n_ref + 1], gold["t_rp"])
    assert np.array_equal(tci, gold["t_col"])


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_oracle_spmv_matches_reference_naive(name):
    gold = load(name)
    rp, ci, v = gold["t_rp"], gold["t_col"], gold["t_val"]
    y = O.spmv_minplus_u32(rp, ci, v, gold["spmv_mp_x"])
    assert np.array_equal(y, gold["spmv_mp_y"])
    yf = O.spmv_plustimes_f32(rp, ci, v.astype(np.float32), gold["spmv_pt_x"])
    assert np.array_equal(yf, gold["spmv_pt_y"])  # same sequential fp32 order


@pytest.mark.parametrize("name", ["rmat8_sym", "rmat9_dir", "grid16"])
def test_oracle_sssp_matches_reference_engine(name):
    gold = load(name)
    src = int(gold["sssp_src"])
    d, it = O.sssp_blas_u32(gold["t_rp"], gold["t_col"], gold["t_val"], src)
    assert np.array_equal(d, gold["sssp_dist"])
    assert it == int(gold["sssp_iters"])
    d2, _ = O.sssp_advance_u32(gold["n_rp"], gold["n_col"], gold["n_val"], src)
    assert np.array_equal(d2, gold["sssp_dist"])
    d3 = O.dijkstra_u32(gold["n_rp"], gold["n_col"], gold["n_val"], src)
    assert np.array_equal(d3, gold["sssp_dist"])


def test_oracle_sssp_matches_scipy():
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import dijkstra
    g = gen.rmat(10, 8, False, (1, 64))
    rp, ci, v = g.np("n")
    A = csr_matrix((v.astype(np.float64), ci, rp), shape=(g.n, g.n))
    for src in (0, 3, 17):
        ref = dijkstra(A, indices=src)
        d = O.dijkstra_u32(rp, ci, v, src)
        exp = np.where(np.isinf(ref), O.U32_MAX, ref).astype(np.uint32)
        assert np.array_equal(d, exp)
        trp, tci, tv = g.np("t")
        d2, _ = O.sssp_blas_u32(trp, tci, tv, src)
        assert np.array_equal(d2, exp)


def test_oracle_bfs_is_unit_weight_sssp():
    g = gen.rmat(10, 8, True, (1, 64))
    rp, ci, v = g.np("n")
    for src in (0, 5):
        lv = O.bfs(rp, ci, src)
        d, _ = O.sssp_blas_u32(rp, ci, np.ones_like(v), src)
        assert np.array_equal(lv, d)


def test_oracle_pagerank_matches_reference_fp32_and_power_iteration():
    gold = load("rmat8_pr")
    rp, ci = gold["t_rp"], gold["t_col"]
    v = gold["t_val"].astype(np.float32)
    for mode in (0, 1):
        r64 = O.pagerank_f64(rp, ci, v, 0.85, 30, mode)
        assert O.rel_l1(gold[f"pr{mode}_rank"], r64) < 1e-6
    # independent dense power iteration (mode 1: column-stochastic with
    # dangling columns replaced by the uniform vector)
    n = len(rp) - 1
    A = np.zeros((n, n))
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            A[r, ci[k]] += v[k]
    outw = A.sum(axis=0)
    M = np.where(outw > 0, A / np.where(outw > 0, outw, 1), 1.0 / n)
    x = np.full(n, 1.0 / n)
    for _ in range(30):
        x = 0.85 * M @ x + 0.15 / n
    assert O.rel_l1(O.pagerank_f64(rp, ci, v, 0.85, 30, 1), x) < 1e-12


def test_oracle_ppr_mass_is_conserved():
    g = gen.rmat(9, 8, False, float_values=True)
    rp, ci, v = g.np("t")
    r = O.ppr_f64(rp, ci, v, src=3, alpha=0.85, iters=20)
    assert abs(r.sum() - 1.0) < 1e-9
    assert r[3] > 0.15


def test_golden_fixtures_present():
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    assert set(GRAPHS) <= set(names)


@pytest.mark.parametrize("float_values", [False, True])
def test_write_adj_lists_each_undirected_edge_once(tmp_path, float_values):
    """The .adj writer (GraphOne's `src dst w` edge list, read by the unchanged
    apps) lists each undirected edge once, u < v, with its weight."""
    g = gen.rmat(9, 16, True, (1, 64), float_values=float_values)
    path = tmp_path / "g.adj"
    gen.write_adj(g, str(path), False)
    lines = path.read_text().splitlines()
    assert lines[0].startswith("%")
    rows = np.array([l.split() for l in lines[1:]], dtype=np.float64)
    rp, ci, v = g.np("n")
    src = np.repeat(np.arange(g.n), np.diff(rp.astype(np.int64)))
    keep = src < ci
    assert rows.shape == (int(keep.sum()), 3)
    assert np.array_equal(rows[:, 0], src[keep]) and np.array_equal(rows[:, 1], ci[keep])
    assert np.array_equal(rows[:, 2].astype(v.dtype), v[keep])
