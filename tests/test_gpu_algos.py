"""SSSP / BFS bit-exact and PageRank within 1e-6 relative L1 of the FP64
oracle, on the GPU through the C ABI."""
import numpy as np
import pytest

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O
from tests.gpu_util import edge_case_graphs

pytestmark = pytest.mark.gpu

GRAPHS = edge_case_graphs()
ENGINES = [g1.ENGINE_BLAS, g1.ENGINE_ADVANCE, g1.ENGINE_AUTO, g1.ENGINE_NEARFAR]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_sssp_bit_exact(cuda, name, engine):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    rp, ci, v = g.np("n")
    srcs = sorted({0, g.n // 2, g.n - 1})
    for s in srcs:
        d = G.sssp(s, engine)
        assert np.array_equal(d, O.dijkstra_u32(rp, ci, v, s)), (name, s, engine)


SPARSE_STEP_GRAPHS = {  # 2^20 edges or more: the BLAS engine's sparse steps apply
    "rmat16_sym": lambda: gen.rmat(16, 16, True, (1, 64)),
    "rmat17_dir": lambda: gen.rmat(17, 16, False, (1, 64)),
}


@pytest.mark.parametrize("push_div", [1, 16, 1 << 30])
@pytest.mark.parametrize("name", ["rmat10_sym", "grid32", "path3000", "rmat16_sym", "rmat17_dir"])
def test_sssp_blas_iterations_match_reference_engine(cuda, name, push_div):
    """The BLAS engine's distances and iteration count are the reference
    loop's whether its steps pull every row (push_div 2^30: never sparse) or
    are computed from the frontier's out-edges (push_div 1: nearly always,
    on the graphs of 2^20 edges or more)."""
    g = GRAPHS[name] if name in GRAPHS else SPARSE_STEP_GRAPHS[name]()
    if name in SPARSE_STEP_GRAPHS:
        assert g.m >= 1 << 20
    G = g1.Graph.from_gen(g)
    G.set_traversal_thresholds(push_div=push_div)
    trp, tci, tv = g.np("t")
    rp, ci, _ = g.np("n")
    for s in sorted({0, g.n // 3, g.n - 1}):
        d, it = G.sssp(s, g1.ENGINE_BLAS, return_iters=True)
        d_o, it_o = O.sssp_blas_u32(trp, tci, tv, s)
        assert np.array_equal(d, d_o) and it == it_o, (name, s)
        assert np.array_equal(G.bfs(s, g1.ENGINE_BLAS), O.bfs(rp, ci, s)), (name, s)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_bfs_bit_exact(cuda, name, engine):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    rp, ci, _ = g.np("n")
    for s in sorted({0, g.n - 1}):
        assert np.array_equal(G.bfs(s, engine), O.bfs(rp, ci, s)), (name, s, engine)


def test_sssp_golden_fixtures(cuda):
    for name in ("rmat8_sym", "rmat9_dir", "grid16"):
        gold = dict(np.load(f"tests/golden/{name}.npz"))
        G = g1.Graph.from_csr(gold["n_rp"], gold["n_col"], gold["n_val"])
        for e in ENGINES:
            assert np.array_equal(G.sssp(int(gold["sssp_src"]), e), gold["sssp_dist"])


@pytest.mark.parametrize("mode", [g1.PR_REFERENCE, g1.PR_DANGLING])
@pytest.mark.parametrize("scale", [8, 12, 16])
def test_pagerank_within_1e6_of_fp64(cuda, scale, mode):
    g = gen.rmat(scale, 16, False, float_values=True)
    G = g1.Graph.from_gen(g)
    trp, tci, tv = g.np("t")
    r = G.pagerank(0.85, 30, mode)
    r64 = O.pagerank_f64(trp, tci, tv, 0.85, 30, mode)
    err = O.rel_l1(r, r64)
    assert err < 1e-6, err  # tolerance: relative L1 vs the FP64 oracle


def test_pagerank_golden(cuda):
    gold = dict(np.load("tests/golden/rmat8_pr.npz"))
    G = g1.Graph.from_csr(gold["n_rp"], gold["n_col"], gold["n_val"].astype(np.float32))
    for mode in (0, 1):
        r = G.pagerank(0.85, 30, mode)
        assert O.rel_l1(r, gold[f"pr{mode}_rank"]) < 1e-6


@pytest.mark.parametrize("iters", [1, 2, 3, 30])
def test_pagerank_isolated_vertices_every_nnz_variant(cuda, iters):
    """Isolated vertices (no in- or out-edges) are skipped by the nnz fixup
    before the last iteration and counted into the dangling mass instead;
    rank is written only in the last iteration.  Results must match the FP64
    oracle, and every nnz variant (same fold order) must give the same bits."""
    import torch
    g0 = gen.rmat(12, 16, False, float_values=True)
    rp0, ci0, _ = g0.np("n")
    n = g0.n + 5000  # 5000 extra isolated vertices at the end
    src = torch.from_numpy(np.repeat(np.arange(g0.n), np.diff(rp0)).astype(np.int64))
    dst = torch.from_numpy(ci0.astype(np.int64))
    g = gen.from_edges(src, dst, n, False, (1, 64), float_values=True)
    trp, tci, tv = g.np("t")
    rp, ci, v = g.np("n")
    G = g1.Graph.from_csr(rp, ci, v, relabel=True)
    nnz_variants = [i for i, k in enumerate(g1.MERGE_VARIANTS) if k == "nnz"]
    # tiles of 32 x 8, 16, 24 nonzeros: another fold grouping, same plan logic
    nnz2_variants = [i for i, k in enumerate(g1.MERGE_VARIANTS) if k == "nnz2"]
    for mode in (g1.PR_REFERENCE, g1.PR_DANGLING):
        ref = O.pagerank_f64(trp, tci, tv, 0.85, iters, mode)
        first = None
        for var in nnz_variants:
            G.set_schedule(g1.SCHED_MERGE, var, transpose=1)
            r = G.pagerank(0.85, iters, mode)
            assert O.rel_l1(r, ref) < 1e-6, (mode, var)  # tolerance: relative L1 vs FP64
            if first is None:
                first = r
                assert np.array_equal(G.pagerank(0.85, iters, mode), r)  # run to run
            else:
                assert np.array_equal(r, first), (mode, var)
        for var in nnz2_variants:
            G.set_schedule(g1.SCHED_MERGE, var, transpose=1)
            r = G.pagerank(0.85, iters, mode)
            assert O.rel_l1(r, ref) < 1e-6, (mode, var)  # tolerance: relative L1 vs FP64
            assert np.array_equal(G.pagerank(0.85, iters, mode), r), (mode, var)  # run to run


def test_pagerank_device_output_and_zero_iterations(cuda):
    import torch
    g = gen.rmat(10, 16, False, float_values=True)
    G = g1.Graph.from_gen(g)
    out = torch.empty(g.n, dtype=torch.float32, device="cuda")
    G.pagerank(0.85, 0, g1.PR_DANGLING, out=out)
    torch.cuda.synchronize()
    assert torch.allclose(out, torch.full_like(out, 1.0 / g.n))


def test_invalid_source(cuda):
    G = g1.Graph.from_gen(GRAPHS["grid32"])
    with pytest.raises(g1.G1Error):
        G.sssp(10**6)


@pytest.mark.parametrize("name", ["rmat10_sym", "rmat11_dir", "star20k", "grid7x13", "single"])
def test_relabelled_graph_results_in_caller_order(cuda, name):
    """G1_GRAPH_RELABEL stores vertices by decreasing out-degree internally;
    every result must still come back bit-exact in the caller's order."""
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g, relabel=True)
    rp, ci, v = g.np("n")
    for e in ENGINES:
        for s in sorted({0, g.n - 1}):
            assert np.array_equal(G.sssp(s, e), O.dijkstra_u32(rp, ci, v, s)), (name, e, s)
            assert np.array_equal(G.bfs(s, e), O.bfs(rp, ci, s)), (name, e, s)


@pytest.mark.parametrize("variant", [0, 2, 5])
def test_relabelled_pagerank(cuda, variant):
    g = gen.rmat(14, 16, False, float_values=True)
    trp, tci, tv = g.np("t")
    rp, ci, v = g.np("n")
    G = g1.Graph.from_csr(rp, ci, v, relabel=True)
    G.set_schedule(g1.SCHED_MERGE, variant, transpose=1)
    for mode in (g1.PR_REFERENCE, g1.PR_DANGLING):
        r = G.pagerank(0.85, 30, mode)
        assert O.rel_l1(r, O.pagerank_f64(trp, tci, tv, 0.85, 30, mode)) < 1e-6


def test_relabelled_spmv_caller_order(cuda):
    import torch
    g = gen.rmat(12, 16, True, (1, 64))
    G = g1.Graph.from_gen(g, relabel=True)
    rp, ci, v = g.np("t")
    x = np.full(g.n, O.U32_MAX, np.uint32)
    x[::7] = np.arange(len(x[::7]), dtype=np.uint32)
    xd = torch.from_numpy(x.view(np.int32)).cuda()
    yd = torch.empty(g.n, dtype=torch.int32, device="cuda")
    G.spmv(xd, yd, g1.SR_MINPLUS_U32, transpose=1)
    assert np.array_equal(yd.cpu().numpy().view(np.uint32), O.spmv_minplus_u32(rp, ci, v, x))


@pytest.mark.parametrize("k", [1, 37, 256, 300])
@pytest.mark.parametrize("name", ["rmat10_sym", "rmat11_dir", "grid32", "star20k", "single"])
def test_batched_bfs_and_sssp_bit_exact(cuda, name, k):
    """k sources in one multi-source pass == k single-source runs."""
    g = GRAPHS[name]
    rp, ci, v = g.np("n")
    rng = np.random.default_rng(k)
    srcs = rng.choice(g.n, size=min(k, g.n), replace=False).astype(np.uint32)
    if len(srcs) < k:
        srcs = np.resize(srcs, k)  # repeats are allowed
    for relabel in (False, True):
        G = g1.Graph.from_gen(g, relabel=relabel)
        lv = G.bfs_batch(srcs)
        d = G.sssp_batch(srcs)
        for j in sorted(set(range(min(12, k))) | set(range(max(0, k - 3), k))):
            assert np.array_equal(lv[j], O.bfs(rp, ci, int(srcs[j]))), (name, k, j, relabel)
            assert np.array_equal(d[j], O.dijkstra_u32(rp, ci, v, int(srcs[j]))), (name, k, j, relabel)


@pytest.mark.parametrize("relabel", [False, True])
def test_pagerank_rmat20_within_1e6_of_fp64(cuda, relabel):
    """fp32 error grows with hub degree and graph size: the headline's error
    bound checked on a graph of a million vertices (RMAT-20 directed, 16.7M
    samples), both layouts, 30 iterations, dangling mass redistributed."""
    g = gen.rmat(20, 16, False, float_values=True, device="cuda")
    trp, tci, tv = g.np("t")
    G = g1.Graph.from_csr(trp, tci, tv, input_transpose=True, build_other=False, relabel=relabel)
    r = G.pagerank(0.85, 30, g1.PR_DANGLING)
    err = O.rel_l1(r, O.pagerank_f64(trp, tci, tv, 0.85, 30, 1))
    assert err < 1e-6, err  # tolerance: relative L1 vs the FP64 oracle


def test_pagerank_outweights_summed_during_upload(cuda):
    """A directed in-edge CSR of 2^22 edges or more with f32 values, from
    host memory, has its out-weights summed and its hot-column copy built
    chunk by chunk while it is copied.  Same ranks as a graph built from
    device arrays (both made at PageRank's first call; the integer-valued
    weights sum exactly in any order, and any column order gives the same
    bits), within 1e-6 of FP64; a column out of range is still rejected (the
    chunk histograms skip it)."""
    import torch
    g = gen.rmat(19, 16, False, float_values=True)
    assert g.m >= 1 << 22
    trp, tci, tv = g.np("t")
    ref = O.pagerank_f64(trp, tci, tv, 0.85, 30, 1)
    runs, created_bytes = [], []
    for host_input, validate in ((True, True), (True, False), (False, True)):
        args = (trp, tci, tv) if host_input else tuple(
            torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda() for a in (trp, tci, tv))
        G = g1.Graph.from_csr(*args, input_transpose=True, build_other=False, validate=validate)
        created_bytes.append(G.device_bytes())
        runs.append(G.pagerank(0.85, 30, g1.PR_DANGLING))
        G.close()
    # from host memory the hot-column copy (4 bytes per edge) was built during
    # the upload too; from device memory at PageRank's first call
    assert created_bytes[0] >= created_bytes[2] + 4 * g.m
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])
    assert O.rel_l1(runs[0], ref) < 1e-6  # tolerance: relative L1 vs the FP64 oracle
    bad = tci.copy()
    bad[len(bad) // 2] = g.n + 7
    with pytest.raises(g1.G1Error):
        g1.Graph.from_csr(trp, bad, tv, input_transpose=True, build_other=False)
    # the device still answers correctly afterwards
    G = g1.Graph.from_csr(trp, tci, tv, input_transpose=True, build_other=False)
    assert np.array_equal(G.pagerank(0.85, 30, g1.PR_DANGLING), runs[0])


@pytest.mark.parametrize("relabel", [False, True])
def test_pagerank_hot_columns_same_bits(cuda, relabel):
    """The hot-column layout renames the in-edge CSR's columns by decreasing
    out-degree and keeps x in that order; rows keep their nonzeros' order, so
    on every schedule the ranks are the same bits as on the plain layout."""
    g = gen.rmat(16, 16, False, float_values=True)
    trp, tci, tv = g.np("t")
    plain = g1.Graph.from_csr(trp, tci, tv, input_transpose=True, build_other=False, relabel=relabel)
    hot = g1.Graph.from_csr(trp, tci, tv, input_transpose=True, build_other=False, relabel=relabel)
    plain.set_hot_columns(g1.HOT_COLUMNS_OFF)
    hot.set_hot_columns(g1.HOT_COLUMNS_ON)
    bytes_plain = plain.device_bytes()
    ref = O.pagerank_f64(trp, tci, tv, 0.85, 30, 1)
    cases = [(g1.SCHED_VECTOR, 0)] + [(g1.SCHED_MERGE, v) for v in range(len(g1.MERGE_VARIANTS))]
    for sched, var in cases:
        for G in (plain, hot):
            G.set_schedule(sched, var, transpose=1)
        for iters in (1, 30):
            a = plain.pagerank(0.85, iters, g1.PR_DANGLING)
            b = hot.pagerank(0.85, iters, g1.PR_DANGLING)
            assert np.array_equal(a, b), (sched, var, iters)
        assert O.rel_l1(b, ref) < 1e-6, (sched, var)  # tolerance: relative L1 vs FP64
    # the copy of the column array (4 bytes per edge) and the hot ids
    assert hot.device_bytes() >= bytes_plain + 4 * g.m


@pytest.mark.parametrize("name", ["rmat10_sym", "rmat11_dir", "star20k", "grid32"])
def test_autotune_traversal_keeps_results_exact(cuda, name):
    """g1_autotune_traversal picks the push/pull divisors among its
    candidates; SSSP and BFS (single-source AUTO and batched) stay bit-exact."""
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g, relabel=(name == "rmat10_sym"))
    rp, ci, v = g.np("n")
    push_div, slot_div = G.autotune_traversal(8)
    assert push_div in (4, 8, 16, 32, 64, 128) and slot_div in (2, 4, 8, 16, 32)
    srcs = sorted({0, g.n // 3, g.n - 1})
    for s in srcs:
        assert np.array_equal(G.sssp(s, g1.ENGINE_AUTO), O.dijkstra_u32(rp, ci, v, s)), (name, s)
        assert np.array_equal(G.bfs(s, g1.ENGINE_AUTO), O.bfs(rp, ci, s)), (name, s)
    d = G.sssp_batch(np.array(srcs, np.uint32))
    for j, s in enumerate(srcs):
        assert np.array_equal(d[j], O.dijkstra_u32(rp, ci, v, s)), (name, s)
