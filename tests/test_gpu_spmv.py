"""Semiring SpMV on the GPU against the oracle (bit-exact for integer
semirings; plus-times fp32 within 1e-6 relative L1 of FP64)."""
import numpy as np
import pytest
import torch

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O
from tests.gpu_util import edge_case_graphs

pytestmark = pytest.mark.gpu

GRAPHS = edge_case_graphs()


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR, g1.SCHED_AUTO])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_minplus_u32_bit_exact(cuda, name, sched):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    rng = np.random.default_rng(11)
    for t in (0, 1):
        rp, ci, v = g.np("t" if t else "n")
        for density in (0.02, 0.5, 1.0):
            x = np.full(g.n, O.U32_MAX, np.uint32)
            sel = rng.random(g.n) < density
            x[sel] = rng.integers(0, 1 << 20, size=int(sel.sum()), dtype=np.uint32)
            xd = torch.from_numpy(x.view(np.int32)).cuda()
            yd = torch.empty(g.n, dtype=torch.int32, device="cuda")
            G.spmv(xd, yd, g1.SR_MINPLUS_U32, transpose=t, schedule=sched)
            y = yd.cpu().numpy().view(np.uint32)
            assert np.array_equal(y, O.spmv_minplus_u32(rp, ci, v, x)), (name, t, density)


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_bfs_semiring_bit_exact(cuda, name, sched):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    rp, ci, v = g.np("t")
    x = np.full(g.n, O.U32_MAX, np.uint32)
    x[:: 3] = np.arange(len(x[::3]), dtype=np.uint32)
    xd = torch.from_numpy(x.view(np.int32)).cuda()
    yd = torch.empty(g.n, dtype=torch.int32, device="cuda")
    G.spmv(xd, yd, g1.SR_BFS_U32, transpose=1, schedule=sched)
    exp = O.spmv_minplus_u32(rp, ci, np.ones_like(v), x)
    assert np.array_equal(yd.cpu().numpy().view(np.uint32), exp)


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR])
@pytest.mark.parametrize("scale", [10, 14])
def test_plustimes_f32_within_1e6_of_fp64(cuda, scale, sched):
    g = gen.rmat(scale, 16, False, float_values=True)
    G = g1.Graph.from_gen(g)
    rp, ci, v = g.np("t")
    x = np.random.default_rng(3).random(g.n).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty(g.n, dtype=torch.float32, device="cuda")
    G.spmv(xd, yd, g1.SR_PLUSTIMES_F32, transpose=1, schedule=sched)
    y64 = O.spmv_plustimes_f64(rp, ci, v.astype(np.float64), x.astype(np.float64))
    err = O.rel_l1(yd.cpu().numpy(), y64)
    assert err < 1e-6, err  # tolerance: relative L1 vs FP64


def test_golden_spmv_fixtures(cuda):
    for name in ("rmat8_sym", "rmat9_dir", "grid16"):
        gold = dict(np.load(f"tests/golden/{name}.npz"))
        n = int(gold["n"])
        G = g1.Graph.from_csr(gold["t_rp"], gold["t_col"], gold["t_val"], input_transpose=True)
        xd = torch.from_numpy(gold["spmv_mp_x"].view(np.int32)).cuda()
        yd = torch.empty(n, dtype=torch.int32, device="cuda")
        G.spmv(xd, yd, g1.SR_MINPLUS_U32, transpose=1)
        assert np.array_equal(yd.cpu().numpy().view(np.uint32), gold["spmv_mp_y"])


def test_transpose_built_on_gpu_matches_host(cuda):
    g = gen.rmat(12, 16, False, (1, 64))
    G = g1.Graph.from_gen(g)
    import ctypes as C
    rp_p, ci_p, v_p = C.c_void_p(), C.c_void_p(), C.c_void_p()
    g1.check(g1.lib().g1_graph_arrays(G.handle, 1, C.byref(rp_p), C.byref(ci_p), C.byref(v_p)))
    trp, tci, tv = g.np("t")
    def fetch(ptr, count):
        out = np.empty(count, np.uint32)
        g1.check(g1.lib().g1_mem_copy(out.ctypes.data, ptr.value, count * 4, 1, None))
        return out
    assert np.array_equal(fetch(rp_p, g.n + 1), trp)
    assert np.array_equal(fetch(ci_p, g.m), tci)
    assert np.array_equal(fetch(v_p, g.m), tv)


def test_malformed_csr_is_rejected(cuda):
    rp = np.array([0, 2, 1, 3], np.uint32)  # not monotone
    ci = np.array([1, 2, 0], np.uint32)
    v = np.ones(3, np.uint32)
    with pytest.raises(g1.G1Error) as e:
        g1.Graph.from_csr(rp, ci, v)
    assert e.value.status == 1
    rp = np.array([0, 1, 2, 3], np.uint32)
    ci = np.array([1, 7, 0], np.uint32)  # column out of range
    with pytest.raises(g1.G1Error) as e:
        g1.Graph.from_csr(rp, ci, v)
    assert e.value.status == 1


@pytest.mark.parametrize("variant", list(range(len(g1.MERGE_VARIANTS))))
@pytest.mark.parametrize("name", ["star20k", "rmat10_sym", "rmat11_dir", "path3000", "empty5"])
def test_every_merge_variant(cuda, name, variant):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    G.set_schedule(g1.SCHED_MERGE, variant, transpose=1)
    rp, ci, v = g.np("t")
    rng = np.random.default_rng(5)
    x = np.full(g.n, O.U32_MAX, np.uint32)
    sel = rng.random(g.n) < 0.3
    x[sel] = rng.integers(0, 1 << 20, size=int(sel.sum()), dtype=np.uint32)
    xd = torch.from_numpy(x.view(np.int32)).cuda()
    yd = torch.empty(g.n, dtype=torch.int32, device="cuda")
    G.spmv(xd, yd, g1.SR_MINPLUS_U32, transpose=1, schedule=g1.SCHED_MERGE)
    assert np.array_equal(yd.cpu().numpy().view(np.uint32), O.spmv_minplus_u32(rp, ci, v, x))
    # plus-times on the same graph, fp32 vs fp64
    xf = rng.random(g.n).astype(np.float32)
    vf = v.astype(np.float32)
    Gf = g1.Graph.from_csr(rp, ci, vf, input_transpose=True, build_other=False)
    Gf.set_schedule(g1.SCHED_MERGE, variant, transpose=1)
    yf = torch.empty(g.n, dtype=torch.float32, device="cuda")
    Gf.spmv(torch.from_numpy(xf).cuda(), yf, g1.SR_PLUSTIMES_F32, transpose=1,
            schedule=g1.SCHED_MERGE)
    y64 = O.spmv_plustimes_f64(rp, ci, vf.astype(np.float64), xf.astype(np.float64))
    assert O.rel_l1(yf.cpu().numpy(), y64) < 1e-6


@pytest.mark.parametrize("variant", list(range(len(g1.MERGE_VARIANTS))))
def test_pagerank_every_merge_variant(cuda, variant):
    g = gen.rmat(13, 16, False, float_values=True)
    G = g1.Graph.from_gen(g)
    G.set_schedule(g1.SCHED_MERGE, variant, transpose=1)
    trp, tci, tv = g.np("t")
    r = G.pagerank(0.85, 20, g1.PR_DANGLING)
    assert O.rel_l1(r, O.pagerank_f64(trp, tci, tv, 0.85, 20, 1)) < 1e-6


@pytest.mark.parametrize("relabel", [False, True])
def test_autotune_picks_a_variant_and_keeps_parity(cuda, relabel):
    g = gen.rmat(14, 16, False, float_values=True)
    G = g1.Graph.from_gen(g, relabel=relabel)
    merge_ms, vector_ms, variant = G.autotune()
    assert 0 <= variant < len(g1.MERGE_VARIANTS)
    assert merge_ms > 0 and vector_ms > 0
    trp, tci, tv = g.np("t")
    r = G.pagerank(0.85, 20, g1.PR_DANGLING)
    assert O.rel_l1(r, O.pagerank_f64(trp, tci, tv, 0.85, 20, 1)) < 1e-6
