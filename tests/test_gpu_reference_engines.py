"""GraphOne's own GPU engines, built from the reference sources into
oracle/_ref/libgraphone_refgpu.so (the reference GPU baseline the bench times
beside this library), checked on small graphs against the oracle and against
this library's results, so that the baseline computes what it is said to."""
import numpy as np
import pytest

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O
from tests.gpu_util import edge_case_graphs

pytestmark = pytest.mark.gpu

GRAPHS = edge_case_graphs()


def _need_refgpu():
    if O.refgpu() is None:
        pytest.skip("oracle/_ref/libgraphone_refgpu.so was not built (reference tree absent)")


@pytest.mark.parametrize("name", ["rmat10_sym", "rmat11_dir", "grid32", "path3000"])
def test_reference_gpu_sssp_engines_match_dijkstra(cuda, name):
    _need_refgpu()
    g = GRAPHS[name]
    rp, ci, v = g.np("n")
    trp, tci, tv = g.np("t")
    G = g1.Graph.from_gen(g)
    for s in sorted({0, g.n // 2}):
        ref = O.dijkstra_u32(rp, ci, v, s)
        d_blas, _, it_blas = O.refgpu_sssp_blas(trp, tci, tv, [s])
        d_adv, _, _ = O.refgpu_sssp_adv(rp, ci, v, [s])
        assert np.array_equal(d_blas, ref), (name, s)
        assert np.array_equal(d_adv, ref), (name, s)
        # the sparse-frontier BLAS engine's loop: same iteration count as ours
        _, it = G.sssp(s, g1.ENGINE_BLAS, return_iters=True)
        assert int(it_blas[0]) == it, (name, s)


@pytest.mark.parametrize("scale", [10, 14])
def test_reference_gpu_pagerank_matches_fp64_and_ours(cuda, scale):
    _need_refgpu()
    g = gen.rmat(scale, 16, False, float_values=True)
    rp, ci, v = g.np("n")
    trp, tci, tv = g.np("t")
    rank, ms, ms_spmv = O.refgpu_pagerank(rp, ci, v, trp, tci, tv, 0.85, 30, reps=2, spmv_reps=2)
    r64 = O.pagerank_f64(trp, tci, tv, 0.85, 30, 0)
    assert O.rel_l1(rank, r64) < 1e-6  # tolerance: relative L1 vs the FP64 oracle
    ours = g1.Graph.from_gen(g).pagerank(0.85, 30, g1.PR_REFERENCE)
    assert O.rel_l1(ours, r64) < 1e-6
    assert len(ms) == 2 and len(ms_spmv) == 2 and (ms > 0).all() and (ms_spmv > 0).all()
