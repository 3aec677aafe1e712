"""Bounded device waits run out cleanly: with g1_test_set_wait_polls(0)
every wait gives up at its first poll -- the near-far engine's grid barrier
and the waits on bulk copies of the TMA-staged SpMV variants (block tiles,
warp tiles, nnz tiles) -- the call returns G1_ERR_TIMEOUT, the kernels still
let their copies in flight land before leaving, and afterwards, with the
defaults back, the same graphs give exact results in the same process.

No GPU fault is involved: a wait that runs out is an ordinary return path.
Collected late (file name) so that a failure here cannot hide the others."""
import numpy as np
import pytest

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TMA_VARIANTS = (3, 4, 6, 24, 26)  # block tiles (2 and 1 stages), warp tiles, nnz tiles (col+val, col)


def test_bounded_waits_run_out_and_the_process_stays_usable(cuda):
    grid = gen.grid2d(64, 64, (1, 100))
    G = g1.Graph.from_gen(grid)
    rp, ci, v = grid.np("n")
    ref = O.dijkstra_u32(rp, ci, v, 0)
    ref_bfs = O.bfs(rp, ci, 0)
    rm = gen.rmat(12, 16, False, float_values=True)
    trp, tci, tv = rm.np("t")
    R = g1.Graph.from_gen(rm)
    pr64 = O.pagerank_f64(trp, tci, tv, 0.85, 3, 1)
    try:
        g1.test_set_wait_polls(0)
        for fn in (G.sssp, G.bfs):
            with pytest.raises(g1.G1Error) as e:
                fn(0, g1.ENGINE_NEARFAR)
            assert e.value.status == 4, fn  # G1_ERR_TIMEOUT
        for var in TMA_VARIANTS:
            R.set_schedule(g1.SCHED_MERGE, var)
            with pytest.raises(g1.G1Error) as e:
                R.pagerank(0.85, 3, g1.PR_DANGLING)
            assert e.value.status == 4, var
    finally:
        g1.test_set_wait_polls(-1)
    # defaults back: exact results from the same graphs
    assert np.array_equal(G.sssp(0, g1.ENGINE_NEARFAR), ref)
    assert np.array_equal(G.bfs(0, g1.ENGINE_NEARFAR), ref_bfs)
    for var in TMA_VARIANTS:
        R.set_schedule(g1.SCHED_MERGE, var)
        assert O.rel_l1(R.pagerank(0.85, 3, g1.PR_DANGLING), pr64) < 1e-6, var
    G.close()
    R.close()
