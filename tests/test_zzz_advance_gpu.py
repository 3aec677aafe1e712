"""g1_advance_run, one push relax step of the advance/filter engine over
caller-owned device arrays, iterated to convergence from a source: the
distances (BFS levels with unit=1) bit-exact against the oracle's Dijkstra /
BFS on every edge-case graph (short adjacency lists take the lanes-per-vertex
kernel, graphs with hubs the edge-balanced one).

Collected last (file name) so that a failure here cannot hide the others."""
import numpy as np
import pytest
import torch

import graphone_b200 as g1
from oracle import oracle as O
from tests.gpu_util import edge_case_graphs

pytestmark = pytest.mark.gpu

GRAPHS = edge_case_graphs()


def traverse_by_steps(G, n, src, unit):
    dev = torch.device("cuda:0")
    dist = torch.full((n,), -1, dtype=torch.int32, device=dev)  # UINT32_MAX
    dist[src] = 0
    visited = torch.zeros(n, dtype=torch.int32, device=dev)
    fr = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
    fr[0] = src
    out = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    n_f, it = 1, 0
    while n_f:
        it += 1
        assert it <= n + 1
        n_f = G.advance_run(fr, n_f, dist, visited, it, out, unit=unit)
        fr, out = out, fr
    return dist.cpu().numpy().view(np.uint32), it


@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_advance_steps_match_oracle(cuda, name, unit):
    g = GRAPHS[name]
    rp, ci, v = g.np("n")
    G = g1.Graph.from_gen(g)
    src = 0
    got, _ = traverse_by_steps(G, g.n, src, unit)
    ref = O.bfs(rp, ci, src) if unit else O.dijkstra_u32(rp, ci, v, src)
    assert np.array_equal(got, ref)
    G.close()


def test_advance_run_rejects_host_arrays_and_relabelled_graphs(cuda):
    g = GRAPHS["grid32"]
    G = g1.Graph.from_gen(g)
    host = np.zeros(g.n, np.uint32)
    with pytest.raises(g1.G1Error):
        G.advance_run(host, 1, host, host, 1, host)
    G.close()
    R = g1.Graph.from_gen(g, relabel=True)
    d = torch.zeros(g.n, dtype=torch.int32, device="cuda:0")
    with pytest.raises(g1.G1Error):
        R.advance_run(d, 1, d, d, 1, d)
    R.close()


@pytest.mark.parametrize("name", ["grid32", "star20k"])
def test_advance_run_out_of_range_ids_and_unreached_vertices(cuda, name):
    """Frontier ids come from the caller: an id >= n is skipped on the device
    and reported as G1_ERR_INVALID (the graph stays usable), and a frontier
    vertex whose distance is still UINT32_MAX pushes nothing (MAX + w would
    wrap).  grid32 takes the lanes-per-vertex kernel, star20k (a hub) the
    edge-balanced one."""
    g = GRAPHS[name]
    rp, ci, v = g.np("n")
    G = g1.Graph.from_gen(g)
    dev = torch.device("cuda:0")
    n = g.n
    for unit in (False, True):
        dist = torch.full((n,), -1, dtype=torch.int32, device=dev)
        dist[0] = 0
        visited = torch.zeros(n, dtype=torch.int32, device=dev)
        out = torch.empty(n, dtype=torch.int32, device=dev)
        bad = torch.tensor([0, n, n + 12345, 0x7FFFFFFF], dtype=torch.int32, device=dev)
        with pytest.raises(g1.G1Error) as e:
            G.advance_run(bad, 4, dist, visited, 1, out, unit=unit)
        assert e.value.status == 1  # G1_ERR_INVALID
        # an unreached vertex in the frontier changes nothing
        dist2 = torch.full((n,), -1, dtype=torch.int32, device=dev)
        fr = torch.tensor([n - 1], dtype=torch.int32, device=dev)
        assert G.advance_run(fr, 1, dist2, visited, 2, out, unit=unit) == 0
        assert bool((dist2 == -1).all())
    # the graph is still usable: a full traversal by steps is exact
    got, _ = traverse_by_steps(G, n, 0, False)
    assert np.array_equal(got, O.dijkstra_u32(rp, ci, v, 0))
    G.close()
