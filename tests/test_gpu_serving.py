"""Personalized PageRank, continuous multi-source batching and the serving
loop (g1_ppr*, g1_server_*) against the oracle and against themselves:
every query's result is the same alone, in a batch and in the served mix.

Tolerances: BFS levels and SSSP distances bit-exact (u32); PPR within 1e-6
relative L1 of the FP64 oracle on every path.  PPR results of one engine
are bit-identical wherever the query runs: a slot engine query alone, in a
batch or served on a small graph; g1_ppr (the SpMV schedules) alone or
served solo on a graph of 2^22 edges or more."""
import threading
import time

import numpy as np
import pytest
import torch

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O
from tests.gpu_util import edge_case_graphs

pytestmark = pytest.mark.gpu

GRAPHS = edge_case_graphs()
PPR_TOL = 1e-6


def ppr_oracle(g, src, alpha=0.85, iters=20):
    trp, tci, _ = g.np("t")
    return O.ppr_f64(trp, tci, np.ones(len(tci), np.float32), src, alpha, iters)


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_ppr_matches_fp64_oracle(cuda, name, sched):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    G.set_schedule(sched, g1.DEFAULT_MERGE_VARIANT)
    for src in sorted({0, g.n // 2, g.n - 1}):
        r = G.ppr(src, 0.85, 20)
        ref = ppr_oracle(g, src)
        assert O.rel_l1(r, ref) < PPR_TOL, (name, src)


def small_directed():
    """0->1->2->0 (a cycle), 3->0 (3 has no in-edges), 2->4 (4 has no
    out-edges), 5 isolated, plus 6 with both a self loop and an edge to 4."""
    src = torch.tensor([0, 1, 2, 3, 2, 6, 6])
    dst = torch.tensor([1, 2, 0, 0, 4, 6, 4])
    return gen.from_edges(src, dst, 7, False, (1, 9), name="small_directed")


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR])
def test_ppr_sources_without_in_or_out_edges(cuda, sched):
    """The source's own row empty (the nnz fixup emits it by itself before
    the last iteration), a dangling source (its mass teleports back to it),
    an isolated source (rank 1 at the source forever) and a self loop."""
    g = small_directed()
    G = g1.Graph.from_gen(g)
    G.set_schedule(sched, g1.DEFAULT_MERGE_VARIANT)
    for src in range(g.n):
        for iters in (1, 2, 3, 20):
            r = G.ppr(src, 0.85, iters)
            ref = O.ppr_f64(*g.np("t")[:2], np.ones(g.m, np.float32), src, 0.85, iters)
            assert O.rel_l1(r, ref) < PPR_TOL, (src, iters)
    r = G.ppr(5, 0.85, 20)
    assert r[5] == 1.0 and np.count_nonzero(r) == 1


def test_ppr_directed_rmat_sources_with_empty_rows(cuda):
    g = GRAPHS["rmat11_dir"]
    G = g1.Graph.from_gen(g, relabel=True)
    rp, _, _ = g.np("n")
    trp, _, _ = g.np("t")
    indeg, outdeg = np.diff(trp), np.diff(rp)
    picks = [int(np.flatnonzero((indeg == 0) & (outdeg > 0))[0]),
             int(np.flatnonzero((indeg > 0) & (outdeg == 0))[0]),
             int(np.flatnonzero((indeg == 0) & (outdeg == 0))[0]),
             int(np.argmax(indeg))]
    for src in picks:
        assert O.rel_l1(G.ppr(src, 0.85, 20), ppr_oracle(g, src)) < PPR_TOL, src
        assert O.rel_l1(G.ppr(src, 0.5, 7), ppr_oracle(g, src, 0.5, 7)) < PPR_TOL, src


SPARSE_GRAPHS = {
    "grid1024": lambda: gen.grid2d(1024, 1024, (1, 100)),
    "rmat16_sym": lambda: gen.rmat(16, 16, True, (1, 64)),
    "rmat17_dir": lambda: gen.rmat(17, 16, False, (1, 64)),
    # uniform random (no hubs): sparse until the reach covers m / 16 edges
    "uniform17": lambda: gen.from_edges(*gen.rmat_samples(17, 8, 0.25, 0.25, 0.25), 1 << 17, True,
                                        (1, 64), name="uniform17"),
}


@pytest.mark.parametrize("sched", [g1.SCHED_MERGE, g1.SCHED_VECTOR])
@pytest.mark.parametrize("name", sorted(SPARSE_GRAPHS))
def test_ppr_sparse_steps_match_oracle(cuda, name, sched):
    """Graphs of 2^20 edges or more, where g1_ppr's first steps compute only
    the rows the source's neighbourhood reaches: every step of 20 on the
    grid, a few on the uniform graph before the full SpMV takes over, at
    most the first three on RMAT (whose hubs end them at once).
    Sources of every kind: a hub, a leaf, no out-edges, no in-edges,
    isolated; the last step sparse (1-3 iterations) or dense."""
    g = SPARSE_GRAPHS[name]()
    assert g.m >= 1 << 20
    G = g1.Graph.from_gen(g, relabel=name != "grid1024")
    G.set_schedule(sched, g1.DEFAULT_MERGE_VARIANT)
    rp, _, _ = g.np("n")
    trp, _, _ = g.np("t")
    indeg, outdeg = np.diff(trp), np.diff(rp)
    picks = {0, g.n // 2 + 17, g.n - 1, int(np.argmax(indeg))}
    for mask in ((outdeg == 1), (outdeg == 0) & (indeg > 0), (indeg == 0) & (outdeg > 0),
                 (indeg == 0) & (outdeg == 0)):
        hit = np.flatnonzero(mask)
        if len(hit):
            picks.add(int(hit[len(hit) // 2]))
    for src in sorted(picks):
        for iters in (1, 2, 3, 20):
            r = G.ppr(src, 0.85, iters)
            assert O.rel_l1(r, ppr_oracle(g, src, 0.85, iters)) < PPR_TOL, (src, iters)
        # the same bits again (the store's lists and flags reset per query)
        assert np.array_equal(G.ppr(src, 0.85, 20), r), src


@pytest.mark.parametrize("name", ["rmat16_sym", "rmat17_dir"])
def test_ppr_hot_columns_same_bits(cuda, name):
    """g1_ppr on the hot-column copy of the in-edge CSR (x stored by hot id,
    the full SpMV and the sparse steps) gives the same bits as on the plain
    layout, whichever of PageRank and PPR built the copy."""
    g = SPARSE_GRAPHS[name]()
    plain = g1.Graph.from_gen(g)
    hot = g1.Graph.from_gen(g)
    plain.set_hot_columns(g1.HOT_COLUMNS_OFF)
    hot.set_hot_columns(g1.HOT_COLUMNS_ON)
    srcs = [int(s) for s in gen.pick_sources(g, 4)]
    for sched in (g1.SCHED_MERGE, g1.SCHED_VECTOR):
        for G in (plain, hot):
            G.set_schedule(sched, g1.DEFAULT_MERGE_VARIANT)
        for src in srcs:
            for iters in (1, 3, 20):
                a = plain.ppr(src, 0.85, iters)
                b = hot.ppr(src, 0.85, iters)
                assert np.array_equal(a, b), (sched, src, iters)
        assert O.rel_l1(b, ppr_oracle(g, srcs[-1])) < PPR_TOL
    # a copy built by PageRank (out-weight order; the same edges with f32
    # values, which PPR does not read) serves PPR as well
    if not g.symmetric:
        gf = gen.rmat(17, 16, False, (1, 64), float_values=True)
        assert gf.m == g.m
        pr = g1.Graph.from_gen(gf)
        pr.set_hot_columns(g1.HOT_COLUMNS_ON)
        pr.pagerank(0.85, 2, g1.PR_DANGLING)
        plain.set_schedule(g1.SCHED_AUTO, g1.DEFAULT_MERGE_VARIANT)
        assert np.array_equal(pr.ppr(srcs[0], 0.85, 20), plain.ppr(srcs[0], 0.85, 20))


def test_ppr_zero_iterations_is_the_indicator(cuda):
    g = GRAPHS["rmat10_sym"]
    G = g1.Graph.from_gen(g)
    r = G.ppr(5, 0.85, 0)
    e = np.zeros(g.n, np.float32)
    e[5] = 1.0
    assert np.array_equal(r, e)


@pytest.mark.parametrize("name", ["rmat11_dir", "star20k", "grid32", "path3000"])
@pytest.mark.parametrize("k", [1, 37, 300])
def test_ppr_batch_bit_identical_wherever_a_query_sits(cuda, name, k):
    g = GRAPHS[name]
    G = g1.Graph.from_gen(g)
    rng = np.random.default_rng(k)
    srcs = rng.integers(0, g.n, size=k).astype(np.uint32)
    batch = G.ppr_batch(srcs, 0.85, 20)
    for i in sorted({0, k // 2, k - 1}):
        one = G.ppr_batch(srcs[i:i + 1], 0.85, 20)[0]
        assert np.array_equal(batch[i], one), (name, k, i)
        assert O.rel_l1(batch[i], G.ppr(int(srcs[i]), 0.85, 20)) < PPR_TOL
    assert O.rel_l1(batch[k - 1], ppr_oracle(g, int(srcs[k - 1]))) < PPR_TOL


def test_ppr_batch_device_output_and_relabelled_graph(cuda):
    g = gen.rmat(12, 16, True, (1, 100))
    G = g1.Graph.from_gen(g, relabel=True)
    srcs = gen.pick_sources(g, 40)
    out = torch.empty((40, g.n), dtype=torch.float32, device="cuda")
    G.ppr_batch(srcs, 0.85, 20, out=out)
    torch.cuda.synchronize()
    host = out.cpu().numpy()
    for i in (0, 39):
        assert O.rel_l1(host[i], ppr_oracle(g, int(srcs[i]))) < PPR_TOL


def test_ppr_rejects_bad_damping(cuda):
    G = g1.Graph.from_gen(GRAPHS["rmat10_sym"])
    with pytest.raises(g1.G1Error):
        G.ppr(0, 1.5, 20)


# ----------------------------------------------------------------- serving

def serving_graphs():
    """Small stand-ins for the serving mix: RMAT graphs and grids with
    uint32 weights in [1, 100]."""
    return [gen.rmat(10, 16, True, (1, 100)), gen.rmat(12, 16, True, (1, 100)),
            gen.grid2d(24, 24, (1, 100)), gen.grid2d(40, 17, (1, 100))]


def request_mix(graphs, count, seed):
    """(graph index, kind, source): 60% SSSP, 25% BFS, 15% PPR, graph and
    source uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        gi = int(rng.integers(0, len(graphs)))
        u = rng.random()
        kind = g1.QUERY_SSSP if u < 0.60 else (g1.QUERY_BFS if u < 0.85 else g1.QUERY_PPR)
        out.append((gi, kind, int(rng.integers(0, graphs[gi].n))))
    return out


def alone(G, kind, src):
    """The query run by itself on each engine the server may give it: the
    single-source engine first, then a slot engine (PPR only; distances and
    levels are the same on every engine)."""
    if kind == g1.QUERY_SSSP:
        return [G.sssp(src).view(np.uint32)]
    if kind == g1.QUERY_BFS:
        return [G.bfs(src).view(np.uint32)]
    return [G.ppr(src, 0.85, 20), G.ppr_batch(np.array([src], np.uint32), 0.85, 20)[0]]


def same_as_alone(res, G, kind, src, batched_only=False):
    """Bit-identical to the query run alone on one of its engines (on the
    slot engine when the server batches every query)."""
    cands = alone(G, kind, src)
    if batched_only:
        cands = cands[-1:]
    return any(np.array_equal(res.view(np.uint32), c.view(np.uint32)) for c in cands)


def check_against_oracle(g, kind, src, res):
    rp, ci, v = g.np("n")
    if kind == g1.QUERY_SSSP:
        assert np.array_equal(res.view(np.uint32), O.dijkstra_u32(rp, ci, v, src))
    elif kind == g1.QUERY_BFS:
        assert np.array_equal(res.view(np.uint32), O.bfs(rp, ci, src))
    else:
        assert O.rel_l1(res.view(np.float32), ppr_oracle(g, src)) < PPR_TOL


def host_out(g, kind):
    return np.empty(g.n, np.float32 if kind == g1.QUERY_PPR else np.uint32)


@pytest.mark.parametrize("max_batch,solo_queue_ms,lanes",
                         [(32, -1, 0), (256, -1, 0), (256, 0, 0), (64, 1000, 0), (256, 1000, 3)])
def test_served_mix_equals_each_query_alone(cuda, max_batch, solo_queue_ms, lanes):
    """solo_queue_ms -1: SSSP / BFS always batched on the slot engines; 0:
    the default hybrid (one at a time on the single-source engines while the
    queue is short); 1000: mostly one at a time, on one lane or three."""
    graphs = serving_graphs()
    Gs = [g1.Graph.from_gen(g) for g in graphs]
    reqs = request_mix(graphs, 400, seed=max_batch + solo_queue_ms + lanes)
    with g1.Server(max_batch=max_batch, solo_queue_ms=solo_queue_ms, solo_lanes=lanes) as srv:
        gids = [srv.add_graph(G) for G in Gs]
        outs = [host_out(graphs[gi], kind) for gi, kind, _ in reqs]
        # arrivals in waves, so later queries join batches already running
        tickets = []
        for i, (gi, kind, src) in enumerate(reqs):
            tickets.append(srv.submit(gids[gi], kind, src, outs[i]))
            if i % 50 == 49:
                time.sleep(0.002)
        lat = [srv.wait(t, 60000) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    if solo_queue_ms < 0:
        assert st["max_occupancy"] > 1  # queries did share engine steps
    assert all(x > 0 for x in lat)
    for i, (gi, kind, src) in enumerate(reqs):
        assert same_as_alone(outs[i], Gs[gi], kind, src, solo_queue_ms < 0), (i, gi, kind, src)
    for i in range(0, len(reqs), 37):
        gi, kind, src = reqs[i]
        check_against_oracle(graphs[gi], kind, src, outs[i])


def test_served_queries_run_solo_while_few_wait(cuda):
    """A handful of PPR and SSSP queries on one graph are served one at a
    time on the single-source engines: the same bits as g1_ppr / g1_sssp."""
    g = gen.rmat(18, 16, True, (1, 100), device="cuda")
    G = g1.Graph.from_gen(g, relabel=True)
    srcs = [int(s) for s in gen.pick_sources(g, 6)]
    with g1.Server() as srv:
        gid = srv.add_graph(G)
        pp = [np.empty(g.n, np.float32) for _ in srcs]
        ss = [np.empty(g.n, np.uint32) for _ in srcs]
        ts = []
        for i, s in enumerate(srcs):
            ts.append(srv.submit(gid, g1.QUERY_PPR, s, pp[i]))
            ts.append(srv.submit(gid, g1.QUERY_SSSP, s, ss[i]))
        for t in ts:
            srv.wait(t, 120000)
    for i, s in enumerate(srcs):
        assert np.array_equal(pp[i], G.ppr(s, 0.85, 20)), i
        assert np.array_equal(ss[i], G.sssp(s)), i
    assert O.rel_l1(pp[0], ppr_oracle(g, srcs[0])) < PPR_TOL


@pytest.mark.parametrize("stretch", [4.0, -1.0])
def test_lane_takes_short_queries_first_unless_told_oldest_first(cuda, stretch):
    """While a long grid traversal runs on the lane, a second long one (another
    grid) and then twelve short ones (a small RMAT graph) arrive.  With
    lane_stretch > 0 the lane takes the short ones first (their expected
    time is far lower and none has waited long); with a negative stretch it
    takes the oldest, the second grid.  Every result is the plain call's."""
    grids = [g1.Graph.from_gen(gen.grid2d(700, 700, (1, 100), seed=s)) for s in (1, 2)]
    g = gen.rmat(10, 16, True, (1, 100))
    small = g1.Graph.from_gen(g)
    srcs = [int(x) for x in gen.pick_sources(g, 12)]
    with g1.Server(lane_stretch=stretch) as srv:
        gids = [srv.add_graph(G) for G in grids + [small]]
        # a few queries per executor first: the lane's time estimates (its
        # first query, which pays one-time costs, sets none)
        warm = [np.empty(G.n, np.uint32) for G in grids + [small]]
        for _ in range(3):
            for gid, w in zip(gids, warm):
                srv.wait(srv.submit(gid, g1.QUERY_SSSP, 0, w), 120000)
        outs = [np.empty(grids[0].n, np.uint32), np.empty(grids[1].n, np.uint32)]
        t_long = [srv.submit(gids[0], g1.QUERY_SSSP, 5, outs[0])]
        # the first long query takes the idle lane at once (it runs ~8 ms);
        # the rest arrive while it runs
        time.sleep(0.003)
        t_long.append(srv.submit(gids[1], g1.QUERY_SSSP, 7, outs[1]))
        so = [np.empty(g.n, np.uint32) for _ in srcs]
        t_short = [srv.submit(gids[2], g1.QUERY_SSSP, s, so[i]) for i, s in enumerate(srcs)]
        lat_long = [srv.wait(t, 120000) for t in t_long]
        lat_short = [srv.wait(t, 120000) for t in t_short]
    for i, s in enumerate(srcs):
        assert np.array_equal(so[i], small.sssp(s)), i
    assert np.array_equal(outs[0], grids[0].sssp(5)) and np.array_equal(outs[1], grids[1].sssp(7))
    if stretch > 0:
        assert max(lat_short) < lat_long[1], (lat_short, lat_long)
    else:
        assert min(lat_short) > lat_long[1], (lat_short, lat_long)


def test_served_device_and_pinned_outputs(cuda):
    g = gen.rmat(11, 16, True, (1, 100))
    G = g1.Graph.from_gen(g)
    srcs = gen.pick_sources(g, 64)
    dev = torch.empty((64, g.n), dtype=torch.int32, device="cuda")
    pin = torch.empty((64, g.n), dtype=torch.int32).pin_memory()
    with g1.Server() as srv:
        gid = srv.add_graph(G)
        ts = [srv.submit(gid, g1.QUERY_SSSP, int(s), dev[i]) for i, s in enumerate(srcs)]
        ts += [srv.submit(gid, g1.QUERY_BFS, int(s), pin[i]) for i, s in enumerate(srcs)]
        for t in ts:
            srv.wait(t, 60000)
    torch.cuda.synchronize()
    d = dev.cpu().numpy().view(np.uint32)
    p = pin.numpy().view(np.uint32)
    for i in (0, 31, 63):
        assert np.array_equal(d[i], G.sssp(int(srcs[i])))
        assert np.array_equal(p[i], G.bfs(int(srcs[i])))


def test_admission_by_memory_limit(cuda):
    """A memory limit below one 256-slot engine: the engines shrink to fit
    and queries wait for memory; every result is still exact."""
    graphs = serving_graphs()[:2]
    Gs = [g1.Graph.from_gen(g) for g in graphs]
    n_max = max(g.n for g in graphs)
    limit = 4 * n_max * 64 * 4  # room for engines of about 32-64 slots
    reqs = request_mix(graphs, 200, seed=7)
    with g1.Server(max_batch=256, memory_limit=limit, idle_release_ms=1, solo_queue_ms=-1) as srv:
        gids = [srv.add_graph(G) for G in Gs]
        outs = [host_out(graphs[gi], kind) for gi, kind, _ in reqs]
        ts = [srv.submit(gids[gi], kind, src, outs[i]) for i, (gi, kind, src) in enumerate(reqs)]
        for t in ts:
            srv.wait(t, 60000)
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["max_occupancy"] <= 64
    for i, (gi, kind, src) in enumerate(reqs):
        assert same_as_alone(outs[i], Gs[gi], kind, src, batched_only=True), (i, gi, kind, src)


def test_server_rejects_bad_requests(cuda):
    g = GRAPHS["rmat10_sym"]
    G = g1.Graph.from_gen(g)
    gf = gen.rmat(9, 8, False, float_values=True)
    Gf = g1.Graph.from_gen(gf)
    out = np.empty(g.n, np.uint32)
    with g1.Server() as srv:
        gid = srv.add_graph(G)
        fid = srv.add_graph(Gf)
        with pytest.raises(g1.G1Error):
            srv.submit(gid + 5, g1.QUERY_BFS, 0, out)
        with pytest.raises(g1.G1Error):
            srv.submit(gid, g1.QUERY_BFS, g.n, out)
        with pytest.raises(g1.G1Error):
            srv.submit(fid, g1.QUERY_SSSP, 0, out)  # SSSP needs u32 weights
        with pytest.raises(g1.G1Error):
            srv.poll(12345)
        t = srv.submit(gid, g1.QUERY_BFS, 0, out)
        srv.wait(t, 60000)
    assert np.array_equal(out, O.bfs(*g.np("n")[:2], 0))


def test_concurrent_submitters(cuda):
    """Queries from several host threads; results as alone."""
    g = gen.rmat(11, 16, True, (1, 100))
    G = g1.Graph.from_gen(g)
    srcs = gen.pick_sources(g, 96)
    outs = np.empty((96, g.n), np.uint32)
    with g1.Server(max_batch=64) as srv:
        gid = srv.add_graph(G)

        def worker(lo, hi):
            ts = [srv.submit(gid, g1.QUERY_SSSP, int(srcs[i]), outs[i]) for i in range(lo, hi)]
            for t in ts:
                srv.wait(t, 60000)

        th = [threading.Thread(target=worker, args=(i * 24, i * 24 + 24)) for i in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for i in (0, 50, 95):
        assert np.array_equal(outs[i], G.sssp(int(srcs[i])))


@pytest.mark.parametrize("kind", [g1.QUERY_SSSP, g1.QUERY_BFS])
@pytest.mark.parametrize("relabel", [False, True])
def test_served_grid_sssp_runs_on_the_nearfar_engine(cuda, relabel, kind):
    """SSSP and BFS on a grid go to the near-far engine one query at a time;
    the results equal every other engine's, in caller vertex order."""
    g = gen.grid2d(48, 37, (1, 100))
    G = g1.Graph.from_gen(g, relabel=relabel)
    rp, ci, v = g.np("n")
    srcs = [0, 5, 1000, g.n - 1]
    host = [np.empty(g.n, np.uint32) for _ in srcs]
    dev = torch.empty((len(srcs), g.n), dtype=torch.int32, device="cuda")
    with g1.Server() as srv:
        gid = srv.add_graph(G)
        ts = [srv.submit(gid, kind, s, host[i]) for i, s in enumerate(srcs)]
        ts += [srv.submit(gid, kind, s, dev[i]) for i, s in enumerate(srcs)]
        for t in ts:
            srv.wait(t, 60000)
    d = dev.cpu().numpy().view(np.uint32)
    for i, s in enumerate(srcs):
        if kind == g1.QUERY_SSSP:
            ref = O.dijkstra_u32(rp, ci, v, s)
            assert np.array_equal(G.sssp(s, g1.ENGINE_NEARFAR), ref)
        else:
            ref = O.bfs(rp, ci, s)
            assert np.array_equal(G.bfs(s, g1.ENGINE_NEARFAR), ref)
        assert np.array_equal(host[i], ref)
        assert np.array_equal(d[i], ref)
