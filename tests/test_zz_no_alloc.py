"""g1_spmv_noalloc: the SpMV entry point for callers that cannot call
cudaMalloc (processes whose device memory comes only from their own arena or
caching pool, plugins inside such hosts, loops that cannot take cudaMalloc's
implicit synchronisation).  It keeps its scratch in one static device array
instead of graph-owned buffers; its results must equal those of g1_spmv on the
same inputs, and the oracle's, call after call, for every semiring.

Graphs: small edge cases (a hub row spanning many tiles with many empty rows,
a grid), RMAT-18 symmetrised (about 35k warp tiles, more than one resident
wave, so the tile kernel's grid-stride loop runs), and a 3400 x 3400 grid
whose n + m (57.8M) sits just under the scratch limit of 58,720,256.

Collected last (file name) so that a failure here cannot hide the others; it
must pass alone in a fresh process as well as after the other tests."""
import numpy as np
import pytest
import torch

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SEMIRINGS = [g1.SR_MINPLUS_U32, g1.SR_MINPLUS_F32, g1.SR_PLUSTIMES_F32, g1.SR_BFS_U32]
F32_MAX = np.finfo(np.float32).max


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


def _graph(name):
    if name == "rmat12_sym":
        return gen.rmat(12, 16, True, (1, 64), device="cuda")
    if name == "star":  # one row spanning many tiles, many empty rows
        n = 30000
        src = torch.cat([torch.zeros(n - 1, dtype=torch.int64), torch.arange(1, 40)])
        dst = torch.cat([torch.arange(1, n), torch.zeros(39, dtype=torch.int64)])
        return gen.from_edges(src.cuda(), dst.cuda(), n, False, (1, 64))
    if name == "grid61x67":
        return gen.grid2d(61, 67, (1, 100), device="cuda")
    if name == "rmat18_sym":
        return gen.rmat(18, 16, True, (1, 64), device="cuda")
    if name == "grid3400":
        return gen.grid2d(3400, 3400, (1, 100), device="cuda")
    raise KeyError(name)


def _inputs(sr, n, vals, rng):
    """x for the semiring (about 40% of entries reached) and the edge values
    in the semiring's type."""
    sel = rng.random(n) < 0.4
    if sr in (g1.SR_MINPLUS_U32, g1.SR_BFS_U32):
        x = np.full(n, O.U32_MAX, np.uint32)
        x[sel] = rng.integers(0, 1 << 20, size=int(sel.sum()), dtype=np.uint32)
        return x, vals.astype(np.uint32)
    if sr == g1.SR_MINPLUS_F32:
        x = np.full(n, F32_MAX, np.float32)
        x[sel] = rng.integers(0, 1 << 20, size=int(sel.sum())).astype(np.float32)
        return x, vals.astype(np.float32)
    return rng.random(n).astype(np.float32), vals.astype(np.float32)


def _oracle(sr, rp, ci, v, x):
    if sr == g1.SR_MINPLUS_U32:
        return O.spmv_minplus_u32(rp, ci, v, x)
    if sr == g1.SR_BFS_U32:
        return O.spmv_minplus_u32(rp, ci, np.ones(len(ci), np.uint32), x)
    if sr == g1.SR_PLUSTIMES_F32:
        return O.spmv_plustimes_f64(rp, ci, v, x)
    return None  # min-plus over fp32: checked bit for bit against g1_spmv


@pytest.mark.parametrize("name", ["rmat12_sym", "star", "grid61x67", "rmat18_sym", "grid3400"])
def test_noalloc_matches_g1_spmv_and_oracle_twice(cuda, name):
    g = _graph(name)
    rp, ci, v = g.np("t")
    del g
    assert len(rp) - 1 + len(ci) <= 58_720_256
    d_rp, d_ci = _dev(rp, np.int32), _dev(ci, np.int32)
    L = g1.lib()
    rng = np.random.default_rng(len(ci))
    n, m = len(rp) - 1, len(ci)
    for sr in SEMIRINGS:
        x0, vv = _inputs(sr, n, v, rng)
        G = g1.Graph.from_csr(rp, ci, vv, input_transpose=True, build_other=False)
        # the caller's own device CSR: exact sizes, no padding
        d_v = _dev(vv, np.int32)
        for call in range(2):  # two calls in a row share (and rewrite) the scratch
            x = x0 if call == 0 else _inputs(sr, n, v, rng)[0]
            xd = _dev(x, np.int32)
            y_ref = torch.empty(n, dtype=torch.int32, device="cuda")
            y_na = torch.full((n,), 7, dtype=torch.int32, device="cuda")
            G.spmv(xd, y_ref, sr, transpose=1)
            g1.check(L.g1_spmv_noalloc(d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), n, m,
                                       sr, xd.data_ptr(), y_na.data_ptr(), None))
            torch.cuda.synchronize()
            got = y_na.cpu().numpy()
            ref = y_ref.cpu().numpy()
            orc = _oracle(sr, rp, ci, vv, x)
            if sr == g1.SR_PLUSTIMES_F32:
                # fp32 accumulation: relative L1 within 1e-6, the SpMV tests' tolerance
                assert O.rel_l1(got.view(np.float32), ref.view(np.float32)) < 1e-6, (name, sr, call)
                assert O.rel_l1(got.view(np.float32), orc) < 1e-6, (name, sr, call)
            else:
                # min-plus: every candidate is exact and min is order-free: bit-exact
                assert np.array_equal(got, ref), (name, sr, call)
                if orc is not None:
                    assert np.array_equal(got.view(np.uint32), orc), (name, sr, call)
        G.close()


def test_noalloc_rejects_sizes_beyond_scratch(cuda):
    L = g1.lib()
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    st = L.g1_spmv_noalloc(p, p, p, 40_000_000, 40_000_000, g1.SR_MINPLUS_U32, p, p, None)
    assert st == 1
    assert b"scratch limit" in L.g1_last_error()
    # one merge item over the limit is rejected too
    st = L.g1_spmv_noalloc(p, p, p, 1, 58_720_256, g1.SR_MINPLUS_U32, p, p, None)
    assert st == 1
