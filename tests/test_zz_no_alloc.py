"""g1_spmv_noalloc: the SpMV entry point for callers that cannot call
cudaMalloc (processes whose device memory comes only from their own arena or
caching pool, plugins inside such hosts, loops that cannot take cudaMalloc's
implicit synchronisation).  It keeps its scratch in one static device array
instead of graph-owned buffers; its results must equal those of g1_spmv on the
same inputs, call after call.

Collected last (file name) so that a failure here cannot hide the others; it
must pass alone in a fresh process as well as after the other tests."""
import ctypes as C

import numpy as np
import pytest
import torch

import graphone_b200 as g1
from graphone_b200 import gen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


@pytest.mark.parametrize("name", ["rmat12_sym", "star", "grid"])
def test_noalloc_matches_g1_spmv_twice(cuda, name):
    if name == "rmat12_sym":
        g = gen.rmat(12, 16, True, (1, 64))
    elif name == "star":  # one row spanning many tiles, many empty rows
        n = 30000
        src = torch.cat([torch.zeros(n - 1, dtype=torch.int64), torch.arange(1, 40)])
        dst = torch.cat([torch.arange(1, n), torch.zeros(39, dtype=torch.int64)])
        g = gen.from_edges(src, dst, n, False, (1, 64))
    else:
        g = gen.grid2d(61, 67, (1, 100))
    rp, ci, v = g.np("t")
    G = g1.Graph.from_csr(rp, ci, v, input_transpose=True, build_other=False)
    # the caller's own device CSR: exact sizes, no padding
    d_rp, d_ci, d_v = _dev(rp, np.int32), _dev(ci, np.int32), _dev(v, np.int32)
    L = g1.lib()
    rng = np.random.default_rng(1)
    for call in range(2):  # two calls in a row share (and rewrite) the scratch
        x = np.full(g.n, O.U32_MAX, np.uint32)
        sel = rng.random(g.n) < 0.4
        x[sel] = rng.integers(0, 1 << 20, size=int(sel.sum()), dtype=np.uint32)
        xd = _dev(x, np.int32)
        y_ref = torch.empty(g.n, dtype=torch.int32, device="cuda")
        y_na = torch.full((g.n,), 7, dtype=torch.int32, device="cuda")
        G.spmv(xd, y_ref, g1.SR_MINPLUS_U32, transpose=1)
        g1.check(L.g1_spmv_noalloc(d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), g.n, g.m,
                                   g1.SR_MINPLUS_U32, xd.data_ptr(), y_na.data_ptr(), None))
        torch.cuda.synchronize()
        assert torch.equal(y_na, y_ref), (name, call)
        # plus-times in fp32: same tolerance as the other SpMV tests
        vf = v.astype(np.float32)
        Gf = g1.Graph.from_csr(rp, ci, vf, input_transpose=True, build_other=False)
        d_vf = _dev(vf, np.float32)
        xf = torch.from_numpy(rng.random(g.n).astype(np.float32)).cuda()
        yf_ref = torch.empty(g.n, dtype=torch.float32, device="cuda")
        yf_na = torch.empty(g.n, dtype=torch.float32, device="cuda")
        Gf.spmv(xf, yf_ref, g1.SR_PLUSTIMES_F32, transpose=1)
        g1.check(L.g1_spmv_noalloc(d_rp.data_ptr(), d_ci.data_ptr(), d_vf.data_ptr(), g.n, g.m,
                                   g1.SR_PLUSTIMES_F32, xf.data_ptr(), yf_na.data_ptr(), None))
        torch.cuda.synchronize()
        assert O.rel_l1(yf_na.cpu().numpy(), yf_ref.cpu().numpy()) < 1e-6, (name, call)


def test_noalloc_rejects_sizes_beyond_scratch(cuda):
    L = g1.lib()
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    st = L.g1_spmv_noalloc(p, p, p, 40_000_000, 40_000_000, g1.SR_MINPLUS_U32, p, p, None)
    assert st == 1
    assert b"scratch limit" in L.g1_last_error()
