"""Shared helpers of the GPU parity tests."""
import numpy as np
import torch

import graphone_b200 as g1
from graphone_b200 import gen


def edge_case_graphs():
    """Small graphs with the shapes the reference's loader can produce plus
    the corner cases of the merge-path split."""
    out = {}
    out["rmat10_sym"] = gen.rmat(10, 16, True, (1, 64))
    out["rmat11_dir"] = gen.rmat(11, 8, False, (1, 64))
    out["grid32"] = gen.grid2d(32, 32, (1, 100))
    out["grid7x13"] = gen.grid2d(7, 13, (1, 100))
    # one hub row spanning many merge tiles + many empty rows
    n = 20000
    src = torch.cat([torch.zeros(n - 1, dtype=torch.int64), torch.arange(1, 50)])
    dst = torch.cat([torch.arange(1, n), torch.zeros(49, dtype=torch.int64)])
    out["star20k"] = gen.from_edges(src, dst, n, False, (1, 64), name="star20k")
    # isolated vertices only
    out["empty5"] = gen.from_edges(torch.zeros(0, dtype=torch.int64),
                                   torch.zeros(0, dtype=torch.int64), 5, True, (1, 64),
                                   name="empty5")
    # single vertex
    out["single"] = gen.from_edges(torch.zeros(0, dtype=torch.int64),
                                   torch.zeros(0, dtype=torch.int64), 1, True, (1, 64),
                                   name="single")
    # path graph: long chain (many iterations)
    n = 3000
    a = torch.arange(0, n - 1)
    out["path3000"] = gen.from_edges(a, a + 1, n, True, (1, 64), name="path3000")
    return out


def device_graph(g):
    return g1.Graph.from_gen(g)


def to_dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()
