"""Seeded synthetic graphs with the shapes of the GraphOne workloads.

GraphOne reads ``.adj`` edge lists (loader/graph_loader.h:32-122) and turns
them into CSR with a host counting sort (loader/edge_cache.h:50-105): self
loops dropped (graph_loader.h:256-259), undirected inputs symmetrised
(:281-288), duplicates merged after a sort by (src, dst) (:290-296).  The
generators here produce that final CSR directly, on any torch device, from a
counter-based splitmix64 stream so that every element is a pure function of
(seed, index):

* RMAT (Chakrabarti et al.): sample i, level l draws
  ``r = mix64(seed + (i*scale + l + 1) * GOLDEN) >> 11`` and picks the
  quadrant by comparing r with floor(p * 2**53) of the cumulative a, a+b,
  a+b+c.
* 2-D grids: vertex id r*cols + c, 4-neighbour.
* Weights: an undirected edge {u, v} gets
  ``wlo + ((mix64(wseed + (key + 1) * GOLDEN) >> 11) % (whi - wlo + 1))``
  with key = min*n + max, so w(u, v) == w(v, u); a directed edge uses
  key = src*n + dst.

Rows of both the CSR and its transpose list columns in increasing order,
exactly like EdgeCache::ToCsr on the sorted, deduplicated edge cache.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

GOLDEN = 0x9E3779B97F4A7C15
MIX1 = 0xBF58476D1CE4E5B9
MIX2 = 0x94D049BB133111EB
SEED = 20261203
WEIGHT_SEED_XOR = 0x5EED5EED
SOURCE_SEED_ADD = 1


def _s64(c: int) -> int:
    """Two's-complement int64 view of an unsigned 64-bit constant."""
    c &= (1 << 64) - 1
    return c - (1 << 64) if c >= (1 << 63) else c


def _lsr(x: torch.Tensor, k: int) -> torch.Tensor:
    """Logical right shift of int64 bit patterns."""
    return (x >> k) & ((1 << (64 - k)) - 1)


def mix64(z: torch.Tensor) -> torch.Tensor:
    """splitmix64 finaliser on int64 bit patterns (wrapping arithmetic)."""
    z = (z ^ _lsr(z, 30)) * _s64(MIX1)
    z = (z ^ _lsr(z, 27)) * _s64(MIX2)
    return z ^ _lsr(z, 31)


def rng(seed: int, ctr: torch.Tensor) -> torch.Tensor:
    """ctr-th output of the splitmix64 stream that starts at ``seed``."""
    return mix64((ctr + 1) * _s64(GOLDEN) + _s64(seed))


def rmat_thresholds(a: float, b: float, c: float):
    two53 = float(1 << 53)
    return int(a * two53), int((a + b) * two53), int((a + b + c) * two53)


@dataclass
class CsrGraph:
    """A graph held as CSR (out-edges) and its transpose (in-edges).

    Arrays are torch tensors on ``device``: ``row_ptr``/``t_row_ptr`` int64 of
    n+1 entries, ``col``/``t_col`` int64, ``val``/``t_val`` int64 (integer
    weights) or float32.  ``to_u32()`` gives the uint32 / float32 numpy
    arrays the C ABI takes.
    """

    n: int
    m: int
    row_ptr: torch.Tensor
    col: torch.Tensor
    val: torch.Tensor
    t_row_ptr: torch.Tensor
    t_col: torch.Tensor
    t_val: torch.Tensor
    symmetric: bool
    name: str = ""

    def out_degree(self) -> torch.Tensor:
        return self.row_ptr[1:] - self.row_ptr[:-1]

    def np(self, which: str = "t"):
        """(row_ptr, col, val) as contiguous numpy uint32 (+ float32 values)."""
        rp, ci, v = ((self.t_row_ptr, self.t_col, self.t_val) if which == "t"
                     else (self.row_ptr, self.col, self.val))
        vv = v.cpu().numpy()
        vv = vv.astype(np.float32) if vv.dtype.kind == "f" else vv.astype(np.uint32)
        return (np.ascontiguousarray(rp.cpu().numpy().astype(np.uint32)),
                np.ascontiguousarray(ci.cpu().numpy().astype(np.uint32)),
                np.ascontiguousarray(vv))


def _csr_from_sorted_keys(keys: torch.Tensor, n: int):
    rows = keys // n
    cols = keys - rows * n
    counts = torch.bincount(rows, minlength=n)
    rp = torch.zeros(n + 1, dtype=torch.int64, device=keys.device)
    rp[1:] = torch.cumsum(counts, 0)
    return rp, cols


def _weights(src: torch.Tensor, dst: torch.Tensor, n: int, symmetric: bool,
             wseed: int, wlo: int, whi: int) -> torch.Tensor:
    if symmetric:
        key = torch.minimum(src, dst) * n + torch.maximum(src, dst)
    else:
        key = src * n + dst
    r = _lsr(rng(wseed, key), 11)
    return wlo + torch.remainder(r, whi - wlo + 1)


def from_edges(src: torch.Tensor, dst: torch.Tensor, n: int, symmetric: bool,
               weights: Optional[tuple] = (1, 64), seed: int = SEED,
               float_values: bool = False, name: str = "") -> CsrGraph:
    """Self-loops dropped, symmetrised if asked, deduplicated, both CSRs."""
    src = src.to(torch.int64)
    dst = dst.to(torch.int64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    if symmetric:
        src, dst = torch.cat([src, dst]), torch.cat([dst, src])
    keys = torch.unique(src * n + dst)          # sorted by (src, dst)
    rp, cols = _csr_from_sorted_keys(keys, n)
    rows = keys // n
    tkeys = torch.sort(cols * n + rows).values  # sorted by (dst, src)
    trp, tcols = _csr_from_sorted_keys(tkeys, n)
    trows = tkeys // n
    m = int(keys.numel())
    if float_values:
        val = torch.ones(m, dtype=torch.float32, device=keys.device)
        tval = torch.ones(m, dtype=torch.float32, device=keys.device)
    else:
        wseed = seed ^ WEIGHT_SEED_XOR
        wlo, whi = weights
        val = _weights(rows, cols, n, symmetric, wseed, wlo, whi)
        tval = _weights(tcols, trows, n, symmetric, wseed, wlo, whi)
    return CsrGraph(n, m, rp, cols, val, trp, tcols, tval, symmetric, name)


def rmat_samples(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19,
                 seed: int = SEED, device="cpu", chunk: int = 1 << 24):
    """Raw RMAT (src, dst) samples, int64 tensors of edge_factor * 2**scale."""
    tA, tAB, tABC = rmat_thresholds(a, b, c)
    ns = edge_factor << scale
    src = torch.empty(ns, dtype=torch.int64, device=device)
    dst = torch.empty(ns, dtype=torch.int64, device=device)
    for lo in range(0, ns, chunk):
        hi = min(ns, lo + chunk)
        i = torch.arange(lo, hi, dtype=torch.int64, device=device)
        s = torch.zeros_like(i)
        d = torch.zeros_like(i)
        for lvl in range(scale):
            r = _lsr(rng(seed, i * scale + lvl), 11)
            rb = (r >= tAB).to(torch.int64)
            cb = ((r >= tA) & (r < tAB)).to(torch.int64) | (r >= tABC).to(torch.int64)
            s = (s << 1) | rb
            d = (d << 1) | cb
        src[lo:hi] = s
        dst[lo:hi] = d
    return src, dst


def rmat(scale: int, edge_factor: int = 16, symmetric: bool = True,
         weights=(1, 64), seed: int = SEED, float_values: bool = False,
         device="cpu") -> CsrGraph:
    src, dst = rmat_samples(scale, edge_factor, seed=seed, device=device)
    g = from_edges(src, dst, 1 << scale, symmetric, weights, seed, float_values,
                   name=f"rmat{scale}{'s' if symmetric else 'd'}")
    return g


def grid2d(rows: int, cols: int, weights=(1, 100), seed: int = SEED,
           device="cpu") -> CsrGraph:
    n = rows * cols
    v = torch.arange(n, dtype=torch.int64, device=device)
    r, c = v // cols, v % cols
    right = c + 1 < cols
    down = r + 1 < rows
    src = torch.cat([v[right], v[down]])
    dst = torch.cat([v[right] + 1, v[down] + cols])
    return from_edges(src, dst, n, True, weights, seed, name=f"grid{rows}x{cols}")


def pick_sources(g: CsrGraph, k: int, seed: int = SEED) -> np.ndarray:
    """k distinct vertices with out-degree > 0, ordered by a seeded hash."""
    deg = g.out_degree()
    cand = torch.nonzero(deg > 0).flatten()
    h = _lsr(rng(seed + SOURCE_SEED_ADD, cand), 11)
    order = torch.argsort(h, stable=True)
    return cand[order[:k]].cpu().numpy().astype(np.uint32)


def write_adj(g: CsrGraph, path: str, directed: bool) -> None:
    """Writes the graph as a GraphOne ``.adj`` edge list (src dst w per line).

    For an undirected graph only the u < v half is written; GraphOne's loader
    symmetrises it again (graph_loader.h:281-288).
    """
    rp, ci, v = g.np("n")
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(rp.astype(np.int64)))
    if not directed:
        keep = src < ci
        src, ci, v = src[keep], ci[keep], v[keep]
    import pandas as pd  # vectorised text output (tens of millions of lines)
    with open(path, "w") as f:
        f.write("% generated\n")
    df = pd.DataFrame({"s": src, "d": ci, "w": v})
    df.to_csv(path, mode="a", sep=" ", header=False, index=False,
              float_format="%g" if v.dtype.kind == "f" else None, lineterminator="\n")
