"""Result files of GraphOne's apps and a comparator for them.

GraphOne's apps write their result as text (apps/sssp_blas.cu:123-134,
apps/sssp_adv.cu:111-122, apps/pagerank_blas.cu:163-174):

    Elapsed time: <ms> ms
    <vid>-<value>          one line per vertex, value printed with "%f"

SSSP distances are floats there (unreachable = FLT_MAX, printed as
340282346638528859811704183484516925440.000000); PageRank ranks are floats.
This module reads and writes that format and compares two result files (or a
result file and an array) the way the parity tests do: distances bit for bit
after rounding to float32 (every distance below 2^24 is an exact float), ranks
within a relative L1 tolerance.

    python -m graphone_b200.results compare ours.txt theirs.txt [--kind sssp|pagerank]
                                            [--tol 1e-6] [--limit N]

exits 0 when the files agree, 1 when they differ (the first differences are
printed), 2 when a file cannot be read.
"""
from __future__ import annotations

import argparse
import sys
from dataclasses import dataclass
from typing import Optional

import numpy as np

FLT_MAX = float(np.finfo(np.float32).max)
U32_MAX = 0xFFFFFFFF


@dataclass
class AppResult:
    elapsed_ms: Optional[float]
    values: np.ndarray  # float64, indexed by vertex id


def read_result(path: str) -> AppResult:
    """Parses an app result file.  Vertex ids may come in any order; a
    missing id reads as NaN."""
    elapsed = None
    ids, vals = [], []
    with open(path) as f:
        for ln, line in enumerate(f, 1):
            line = line.strip()
            if not line:
                continue
            if line.startswith("Elapsed time:"):
                tok = line[len("Elapsed time:"):].split()
                elapsed = float(tok[0]) if tok else None
                continue
            vid, sep, val = line.partition("-")
            if not sep:
                raise ValueError(f"{path}:{ln}: expected '<vid>-<value>', got {line!r}")
            ids.append(int(vid))
            vals.append(float(val))
    n = (max(ids) + 1) if ids else 0
    out = np.full(n, np.nan, np.float64)
    out[np.asarray(ids, dtype=np.int64)] = np.asarray(vals, dtype=np.float64)
    return AppResult(elapsed, out)


def write_result(path: str, values, elapsed_ms: Optional[float] = None) -> None:
    """Writes values in the apps' format.  uint32 distances are written as the
    apps' float distances (UINT32_MAX -> FLT_MAX)."""
    v = np.asarray(values)
    if v.dtype == np.uint32:
        f = v.astype(np.float64)
        f[v == U32_MAX] = FLT_MAX
        v = f
    v = v.astype(np.float32)
    with open(path, "w") as fh:
        fh.write(f"Elapsed time: {int(round(elapsed_ms or 0))} ms\n")
        fh.writelines(f"{i}-{x:f}\n" for i, x in enumerate(v.tolist()))


def as_app_values(values) -> np.ndarray:
    """An array as the apps would print it: float32, unreachable = FLT_MAX."""
    v = np.asarray(values)
    if v.dtype == np.uint32:
        f = v.astype(np.float64)
        f[v == U32_MAX] = FLT_MAX
        return f.astype(np.float32).astype(np.float64)
    return v.astype(np.float32).astype(np.float64)


@dataclass
class Comparison:
    same: bool
    n_compared: int
    n_different: int
    rel_l1: float
    first_differences: list  # (vid, a, b)
    size_a: int
    size_b: int


def compare(a, b, kind: str = "sssp", tol: float = 1e-6, limit: Optional[int] = None) -> Comparison:
    """Compares two results (AppResult, or arrays in vertex order).

    kind "sssp" (also BFS levels): float32 values must be identical.
    kind "pagerank": relative L1 of a against b within `tol`.
    Only the first `limit` vertices are compared when given; otherwise both
    must have the same length (GraphOne's loader drops trailing isolated
    vertices, so compare with limit = its vertex count when that applies)."""
    va = a.values if isinstance(a, AppResult) else as_app_values(a)
    vb = b.values if isinstance(b, AppResult) else as_app_values(b)
    size_a, size_b = len(va), len(vb)
    if limit is not None:
        va, vb = va[:limit], vb[:limit]
    elif size_a != size_b:
        return Comparison(False, 0, abs(size_a - size_b), float("inf"), [], size_a, size_b)
    if len(va) != len(vb):
        return Comparison(False, 0, abs(len(va) - len(vb)), float("inf"), [], size_a, size_b)
    fa, fb = va.astype(np.float32), vb.astype(np.float32)
    diff = ~((fa == fb) | (np.isnan(fa) & np.isnan(fb)))
    den = np.abs(vb).sum()
    rel = float(np.abs(va - vb).sum() / den) if den > 0 else (0.0 if not diff.any() else float("inf"))
    idx = np.nonzero(diff)[0][:10]
    first = [(int(i), float(va[i]), float(vb[i])) for i in idx]
    if kind == "pagerank":
        same = bool(rel <= tol) and not np.isnan(va).any() and not np.isnan(vb).any()
    elif kind == "sssp":
        same = not bool(diff.any())
    else:
        raise ValueError(f"unknown kind {kind!r}")
    return Comparison(same, len(va), int(diff.sum()), rel, first, size_a, size_b)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m graphone_b200.results")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("compare", help="compare two app result files")
    c.add_argument("a")
    c.add_argument("b")
    c.add_argument("--kind", choices=["sssp", "pagerank"], default="sssp")
    c.add_argument("--tol", type=float, default=1e-6, help="relative L1 tolerance (pagerank)")
    c.add_argument("--limit", type=int, default=None, help="compare the first N vertices only")
    args = ap.parse_args(argv)
    try:
        ra, rb = read_result(args.a), read_result(args.b)
    except (OSError, ValueError) as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    r = compare(ra, rb, args.kind, args.tol, args.limit)
    print(f"{args.kind}: {r.n_compared} vertices compared ({r.size_a} vs {r.size_b}), "
          f"{r.n_different} differ, relative L1 {r.rel_l1:.3g}, elapsed {ra.elapsed_ms} vs {rb.elapsed_ms} ms")
    for vid, x, y in r.first_differences:
        print(f"  vertex {vid}: {x!r} vs {y!r}")
    print("same" if r.same else "DIFFERENT")
    return 0 if r.same else 1


if __name__ == "__main__":
    sys.exit(main())
