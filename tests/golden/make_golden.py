"""Generates tests/golden/*.npz from GraphOne's own host code.

Run here, where the reference tree is present (it is not on GPU machines):

    make -C oracle ref && python tests/golden/make_golden.py

For each small synthetic graph it writes the graph as a GraphOne ``.adj``
file, loads it back with the reference's GraphLoader + EdgeCache::ToCsr
(oracle/_ref/libgraphone_ref.so, compiled from the reference sources), and
records:
  * the CSR and transpose CSR exactly as the reference builds them,
  * min-plus and plus-times SpMV results of the reference's SpMV_cpu_navie
    on seeded x vectors,
  * SSSP distances of the sparse-frontier BLAS engine loop around
    SpMV_cpu_navie and PageRank ranks (fp32, 30 iterations, both modes) of
    the all-active engine loop around it.
The fixtures pin the oracle (tests/test_oracle.py) and the CUDA path
(tests/test_gpu_*.py) without the reference tree.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import ctypes as C  # noqa: E402

from graphone_b200 import gen  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_csr(path, directed):
    R = O.ref()
    n = C.c_uint32()
    m = C.c_uint64()
    assert R.ref_load_adj(path.encode(), int(directed), C.byref(n), C.byref(m)) == 0
    n, m = n.value, m.value
    out = {}
    for t, tag in ((0, "n"), (1, "t")):
        rp = np.empty(n + 1, np.uint32)
        ci = np.empty(m, np.uint32)
        v = np.empty(m, np.uint32)
        assert R.ref_to_csr(t, _p(rp), _p(ci), _p(v)) == 0
        out[f"{tag}_rp"], out[f"{tag}_col"], out[f"{tag}_val"] = rp, ci, v
    return n, m, out


def make(name, g, directed, float_values=False):
    R = O.ref()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, name + ".adj")
        gen.write_adj(g, path, directed)
        n, m, arrs = ref_csr(path, directed)
    rec = dict(arrs)
    rec["n"] = np.array(n)
    rec["m"] = np.array(m)
    rng = np.random.default_rng(7)
    rp, ci, v = arrs["t_rp"], arrs["t_col"], arrs["t_val"]
    # min-plus SpMV on a sparse "frontier" x
    x = np.full(n, O.U32_MAX, np.uint32)
    sel = rng.choice(n, size=max(1, n // 8), replace=False)
    x[sel] = rng.integers(0, 1000, size=len(sel), dtype=np.uint32)
    y = np.empty(n, np.uint32)
    R.ref_spmv_minplus_u32(n, _p(rp), _p(ci), _p(v), _p(x), _p(y), 1)
    rec["spmv_mp_x"], rec["spmv_mp_y"] = x, y
    # plus-times SpMV (values as float)
    vf = v.astype(np.float32)
    xf = rng.random(n, dtype=np.float32)
    yf = np.empty(n, np.float32)
    R.ref_spmv_plustimes_f32(n, _p(rp), _p(ci), _p(vf), _p(xf), _p(yf), 1)
    rec["spmv_pt_x"], rec["spmv_pt_y"] = xf, yf
    if not float_values:
        dist = np.empty(n, np.uint32)
        src = int(np.argmax(np.diff(arrs["n_rp"].astype(np.int64)) > 0))
        iters = R.ref_sssp_blas_u32(n, _p(rp), _p(ci), _p(v), src, _p(dist), 1, 0)
        rec["sssp_src"], rec["sssp_dist"], rec["sssp_iters"] = np.array(src), dist, np.array(iters)
    else:
        outw = np.zeros(n, np.float32)
        nrp = arrs["n_rp"]
        for u in range(n):
            s = np.float32(0)
            for k in range(nrp[u], nrp[u + 1]):
                s = np.float32(s + np.float32(arrs["n_val"][k]))
            outw[u] = s
        for mode in (0, 1):
            r = np.empty(n, np.float32)
            R.ref_pagerank_f32(n, _p(rp), _p(ci), _p(vf), _p(outw), C.c_float(0.85), 30, mode,
                               _p(r), 1)
            rec[f"pr{mode}_rank"] = r
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    print(name, n, m)


def main():
    O.build(ref=True)
    assert O.ref() is not None, "oracle/_ref was not built"
    make("rmat8_sym", gen.rmat(8, 16, True, (1, 64)), directed=False)
    make("rmat9_dir", gen.rmat(9, 16, False, (1, 64)), directed=True)
    make("grid16", gen.grid2d(16, 16, (1, 100)), directed=False)
    make("rmat8_pr", gen.rmat(8, 16, False, float_values=True), directed=True, float_values=True)


if __name__ == "__main__":
    main()
