"""Register budgets the hot kernels' launch shapes rely on (ptxas, no GPU).

- The default nnz SpMV kernel runs one 1024-thread block per SM (the 128 KB
  x cache plus the segment buffers leave room for one), so it must fit 64
  registers per thread, and a spill would sit on its gather path.
- The near-far engine is one cooperative launch of a 1024-thread block per
  SM, so every instantiation must fit 64 registers per thread.
"""
import os
import re
import shutil
import subprocess

import pytest

from graphone_b200 import build as B

pytestmark = pytest.mark.skipif(shutil.which(B._nvcc()) is None and not os.path.exists(B._nvcc()),
                                reason="nvcc not available")


def _ptxas(src, tmp_path):
    cmd = [B._nvcc(), *B.ARCH, *B.FLAGS, "-Xptxas", "-v", "-c",
           os.path.join(B.CSRC, src), "-o", str(tmp_path / "k.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    # {mangled entry name: (registers, spill store bytes)}
    out, name, spill = {}, None, 0
    for line in r.stderr.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            name, spill = m.group(1), 0
            continue
        m = re.search(r"(\d+) bytes spill stores", line)
        if m and name:
            spill = int(m.group(1))
        m = re.search(r"Used (\d+) registers", line)
        if m and name:
            out[name] = (int(m.group(1)), spill)
            name = None
    return out


def test_default_nnz_kernel_fits_64_registers_without_spills(tmp_path):
    k = _ptxas("pagerank.cu", tmp_path)
    # spmv_nnz_kernel<PlusTimesF32, PrEpilogue, 32 warps, 1 block, 32768 hot, no options,
    # L2 prefetch distance 0 (the default), 1, 2 or 4>
    main = [n for n in k if "spmv_nnz_kernel" in n and "PrEpilogue" in n
            and "Li32ELi1ELi32768ELb0ELb0ELb0ELi0ELi" in n]
    assert len(main) == 4, sorted(k)
    for n in main:
        regs, spill = k[n]
        assert regs <= 64 and spill == 0, (n, regs, spill)
    fix = [n for n in k if "spmv_nnz_fixup_kernel" in n and "PrEpilogue" in n]
    assert fix and all(k[n][1] == 0 for n in fix)


def test_near_far_kernels_fit_a_1024_thread_block(tmp_path):
    k = _ptxas("nearfar.cu", tmp_path)
    nf = [n for n in k if "nf_kernel" in n]
    assert len(nf) == 12, sorted(k)  # {SSSP, BFS} x TPV in {1, 2, 4, 8, 16, 32}
    assert all(k[n][0] <= 64 for n in nf), {n: k[n] for n in nf}
