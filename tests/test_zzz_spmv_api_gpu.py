"""GraphOne's SpMV operator API with the CUDA schedules
(blas::SpmvCudaCsrVector, blas::SpmvCudaCsrMergeBased over the caller's
unpadded device arrays) on the shapes of tests/test_spmv_api.py: the integer
folds bit-exact against the row loop, fp32 plus-times within 1e-6 relative
L1 of FP64.  Each run calls the dispatcher twice on one plan.

Collected last (file name) so that a failure here cannot hide the others."""
import zlib

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_spmv_api import CASES, driver, expected_int, make_csr, run  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["vector", "merge"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_cuda_schedules_match_the_row_loop(driver, tmp_path, kind, case):  # noqa: F811
    csr = make_csr(np.random.default_rng(zlib.crc32(case.encode())), **CASES[case])
    y1, y2, y3 = run(driver, tmp_path, kind, csr)
    e1, e3 = expected_int(csr)
    assert np.array_equal(y1, e1)
    assert np.array_equal(y3, e3)
    rp, ci, _, wf, _, xf = csr
    assert O.rel_l1(y2, O.spmv_plustimes_f64(rp, ci, wf, xf)) <= 1e-6
