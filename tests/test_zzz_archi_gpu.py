"""GraphOne's archi:: primitives with arch_t::cuda (device arrays from
archi::memalloc): the same checks as tests/test_archi.py on the host.

Collected last (file name) so that a failure here cannot hide the others."""
import pytest

from tests.test_archi import archi_driver, check_archi, inputs, run_archi  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 257, 5000, 300000])
def test_archi_primitives_on_the_gpu(archi_driver, tmp_path, n):  # noqa: F811
    arrs = inputs(n, n)
    check_archi(arrs, *run_archi(archi_driver, tmp_path, "cuda", arrs))
