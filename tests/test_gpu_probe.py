"""g1_measure_gather_rate: the random-load probe behind the SpMV's second
roofline.  Rates are positive, ordered by where the buffer lives (L1 above
L2 above HBM), and bad arguments are refused before any device work."""
import pytest

import graphone_b200 as g1

pytestmark = pytest.mark.gpu


def test_gather_rates_are_ordered_by_memory_level(cuda):
    l1 = g1.measure_gather_rate(4, 8, 1, 1 << 16)
    l2 = g1.measure_gather_rate(4, 8, 1, 1 << 24)
    hbm = g1.measure_gather_rate(4, 8, 1, 1 << 30)
    assert l1 > l2 > hbm > 0
    assert g1.measure_gather_rate(16, 4, 2, 1 << 24) > 0


@pytest.mark.parametrize("args", [(8, 8, 1, 1 << 24), (4, 3, 1, 1 << 24), (4, 8, 3, 1 << 24),
                                  (4, 8, 1, 1000), (4, 8, 1, 1 << 12)])
def test_gather_rate_rejects_bad_arguments(cuda, args):
    with pytest.raises(g1.G1Error):
        g1.measure_gather_rate(*args)


def test_smem_gather_rates(cuda):
    """g1_measure_smem_gather_rate: gathers from a block's own shared memory
    outrun L2; distributed shared memory (another block of the cluster) is
    measured for clusters of 2 and 16 blocks."""
    own, blocks = g1.measure_smem_gather_rate(1, False)
    l2 = g1.measure_gather_rate(4, 8, 1, 1 << 24)
    assert own > l2 > 0 and blocks > 0
    for cl in (2, 16):
        r, b = g1.measure_smem_gather_rate(cl, True)
        assert r > 0 and b > 0 and b % cl == 0


@pytest.mark.parametrize("cluster", [0, 3, 32])
def test_smem_gather_rate_rejects_bad_cluster_sizes(cuda, cluster):
    with pytest.raises(g1.G1Error):
        g1.measure_smem_gather_rate(cluster, True)
