"""Host-side pieces of bench.py that need no GPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_summary_is_read_for_the_captured_variant_only():
    import graphone_b200 as g1
    t = bench.measured_traffic(g1.DEFAULT_MERGE_VARIANT)
    alg = bench.spmv_bytes(4194304, 65245678)
    assert alg == 572297076
    # the committed capture: within a few percent of the algorithmic bytes
    assert t is not None and 1.0 <= t / alg < 1.05
    assert bench.measured_traffic(g1.DEFAULT_MERGE_VARIANT + 1) is None
    assert bench.measured_traffic(-1) is None


def test_traffic_summary_missing_or_malformed(tmp_path):
    assert bench.measured_traffic(17, str(tmp_path / "absent.txt")) is None
    p = tmp_path / "s.txt"
    p.write_text("variant: 17\n")
    assert bench.measured_traffic(17, str(p)) is None
    p.write_text("variant: 17\ndram_bytes_per_launch: 123\n")
    assert bench.measured_traffic(17, str(p)) == 123
