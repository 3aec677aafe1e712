"""GraphOne's unchanged apps built on these headers (oracle/_ref/apps_g1)
and on GraphOne's own (oracle/_ref/apps_ref) end with the same exit status
on command lines that fail to parse, or ask for --help: both stop in
CLI11_PARSE, before any CUDA call, so this runs on the CPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G1 = os.path.join(ROOT, "oracle", "_ref", "apps_g1")
REF = os.path.join(ROOT, "oracle", "_ref", "apps_ref")

pytestmark = pytest.mark.skipif(not (os.path.isdir(G1) and os.path.isdir(REF)), reason="apps not built")

ARGV = [["-h"], ["--help"], [], ["--src", "1"], ["-i", "g.adj", "--src"], ["-i", "g.adj", "--src", "x"],
        ["-i", "g.adj", "--src", "-1"], ["-i", "g.adj", "--src", "1", "--src", "2"], ["-i", "g.adj", "--src", "1", "--bogus"],
        ["-i", "g.adj", "--src", "1", "extra"], ["-i", "g.adj", "--src", "1", "--is_directed=maybe"], ["-i"]]


@pytest.mark.parametrize("app", ["sssp_blas", "sssp_adv", "sssp_blas2"])
@pytest.mark.parametrize("argv", ARGV, ids=lambda a: " ".join(a) or "none")
def test_same_exit_status_as_graphone(tmp_path, app, argv):
    codes = []
    for d in (G1, REF):
        r = subprocess.run([os.path.join(d, app), *argv], cwd=tmp_path, capture_output=True, timeout=60)
        codes.append(r.returncode)
    assert codes[0] == codes[1], codes
    assert codes[0] in (0, 104, 106, 109, 114)
