"""The apps' command-line parser (include/GraphOne/utils/cli.hpp) against
GraphOne's own utils/cli.hpp on its vendored CLI11 (oracle/_ref/cli_ref,
when built): the same driver (oracle/cli_driver.cpp) is compiled against
both and run on the same argument vectors; exit code and parsed values must
agree.  Expected results for the common forms are also written out, so the
parser is checked where oracle/_ref is absent.  CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "cli_ref")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")

BASE = ["-i", "g.adj", "--src", "3"]


def cases():
    c = [BASE,
         ["--input_graph=g.adj", "--src=3", "-d", "-r", "--keep_self", "--keep_dup", "-o", "out.txt"],
         ["--src", "3"], ["-i", "g.adj"], BASE + ["--foo"], ["-i", "g.adj", "--src"],
         ["-i", "g.adj", "--src", "abc"], BASE + ["--alpha", "0.9"], ["-h"], ["--help"], BASE + ["-dr"],
         ["-i", "g.adj", "--src", "-1"], ["-i", "g.adj", "--src", "1", "--src", "2"], ["-ig.adj", "--src", "3"],
         BASE + ["--line_sep", ","], BASE + ["extra"],
         ["--src", "3", "-i", "g.adj", "--comment_prefix", "#", "--file_ext", ".txt"],
         BASE + ["-d", "-d"], BASE + ["--", "x"], BASE + ["-o"], ["-i", "", "--src", "3"],
         ["-i", "a", "-i", "b", "--src", "3"], BASE + ["--alpha=0.5"], BASE + ["-r", "--reorder"],
         BASE + ["--src=4"], ["-i", "g.adj", "--src=", "3"], ["-d=false"] + BASE, ["-i", "-d", "--src", "3"],
         ["-i", "g.adj", "--src", "--alpha", "0.5"], BASE + ["-o", "-x"], BASE + ["--output", "--src"],
         ["-i", "g.adj", "--", "--src", "3"], ["-dri", "g.adj", "--src", "3"],
         ["-rdo", "out.txt", "-i", "g.adj", "--src", "3"], ["--src", "abc", "-h"], ["-h", "--foo"], ["-dh"],
         ["--foo", "--src", "abc"], ["--foo"], [], ["-"], ["-1"], ["--src", "3", "-i"],
         BASE + ["--alpha", "1", "--alpha", "2"], BASE + ["--is_directed=1", "--is_directed=0"],
         BASE + ["--keep_self=no", "-d"], ["-i=g.adj", "--src", "3"], ["--i", "g.adj", "--src", "3"],
         BASE + ["--line_sep="], BASE + ["--line_sep=", "x"]]
    for v in ["1", "0", "yes", "no", "on", "off", "TRUE", "abc", "2", "-1", "", "t", "f", "enable",
              "disabled", "+", "-", "y", "n", "disable", "enabled", "2.5", "0x1", "Yes", "OFF", "00",
              "-0", "+1", " 1", "1 "]:
        c.append(BASE + ["--is_directed=" + v])
    for v in ["0b101", "0o17", "0B11", "0X1F", "010", "00", " 3", "3 ", "+3", "0x", "0x10", "1e3", "-0",
              "3.5", "3abc", "4294967295", "4294967296", "99999999999999999999999", "0b", "0b2", "+0x10",
              "0b-1", "+ 3", "", "0x-1", "08", "0b1111111111111111111111111111111111"]:
        c.append(["-i", "g.adj", "--src", v])
    for v in [" 0.5", "0.5 ", "inf", "0x1p-2", "1e99", "-0.5", "1,5", "nan", "-1e99", ".5", "5.", "1e-50",
              "abc", "", "1e-1", "0.5x"]:
        c.append(BASE + ["--alpha", v])
    return c


def is_help(argv):
    return any(a in ("-h", "--help", "-dh") for a in argv)


@pytest.fixture(scope="module")
def ours(tmp_path_factory):
    exe = tmp_path_factory.mktemp("cli") / "cli_ours"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                        "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "oracle", "cli_driver.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


def run(exe, argv):
    r = subprocess.run([exe, *argv], capture_output=True, text=True, timeout=30)
    vals = dict(ln.split("=", 1) for ln in r.stdout.splitlines() if "=" in ln) if r.returncode == 0 else {}
    return r.returncode, r.stdout, vals


# (argv, exit code, {value: expected}) of the forms users type
EXPECTED = [
    (BASE, 0, {"input": "g.adj", "src": "3", "directed": "0", "reorder": "0", "alpha": "0.850000024"}),
    (["--input_graph=g.adj", "--src=3", "-d", "-r", "--keep_self", "--keep_dup", "-o", "out.txt"], 0,
     {"directed": "1", "reorder": "1", "keep_self": "1", "keep_dup": "1", "output": "out.txt"}),
    (BASE + ["-dr"], 0, {"directed": "1", "reorder": "1"}),
    (["-ig.adj", "--src", "3"], 0, {"input": "g.adj"}),
    (["-rdo", "out.txt", "-i", "g.adj", "--src", "3"], 0, {"output": "out.txt", "directed": "1"}),
    (BASE + ["--is_directed=false"], 0, {"directed": "0"}),
    (BASE + ["--keep_dup=0"], 0, {"keep_dup": "0"}),
    (BASE + ["--is_directed=yes"], 0, {"directed": "1"}),
    (BASE + ["--alpha", "0.9"], 0, {"alpha": "0.899999976"}),
    (["-i", "g.adj", "--src", "0x10"], 0, {"src": "16"}),
    (["-i", "g.adj", "--src", "010"], 0, {"src": "8"}),
    (["-i", "g.adj", "--src", "0b101"], 0, {"src": "5"}),
    (["-i", "g.adj", "--src", "4294967295"], 0, {"src": "4294967295"}),
    (["-i", "-d", "--src", "3"], 0, {"input": "-d", "directed": "0"}),
    (["-h"], 0, {}),
    (["-i", "g.adj", "--src", "-1"], 104, {}),
    (["-i", "g.adj", "--src", "3.5"], 104, {}),
    (["-i", "g.adj", "--src", "4294967296"], 104, {}),
    (BASE + ["--alpha", "abc"], 104, {}),
    (BASE + ["--is_directed=abc"], 104, {}),
    (["--src", "3"], 106, {}),
    (["-i", "g.adj"], 106, {}),
    (["-i", "g.adj", "--", "--src", "3"], 106, {}),
    (BASE + ["--foo"], 109, {}),
    (BASE + ["extra"], 109, {}),
    (["-d=false"] + BASE, 109, {}),
    (["-i", "g.adj", "--src"], 114, {}),
    (["-i", "g.adj", "--src", "1", "--src", "2"], 114, {}),
]


@pytest.mark.parametrize("argv,code,vals", EXPECTED)
def test_cli_written_expectations(ours, argv, code, vals):
    rc, _, got = run(ours, argv)
    assert rc == code, (argv, rc)
    for k, v in vals.items():
        assert got[k] == v, (argv, k, got[k], v)


@pytest.mark.skipif(not os.path.exists(REF_CLI), reason="oracle/_ref/cli_ref not built")
def test_cli_matches_graphone_cli11_on_every_case(ours):
    bad = []
    for argv in cases():
        ra, oa, _ = run(REF_CLI, argv)
        rb, ob, _ = run(ours, argv)
        if ra != rb or (oa != ob and not is_help(argv)):
            bad.append((argv, ra, rb))
    assert not bad, bad[:10]
    assert len(cases()) >= 120
