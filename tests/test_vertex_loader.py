"""GraphLoader's vertex-file readers (include/GraphOne/loader/loader.h:
LoadVertexStatusFromTxt with token and raw-string parsers,
LoadVertexVecFromTxt) against GraphOne's own (oracle/_ref/tests_ref/
vertex_loader, when built): the same driver (oracle/vertex_loader_driver.cpp)
on both header trees writes the same results, with and without renumbering.
CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "tests_ref", "vertex_loader")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")

FILES = {
    "mixed": "% vertex file\n3 10 20\n0 5\n7 1 2 3\n\n  2\t4 8\n5\n1 2.5 x\n0 9\n",
    "crlf": "0 1\r\n1 2 3\r\n% c\r\n2 7\r\n",
    "no_final_newline": "4 4\n2 2\n0 1.25",
    "sparse_ids": "900 1\n17 2\n900 3\n5 4\n",
}
N = {"mixed": 8, "crlf": 3, "no_final_newline": 5, "sparse_ids": 1000}


@pytest.fixture(scope="module")
def ours(tmp_path_factory):
    lib = os.path.join(ROOT, "graphone_b200")
    exe = tmp_path_factory.mktemp("vl") / "vertex_loader"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "oracle", "vertex_loader_driver.cpp"), "-o", str(exe),
                        "-L", lib, "-lgraphone_b200", f"-Wl,-rpath,{lib}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


def run(exe, path, reorder, n, out):
    r = subprocess.run([exe, str(path), "1" if reorder else "0", str(n), str(out)],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr[-2000:]
    return out.read_text()


def test_written_expectations(ours, tmp_path):
    p = tmp_path / "v.txt"
    p.write_text(FILES["mixed"])
    got = run(ours, p, False, 8, tmp_path / "o.txt").splitlines()
    assert got[0] == "T 3 10 20" and "S 5 []" in got and "D 1 2.5 0" in got
    assert got[-1] == "V 9 2.5 4 10 0 0 0 1"
    got = run(ours, p, True, 8, tmp_path / "o2.txt").splitlines()
    assert got[0] == "T 0 10 20" and got[1] == "T 1 5"  # first-seen renumbering


@pytest.mark.skipif(not os.path.exists(REF), reason="reference vertex_loader not built")
@pytest.mark.parametrize("reorder", [False, True])
@pytest.mark.parametrize("name", sorted(FILES))
def test_same_results_as_graphone(ours, tmp_path, name, reorder):
    p = tmp_path / f"{name}.txt"
    p.write_bytes(FILES[name].encode())
    a = run(ours, p, reorder, N[name], tmp_path / "a.txt")
    b = run(REF, p, reorder, N[name], tmp_path / "b.txt")
    assert a == b
