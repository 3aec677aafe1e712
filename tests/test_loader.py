"""The drop-in loader (include/GraphOne/loader/loader.h, host code) against
GraphOne's own GraphLoader + EdgeCache::ToCsr (oracle/_ref, when built) and
the oracle's counting sort, on .adj files with comments, blank lines, tabs,
self loops, missing weights, duplicates and isolated vertices, with each of
the loader's switches (directed, first-seen renumbering, self loops and
duplicates kept).  CPU only."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")

TRICKY = """% a comment line
% another one

0 1 5
  0\t2 7   
1 1 9
2 4
3 0 4
0 1 5
% duplicate above, self loop 1-1 dropped
6 3 2
\t
7\t6\t1
5
9 9 3
"""


def random_adj(rng, n, m):
    """Weighted lines over vertices [0, n), weightless ones over [n, n + 50);
    duplicates (in either direction) carry the same weight, because the
    reference keeps an unspecified one of differing duplicates."""
    a = rng.integers(0, n, m)
    b = rng.integers(0, n, m)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    w = (lo * 7919 + hi * 104729) % 97 + 1
    lines = [f"{x} {y} {z}" for x, y, z in zip(a, b, w)]
    c = rng.integers(n, n + 50, (m // 5, 2))
    lines += [f"{x}\t{y}" for x, y in c]
    lines += lines[: m // 10]  # verbatim repeats
    order = rng.permutation(len(lines))
    return "\n".join(lines[i] for i in order)  # no newline after the last line


def parse(text, directed, reorder=False, keep_self=False, keep_dup=False):
    """The reference's reading rules restated (loader/graph_loader.h:32-122,
    255-296, edge_cache.h:50-105): edges in file order, self loops dropped
    unless kept, ids renumbered in first-seen order when asked (after the
    self-loop check), reverse edges for undirected input, duplicates merged
    after sorting by (src, dst) unless kept."""
    edges, vmap = [], {}

    def rn(x):
        if not reorder:
            return x
        if x not in vmap:
            vmap[x] = len(vmap)
        return vmap[x]

    for line in text.split("\n"):
        s = line.strip()
        if not s or s.startswith("%"):
            continue
        tok = s.replace("\t", " ").split()
        if len(tok) < 2:
            continue
        u, v = int(tok[0]), int(tok[1])
        w = int(tok[2]) if len(tok) > 2 else 1
        if u == v and not keep_self:
            continue
        u, v = rn(u), rn(v)
        edges.append((u, v, w))
        if not directed and u != v:
            edges.append((v, u, w))
    if not keep_dup:
        edges = sorted(set(edges), key=lambda e: (e[0], e[1]))
    n = max([max(u, v) for u, v, _ in edges], default=0) + 1
    src = np.array([e[0] for e in edges], np.uint32)
    dst = np.array([e[1] for e in edges], np.uint32)
    w = np.array([e[2] for e in edges], np.uint32)
    return n, src, dst, w


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("loader") / "loader_driver"
    lib = os.path.join(ROOT, "graphone_b200")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "loader_driver.cpp"), "-o", str(exe),
                        "-L", lib, "-lgraphone_b200", f"-Wl,-rpath,{lib}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


def ours(driver, path, flags):
    r = subprocess.run([driver, path, *("1" if f else "0" for f in flags)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    # the loader's warnings ("[WARN] ...", the one-token line) share stdout
    lines = [ln for ln in r.stdout.split("\n") if not ln.startswith("[")]
    out = []
    for t in range(3):  # out-edge CSR, in-edge CSR, LoadCsrFromTxt's CSR
        n, m = map(int, lines[4 * t].split())
        arr = [np.array(lines[4 * t + k].split(), dtype=np.int64).astype(np.uint32) for k in (1, 2, 3)]
        out.append((n, m, *arr))
    # LoadCsrFromTxt<arch> alone (edge data double by default): same shape
    assert lines[12].split() == ["default-edata", str(out[2][0]), str(out[2][1]), "1"]
    return out


def reference(path, flags):
    R = O.ref()
    if R is None:
        return None
    n, m = C.c_uint32(), C.c_uint64()
    assert R.ref_load_adj_opts(path.encode(), *(int(f) for f in flags), C.byref(n), C.byref(m)) == 0
    out = []
    for t in range(2):
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(max(1, m.value), np.uint32)
        v = np.zeros(max(1, m.value), np.uint32)
        assert R.ref_to_csr(t, O._ptr(rp), O._ptr(ci), O._ptr(v)) == 0
        out.append((n.value, m.value, rp, ci[: m.value], v[: m.value]))
    return out


CASES = {"tricky": lambda: TRICKY,
         "random": lambda: random_adj(np.random.default_rng(7), 300, 4000),
         "one_edge": lambda: "4 2 3",
         "only_comments": lambda: "% nothing\n\n% here\n"}


# (directed, reorder, keep_self, keep_dup); the reference's own loader test
# (test/loader_test.cpp) reads a directed file with renumbering on
FLAGS = [(True, False, False, False), (False, False, False, False), (True, True, False, False),
         (False, True, False, False), (True, False, True, False), (False, False, True, True),
         (True, True, True, True), (False, True, False, True)]


@pytest.mark.parametrize("flags", FLAGS, ids=lambda f: "".join("dRsD"[i] if x else "-" for i, x in enumerate(f)))
@pytest.mark.parametrize("case", sorted(CASES))
def test_loader_matches_graphone_loader_and_oracle(driver, tmp_path, case, flags):
    text = CASES[case]()
    path = str(tmp_path / f"{case}.adj")
    with open(path, "w") as f:
        f.write(text)
    got = ours(driver, path, flags)
    n, src, dst, w = parse(text, *flags)
    for t, (gn, gm, rp, ci, v) in enumerate(got):
        assert (gn, gm) == (n, len(src))
        erp, eci, ev = O.csr_build(n, src, dst, w, transpose=t == 1)
        assert np.array_equal(rp, erp) and np.array_equal(ci, eci) and np.array_equal(v, ev)
    ref = reference(path, flags)
    if ref is not None:
        for g, r in zip(got[:2], ref):
            assert g[:2] == r[:2]
            for a, b in zip(g[2:], r[2:]):
                assert np.array_equal(a, b)


def run_threads(driver, path, flags, threads):
    env = dict(os.environ, G1_LOADER_THREADS=str(threads))
    r = subprocess.run([driver, path, *("1" if f else "0" for f in flags)], capture_output=True, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


@pytest.mark.parametrize("flags", [(True, False, False, False), (False, True, False, False),
                                   (True, True, True, True)],
                         ids=lambda f: "".join("dRsD"[i] if x else "-" for i, x in enumerate(f)))
def test_parallel_read_of_a_large_file_equals_the_one_thread_read(driver, tmp_path, flags):
    """A file of several MiB is parsed by several threads (parts cut at line
    ends) and its duplicates merged by a parallel stable sort: the output,
    warnings included, is the same bytes as with one thread, and matches the
    restated reading rules.  Duplicates with different weights check that
    the first one in file order keeps its weight either way."""
    rng = np.random.default_rng(11)
    body = random_adj(rng, 200_000, 400_000).split("\n")
    # comments, blank lines, one-token lines (a warning each) and
    # conflicting duplicates, spread over the file (and so over the parts)
    extra = ["% comment", "", "   ", "12345", "7 8 1", "7 8 2", "8 7 3"]
    for k, pos in enumerate(rng.integers(0, len(body), 400)):
        body.insert(int(pos), extra[k % len(extra)])
    text = "\n".join(body) + "\n"
    path = str(tmp_path / "large.adj")
    with open(path, "w") as f:
        f.write(text)
    assert len(text) > 6 << 20
    one = run_threads(driver, path, flags, 1)
    many = run_threads(driver, path, flags, 6)
    assert one == many
    assert one.count(b"[WARN]") >= 50
    if not flags[3]:
        # without the conflicting duplicates the restated rules apply too
        clean = "\n".join(ln for ln in body if ln not in ("7 8 2", "8 7 3")) + "\n"
        cpath = str(tmp_path / "clean.adj")
        with open(cpath, "w") as f:
            f.write(clean)
        got = ours(driver, cpath, flags)
        n, src, dst, w = parse(clean, *flags)
        for t, (gn, gm, rp, ci, v) in enumerate(got):
            assert (gn, gm) == (n, len(src))
            erp, eci, ev = O.csr_build(n, src, dst, w, transpose=t == 1)
            assert np.array_equal(rp, erp) and np.array_equal(ci, eci) and np.array_equal(v, ev)
