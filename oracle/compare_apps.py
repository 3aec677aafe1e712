"""GraphOne's unchanged SSSP apps, built against GraphOne's own headers
(oracle/_ref/apps_ref) and against this repository's include/
(oracle/_ref/apps_g1) by `make -C oracle refapps dropin`, run on the same
generated inputs; prints each app's own "Elapsed" line, wall time and parity
with the oracle's Dijkstra.  A checker, not part of the library.

    python oracle/compare_apps.py              # rmat14 and grid256, three apps
    python oracle/compare_apps.py --grid4096   # also sssp_adv on the 4096^2 grid
"""
import os, subprocess, sys, time, tempfile
import numpy as np
_HERE = os.path.dirname(os.path.abspath(__file__))
# the repository root, not this directory (whose oracle.py would shadow the package)
sys.path[:] = [os.path.dirname(_HERE)] + [q for q in sys.path if os.path.abspath(q or ".") != _HERE]
from graphone_b200 import gen
from oracle import oracle as O
tmp = tempfile.mkdtemp()
APPS = ["sssp_blas", "sssp_blas2", "sssp_adv"]
cases = {"rmat14": (gen.rmat(14, 16, True, (1, 64)), False, APPS),
         "grid256": (gen.grid2d(256, 256, (1, 100)), False, APPS)}
if "--grid4096" in sys.argv:
    # the advance-engine configuration: 16.7M vertices, source at the corner
    cases["grid4096"] = (gen.grid2d(4096, 4096, (1, 100)), False, ["sssp_adv"])
for name, (g, directed, apps) in cases.items():
    adj = os.path.join(tmp, name + ".adj")
    gen.write_adj(g, adj, directed)
    rp, ci, v = g.np("n")
    exp = O.dijkstra_u32(rp, ci, v, 0)
    for app in apps:
        for kind in ["ref", "g1"]:
            path = O.app(kind, app)
            if not path: continue
            out = os.path.join(tmp, f"{name}_{app}_{kind}.txt")
            t0 = time.time()
            r = subprocess.run([path, "-i", adj, "--src", "0", "-o", out], capture_output=True, text=True, timeout=1200)
            wall = time.time() - t0
            if r.returncode != 0:
                print(name, app, kind, "FAILED rc", r.returncode, r.stdout[-300:], r.stderr[-300:]); continue
            lines = open(out).read().splitlines()
            vals = np.array([float(l.split("-",1)[1]) for l in lines[1:]], dtype=np.float64)
            e = exp[:len(vals)].astype(np.float64); e[exp[:len(vals)] == O.U32_MAX] = float(np.float32(3.4028234663852886e38))
            ok = np.array_equal(vals.astype(np.float32), e.astype(np.float32))
            print(f"{name:8s} {app:11s} {kind:4s} {lines[0]:28s} wall={wall:.2f}s parity={ok}")
