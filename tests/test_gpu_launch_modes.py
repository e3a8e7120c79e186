"""The PCG loop's three launch modes give the same bits.

The loop normally runs inside a CUDA graph with a conditional while node.
HS_GRAPH=0 launches the same kernels one by one from the host (the mode
profilers need), and HS_PDL=1 launches them with programmatic dependent
launch.  Each mode is chosen once per process, so each runs in a child
process here, on the same seeded problem: an N=96 lognormal field, 6 steps,
ABFT on, the clean run (kept as the reference) and two faulted runs (a
level-R fault at step 2, a p-vector fault at step 4).  Fields, per-step CG
counts, detector values and E(t) must agree bit for bit across the modes.
"""
import json
import os
import subprocess
import sys

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, %r)
from mnhack8_b200 import _lib
from mnhack8_b200.fields import FieldSpec, make_field
k, r, _ = make_field(FieldSpec(n=96, model="lognormal", sigma=1.0, L=0.1, seed=5))
g = _lib.Solver(96, 1e-4, k.ravel(), r.ravel(), kernel="wht", scatter="colored", detect=True,
                no_source=True, ic="gaussian", ic_sigma=0.15, rtol=1e-10, max_iter=500)
out = []
for fi in (None, dict(level=2, step=2, target=12345, bit=52), dict(level=5, step=4, target=20000, bit=50, iter=3)):
    res = g.run_case(6, snap_every=1, fi=fi, keep_reference=fi is None)
    out.append(dict(T=res["T"].view(np.uint64).tolist()[::97],
                    steps=[[s["cg_iters"], float(s["d1"]).hex(), float(s["d2"]).hex(), float(s["tmin"]).hex(),
                            float(s["tmax"]).hex(), float(s["E"]).hex()] for s in res["steps"]]))
g.close()
print(json.dumps(out))
"""


def _run(env_extra):
    env = dict(os.environ)
    env.pop("HS_GRAPH", None)
    env.pop("HS_PDL", None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD % ROOT], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_graph_direct_and_programmatic_launches_agree():
    base = _run({})
    assert _run({"HS_GRAPH": "0"}) == base
    assert _run({"HS_PDL": "1"}) == base
    assert _run({"HS_GRAPH": "0", "HS_PDL": "1"}) == base
