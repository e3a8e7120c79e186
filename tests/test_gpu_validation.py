"""GPU runs of the reference's validation checks against its recorded values.

* V0 (scripts/validations/v0_convergence.py, recorded in
  tests/baseline_validation/v10/v0_fast_colored_np1/verify.csv): the
  relative L2 error of the sin^3 eigenmode after hs_verify, homogeneous
  k = rho*c = 1, source off, for the spatial series (N = 8, 16, 32 at t =
  0.02, dt = 1e-5) and the temporal series (N = 32, t = 0.04, dt = 4e-3 ..
  5e-4): every printed digit, the average CG count, and the observed orders
  of convergence the script gates on (het.cu:1293-1338).
* V3 boundary control (scripts/validations/v3_injection.py, het.cu:1192-1196):
  a level-G bit-62 flip of a boundary node at step 10, with and without
  --reproject-bc; E_max, E_final and the class to their printed digits, and
  the reduction factor the script gates on (>= 100).
"""
import math

import pytest

from mnhack8_b200 import _lib
from tests.helpers import field

pytestmark = pytest.mark.gpu

SPATIAL = [(8, 0.02, 1e-5), (16, 0.02, 1e-5), (32, 0.02, 1e-5)]
TEMPORAL = [(32, 0.04, 4e-3), (32, 0.04, 2e-3), (32, 0.04, 1e-3), (32, 0.04, 5e-4)]


def _verify(N, t, dt, form):
    k, r = field(N, "homogeneous")
    g = _lib.Solver(N, dt, k, r, kernel=form, scatter="colored", verify=True)
    steps = int(t / dt + 0.5)
    rel, tot, _ = g.verify(steps)
    g.close()
    return rel, tot / steps


@pytest.mark.parametrize("form,combo", [("fast", "fast_colored"), ("gauss", "gauss_colored")])
def test_v0_verify_goldens(golden, form, combo):
    errs = {}
    for case in SPATIAL + TEMPORAL:
        N, t, dt = case
        recs = [r for r in golden["v0_verify"][combo] if r["N"] == N and abs(r["dt"] - dt) < 1e-15]
        rel, avg = _verify(N, t, dt, form)
        errs[case] = rel
        if recs:
            assert "%.10e" % rel == recs[0]["rel_L2_err"], (case, rel)
            assert avg == pytest.approx(recs[0]["avg_cg_iters"], abs=1e-9)
    # the orders v0_convergence.py gates on
    es = [errs[c] for c in SPATIAL]
    so = [math.log2(es[i] / es[i + 1]) for i in range(2)]
    assert 1.7 <= so[0] <= 2.3 and so[1] >= 1.6
    et = [errs[c] for c in TEMPORAL]
    assert all(0.85 <= math.log2(et[i] / et[i + 1]) <= 1.15 for i in range(3))


def test_v0_verify_wht_within_rounding(golden):
    """The wht form computes the same matrix through its eigen-structure: the
    eigenmode error agrees with the recorded fast-form digits to 2e-10."""
    for case in SPATIAL[:1] + TEMPORAL:
        N, t, dt = case
        rec = [r for r in golden["v0_verify"]["fast_colored"] if r["N"] == N and abs(r["dt"] - dt) < 1e-15][0]
        rel, _ = _verify(N, t, dt, "wht")
        assert abs(rel - float(rec["rel_L2_err"])) <= 2e-10 * float(rec["rel_L2_err"])


def test_v3_boundary_control_reproject(golden):
    g = golden["v3"]["boundary_control"]
    N = 32
    k, r = field(N, "lognormal", sigma=1.0, L=0.125, seed=7)
    s = _lib.Solver(N, 5e-4, k, r, kernel="fast", scatter="colored")
    rA = s.run_case(40, snap_every=1, keep_reference=True)
    rB = s.run_case(40, snap_every=1)
    bnode = (N // 2) * (N + 1) + N // 2
    fi = (_lib.LEVELS["G"], 10, bnode, 62, 0)
    assert s.target_on_boundary(fi) == 1
    out = {}
    for key, rep in (("no_reproject", False), ("reproject", True)):
        rF = s.run_case(40, snap_every=1, fi=fi, reproject=rep)
        c = _lib.classify(rA["steps"], rB["steps"], rF["steps"], 1, 5e-4)
        assert c["cls"] == g[key]["class"]
        assert "%.6e" % c["E_fault_max"] == "%.6e" % g[key]["E_max"]
        assert "%.6e" % c["E_fault_final"] == "%.6e" % g[key]["E_final"]
        out[key] = c["E_fault_final"]
    assert out["no_reproject"] / out["reproject"] >= 100
    s.close()
