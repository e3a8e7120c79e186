"""Fault-injection campaign (hs_campaign): every flip's resumed trajectory and
twin-run outcome equal the oracle's full faulted run of the same site.

The campaign resumes each faulted run at its flip step from the kept clean
field; the oracle reruns the whole trajectory from the initial condition.
Equality of class, detectors, E and iteration counts shows that the resume is
exact and that the sites are what the records say.
"""
import pytest

from mnhack8_b200 import _lib
from mnhack8_b200.campaign import coverage
from tests.helpers import field


@pytest.mark.gpu
def test_campaign_matches_oracle_runs(oracle):
    N, steps, dt = 10, 8, 5e-4
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=3)
    g = _lib.Solver(N, dt, k, r, kernel="wht", scatter="colored", detect=True)
    clean, flips = g.campaign(steps, 1, 14, seed=11)
    g.close()
    o = oracle.Oracle(N, dt, k, r, form="wht", detect=True)
    rA = o.run_case(steps, snap_every=1, keep_snaps=True)
    rB = o.run_case(steps, snap_every=1, ref_snaps=rA["snaps"])
    assert [s["cg_iters"] for s in clean] == [s["cg_iters"] for s in rA["steps"]]
    total = sum(s["cg_iters"] for s in clean)
    levels = set()
    for f in flips:
        assert 0 <= f["step"] < steps and 0 <= f["iter"] < clean[f["step"]]["cg_iters"]
        assert 0 <= f["idx"] < (N + 1) ** 3 and 0 <= f["bit"] < 64 and f["level"] in (5, 6, 7)
        levels.add(f["level"])
        fi = (f["level"], f["step"], f["idx"], f["bit"], f["iter"])
        rF = o.run_case(steps, snap_every=1, fi=fi, ref_snaps=rA["snaps"])
        want = oracle.classify(rA, rB, rF, f["level"], dt, detect=True)
        got = f["summary"]
        assert got["cls"] == want["cls"], fi
        assert got["detected_by"] == want["detected_by"], fi
        for key in ("E_fault_max", "E_fault_final", "iters_delta_max", "d1_first", "d2_first", "d3_first"):
            assert got[key] == want[key] or (got[key] != got[key] and want[key] != want[key]), (fi, key)
        assert f["nonfinite"] == rF["nonfinite"]
        assert f["iters_total_delta"] == sum(s["cg_iters"] for s in rF["steps"]) - total
    assert len(levels) >= 2
    cov = coverage(flips, clean)
    assert cov["flips"] == 14 and sum(cov["classes"].values()) == 14


@pytest.mark.gpu
def test_campaign_is_reproducible_and_rejects_atomic():
    N = 8
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=2)
    g = _lib.Solver(N, 1e-3, k, r, kernel="wht", scatter="colored", detect=True)
    _, a = g.campaign(4, 1, 6, seed=3)
    _, b = g.campaign(4, 1, 6, seed=3)
    assert [(x["step"], x["iter"], x["level"], x["idx"], x["bit"]) for x in a] == \
           [(x["step"], x["iter"], x["level"], x["idx"], x["bit"]) for x in b]
    assert [x["summary"]["cls"] for x in a] == [x["summary"]["cls"] for x in b]
    g.close()
    ga = _lib.Solver(N, 1e-3, k, r, kernel="wht", scatter="atomic", detect=True)
    with pytest.raises(_lib.HeatError):
        ga.campaign(4, 1, 2, seed=1)
    ga.close()


def _flip(level, bit, cls, by, d1_first, E=0.0):
    return dict(level=level, bit=bit, summary=dict(cls=cls, detected_by=by, d1_first=d1_first, E_fault_max=E))


def test_coverage_arithmetic():
    """Coverage shares, counted on hand-made records (no GPU)."""
    flips = [_flip(5, 10, "benign", "none", -1), _flip(5, 60, "persistent", "D1+D2", 3, E=0.2),
             _flip(6, 63, "transient", "none", -1, E=1e-11), _flip(7, 55, "detected", "D1+D2+D3", 2, E=float("nan"))]
    clean = [dict(d1=1e-17), dict(d1=3e-17)]
    c = coverage(flips, clean)
    assert c["classes"] == {"benign": 1, "transient": 1, "persistent": 1, "detected": 1}
    assert c["harmful"] == 3 and c["missed_harmful"] == 1
    assert c["abft_d1_rate"] == 0.5 and abs(c["abft_d1_coverage_of_harmful"] - 2 / 3) < 1e-15
    assert c["by_vector"]["p"]["flips"] == 2 and c["by_vector"]["Ap"]["any_detector_rate"] == 1.0
    assert c["by_bit_field"]["exponent"]["flips"] == 2 and c["by_bit_field"]["sign"]["missed_harmful"] == 1
    assert c["abft_noise_floor_clean_max_d1"] == 3e-17
    assert c["significant"] == 2 and c["any_detector_coverage_of_significant"] == 1.0 and c["missed_significant"] == 0
