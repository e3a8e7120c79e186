"""The CPU oracle against the reference's own recorded test outputs (no GPU).

Pins: V0 eigenmode errors (verify.csv), V1 MNHack7 regression norm, V5
gauss-vs-fast equivalence, V6 clean detector traces (CG iterations, D2, D3)
and a level-R fault trajectory, and the V3 injector magnitudes.
"""
import math

import numpy as np
import pytest

from tests.helpers import field


@pytest.mark.parametrize("form", ["fast", "gauss", "wht"])
@pytest.mark.parametrize("case", [(8, 0.02, 1e-5), (32, 0.04, 4e-3), (32, 0.04, 2e-3), (32, 0.04, 1e-3),
                                  (32, 0.04, 5e-4)])
def test_v0_verify_errors(oracle, golden, form, case):
    """V0: rel-L2 error of the sin^3 eigenmode equals the recorded value to its 11 printed digits."""
    N, t, dt = case
    combo = "gauss_colored" if form == "gauss" else "fast_colored"
    rec = [r for r in golden["v0_verify"][combo] if r["N"] == N and abs(r["dt"] - dt) < 1e-15][0]
    k, r = field(N, "homogeneous")
    o = oracle.Oracle(N, dt, k, r, form=form, verify=True)
    steps = int(t / dt + 0.5)
    rel, tot = o.verify(steps)
    got = "%.10e" % rel
    if form == "wht":
        assert abs(rel - float(rec["rel_L2_err"])) <= 2e-10 * float(rec["rel_L2_err"])
    else:
        assert got == rec["rel_L2_err"]
    assert tot / steps == pytest.approx(rec["avg_cg_iters"], abs=1e-9)


@pytest.mark.parametrize("N", [16])
def test_v0_verify_spatial_16(oracle, golden, N):
    rec = [r for r in golden["v0_verify"]["fast_colored"] if r["N"] == N][0]
    k, r = field(N, "homogeneous")
    o = oracle.Oracle(N, 1e-5, k, r, form="fast", verify=True)
    rel, tot = o.verify(2000)
    assert "%.10e" % rel == rec["rel_L2_err"]


def test_v1_mnhack7_regression(oracle, golden):
    """V1: gauss/atomic on the quadrant field, N=16, t=0.01, dt=1e-4, source on.

    The reference's het gauss/atomic run recorded ||T|| = 0.28362691675518675;
    the oracle reproduces it bit for bit, and the odd-N negative control to
    within rounding."""
    for key in ("even", "odd"):
        g = golden["v1"][key]
        k, r = field(g["N"], "quadrants")
        o = oracle.Oracle(g["N"], 1e-4, k, r, form="gauss", colored=False)
        res = o.run_case(100, snap_every=0)
        nrm = float(np.linalg.norm(res["T"]))
        assert abs(nrm - g["v2_norm"]) <= 1e-15 * g["v2_norm"]
        if key == "even":
            assert abs(nrm - g["ref_norm"]) / g["ref_norm"] <= 1e-6   # the MNHack7 solver's printed norm
        else:
            assert abs(nrm - g["ref_norm"]) / g["ref_norm"] > 1e-6    # negative control must not match


def test_v5_gauss_vs_fast(oracle, golden):
    k, r = field(16, "lognormal", sigma=1.0, L=0.125, seed=7)
    res = {}
    for form in ("gauss", "fast", "wht"):
        o = oracle.Oracle(16, 5e-4, k, r, form=form)
        res[form] = o.run_case(40, snap_every=0)
    rel = np.linalg.norm(res["fast"]["T"] - res["gauss"]["T"]) / np.linalg.norm(res["gauss"]["T"])
    assert rel <= 1e-12
    rel_w = np.linalg.norm(res["wht"]["T"] - res["fast"]["T"]) / np.linalg.norm(res["fast"]["T"])
    assert rel_w <= 1e-12
    for form in res:
        mean = np.mean([s["cg_iters"] for s in res[form]["steps"]])
        # the summary CSV prints the mean with %.2f (het.cu:1575)
        assert float("%.2f" % mean) == golden["v5"]["mean_cg_iters"]["fast"]


@pytest.fixture(scope="module")
def ln32_runs(oracle):
    k, r = field(32, "lognormal", sigma=1.0, L=0.125, seed=7)
    out = {}
    for form in ("fast", "wht"):
        o = oracle.Oracle(32, 5e-4, k, r, form=form, colored=True, detect=True)
        out[form] = (o, o.run_case(40, snap_every=1, keep_snaps=True))
    return out


@pytest.mark.parametrize("form", ["fast", "wht"])
def test_v6_clean_trace(ln32_runs, golden, form):
    """V6 clean colored run: per-step CG iterations, D2 (3 digits), D3 range (7 digits)."""
    _, rA = ln32_runs[form]
    gold = golden["v6"]["clean_colored"]["trace"]
    assert len(gold) == 40
    for g, x in zip(gold, rA["steps"]):
        assert int(g["cg_A"]) == x["cg_iters"]
        assert g["d2_resid_A"] == "%.3e" % x["d2"]
        assert g["d3_tmin_F"] == "%.6e" % x["tmin"]
        assert g["d3_tmax_F"] == "%.6e" % x["tmax"]
        assert x["d1"] < 1e-15 and float(g["d1_abft_A"]) < 1e-15   # rounding-noise floor, by magnitude


def test_v6_level_R_bit55(ln32_runs, golden, oracle):
    """V6 level-R fault, bit 55, element (16,16,16), step 10: E(t) to its 11
    printed digits, spread, D1, D2, class."""
    o, rA = ln32_runs["fast"]
    g = golden["v6"]["L2_b55"]
    sm = g["summary"]
    fi = (2, int(sm["fi_step"]), int(sm["fi_target"]), int(sm["fi_bit"]), 0)
    rF = o.run_case(40, snap_every=1, fi=fi, ref_snaps=rA["snaps"])
    for gt, x in zip(g["trace"], rF["steps"]):
        assert gt["E_fault"] == "%.10e" % x["E"]
        assert gt["spread_F"] == "%.4f" % x["spread"]
        assert int(gt["cg_F"]) == x["cg_iters"]
        assert gt["d2_resid_F"] == "%.3e" % x["d2"]
        if int(gt["step"]) == 10:
            assert gt["d1_abft_F"] == "%.3e" % x["d1"]
    rB = o.run_case(40, snap_every=1, ref_snaps=rA["snaps"])
    s = oracle.classify(rA, rB, rF, 2, 5e-4, detect=True)
    assert s["cls"] == sm["class"]
    assert "%.6e" % s["E_fault_max"] == sm["E_fault_max"]
    assert "%.6e" % s["E_fault_int"] == sm["E_fault_int"]
    assert "%.6e" % s["E_fault_final"] == sm["E_fault_final"]
    assert s["detected_by"] == sm["detected_by"]
    assert (s["d1_first"], s["d2_first"], s["d3_first"]) == (int(sm["d1_first"]), int(sm["d2_first"]),
                                                            int(sm["d3_first"]))


@pytest.mark.parametrize("case", ["L1_b51", "L1_b55", "L2_b51", "L2_b63", "L2_b62", "L1_b62"])
def test_v6_coverage_cases(ln32_runs, golden, oracle, case):
    """V6 coverage rows: fault class, detectors that fire and their first step."""
    o, rA = ln32_runs["fast"]
    sm = golden["v6"][case]["summary"]
    fi = (int(sm["fi_level"]), int(sm["fi_step"]), int(sm["fi_target"]), int(sm["fi_bit"]), 0)
    rF = o.run_case(40, snap_every=1, fi=fi, ref_snaps=rA["snaps"])
    s = oracle.classify(rA, rA, rF, fi[0], 5e-4, detect=True)
    assert s["cls"] == sm["class"]
    assert s["detected_by"] == sm["detected_by"]
    assert s["iters_delta_max"] == int(sm["iters_delta_max"])
    if sm["class"] != "detected":
        assert "%.6e" % s["E_fault_max"] == sm["E_fault_max"]


def test_v3_boundary_control(oracle, golden):
    """V3 boundary control: a level-G bit-62 flip of a boundary node (0, N/2,
    N/2) at step 10 leaves a BC-scheme artifact that --reproject-bc removes.
    E_max / E_final and the class match the recorded run to their printed
    digits, with and without reprojection."""
    g = golden["v3"]["boundary_control"]
    N = 32
    k, r = field(N, "lognormal", sigma=1.0, L=0.125, seed=7)
    o = oracle.Oracle(N, 5e-4, k, r, form="fast", colored=True)
    rA = o.run_case(40, snap_every=1, keep_snaps=True)
    rB = o.run_case(40, snap_every=1, ref_snaps=rA["snaps"])
    bnode = (N // 2) * (N + 1) + N // 2
    for key, rep in (("no_reproject", False), ("reproject", True)):
        rF = o.run_case(40, snap_every=1, fi=(1, 10, bnode, 62, 0), ref_snaps=rA["snaps"], reproject=rep)
        s = oracle.classify(rA, rB, rF, 1, 5e-4)
        assert s["cls"] == g[key]["class"]
        assert "%.6e" % s["E_fault_max"] == "%.6e" % g[key]["E_max"]
        assert "%.6e" % s["E_fault_final"] == "%.6e" % g[key]["E_final"]
