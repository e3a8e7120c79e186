"""Seeded single-bit-flip campaign with ABFT detection coverage.

One transient-heat trajectory is run clean, then faulted once per flip: a
single bit of p (after its formation), r (after its update) or Ap (after the
projection) is flipped at a PCG iteration drawn uniformly over the clean
run's iterations.  Each faulted run is classified with the reference's
twin-run rules (benign / transient / persistent / detected) and its
detectors: D1 is the ABFT checksum on every operator apply, D2 the end-of-step
true residual, D3 the temperature range against the clean run.

The default workload is the N=128 problem: lognormal conductivity ln k ~
N(0, 1) with correlation length 8 elements, Gaussian bump sigma 0.15, dt =
1e-4, 50 steps, PCG to 1e-10, 1000 flips, E(t) at every step.

    python -m mnhack8_b200.campaign --flips 1000 --out campaign_N128
writes <out>.csv (one row per flip) and <out>.json (coverage summary).
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

VEC_NAMES = {5: "p", 6: "r", 7: "Ap"}
HARMFUL = ("transient", "persistent", "detected")


def bit_field(bit: int) -> str:
    return "mantissa" if bit < 52 else ("exponent" if bit < 63 else "sign")


def coverage(flips: list, clean_steps: list, sig_err: float = 1e-6) -> dict:
    """Detection coverage of a campaign: class counts, and (overall, per vector
    and per bit field) the share of flips each detector caught, over all flips,
    over the harmful ones (class other than benign: any final-field change
    above the twin-run threshold, 1e-13 relative) and over the significant ones
    (relative field error above sig_err at some step, i.e. far above the
    changes a flip leaves at the PCG tolerance)."""
    def stats(rows):
        harm = [r for r in rows if r["summary"]["cls"] in HARMFUL]
        sig = [r for r in rows if r["summary"]["cls"] == "detected" or
               not (r["summary"].get("E_fault_max", 0.0) <= sig_err)]

        def share(sel, pool):
            return (sum(1 for r in pool if sel(r)) / len(pool)) if pool else None

        def d1(r):
            return r["summary"]["d1_first"] >= 0

        def anyd(r):
            return r["summary"]["detected_by"] not in ("none", "off")

        return {
            "flips": len(rows),
            "classes": {c: sum(1 for r in rows if r["summary"]["cls"] == c)
                        for c in ("benign", "transient", "persistent", "detected")},
            "abft_d1_rate": share(d1, rows),
            "any_detector_rate": share(anyd, rows),
            "harmful": len(harm),
            "abft_d1_coverage_of_harmful": share(d1, harm),
            "any_detector_coverage_of_harmful": share(anyd, harm),
            "missed_harmful": sum(1 for r in harm if not anyd(r)),
            "significant": len(sig),
            "any_detector_coverage_of_significant": share(anyd, sig),
            "missed_significant": sum(1 for r in sig if not anyd(r)),
        }

    out = stats(flips)
    out["by_vector"] = {v: stats([r for r in flips if VEC_NAMES[r["level"]] == v]) for v in ("p", "r", "Ap")}
    out["by_bit_field"] = {b: stats([r for r in flips if bit_field(r["bit"]) == b])
                           for b in ("mantissa", "exponent", "sign")}
    d1_clean = [s["d1"] for s in clean_steps]
    out["abft_noise_floor_clean_max_d1"] = max(d1_clean) if d1_clean else None
    out["abft_threshold"] = 1e-10
    out["significant_error"] = sig_err
    return out


def run(N=128, steps=50, snap=1, flips=1000, seed=20240601, field_seed=1, dt=1e-4, rtol=1e-10, kernel="wht",
        vectors=("P", "RV", "AP"), out=None, device=0) -> dict:
    from mnhack8_b200 import _lib
    from mnhack8_b200.fields import FieldSpec, make_field

    k, r, _ = make_field(FieldSpec(n=N, model="lognormal", mu=0.0, sigma=1.0, L=8.0 / N, seed=field_seed))
    g = _lib.Solver(N, dt, k.ravel(), r.ravel(), kernel=kernel, scatter="colored", detect=True, no_source=True,
                    ic="gaussian", ic_sigma=0.15, rtol=rtol, max_iter=500, device=device)
    t0 = time.perf_counter()
    clean, recs = g.campaign(steps, snap, flips, seed, vectors)
    wall = time.perf_counter() - t0
    g.close()
    cov = coverage(recs, clean)
    summary = {
        "workload": f"N={N} lognormal k (sigma 1, corr 8 elements, seed {field_seed}), Gaussian IC sigma 0.15, "
                    f"dt={dt}, {steps} steps, PCG rtol {rtol}, {kernel} element form, colored scatter, D1 on",
        "flips": flips, "seed": seed, "snap_every": snap,
        "sampling": "std::mt19937_64(seed), each draw the next output modulo its range: global CG iteration over "
                    "the clean run, vector in {p, r, Ap}, node entry, bit 0..63",
        "clean_cg_iters": sum(s["cg_iters"] for s in clean),
        "wall_s": wall, "coverage": cov,
    }
    if out:
        with open(out + ".csv", "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(["flip", "step", "iter", "vector", "idx", "bit", "bit_field", "class", "detected_by",
                        "d1_first", "d2_first", "d3_first", "E_fault_max", "E_fault_final", "iters_delta_max",
                        "iters_total_delta", "nonfinite"])
            for i, x in enumerate(recs):
                s = x["summary"]
                w.writerow([i, x["step"], x["iter"], VEC_NAMES[x["level"]], x["idx"], x["bit"], bit_field(x["bit"]),
                            s["cls"], s["detected_by"], s["d1_first"], s["d2_first"], s["d3_first"],
                            f"{s['E_fault_max']:.6e}", f"{s['E_fault_final']:.6e}", s["iters_delta_max"],
                            x["iters_total_delta"], x["nonfinite"]])
        with open(out + ".json", "w") as f:
            json.dump(summary, f, indent=1,
                      default=lambda v: None if isinstance(v, float) and math.isnan(v) else v)
    return summary


def _main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--snap", type=int, default=1)
    ap.add_argument("--flips", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=20240601)
    ap.add_argument("--field-seed", type=int, default=1)
    ap.add_argument("--dt", type=float, default=1e-4)
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--kernel", default="wht", choices=["wht", "fast", "gauss"])
    ap.add_argument("--out", default="campaign")
    a = ap.parse_args(argv)
    s = run(a.N, a.steps, a.snap, a.flips, a.seed, a.field_seed, a.dt, a.rtol, a.kernel, out=a.out)
    c = s["coverage"]
    print(json.dumps({"flips": s["flips"], "clean_cg_iters": s["clean_cg_iters"], "wall_s": s["wall_s"],
                      "classes": c["classes"], "abft_d1_rate": c["abft_d1_rate"],
                      "any_detector_coverage_of_harmful": c["any_detector_coverage_of_harmful"],
                      "significant": c["significant"],
                      "any_detector_coverage_of_significant": c["any_detector_coverage_of_significant"]}))
    return 0


if __name__ == "__main__":
    sys.exit(_main())
