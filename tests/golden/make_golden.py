"""Extract the golden vectors of the reference's own recorded test runs.

Reads (only in the development container, where the reference tree is
mounted) the recorded outputs of the reference validation suite
``tests/baseline_validation/v10`` and runs the reference field generator
``scripts/gen_field.py`` to fingerprint its output, then writes
``tests/golden/reference_v10.json``.  The JSON is the fixture the tests use;
nothing at test time reads the reference tree.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT
"""
from __future__ import annotations

import csv
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
ROOT = sys.argv[1]
V10 = os.path.join(ROOT, "tests", "baseline_validation", "v10")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_v10.json")


def rows(path):
    with open(path) as f:
        return list(csv.DictReader(f))


def field_fingerprints():
    """sha256 of the reference generator's k/rhoc files for the specs the tests use."""
    specs = [
        dict(n=32, model="lognormal", sigma=1.0, L=0.125, seed=7),
        dict(n=16, model="lognormal", sigma=1.0, L=0.125, seed=7),
        dict(n=16, model="quadrants"),
        dict(n=15, model="quadrants"),
        dict(n=8, model="homogeneous", k=1.0, rhoc=1.0),
        dict(n=24, model="lognormal", sigma=1.5, L=0.25, seed=3, rhoc_sigma=0.5, upscale=2),
        dict(n=12, model="layered", k=1.0, k2=50.0, period=3),
    ]
    gen = os.path.join(ROOT, "scripts", "gen_field.py")
    out = []
    with tempfile.TemporaryDirectory() as td:
        for i, s in enumerate(specs):
            prefix = os.path.join(td, f"f{i}")
            cmd = [sys.executable, gen, "--n", str(s["n"]), "--model", s["model"], "--out", prefix]
            for k, v in s.items():
                if k not in ("n", "model"):
                    cmd += [f"--{k.replace('_', '-')}", str(v)]
            subprocess.run(cmd, check=True, capture_output=True)
            k = np.fromfile(prefix + "_k.bin")
            r = np.fromfile(prefix + "_rhoc.bin")
            out.append(dict(spec=s, k_sha256=hashlib.sha256(k.tobytes()).hexdigest(),
                            rhoc_sha256=hashlib.sha256(r.tobytes()).hexdigest(),
                            kmin=float(k.min()), kmax=float(k.max())))
    return out


def main():
    g = {"source": "reference tests/baseline_validation/v10 (RTX 3060 recordings) and scripts/gen_field.py"}
    v0 = {}
    for combo in ["fast_colored", "fast_atomic", "gauss_colored", "gauss_atomic"]:
        v0[combo] = [dict(N=int(r["N"]), dt=float(r["dt"]), t_end=float(r["t_end"]), rel_L2_err=r["rel_L2_err"],
                          avg_cg_iters=float(r["avg_cg_iters"]))
                     for r in rows(os.path.join(V10, f"v0_{combo}_np1", "verify.csv"))]
    g["v0_verify"] = v0
    v1 = json.load(open(os.path.join(V10, "v1", "report.json")))["details"]
    g["v1"] = {"even": {k: v1["even"][k] for k in ("N", "ref_norm", "v2_norm")},
               "odd": {k: v1["odd_negative_control"][k] for k in ("N", "ref_norm", "v2_norm")}}
    v5 = json.load(open(os.path.join(V10, "v5", "report.json")))["details"]
    g["v5"] = {"field_rel_diff": v5["field_rel_diff"], "mean_cg_iters": v5["mean_cg_iters"]}
    v6 = {}
    for case in os.listdir(os.path.join(V10, "v6")):
        d = os.path.join(V10, "v6", case)
        if not os.path.isdir(d):
            continue
        tr = rows(os.path.join(d, "fi_trace_det.csv"))
        sm = rows(os.path.join(d, "fi_summary_det.csv"))[0]
        keep = ["step", "E_fault", "spread_F", "cg_A", "cg_F", "d1_abft_A", "d1_abft_F", "d2_resid_A", "d2_resid_F",
                "d3_tmin_F", "d3_tmax_F"]
        v6[case] = {"trace": [{k: r[k] for k in keep} for r in tr],
                    "summary": {k: sm[k] for k in ("fi_level", "fi_step", "fi_target", "fi_bit", "E_fault_max",
                                                   "step_at_max", "E_fault_int", "E_fault_final", "class",
                                                   "iters_delta_max", "d1_first", "d2_first", "d3_first",
                                                   "detected_by", "mean_cg_iters_A", "kmin", "kmax",
                                                   "target_on_boundary")}}
    g["v6"] = v6
    v3 = json.load(open(os.path.join(V10, "v3", "report.json")))["details"]
    g["v3"] = {"runs": v3["runs"], "boundary_control": v3.get("boundary_control")}
    meta = json.load(open(os.path.join(V10, "v6", "ln32_meta.json")))
    g["ln32_meta"] = {k: meta[k] for k in ("n", "sigma", "L", "seed", "kmin", "kmax")}
    g["fields"] = field_fingerprints()
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
