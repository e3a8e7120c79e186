#!/usr/bin/env python3
"""Run the reference's validation battery against heat_solver_b200.

The reference ships its validation scripts (``scripts/validations/v0..v6``
and the field generator ``scripts/gen_field.py``); they drive a solver binary
through its CLI and write one ``report.json`` per check.  This runner executes
the same sequence as the reference's ``run_validations.sh`` (V0 for the four
kernel/scatter combinations, V2, V3, V4/V5, V6) with the binary of this
package and one rank (``--mpi 1``: the MPI cases of V3/V4 are skipped by the
scripts themselves), then prints one line per report and exits non-zero when
any report says FAIL.

V1 is not run: it compares against the reference's previous solver binary
(``src/heat_solver.cu``), which needs MPI to build.

The scripts are not part of this repository.  Point ``--validations`` at a
directory that holds them (the reference's ``scripts/validations``) and
``--gen`` at its ``scripts/gen_field.py``.

Usage:
    python tests/reference_validations.py --validations DIR --gen GEN_FIELD_PY --out OUTDIR
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mnhack8_b200", "heat_solver_b200")


def battery(vdir, gen, binary, out):
    """(name, argv) of every check, in the reference runner's order."""
    py = sys.executable
    common = ["--bin", binary, "--gen", gen, "--out", out]
    runs = []
    for k in ("fast", "gauss"):
        for s in ("colored", "atomic"):
            runs.append((f"V0 {k}/{s}", [py, os.path.join(vdir, "v0_convergence.py")] + common
                         + ["--kernel", k, "--scatter", s]))
    runs.append(("V2", [py, os.path.join(vdir, "v2_noise_floor.py")] + common))
    runs.append(("V3", [py, os.path.join(vdir, "v3_injection.py")] + common + ["--mpi", "1"]))
    runs.append(("V4/V5", [py, os.path.join(vdir, "v4_v5_equivalence.py")] + common + ["--mpi", "1"]))
    runs.append(("V6", [py, os.path.join(vdir, "v6_detection.py")] + common + ["--mpi", "1"]))
    return runs


def reports(out):
    """(relative path, pass, status) of every report.json under out, sorted."""
    rows = []
    for d, _, files in os.walk(out):
        if "report.json" in files:
            p = os.path.join(d, "report.json")
            with open(p) as f:
                r = json.load(f)
            rows.append((os.path.relpath(p, out), bool(r.get("pass")), r.get("details", {}).get("status", "")))
    return sorted(rows)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--validations", required=True, help="directory holding the reference's v*.py and vlib.py")
    ap.add_argument("--gen", required=True, help="the reference's scripts/gen_field.py")
    ap.add_argument("--out", required=True)
    ap.add_argument("--bin", default=BIN)
    ap.add_argument("--timeout", type=int, default=900, help="seconds per script")
    args = ap.parse_args(argv)
    os.makedirs(args.out, exist_ok=True)
    log = open(os.path.join(args.out, "runner.log"), "w")
    for name, cmd in battery(args.validations, args.gen, args.bin, args.out):
        log.write(f"== {name}: {' '.join(cmd)}\n")
        log.flush()
        try:
            r = subprocess.run(cmd, stdout=log, stderr=subprocess.STDOUT, timeout=args.timeout)
            log.write(f"-- exit {r.returncode}\n")
        except subprocess.TimeoutExpired:
            log.write(f"-- timed out after {args.timeout} s\n")
    log.close()
    rows = reports(args.out)
    for path, ok, status in rows:
        print(f"{path:60s} {'PASS' if ok else 'FAIL'} {status}")
    if not rows:
        print("no report.json written")
        return 1
    return 0 if all(ok for _, ok, _ in rows) else 1


if __name__ == "__main__":
    sys.exit(main())
