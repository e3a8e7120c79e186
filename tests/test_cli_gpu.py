"""The command-line drop-in on the GPU: the reference's V6 level-R bit-55 case
(ln32 field, seed 7; N=32, t 0.02, dt 5e-4, --kernel fast --scatter colored
--detect --snap 1, fault at step 10 in element (16,16,16)) run through
heat_solver_b200's entry point.  The files the reference's validation scripts
parse carry the reference's recorded values to their printed digits."""
import csv
import os

import numpy as np
import pytest

from mnhack8_b200 import _lib
from mnhack8_b200.fields import FieldSpec, make_field, write_field

pytestmark = pytest.mark.gpu


def test_v6_level_R_case_through_the_cli(tmp_path, golden):
    g = golden["v6"]["L2_b55"]
    sm = g["summary"]
    k, r, meta = make_field(FieldSpec(n=32, model="lognormal", sigma=1.0, L=0.125, seed=7))
    prefix = str(tmp_path / "ln32")
    write_field(prefix, k, r, meta)
    out = tmp_path / "out"
    rc = _lib.cli(["32", "0.02", "5e-4", prefix, str(out), "--kernel", "fast", "--scatter", "colored", "--detect",
                   "--snap", "1", "--tag", "det", "--fi", sm["fi_level"], sm["fi_step"], sm["fi_target"],
                   sm["fi_bit"]])
    assert rc == 0
    with open(out / "fi_trace_det.csv") as f:
        trace = list(csv.DictReader(f))
    assert len(trace) == len(g["trace"]) == 40
    assert set(g["trace"][0]) <= set(trace[0])           # every column the reference recorded
    for want, got in zip(g["trace"], trace):
        for key in ("step", "E_fault", "spread_F", "cg_A", "cg_F", "d2_resid_A", "d2_resid_F", "d3_tmin_F",
                    "d3_tmax_F"):
            assert got[key] == want[key], (want["step"], key)
        if want["step"] == sm["fi_step"]:
            assert got["d1_abft_F"] == want["d1_abft_F"]
    with open(out / "fi_summary_det.csv") as f:
        summary = list(csv.DictReader(f))[0]
    for key in ("fi_level", "fi_step", "fi_target", "fi_bit", "class", "E_fault_max", "step_at_max",
                "E_fault_int", "E_fault_final", "iters_delta_max", "d1_first", "d2_first", "d3_first",
                "detected_by", "mean_cg_iters_A", "kmin", "kmax", "target_on_boundary"):
        assert summary[key] == sm[key], key
    assert os.path.exists(out / "meta_det.txt")
    Tc = np.fromfile(out / "T_final_det_clean_rank0.bin")
    Tf = np.fromfile(out / "T_final_det_fault_rank0.bin")
    assert Tc.size == Tf.size == 33 ** 3
    assert np.linalg.norm(Tf - Tc) / np.linalg.norm(Tc) == pytest.approx(float(sm["E_fault_final"]), rel=1e-5)
