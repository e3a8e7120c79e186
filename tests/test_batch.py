"""Batched mixed-precision solves (hs_batch_*).

* Accuracy: FP32 inner solves with FP64 defect correction reach the FP64
  solution (the oracle's PCG to 1e-13) within the outer tolerance.
* Isolation: every reduction of an instance runs over its own tiles and
  blocks in a fixed order, and its convergence decisions are its own, so an
  instance gives the same bits alone, in a mixed batch, and when it joins a
  batch that is already running (continuous batching).
"""
import numpy as np
import pytest

from mnhack8_b200 import _lib
from tests.helpers import bits, field

pytestmark = pytest.mark.gpu


def gaussian_T0(oracle, N, dt, k, r):
    return oracle.Oracle(N, dt, k, r, form="wht", no_source=True, ic="gaussian", ic_sigma=0.15).initial_condition()


def test_mixed_precision_reaches_fp64(oracle):
    N, dt, steps = 12, 5e-4, 6
    k, r = field(N, "lognormal", sigma=1.5, L=0.25, seed=4)
    o = oracle.Oracle(N, dt, k, r, form="wht", no_source=True, ic="gaussian", ic_sigma=0.15)
    ref = o.run_case(steps, snap_every=0, tol=1e-13)["T"]
    b = _lib.Batch(rtol=1e-10, inner_tol=1e-4)
    s = b.add(N, dt, k, r, T0=o.initial_condition(), steps=steps)
    while b.step()[0]:
        pass
    T = b.field(s)
    inf = b.info(s)
    b.close()
    assert np.linalg.norm(T - ref) <= 1e-9 * np.linalg.norm(ref)
    assert inf["steps_done"] == steps and inf["rel_residual"] < 1e-10
    assert inf["outer_iters"] >= steps and inf["inner_iters"] > 0
    assert inf["d1_max64"] < 1e-10                 # clean FP64 applies pass the ABFT test
    assert 0.0 < inf["d1_max32"] < 1e-4            # FP32 applies: their rounding noise floor


CASES = [(8, 1e-3, 4, 1), (13, 5e-4, 6, 2), (20, 2e-4, 3, 3), (5, 2e-3, 5, 4)]


def _solo(oracle, N, dt, steps, seed, planes=0):
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=seed)
    b = _lib.Batch(rtol=1e-8, tile_planes=planes)
    s = b.add(N, dt, k, r, T0=gaussian_T0(oracle, N, dt, k, r), steps=steps)
    while b.step()[0]:
        pass
    T, inf = b.field(s), b.info(s)
    b.close()
    return T, inf


def test_alone_equals_in_the_mix(oracle):
    solo = [_solo(oracle, *c) for c in CASES]
    b = _lib.Batch(rtol=1e-8)
    slots = []
    for N, dt, steps, seed in CASES:
        k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=seed)
        slots.append(b.add(N, dt, k, r, T0=gaussian_T0(oracle, N, dt, k, r), steps=steps))
    n_steps = 0
    while b.step()[0]:
        n_steps += 1
    assert n_steps == max(c[2] for c in CASES)
    for s, (T, inf) in zip(slots, solo):
        assert np.array_equal(bits(b.field(s)), bits(T))
        got = b.info(s)
        assert (got["inner_iters"], got["outer_iters"]) == (inf["inner_iters"], inf["outer_iters"])
    b.close()


def test_join_running_batch_and_reuse_slot(oracle):
    (N1, dt1, st1, sd1), (N2, dt2, st2, sd2), (N3, dt3, st3, sd3) = CASES[1], CASES[0], CASES[2]
    ref1, ref2, ref3 = (_solo(oracle, *CASES[1])[0], _solo(oracle, *CASES[0])[0], _solo(oracle, *CASES[2])[0])
    b = _lib.Batch(rtol=1e-8)
    k, r = field(N1, "lognormal", sigma=1.0, L=0.25, seed=sd1)
    a = b.add(N1, dt1, k, r, T0=gaussian_T0(oracle, N1, dt1, k, r), steps=st1)
    b.step(); b.step()
    k, r = field(N2, "lognormal", sigma=1.0, L=0.25, seed=sd2)
    c = b.add(N2, dt2, k, r, T0=gaussian_T0(oracle, N2, dt2, k, r), steps=st2)   # joins mid-run
    while b.info(c)["steps_left"] > 0:
        b.step()
    assert np.array_equal(bits(b.field(c)), bits(ref2))
    b.remove(c)
    k, r = field(N3, "lognormal", sigma=1.0, L=0.25, seed=sd3)
    d = b.add(N3, dt3, k, r, T0=gaussian_T0(oracle, N3, dt3, k, r), steps=st3)  # reuses the slot
    assert d == c
    while b.step()[0]:
        pass
    assert np.array_equal(bits(b.field(a)), bits(ref1))
    assert np.array_equal(bits(b.field(d)), bits(ref3))
    b.close()


def test_admission_during_a_step_in_flight(oracle):
    """hs_batch_step_begin / _end: instances added while a step runs join at
    the next step, a slot removed during a step is not reused before it ends,
    and every instance gives the bits of its solo run."""
    (N1, dt1, st1, sd1), (N2, dt2, st2, sd2), (N3, dt3, st3, sd3) = CASES[1], CASES[0], CASES[2]
    ref1, ref2, ref3 = (_solo(oracle, *CASES[1])[0], _solo(oracle, *CASES[0])[0], _solo(oracle, *CASES[2])[0])
    b = _lib.Batch(rtol=1e-8)
    k, r = field(N1, "lognormal", sigma=1.0, L=0.25, seed=sd1)
    a = b.add(N1, dt1, k, r, T0=gaussian_T0(oracle, N1, dt1, k, r), steps=st1)
    k, r = field(N2, "lognormal", sigma=1.0, L=0.25, seed=sd2)
    c = b.add(N2, dt2, k, r, T0=gaussian_T0(oracle, N2, dt2, k, r), steps=st2)
    assert b.step_begin() == 2
    with pytest.raises(_lib.HeatError):
        b.step_begin()                                  # one step in flight at a time
    k, r = field(N3, "lognormal", sigma=1.0, L=0.25, seed=sd3)
    d = b.add(N3, dt3, k, r, T0=gaussian_T0(oracle, N3, dt3, k, r), steps=st3)   # set up beside the step
    assert b.step_end()[0] == 2                         # d was not part of it
    assert b.info(d)["steps_done"] == 0 and b.info(a)["steps_done"] == 1
    while b.info(c)["steps_left"] > 0:
        b.step_begin()
        b.step_end()
    assert np.array_equal(bits(b.field(c)), bits(ref2))
    b.step_begin()
    b.remove(c)                                         # freed after the step; its slot is held
    e = b.add(N2, dt2, np.ones(N2 ** 3), np.ones(N2 ** 3), steps=1)
    assert e not in (a, c, d)
    b.step_end()
    b.remove(e)
    while b.step()[0]:
        pass
    assert np.array_equal(bits(b.field(a)), bits(ref1))
    assert np.array_equal(bits(b.field(d)), bits(ref3))
    assert b.step_end() == (0, 0.0)                     # nothing in flight
    b.close()


def test_tile_depth_changes_only_rounding(oracle):
    T1, _ = _solo(oracle, 20, 2e-4, 3, 3, planes=0)
    T4, _ = _solo(oracle, 20, 2e-4, 3, 3, planes=5)
    assert np.linalg.norm(T1 - T4) <= 1e-7 * np.linalg.norm(T1)


def test_bad_arguments():
    b = _lib.Batch()
    with pytest.raises(_lib.HeatError):
        b.add(0, 1e-3, np.ones(1), np.ones(1))
    with pytest.raises(_lib.HeatError):
        b.remove(3)
    assert b.step() == (0, 0.0)
    b.close()


def test_inner_fault_fires_is_detected_and_corrected(oracle):
    """A flip in an FP32 inner vector fires once, an exponent flip of Ap
    shows in the FP32 checksum, and the FP64 defect correction still brings
    the step to the clean answer; a site past the inner solve never fires."""
    N, dt, steps = 12, 5e-4, 3
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=9)
    T0 = gaussian_T0(oracle, N, dt, k, r)
    b = _lib.Batch(rtol=1e-8)
    clean = b.add(N, dt, k, r, T0=T0, steps=steps)
    hit = b.add(N, dt, k, r, T0=T0, steps=steps)
    miss = b.add(N, dt, k, r, T0=T0, steps=steps)
    mid = 6 * 169 + 6 * 13 + 6
    b.arm_fault(hit, "AP", 1, 1, 2, mid, 29)        # exponent bit of Ap32
    b.arm_fault(miss, "P", 1, 1, 10000, mid, 29)    # iteration never reached
    while b.step()[0]:
        pass
    c, h, m = b.info(clean), b.info(hit), b.info(miss)
    assert h["fault_fired"] == 1 and m["fault_fired"] == 0 and c["fault_fired"] == 0
    assert h["d1_max32"] > 1e3 * c["d1_max32"]
    Tc, Th = b.field(clean), b.field(hit)
    assert np.linalg.norm(Th - Tc) <= 1e-7 * np.linalg.norm(Tc)
    assert h["rel_residual"] < 1e-8 and h["stalls"] == 0
    assert np.array_equal(bits(b.field(miss)), bits(Tc))
    b.close()


def test_boundary_and_nonfinite_faults_heal(oracle):
    """Flips the FP64 residual cannot see (a Dirichlet entry) or that make the
    inner solve non-finite (an r exponent flip) leave the answer at the clean
    one: corrections never touch Dirichlet nodes, and a non-finite inner solve
    is discarded and solved again."""
    N, dt, steps = 12, 5e-4, 3
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=9)
    T0 = gaussian_T0(oracle, N, dt, k, r)
    b = _lib.Batch(rtol=1e-8)
    clean = b.add(N, dt, k, r, T0=T0, steps=steps)
    bnd = b.add(N, dt, k, r, T0=T0, steps=steps)
    nf = b.add(N, dt, k, r, T0=T0, steps=steps)
    b.arm_fault(bnd, "P", 1, 1, 3, 5, 30)                        # node 5 lies on the x = 0 face
    b.arm_fault(nf, "RV", 1, 1, 3, 6 * 169 + 6 * 13 + 6, 30)     # r exponent flip: z overflows
    while b.step()[0]:
        pass
    Tc = b.field(clean)
    for s in (bnd, nf):
        inf = b.info(s)
        assert inf["fault_fired"] == 1 and inf["stalls"] == 0 and inf["rel_residual"] < 1e-8
        T = b.field(s)
        assert np.all(np.isfinite(T))
        assert np.linalg.norm(T - Tc) <= 1e-7 * np.linalg.norm(Tc)
    assert b.info(nf)["inner_faults"] >= 1
    b.close()


_DIRECT = r"""
import sys, hashlib
sys.path.insert(0, {root!r})
import numpy as np
from mnhack8_b200 import _lib
from tests.helpers import field
k, r = field(10, "lognormal", sigma=1.0, L=0.25, seed=6)
b = _lib.Batch(rtol=1e-8)
s = b.add(10, 1e-3, k, r, T0=_lib.gaussian_ic(10, 0.15), steps=3)
while b.step()[0]:
    pass
print(hashlib.sha256(b.field(s).tobytes()).hexdigest(), b.info(s)["inner_iters"])
"""


def test_direct_launches_equal_graph():
    """HS_GRAPH=0 (direct launches, for profilers) computes the same bits as the graph."""
    import hashlib
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    k, r = field(10, "lognormal", sigma=1.0, L=0.25, seed=6)
    b = _lib.Batch(rtol=1e-8)
    s = b.add(10, 1e-3, k, r, T0=_lib.gaussian_ic(10, 0.15), steps=3)
    while b.step()[0]:
        pass
    want = f"{hashlib.sha256(b.field(s).tobytes()).hexdigest()} {b.info(s)['inner_iters']}"
    b.close()
    env = dict(os.environ, HS_GRAPH="0")
    out = subprocess.run([sys.executable, "-c", _DIRECT.format(root=root)], env=env, capture_output=True,
                         text=True, timeout=300, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().splitlines()[-1] == want


def test_extrapolated_start_same_answer_fewer_iterations(oracle):
    """Starting each step from 2 T - T_prev changes where the solve starts, not
    what it converges to: the fields agree within the tolerance and the inner
    iterations do not grow."""
    N, dt, steps = 16, 5e-4, 8
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=12)
    T0 = gaussian_T0(oracle, N, dt, k, r)
    out = {}
    for ex in (False, True):
        b = _lib.Batch(rtol=1e-9, extrapolate=ex)
        s = b.add(N, dt, k, r, T0=T0, steps=steps)
        while b.step()[0]:
            pass
        out[ex] = (b.field(s), b.info(s))
        b.close()
    (T0f, i0), (T1f, i1) = out[False], out[True]
    assert np.linalg.norm(T1f - T0f) <= 1e-8 * np.linalg.norm(T0f)
    assert i1["rel_residual"] < 1e-9 and i0["rel_residual"] < 1e-9
    assert i1["inner_iters"] <= i0["inner_iters"]
