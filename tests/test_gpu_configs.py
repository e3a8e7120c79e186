"""GPU parity at the configurations the measurements are quoted on.

Each test runs a named workload through the C ABI and compares it with the CPU
oracle on the same seeded inputs:

* config 1 exactly: 8^3 unit-cube Q1 elements, homogeneous k = rho*c = 1,
  Dirichlet T = 0, Gaussian bump (sigma 0.15), implicit Euler dt = 1e-3 for 10
  steps, Jacobi-PCG rtol 1e-10, colored scatter, ABFT on, no injection -- the
  field, every step's CG count and the detector values d1, d2, tmin, tmax bit
  for bit (both the reference's dense element form and the wht form);
* the bench trajectory (config 2's problem: N=128, lognormal sigma 1,
  correlation 8 elements, seed 1, dt 1e-4, rtol 1e-10, ABFT on, source off):
  its first implicit-Euler steps bit for bit, through the records path
  (hs_run_case) and through the path the bench times (hs_advance);
* config 3's problem in the plain FP64 drop-in (N=256, lognormal sigma 1.5,
  correlation 16 elements, dt 1e-4, rtol 1e-8): one step, its CG count equal
  and the field within rel-L2 1e-10 (it is in fact compared bit for bit).

The PCG recurrence is het.cu:994-1039 and the step driver het.cu:1161-1162.
"""
import numpy as np
import pytest

from mnhack8_b200 import _lib
from mnhack8_b200.fields import FieldSpec, make_field
from tests.helpers import bits

pytestmark = pytest.mark.gpu


def _fields(N, model, **kw):
    k, r, _ = make_field(FieldSpec(n=N, model=model, **kw))
    return k.ravel(), r.ravel()


def _cmp_steps(got, want):
    assert len(got["steps"]) == len(want["steps"])
    for s, (a, b) in enumerate(zip(got["steps"], want["steps"])):
        assert a["cg_iters"] == b["cg_iters"], (s, a["cg_iters"], b["cg_iters"])
        for key in ("d1", "d2", "tmin", "tmax"):
            assert np.float64(a[key]).view(np.uint64) == np.float64(b[key]).view(np.uint64), (s, key, a[key], b[key])


@pytest.mark.parametrize("form", ["fast", "wht"])
def test_config1_exact(oracle, form):
    N, dt, steps = 8, 1e-3, 10
    k, r = _fields(N, "homogeneous", k=1.0, rhoc=1.0)
    assert np.all(k == 1.0) and np.all(r == 1.0)
    opts = dict(detect=True, ic="gaussian", ic_sigma=0.15)
    o = oracle.Oracle(N, dt, k, r, form=form, colored=True, **opts)
    g = _lib.Solver(N, dt, k, r, kernel=form, scatter="colored", rtol=1e-10, **opts)
    want = o.run_case(steps, snap_every=1, tol=1e-10)
    got = g.run_case(steps, snap_every=1, keep_reference=True)
    _cmp_steps(got, want)
    assert np.array_equal(bits(got["T"]), bits(want["T"]))
    assert all(s["d1"] <= 1e-10 for s in got["steps"])      # clean run: no detection
    g.close()


@pytest.fixture(scope="module")
def bench_problem():
    import bench

    N = bench.N_DEFAULT
    k, r = bench.make_field(N, 1)
    return N, k, r, bench


def test_bench_trajectory_first_steps(oracle, bench_problem):
    N, k, r, bench = bench_problem
    steps = 2
    opts = dict(detect=True, no_source=True, ic="gaussian", ic_sigma=bench.IC_SIGMA)
    o = oracle.Oracle(N, bench.DT, k, r, form="wht", colored=True, **opts)
    g = _lib.Solver(N, bench.DT, k, r, kernel="wht", scatter="colored", rtol=bench.RTOL, max_iter=500, **opts)
    want = o.run_case(steps, snap_every=1, tol=bench.RTOL)
    got = g.run_case(steps, snap_every=1, keep_reference=True)
    _cmp_steps(got, want)
    assert np.array_equal(bits(got["T"]), bits(want["T"]))
    # the path the bench times: the same steps without records
    it, _ = g.advance(steps, from_ic=True)
    assert it == sum(s["cg_iters"] for s in want["steps"])
    assert np.array_equal(bits(g.get_field()), bits(want["T"]))
    g.close()


def test_config3_fp64_one_step_N256(oracle):
    N, dt, rtol = 256, 1e-4, 1e-8
    k, r = _fields(N, "lognormal", mu=0.0, sigma=1.5, L=16.0 / N, seed=3)
    opts = dict(detect=True, no_source=True, ic="gaussian", ic_sigma=0.15)
    o = oracle.Oracle(N, dt, k, r, form="wht", colored=True, **opts)
    g = _lib.Solver(N, dt, k, r, kernel="wht", scatter="colored", rtol=rtol, max_iter=500, **opts)
    want = o.run_case(1, snap_every=0, tol=rtol)
    got = g.run_case(1, snap_every=0, keep_reference=True)
    assert got["steps"][0]["cg_iters"] == want["steps"][0]["cg_iters"]
    T, Tw = got["T"], want["T"]
    assert np.linalg.norm(T - Tw) <= 1e-10 * np.linalg.norm(Tw)
    assert np.array_equal(bits(T), bits(Tw))
    g.close()
