"""GPU parity: the library's kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.

The deterministic ("colored") path must reproduce the oracle bit for bit:
every operator value, every reduction, every PCG iterate and every
per-step detector value.  The nondeterministic atomic path is checked within
1e-12 relative.  Grid sizes cover ragged tiles (N-1 not a multiple of the
8x32x16 tile) and the degenerate grids N = 1, 2.
"""
import numpy as np
import pytest

from mnhack8_b200 import _lib
from tests.helpers import Dev, bits, field, random_field, random_nodes

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 5, 8, 17, 33, 40]


@pytest.fixture(scope="module")
def dev():
    return Dev()


def pair(oracle, N, form, detect=True, seed=0, dt=1e-3, scatter="colored", **kw):
    k, r = random_field(N, seed)
    o = oracle.Oracle(N, dt, k, r, form=form if form != "fast" else "fast", colored=(scatter == "colored"),
                      detect=detect, **kw)
    g = _lib.Solver(N, dt, k, r, kernel=form, scatter=scatter, detect=detect, **kw)
    return o, g


@pytest.mark.parametrize("form", ["wht", "fast", "gauss"])
@pytest.mark.parametrize("N", SIZES)
def test_apply_bitwise(oracle, dev, form, N):
    o, g = pair(oracle, N, form, seed=N)
    x = random_nodes(N, 100 + N)          # boundary values too (a G flip can put them there)
    xd, yd = dev.put(x), dev.zeros(o.Nn)
    for dt_eff in (o.dt, 0.0):
        rel = g.apply_ptr(xd.data_ptr(), yd.data_ptr(), dt_eff=dt_eff, project=True)
        y_ref, rel_ref = o.apply(x, dt_eff=dt_eff, project=True, d1=True)
        assert np.array_equal(bits(dev.get(yd)), bits(y_ref))
        assert np.float64(rel).view(np.uint64) == np.float64(rel_ref).view(np.uint64)
        # unprojected (node-parallel kernel)
        g.apply_ptr(xd.data_ptr(), yd.data_ptr(), dt_eff=dt_eff, project=False)
        y_ref, _ = o.apply(x, dt_eff=dt_eff, project=False, d1=False)
        assert np.array_equal(bits(dev.get(yd)), bits(y_ref))
    g.close()


@pytest.mark.parametrize("N", [64, 97, 130])
def test_apply_bitwise_split_tiles(oracle, dev, N):
    """Grids whose slab tiles split in every direction: halo rows, columns and
    planes shared between tiles, short last tiles."""
    lay = oracle.slab_layout(N)
    assert lay["tz"] < N + 1 and lay["ty"] < N + 1 and lay["cx"] < N + 1
    o, g = pair(oracle, N, "wht", seed=N)
    x = random_nodes(N, 200 + N)
    xd, yd = dev.put(x), dev.zeros(o.Nn)
    rel = g.apply_ptr(xd.data_ptr(), yd.data_ptr(), dt_eff=o.dt, project=True)
    y_ref, rel_ref = o.apply(x, dt_eff=o.dt, project=True, d1=True)
    assert np.array_equal(bits(dev.get(yd)), bits(y_ref))
    assert np.float64(rel).view(np.uint64) == np.float64(rel_ref).view(np.uint64)
    g.close()


@pytest.mark.parametrize("N", [128, 256])
def test_apply_bitwise_at_workload_sizes(oracle, dev, N):
    """The operator at the sizes the measurements use (the bench trajectory,
    N=128, and the precision configuration, N=256), on the bench's own seeded
    lognormal field: every value and the checksum bit for bit."""
    import bench

    k, r = bench.make_field(N, 1)
    o = oracle.Oracle(N, 1e-4, k, r, form="wht", colored=True, detect=True)
    g = _lib.Solver(N, 1e-4, k, r, kernel="wht", scatter="colored", detect=True)
    x = random_nodes(N, 300 + N)
    xd, yd = dev.put(x), dev.zeros(o.Nn)
    rel = g.apply_ptr(xd.data_ptr(), yd.data_ptr(), dt_eff=o.dt, project=True)
    y_ref, rel_ref = o.apply(x, dt_eff=o.dt, project=True, d1=True)
    assert np.array_equal(bits(dev.get(yd)), bits(y_ref))
    assert np.float64(rel).view(np.uint64) == np.float64(rel_ref).view(np.uint64)
    g.close()


def test_operator_symmetry_and_linearity_N256(dev):
    """Size-independent properties at N=256: on interior vectors the projected
    operator is symmetric (x.Ay = y.Ax to rounding) and linear
    (A(x + 2y) = Ax + 2Ay to rounding)."""
    import bench

    N = 256
    k, r = bench.make_field(N, 2)
    g = _lib.Solver(N, 1e-4, k, r, kernel="wht", scatter="colored", detect=True)
    x, y = random_nodes(N, 11, boundary=False), random_nodes(N, 12, boundary=False)
    xd, yd, zd = dev.put(x), dev.put(y), dev.put(x + 2.0 * y)
    ax, ay, az = dev.zeros(x.size), dev.zeros(x.size), dev.zeros(x.size)
    for src, dst in ((xd, ax), (yd, ay), (zd, az)):
        g.apply_ptr(src.data_ptr(), dst.data_ptr(), project=True)
    Ax, Ay, Az = dev.get(ax), dev.get(ay), dev.get(az)
    g.close()
    xAy, yAx = float(np.dot(x, Ay)), float(np.dot(y, Ax))
    assert abs(xAy - yAx) <= 1e-12 * max(abs(xAy), np.linalg.norm(x) * np.linalg.norm(Ay))
    lin = Ax + 2.0 * Ay
    assert np.linalg.norm(Az - lin) <= 1e-14 * np.linalg.norm(lin) * 8


def test_apply_rejects_overlap(oracle, dev):
    o, g = pair(oracle, 8, "wht")
    xd = dev.put(random_nodes(8, 1))
    with pytest.raises(_lib.HeatError) as e:
        g.apply_ptr(xd.data_ptr(), xd.data_ptr(), project=True)
    assert e.value.status == 1
    g.close()


@pytest.mark.parametrize("N", SIZES)
def test_setup_vectors_and_dot(oracle, dev, N):
    o, g = pair(oracle, N, "wht", seed=3 * N)
    vec = o.vectors()
    a, b = random_nodes(N, 7), random_nodes(N, 8)
    ad, bd = dev.put(a), dev.put(b)
    assert np.float64(g.dot_ptr(ad.data_ptr(), bd.data_ptr())).view(np.uint64) == np.float64(o.dot(a, b)).view(np.uint64)
    # Jacobi diagonal through the preconditioner: z = r / d with r = 1
    ones, zd = dev.put(np.ones(o.Nn)), dev.zeros(o.Nn)
    g.precond_ptr(ones.data_ptr(), zd.data_ptr())
    assert np.array_equal(bits(dev.get(zd)), bits(1.0 / vec["diag"]))
    g.close()


@pytest.mark.parametrize("form", ["wht", "fast"])
@pytest.mark.parametrize("N", [3, 8, 17, 33])
def test_build_rhs_and_pcg_bitwise(oracle, dev, form, N):
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=N)
    o = oracle.Oracle(N, 5e-4, k, r, form=form, detect=True, ic="gaussian", ic_sigma=0.15)
    g = _lib.Solver(N, 5e-4, k, r, kernel=form, scatter="colored", detect=True, ic="gaussian", ic_sigma=0.15)
    T = o.initial_condition()
    Td, bd = dev.put(T), dev.zeros(o.Nn)
    g.build_rhs_ptr(Td.data_ptr(), bd.data_ptr())
    b_ref = o.build_rhs(T)
    assert np.array_equal(bits(dev.get(bd)), bits(b_ref))
    xd = dev.put(T)
    it = g.pcg_ptr(bd.data_ptr(), xd.data_ptr(), 500, 1e-10)
    it_ref, x_ref, _ = o.pcg(b_ref, T, 500, 1e-10)
    assert it == it_ref
    assert np.array_equal(bits(dev.get(xd)), bits(x_ref))
    g.close()


@pytest.mark.parametrize("max_iter", [1, 2, 5, 6, 7, 9])
def test_pcg_iteration_cap_bitwise(oracle, dev, max_iter):
    """The CUDA graph runs several CG iterations per pass of its while body; a solve
    stopped by the iteration cap in the middle of a pass ends with the oracle's
    iterate and count."""
    N = 17
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=5)
    o = oracle.Oracle(N, 5e-4, k, r, form="wht", detect=True, ic="gaussian", ic_sigma=0.15)
    g = _lib.Solver(N, 5e-4, k, r, kernel="wht", scatter="colored", detect=True, ic="gaussian", ic_sigma=0.15)
    T = o.initial_condition()
    b_ref = o.build_rhs(T)
    bd, xd = dev.put(b_ref), dev.put(T)
    it = g.pcg_ptr(bd.data_ptr(), xd.data_ptr(), max_iter, 1e-14)
    it_ref, x_ref, _ = o.pcg(b_ref, T, max_iter, 1e-14)
    assert it == it_ref == max_iter
    assert np.array_equal(bits(dev.get(xd)), bits(x_ref))
    g.close()


def _cmp_records(got, want, E=True):
    for s, (a, b) in enumerate(zip(got["steps"], want["steps"])):
        assert a["cg_iters"] == b["cg_iters"], s
        for key in ("d1", "d2", "tmin", "tmax") + (("E", "spread") if E else ()):
            assert np.float64(a[key]).view(np.uint64) == np.float64(b[key]).view(np.uint64), (s, key, a[key], b[key])


@pytest.mark.parametrize("form", ["wht", "fast", "gauss"])
def test_run_case_and_faults_bitwise(oracle, form):
    """Full trajectories with detectors, the kept reference and every fault level."""
    N, steps = 12, 12
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=5)
    o = oracle.Oracle(N, 5e-4, k, r, form=form, detect=True)
    g = _lib.Solver(N, 5e-4, k, r, kernel=form, scatter="colored", detect=True)
    ref = o.run_case(steps, snap_every=1, keep_snaps=True)
    got = g.run_case(steps, snap_every=1, keep_reference=True)
    _cmp_records(got, ref, E=False)
    assert np.array_equal(bits(got["T"]), bits(ref["T"]))
    mid = 6 * 169 + 6 * 13 + 6
    faults = [("G", 3, mid, 55, 0), ("G", 3, 5, 62, 0), ("R", 4, 6 * 144 + 6 * 12 + 6, 51, 0),
              ("R", 4, 0, 63, 0), ("P", 2, mid, 52, 3), ("RV", 5, mid, 60, 1), ("AP", 7, mid, 55, 2),
              ("AP", 1, 7, 62, 0), ("P", 6, 3, 62, 0), ("RV", 2, mid, 62, 4)]
    for lv, st, tg, bt, it in faults:
        fi = (_lib.LEVELS[lv], st, tg, bt, it)
        want = o.run_case(steps, snap_every=1, fi=fi, ref_snaps=ref["snaps"])
        have = g.run_case(steps, snap_every=1, fi=fi)
        _cmp_records(have, want)
        assert np.array_equal(bits(have["T"]), bits(want["T"])), (lv, st, tg, bt, it)
        assert have["nonfinite"] == want["nonfinite"]
    g.close()


def test_colored_run_to_run_bitwise(oracle):
    k, r = field(33, "lognormal", sigma=1.0, L=0.125, seed=7)
    g = _lib.Solver(33, 1e-3, k, r, kernel="wht", scatter="colored", detect=True, ic="gaussian", ic_sigma=0.15)
    a = g.run_case(6, snap_every=1, keep_reference=True)
    b = g.run_case(6, snap_every=1)
    assert np.array_equal(bits(a["T"]), bits(b["T"]))
    assert all(s["E"] == 0.0 for s in b["steps"])
    g.close()


@pytest.mark.parametrize("form", ["wht", "fast"])
def test_atomic_within_tolerance(oracle, dev, form):
    N = 17
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=11)
    o = oracle.Oracle(N, 5e-4, k, r, form=form, detect=True)
    g = _lib.Solver(N, 5e-4, k, r, kernel=form, scatter="atomic", detect=True)
    x = random_nodes(N, 3)
    xd, yd = dev.put(x), dev.zeros(o.Nn)
    rel = g.apply_ptr(xd.data_ptr(), yd.data_ptr(), project=True)
    y_ref, rel_ref = o.apply(x, project=True, d1=True)
    y = dev.get(yd)
    assert np.linalg.norm(y - y_ref) <= 1e-13 * np.linalg.norm(y_ref)
    assert rel < 1e-13
    ref = o.run_case(10, snap_every=2)
    got = g.run_case(10, snap_every=2, keep_reference=True)
    assert [s["cg_iters"] for s in got["steps"]] == [s["cg_iters"] for s in ref["steps"]]
    assert np.linalg.norm(got["T"] - ref["T"]) <= 1e-12 * np.linalg.norm(ref["T"])
    g.close()


def test_solve_host_end_to_end(oracle):
    N = 16
    k, r = field(N, "lognormal", sigma=1.0, L=0.125, seed=1)
    o = oracle.Oracle(N, 1e-4, k, r, form="wht", no_source=True, ic="gaussian", ic_sigma=0.15)
    g = _lib.Solver(N, 1e-4, k, r, kernel="wht", scatter="colored", no_source=True, ic="gaussian", ic_sigma=0.15,
                    rtol=1e-10)
    ref = o.run_case(5, snap_every=0, tol=1e-10)
    T0 = o.initial_condition()
    T, tot, ms = g.solve_host(T0, 5)
    assert tot == sum(s["cg_iters"] for s in ref["steps"])
    assert np.array_equal(bits(T), bits(ref["T"]))
    g.close()


def test_diag_cg_log(oracle):
    N = 10
    k, r = field(N, "lognormal", sigma=1.0, L=0.25, seed=4)
    o = oracle.Oracle(N, 1e-3, k, r, form="wht")
    g = _lib.Solver(N, 1e-3, k, r, kernel="wht", scatter="colored")
    it, lg = g.diag_cg(500, 1e-8)
    T = o.initial_condition()
    it_ref, _, lr = o.pcg(o.build_rhs(T), T, 500, 1e-8)
    assert it == it_ref
    assert np.array_equal(bits(lg["rel"]), bits(lr["rel"]))
    assert np.array_equal(bits(lg["alpha"]), bits(lr["alpha"]))
    assert np.array_equal(bits(lg["beta"]), bits(lr["beta"]))
    assert np.float64(lg["rel0"]).view(np.uint64) == np.float64(lr["rel0"]).view(np.uint64)
    g.close()
