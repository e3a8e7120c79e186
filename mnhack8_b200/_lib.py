"""ctypes binding of libheat_b200.so (the C ABI in include/heat_b200.h).

The library is the only compute path: if the shared object is missing or does
not load, every call raises.  There is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libheat_b200.so")
CLI_PATH = os.path.join(HERE, "heat_solver_b200")

KERNELS = {"fast": 0, "gauss": 1, "wht": 2}
SCATTERS = {"atomic": 0, "colored": 1}
LEVELS = {"G": 1, "R": 2, "H": 3, "P": 5, "RV": 6, "AP": 7}
STATUS = {0: "HS_OK", 1: "HS_ERR_ARG", 2: "HS_ERR_MATRIX", 3: "HS_ERR_IO", 4: "HS_ERR_CUDA", 5: "HS_ERR_STATE"}

# every function the header declares (checked by the CPU tests)
EXPORTS = [
    "hs_default_options", "hs_last_error", "hs_api_version", "hs_get_layout", "hs_load_fields", "hs_create",
    "hs_destroy", "hs_num_nodes", "hs_field_stats", "hs_apply", "hs_precond", "hs_build_rhs", "hs_dot", "hs_pcg",
    "hs_arm_fi", "hs_run_case", "hs_verify", "hs_solve_host", "hs_diag_cg", "hs_set_dump", "hs_set_case_tag",
    "hs_target_on_boundary", "hs_classify", "hs_cli_main", "hs_advance", "hs_set_field", "hs_get_field",
    "hs_time_kernel", "hs_dot_noalloc", "hs_campaign", "hs_batch_default_options", "hs_batch_create",
    "hs_batch_destroy", "hs_batch_add", "hs_batch_add_lognormal", "hs_field_lognormal", "hs_batch_arm_flip", "hs_batch_arm_fault", "hs_batch_remove", "hs_batch_step",
    "hs_batch_step_begin", "hs_batch_step_end", "hs_batch_info", "hs_batch_get_field", "hs_gaussian_ic",
]


class Options(C.Structure):
    _fields_ = [("N", C.c_int), ("dt", C.c_double), ("kernel", C.c_int), ("scatter", C.c_int),
                ("detect", C.c_int), ("verify", C.c_int), ("no_source", C.c_int), ("ic_mode", C.c_int),
                ("ic_sigma", C.c_double), ("rtol", C.c_double), ("max_iter", C.c_int), ("device", C.c_int)]


class FiSpec(C.Structure):
    _fields_ = [("level", C.c_int), ("step", C.c_int), ("target", C.c_longlong), ("bit", C.c_int),
                ("iter", C.c_int), ("rank", C.c_int)]


class StepRecord(C.Structure):
    _fields_ = [("cg_iters", C.c_int), ("snap", C.c_int), ("d1", C.c_double), ("d2", C.c_double),
                ("tmin", C.c_double), ("tmax", C.c_double), ("E", C.c_double), ("spread", C.c_double),
                ("solve_ms", C.c_double)]


class LayoutInfo(C.Structure):
    _fields_ = [("cx", C.c_int), ("ty", C.c_int), ("tz", C.c_int), ("rt", C.c_int), ("bpt", C.c_int),
                ("kf", C.c_int)]


class TwinSummary(C.Structure):
    _fields_ = [("E_floor_max", C.c_double), ("E_floor_final", C.c_double), ("E_fault_max", C.c_double),
                ("E_fault_int", C.c_double), ("E_fault_final", C.c_double), ("thr", C.c_double),
                ("spread_at_max", C.c_double), ("spread_final", C.c_double), ("step_at_max", C.c_int),
                ("iters_delta_max", C.c_int), ("d1_first", C.c_int), ("d2_first", C.c_int),
                ("d3_first", C.c_int), ("pad", C.c_int), ("d1_max", C.c_double), ("d2_max", C.c_double),
                ("d1_max_A", C.c_double), ("d2_max_A", C.c_double), ("cls", C.c_char * 16),
                ("detected_by", C.c_char * 16)]


class FlipRecord(C.Structure):
    _fields_ = [("step", C.c_int), ("iter", C.c_int), ("level", C.c_int), ("bit", C.c_int), ("idx", C.c_longlong),
                ("nonfinite", C.c_int), ("iters_total_delta", C.c_int), ("summary", TwinSummary)]


class BatchOptions(C.Structure):
    _fields_ = [("rtol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int), ("max_inner", C.c_int),
                ("detect", C.c_int), ("tile_planes", C.c_int), ("device", C.c_int), ("extrapolate", C.c_int)]


class BatchFault(C.Structure):
    _fields_ = [("level", C.c_int), ("step", C.c_int), ("outer", C.c_int), ("iter", C.c_int), ("idx", C.c_longlong),
                ("bit", C.c_int), ("pad", C.c_int)]


class BatchInstInfo(C.Structure):
    _fields_ = [("N", C.c_int), ("steps_done", C.c_int), ("steps_left", C.c_int), ("pad", C.c_int),
                ("inner_iters", C.c_longlong), ("outer_iters", C.c_longlong), ("applies32", C.c_longlong),
                ("applies64", C.c_longlong), ("tiles", C.c_longlong), ("fault_fired", C.c_int),
                ("stalls", C.c_int), ("inner_faults", C.c_int), ("pad2", C.c_int), ("rel_residual", C.c_double),
                ("d1_max64", C.c_double), ("d1_max32", C.c_double)]


_lib = None


class HeatError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Load libheat_b200.so (raises if it is absent: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mnhack8_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
    pd = C.POINTER(C.c_double)
    L.hs_default_options.argtypes = [C.POINTER(Options)]
    L.hs_last_error.restype = C.c_char_p
    L.hs_api_version.restype = i
    L.hs_get_layout.argtypes = [i, C.POINTER(LayoutInfo)]
    L.hs_load_fields.restype = i
    L.hs_load_fields.argtypes = [C.c_char_p, i, vp, vp]
    L.hs_create.restype = i
    L.hs_create.argtypes = [C.POINTER(Options), vp, vp, C.POINTER(vp)]
    L.hs_destroy.argtypes = [vp]
    L.hs_num_nodes.restype = ll
    L.hs_num_nodes.argtypes = [vp]
    L.hs_field_stats.restype = i
    L.hs_field_stats.argtypes = [vp, vp]
    L.hs_apply.restype = i
    L.hs_apply.argtypes = [vp, vp, vp, d, i, i, pd]
    L.hs_precond.restype = i
    L.hs_precond.argtypes = [vp, vp, vp]
    L.hs_build_rhs.restype = i
    L.hs_build_rhs.argtypes = [vp, vp, vp]
    L.hs_dot.restype = i
    L.hs_dot.argtypes = [vp, vp, vp, pd]
    L.hs_pcg.restype = i
    L.hs_pcg.argtypes = [vp, vp, vp, i, d, C.POINTER(i)]
    L.hs_arm_fi.restype = i
    L.hs_arm_fi.argtypes = [vp, C.POINTER(FiSpec)]
    L.hs_run_case.restype = i
    L.hs_run_case.argtypes = [vp, i, i, C.POINTER(FiSpec), i, i, C.POINTER(StepRecord), vp, C.POINTER(i)]
    L.hs_verify.restype = i
    L.hs_verify.argtypes = [vp, i, pd, C.POINTER(ll), pd]
    L.hs_solve_host.restype = i
    L.hs_solve_host.argtypes = [vp, vp, vp, i, C.POINTER(ll), pd]
    L.hs_diag_cg.restype = i
    L.hs_diag_cg.argtypes = [vp, i, d, pd, vp, vp, vp, i, C.POINTER(i)]
    L.hs_set_dump.restype = i
    L.hs_set_dump.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.hs_set_case_tag.restype = i
    L.hs_set_case_tag.argtypes = [vp, C.c_char_p]
    L.hs_target_on_boundary.restype = i
    L.hs_target_on_boundary.argtypes = [vp, C.POINTER(FiSpec)]
    L.hs_classify.restype = i
    L.hs_classify.argtypes = [C.POINTER(StepRecord), C.POINTER(StepRecord), C.POINTER(StepRecord), i, i, i, d, d,
                              i, C.POINTER(TwinSummary)]
    L.hs_advance.restype = i
    L.hs_advance.argtypes = [vp, i, i, C.POINTER(ll), pd]
    L.hs_set_field.restype = i
    L.hs_set_field.argtypes = [vp, vp]
    L.hs_get_field.restype = i
    L.hs_get_field.argtypes = [vp, vp]
    L.hs_time_kernel.restype = i
    L.hs_time_kernel.argtypes = [vp, i, i, pd]
    L.hs_dot_noalloc.restype = i
    L.hs_dot_noalloc.argtypes = [i, vp, vp, vp]
    L.hs_batch_default_options.restype = None
    L.hs_batch_default_options.argtypes = [C.POINTER(BatchOptions)]
    L.hs_batch_create.restype = i
    L.hs_batch_create.argtypes = [C.POINTER(BatchOptions), C.POINTER(vp)]
    L.hs_batch_destroy.restype = None
    L.hs_batch_destroy.argtypes = [vp]
    L.hs_batch_add.restype = i
    L.hs_batch_add.argtypes = [vp, i, C.c_double, vp, vp, vp, i, C.POINTER(i)]
    L.hs_batch_add_lognormal.restype = i
    L.hs_batch_add_lognormal.argtypes = [vp, i, C.c_double, C.c_double, C.c_double, C.c_double, C.c_ulonglong,
                                         C.c_double, vp, i, C.POINTER(i)]
    L.hs_field_lognormal.restype = i
    L.hs_field_lognormal.argtypes = [i, C.c_double, C.c_double, C.c_double, C.c_ulonglong, C.c_double, vp, vp]
    L.hs_batch_arm_flip.restype = i
    L.hs_batch_arm_flip.argtypes = [vp, i, i, C.c_longlong, i]
    L.hs_batch_arm_fault.restype = i
    L.hs_batch_arm_fault.argtypes = [vp, i, C.POINTER(BatchFault)]
    L.hs_batch_remove.restype = i
    L.hs_batch_remove.argtypes = [vp, i]
    L.hs_batch_step.restype = i
    L.hs_batch_step.argtypes = [vp, C.POINTER(i), pd]
    L.hs_batch_step_begin.restype = i
    L.hs_batch_step_begin.argtypes = [vp, C.POINTER(i)]
    L.hs_batch_step_end.restype = i
    L.hs_batch_step_end.argtypes = [vp, C.POINTER(i), pd]
    L.hs_batch_info.restype = i
    L.hs_batch_info.argtypes = [vp, i, C.POINTER(BatchInstInfo)]
    L.hs_batch_get_field.restype = i
    L.hs_batch_get_field.argtypes = [vp, i, vp]
    L.hs_gaussian_ic.restype = i
    L.hs_gaussian_ic.argtypes = [i, C.c_double, vp]
    L.hs_campaign.restype = i
    L.hs_campaign.argtypes = [vp, i, i, i, C.c_ulonglong, i, C.POINTER(StepRecord), C.POINTER(FlipRecord)]
    L.hs_cli_main.restype = i
    L.hs_cli_main.argtypes = [i, C.POINTER(C.c_char_p)]
    _lib = L
    return L


def check(status):
    if status != 0:
        raise HeatError(status, lib().hs_last_error().decode(errors="replace"))


def layout(N=128):
    """Canonical reduction orders the library uses for an N-element grid."""
    li = LayoutInfo()
    lib().hs_get_layout(int(N), C.byref(li))
    return dict(cx=li.cx, ty=li.ty, tz=li.tz, rt=li.rt, bpt=li.bpt, kf=li.kf)


def _host(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fi_spec(fi):
    """(level, step, target, bit[, iter]) tuple or dict -> FiSpec (None -> None)."""
    if fi is None:
        return None
    if isinstance(fi, dict):
        lv = fi["level"]
        return FiSpec(LEVELS.get(lv, lv), fi["step"], fi["target"], fi["bit"], fi.get("iter", 0), fi.get("rank", 0))
    lv, st, tg, bt = fi[:4]
    it = fi[4] if len(fi) > 4 else 0
    return FiSpec(LEVELS.get(lv, lv), st, tg, bt, it, 0)


class Solver:
    """One problem instance on the GPU (the reference's HeatOperator + PCG)."""

    def __init__(self, N, dt, k, rhoc, kernel="wht", scatter="colored", detect=False, verify=False,
                 no_source=False, ic="zero", ic_sigma=0.1, rtol=1e-8, max_iter=500, device=0):
        L = lib()
        o = Options()
        L.hs_default_options(C.byref(o))
        o.N, o.dt = int(N), float(dt)
        o.kernel = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        o.scatter = SCATTERS[scatter] if isinstance(scatter, str) else int(scatter)
        o.detect, o.verify, o.no_source = int(detect), int(verify), int(no_source)
        o.ic_mode = 1 if ic == "gaussian" else 0
        o.ic_sigma, o.rtol, o.max_iter, o.device = float(ic_sigma), float(rtol), int(max_iter), int(device)
        self.opts = o
        self.N = int(N)
        self.Nn = (self.N + 1) ** 3
        kk, rr = _host(k).ravel(), _host(rhoc).ravel()
        if kk.size != self.N ** 3 or rr.size != self.N ** 3:
            raise ValueError("field size mismatch")
        h = C.c_void_p()
        check(L.hs_create(C.byref(o), kk.ctypes.data, rr.ctypes.data, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().hs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def stats(self):
        out = np.zeros(9)
        check(lib().hs_field_stats(self._h, out.ctypes.data))
        return dict(kmin=out[0], kmax=out[1], rhocmin=out[2], rhocmax=out[3], matrix_errors=out[4:].copy())

    # ---- device-pointer operator API (ints are device addresses) ----
    def apply_ptr(self, x_dev, y_dev, dt_eff=None, allow_fi=False, project=True):
        rel = C.c_double(-1.0)
        check(lib().hs_apply(self._h, x_dev, y_dev, self.opts.dt if dt_eff is None else float(dt_eff),
                             int(allow_fi), int(project), C.byref(rel)))
        return rel.value

    def build_rhs_ptr(self, T_dev, b_dev):
        check(lib().hs_build_rhs(self._h, T_dev, b_dev))

    def precond_ptr(self, r_dev, z_dev):
        check(lib().hs_precond(self._h, r_dev, z_dev))

    def dot_ptr(self, x_dev, y_dev):
        out = C.c_double()
        check(lib().hs_dot(self._h, x_dev, y_dev, C.byref(out)))
        return out.value

    def pcg_ptr(self, b_dev, x_dev, max_iter=500, tol=1e-8):
        it = C.c_int()
        check(lib().hs_pcg(self._h, b_dev, x_dev, int(max_iter), float(tol), C.byref(it)))
        return it.value

    def arm_fi(self, fi):
        spec = fi_spec(fi)
        check(lib().hs_arm_fi(self._h, C.byref(spec) if spec is not None else None))

    # ---- trajectories ----
    def run_case(self, n_steps, snap_every=5, fi=None, reproject=False, keep_reference=False, want_T=True):
        recs = (StepRecord * max(n_steps, 1))()
        T = np.zeros(self.Nn) if want_T else None
        nf = C.c_int(0)
        spec = fi_spec(fi)
        check(lib().hs_run_case(self._h, int(n_steps), int(snap_every), C.byref(spec) if spec is not None else None,
                                int(reproject), int(keep_reference), recs, T.ctypes.data if T is not None else None,
                                C.byref(nf)))
        steps = [dict(cg_iters=r.cg_iters, snap=r.snap, d1=r.d1, d2=r.d2, tmin=r.tmin, tmax=r.tmax, E=r.E,
                      spread=r.spread, solve_ms=r.solve_ms) for r in recs[:n_steps]]
        return dict(T=T, steps=steps, nonfinite=nf.value, records=recs)

    def campaign(self, n_steps, snap_every, n_flips, seed, vectors=("P", "RV", "AP")):
        """Seeded single-bit-flip campaign (hs_campaign): the clean run's step
        records and one dict per flip (site and twin-run summary)."""
        mask = sum({"P": 1, "RV": 2, "AP": 4}[v] for v in vectors)
        clean = (StepRecord * max(n_steps, 1))()
        flips = (FlipRecord * max(n_flips, 1))()
        check(lib().hs_campaign(self._h, int(n_steps), int(snap_every), int(n_flips), C.c_ulonglong(seed), mask,
                                clean, flips))
        steps = [dict(cg_iters=r.cg_iters, snap=r.snap, d1=r.d1, d2=r.d2, tmin=r.tmin, tmax=r.tmax, E=r.E,
                      spread=r.spread, solve_ms=r.solve_ms) for r in clean[:n_steps]]
        out = []
        for r in flips[:n_flips]:
            sm = r.summary
            summ = {name: (getattr(sm, name).decode() if name in ("cls", "detected_by") else getattr(sm, name))
                    for name, _ in TwinSummary._fields_ if name != "pad"}
            out.append(dict(step=r.step, iter=r.iter, level=r.level, bit=r.bit, idx=r.idx, nonfinite=r.nonfinite,
                            iters_total_delta=r.iters_total_delta, summary=summ))
        return steps, out

    def verify(self, n_steps):
        rel, ms = C.c_double(), C.c_double()
        tot = C.c_longlong()
        check(lib().hs_verify(self._h, int(n_steps), C.byref(rel), C.byref(tot), C.byref(ms)))
        return rel.value, tot.value, ms.value

    def solve_host(self, T0, n_steps):
        T0 = _host(T0)
        T = np.empty(self.Nn)
        tot, ms = C.c_longlong(), C.c_double()
        check(lib().hs_solve_host(self._h, T0.ctypes.data, T.ctypes.data, int(n_steps), C.byref(tot), C.byref(ms)))
        return T, tot.value, ms.value

    def set_field(self, T):
        T = _host(T)
        check(lib().hs_set_field(self._h, T.ctypes.data))

    def get_field(self):
        T = np.empty(self.Nn)
        check(lib().hs_get_field(self._h, T.ctypes.data))
        return T

    def advance(self, n_steps, from_ic=False):
        """n_steps device-resident steps (optionally restarting from the initial
        condition kept on the device); returns (total CG iterations, device ms)."""
        tot, ms = C.c_longlong(), C.c_double()
        check(lib().hs_advance(self._h, int(n_steps), int(from_ic), C.byref(tot), C.byref(ms)))
        return tot.value, ms.value

    def solve_host_ptr(self, T0_ptr, T_ptr, n_steps):
        """hs_solve_host on caller-owned (e.g. pinned) host buffers given as addresses."""
        tot, ms = C.c_longlong(), C.c_double()
        check(lib().hs_solve_host(self._h, T0_ptr, T_ptr, int(n_steps), C.byref(tot), C.byref(ms)))
        return tot.value, ms.value

    def time_kernel(self, which, reps=20):
        """Average per-launch device ms of one hot-path kernel (L2 flushed before each launch)."""
        ms = C.c_double()
        check(lib().hs_time_kernel(self._h, int(which), int(reps), C.byref(ms)))
        return ms.value

    def diag_cg(self, max_iter=500, tol=1e-8):
        cap = max_iter + 1
        rel, al, be = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        r0 = C.c_double()
        it = C.c_int()
        check(lib().hs_diag_cg(self._h, int(max_iter), float(tol), C.byref(r0), rel.ctypes.data, al.ctypes.data,
                               be.ctypes.data, cap, C.byref(it)))
        n = it.value
        return n, dict(rel0=r0.value, rel=rel[:n], alpha=al[:n], beta=be[:n])

    def target_on_boundary(self, fi):
        spec = fi_spec(fi)
        return lib().hs_target_on_boundary(self._h, C.byref(spec))


def classify(A, B, F, fi_level, dt, thr_user=1e-13, detect=False, F_nonfinite=0):
    """Host-side twin-run summary of the library (records as StepRecord arrays or dict lists)."""
    def arr(x):
        if x is None:
            return None
        if isinstance(x, C.Array):
            return x
        a = (StepRecord * len(x))()
        for i, s in enumerate(x):
            a[i] = StepRecord(int(s["cg_iters"]), int(s["snap"]), s["d1"], s["d2"], s["tmin"], s["tmax"], s["E"],
                              s["spread"], s.get("solve_ms", 0.0))
        return a
    a, b, f = arr(A), arr(B), arr(F)
    out = TwinSummary()
    check(lib().hs_classify(a, b, f, len(a), int(fi_level), int(F_nonfinite), float(dt), float(thr_user),
                            int(detect), C.byref(out)))
    return {name: (getattr(out, name).decode() if name in ("cls", "detected_by") else getattr(out, name))
            for name, _ in TwinSummary._fields_ if name != "pad"}


class Batch:
    """Batched mixed-precision solves (hs_batch_*): instances added to slots
    advance one implicit-Euler step per step() call, all in one graph launch."""

    def __init__(self, rtol=1e-8, inner_tol=1e-4, max_outer=10, max_inner=500, detect=True, tile_planes=0,
                 device=0, extrapolate=True):
        o = BatchOptions()
        lib().hs_batch_default_options(C.byref(o))
        o.rtol, o.inner_tol, o.max_outer, o.max_inner = rtol, inner_tol, max_outer, max_inner
        o.detect, o.tile_planes, o.device = int(detect), int(tile_planes), int(device)
        o.extrapolate = int(extrapolate)
        self._h = C.c_void_p()
        check(lib().hs_batch_create(C.byref(o), C.byref(self._h)))
        self.Nn = {}

    def add_lognormal(self, N, dt, mu, sigma, L, seed, rhoc=1.0, T0=None, steps=1):
        """An instance whose lognormal conductivity is generated on the device
        (hs_batch_add_lognormal): no host field."""
        T0 = None if T0 is None else _host(T0)
        slot = C.c_int(-1)
        check(lib().hs_batch_add_lognormal(self._h, int(N), float(dt), float(mu), float(sigma), float(L),
                                           C.c_ulonglong(seed), float(rhoc),
                                           T0.ctypes.data if T0 is not None else None, int(steps), C.byref(slot)))
        self.Nn[slot.value] = (N + 1) ** 3
        return slot.value

    def add(self, N, dt, k, rhoc, T0=None, steps=1):
        k, rhoc = _host(k), _host(rhoc)
        T0 = None if T0 is None else _host(T0)
        slot = C.c_int(-1)
        check(lib().hs_batch_add(self._h, int(N), float(dt), k.ctypes.data, rhoc.ctypes.data,
                                 T0.ctypes.data if T0 is not None else None, int(steps), C.byref(slot)))
        self.Nn[slot.value] = (N + 1) ** 3
        return slot.value

    def arm_flip(self, slot, step, idx, bit):
        """Flip bit `bit` of the field entry idx before the instance's step `step`."""
        check(lib().hs_batch_arm_flip(self._h, int(slot), int(step), int(idx), int(bit)))

    def arm_fault(self, slot, level, step, outer, it, idx, bit):
        """Flip bit `bit` (0..31) of an FP32 inner vector entry: level 'P', 'RV' or
        'AP' (or 5/6/7), in step `step`, correction `outer` (1-based), inner iteration `it`."""
        f = BatchFault(LEVELS.get(level, level), int(step), int(outer), int(it), int(idx), int(bit), 0)
        check(lib().hs_batch_arm_fault(self._h, int(slot), C.byref(f)))

    def remove(self, slot):
        check(lib().hs_batch_remove(self._h, int(slot)))
        self.Nn.pop(slot, None)

    def step(self):
        """One step of every instance with steps left: (instances stepped, device ms)."""
        n, ms = C.c_int(0), C.c_double(0.0)
        check(lib().hs_batch_step(self._h, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def step_begin(self):
        """Launch one step of every instance with steps left and return at once
        (instances in the step); add() and remove() may run until step_end()."""
        n = C.c_int(0)
        check(lib().hs_batch_step_begin(self._h, C.byref(n)))
        return n.value

    def step_end(self):
        """Wait for the step in flight: (instances stepped, device ms)."""
        n, ms = C.c_int(0), C.c_double(0.0)
        check(lib().hs_batch_step_end(self._h, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def info(self, slot):
        r = BatchInstInfo()
        check(lib().hs_batch_info(self._h, int(slot), C.byref(r)))
        return {name: getattr(r, name) for name, _ in BatchInstInfo._fields_ if name not in ("pad", "pad2")}

    def field(self, slot):
        T = np.empty(self.Nn[slot])
        check(lib().hs_batch_get_field(self._h, int(slot), T.ctypes.data))
        return T

    def close(self):
        if self._h:
            lib().hs_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gaussian_ic(N, sigma=0.15):
    """The library's Gaussian initial condition ((N+1)^3 doubles)."""
    T = np.empty((N + 1) ** 3)
    check(lib().hs_gaussian_ic(int(N), float(sigma), T.ctypes.data))
    return T


def field_lognormal(N, mu, sigma, L, seed, rhoc, k_dev, rhoc_dev):
    """hs_field_lognormal: a lognormal conductivity field generated on the device
    into the N^3-double device buffers at k_dev and rhoc_dev."""
    check(lib().hs_field_lognormal(int(N), float(mu), float(sigma), float(L), C.c_ulonglong(seed), float(rhoc),
                                   k_dev, rhoc_dev))


def dot_noalloc(N, x_dev, y_dev, out_dev):
    """hs_dot_noalloc: x.y into the device double at out_dev, no device allocation."""
    check(lib().hs_dot_noalloc(int(N), x_dev, y_dev, out_dev))


def cli(argv):
    """Run the command line in-process; returns the exit code."""
    args = [b"heat_solver_b200"] + [str(a).encode() for a in argv]
    arr = (C.c_char_p * len(args))(*args)
    return lib().hs_cli_main(len(args), arr)
