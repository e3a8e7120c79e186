"""ctypes front end of the CPU parity oracle (TEST INFRASTRUCTURE ONLY).

The oracle (oracle/heat_oracle.cpp) restates the reference transient-heat
solver src/heat_solver_het.cu on the CPU.  Only the tests, the smoke check and
the CPU-baseline legs of bench.py use this module; the B200 library never
imports it.  ``twin_run`` below restates the reference's twin-run driver and
fault classification (het.cu:1506-1542) on top of ``run_case``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libheat_oracle.so")
_lib = None

FORMS = {"fast": 0, "dense": 0, "gauss": 1, "wht": 2}
LEVELS = {"G": 1, "R": 2, "H": 3, "P": 5, "RV": 6, "AP": 7}


class StepOut(C.Structure):
    _fields_ = [("cg_iters", C.c_int), ("d1", C.c_double), ("d2", C.c_double),
                ("tmin", C.c_double), ("tmax", C.c_double), ("E", C.c_double),
                ("spread", C.c_double), ("snap", C.c_int)]


def build():
    """Compile the oracle with its Makefile (g++ only, no CUDA)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        vp = C.c_void_p
        L.or_create.restype = vp
        L.or_create.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_double, dp, dp, C.POINTER(C.c_int)]
        L.or_destroy.argtypes = [vp]
        L.or_apply.restype = C.c_double
        L.or_apply.argtypes = [vp, dp, dp, C.c_double, C.c_int, C.c_int, C.c_long, C.c_int]
        L.or_dot.restype = C.c_double
        L.or_dot.argtypes = [vp, dp, dp]
        L.or_udot.restype = C.c_double
        L.or_udot.argtypes = [vp, dp, dp]
        L.or_build_rhs.argtypes = [vp, dp, dp]
        L.or_pcg.restype = C.c_int
        L.or_pcg.argtypes = [vp, dp, dp, C.c_int, C.c_double, vp, vp, vp, vp]
        L.or_run_case.restype = C.c_int
        L.or_run_case.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_long,
                                  C.c_int, C.c_int, C.c_int, dp, vp, vp, vp, vp,
                                  C.POINTER(StepOut), C.POINTER(C.c_int)]
        L.or_verify.restype = C.c_double
        L.or_verify.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_long)]
        L.or_get_vectors.argtypes = [vp, vp, vp, vp, vp, vp]
        L.or_get_matrices.argtypes = [vp, vp, vp, vp]
        L.or_set_layout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_slab_layout.restype = C.c_long
        L.or_slab_layout.argtypes = [C.c_int, C.POINTER(C.c_int)]
        L.or_set_threads.restype = C.c_int
        L.or_set_threads.argtypes = [C.c_int]
        L.or_initial_condition.argtypes = [vp, dp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def set_layout(cx: int = 0, ty: int = 0, tz: int = 0, kf: int = 2) -> None:
    """Canonical reduction orders: the apply order's slab tile (planes cx, rows
    ty, columns tz; all 0 for the library's per-N shape slab_layout(N)) and
    the flat order's nodes per thread kf.  The defaults are the library's; a
    block has 256 threads of 4 positions each."""
    lib().or_set_layout(cx, ty, tz, kf)


def slab_layout(N: int) -> dict:
    """The per-N apply tile shape: planes cx, rows ty, columns tz, and the tile count."""
    out = (C.c_int * 3)()
    nt = lib().or_slab_layout(int(N), out)
    return dict(cx=out[0], ty=out[1], tz=out[2], ntiles=int(nt))


def set_threads(n: int) -> int:
    return lib().or_set_threads(n)


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class Oracle:
    """One single-rank solver instance on the CPU."""

    def __init__(self, N, dt, k, rhoc, form="wht", colored=True, detect=False, verify=False,
                 no_source=False, ic="zero", ic_sigma=0.1):
        self.N = int(N)
        self.NN = self.N + 1
        self.Nn = self.NN ** 3
        self.dt = float(dt)
        self.detect = bool(detect)
        k = np.ascontiguousarray(k, dtype=np.float64).ravel()
        rhoc = np.ascontiguousarray(rhoc, dtype=np.float64).ravel()
        if k.size != self.N ** 3 or rhoc.size != self.N ** 3:
            raise ValueError("field size mismatch")
        self.kmin, self.kmax = float(k.min()), float(k.max())
        self.rhocmin, self.rhocmax = float(rhoc.min()), float(rhoc.max())
        st = C.c_int(0)
        self._h = lib().or_create(self.N, self.dt, FORMS[form], int(colored), int(detect), int(verify),
                                  int(no_source), 1 if ic == "gaussian" else 0, float(ic_sigma), k, rhoc,
                                  C.byref(st))
        if not self._h:
            raise OracleError(st.value, "non-positive coefficient" if st.value == 1 else "reference matrices failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().or_destroy(h)
            self._h = None

    def vectors(self):
        n = self.Nn
        d, F, wM, wA = (np.zeros(n) for _ in range(4))
        norms = np.zeros(2)
        lib().or_get_vectors(self._h, _ptr(d), _ptr(F), _ptr(wM), _ptr(wA), _ptr(norms))
        return dict(diag=d, F=F, wM=wM, wA=wA, norm_wM=norms[0], norm_wA=norms[1])

    def matrices(self):
        M, K, e = np.zeros(64), np.zeros(64), np.zeros(5)
        lib().or_get_matrices(self._h, _ptr(M), _ptr(K), _ptr(e))
        return M.reshape(8, 8), K.reshape(8, 8), e

    def apply(self, x, dt_eff=None, project=True, d1=False, fi_elem=-1, fi_bit=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.Nn)
        rel = lib().or_apply(self._h, x, y, self.dt if dt_eff is None else float(dt_eff), int(project),
                             int(d1), int(fi_elem), int(fi_bit))
        return y, rel

    def dot(self, a, b):
        return lib().or_dot(self._h, np.ascontiguousarray(a, dtype=np.float64),
                            np.ascontiguousarray(b, dtype=np.float64))

    def udot(self, a, b):
        """x.y in the PCG update's RUN order."""
        return lib().or_udot(self._h, np.ascontiguousarray(a, dtype=np.float64),
                             np.ascontiguousarray(b, dtype=np.float64))

    def build_rhs(self, T):
        b = np.zeros(self.Nn)
        lib().or_build_rhs(self._h, np.ascontiguousarray(T, dtype=np.float64), b)
        return b

    def pcg(self, b, x0, max_iter=500, tol=1e-8):
        x = np.array(x0, dtype=np.float64, copy=True)
        lr, la, lb = (np.zeros(max_iter + 1) for _ in range(3))
        r0 = np.zeros(1)
        it = lib().or_pcg(self._h, np.ascontiguousarray(b, dtype=np.float64), x, int(max_iter), float(tol),
                          _ptr(lr), _ptr(la), _ptr(lb), _ptr(r0))
        return it, x, dict(rel0=r0[0], rel=lr[:it].copy(), alpha=la[:it].copy(), beta=lb[:it].copy())

    def initial_condition(self):
        T = np.zeros(self.Nn)
        lib().or_initial_condition(self._h, T)
        return T

    def run_case(self, n_steps, snap_every=5, max_iter=500, tol=1e-8, fi=None, reproject=False,
                 ref_snaps=None, keep_snaps=False):
        """One trajectory. fi = (level, step, target, bit, iter) or None."""
        lv, st, tg, bt, itr = fi if fi else (0, -1, 0, 0, 0)
        out = (StepOut * n_steps)()
        nonfinite = C.c_int(0)
        T = np.zeros(self.Nn)
        n_snap = sum(1 for s in range(n_steps) if (snap_every > 0 and s % snap_every == 0) or s == n_steps - 1)
        keep = np.zeros((n_snap, self.Nn)) if keep_snaps else None
        ref = np.ascontiguousarray(ref_snaps, dtype=np.float64) if ref_snaps is not None else None
        lib().or_run_case(self._h, int(n_steps), int(snap_every), int(max_iter), float(tol), int(lv), int(st),
                          int(tg), int(bt), int(itr), int(reproject), T, _ptr(ref), _ptr(keep), None, None,
                          out, C.byref(nonfinite))
        steps = [dict(cg_iters=o.cg_iters, d1=o.d1, d2=o.d2, tmin=o.tmin, tmax=o.tmax, E=o.E,
                      spread=o.spread, snap=o.snap) for o in out]
        return dict(T=T, steps=steps, snaps=keep, nonfinite=nonfinite.value)

    def verify(self, n_steps, max_iter=500, tol=1e-8):
        tot = C.c_long(0)
        rel = lib().or_verify(self._h, int(n_steps), int(max_iter), float(tol), C.byref(tot))
        return rel, tot.value


def classify(rA, rB, rF, fi_level, dt, thr_user=1e-13, detect=False):
    """Twin-run summary and fault class (het.cu:1506-1542, 1585-1595).

    rA/rB/rF are ``run_case`` results of cleanA, cleanB and the fault run
    (rF None without injection).  D3 of B and F is judged against A's
    per-step range with margin 1e-6*|ref_max| + 1e-12 (het.cu:1219-1225).
    """
    snap_steps = [i for i, s in enumerate(rB["steps"]) if s["snap"]]
    EB = [rB["steps"][s]["E"] for s in snap_steps]
    Efl_max, Efl_final = 0.0, 0.0
    Efa_max, Efa_int, Efa_final, step_max = 0.0, 0.0, 0.0, -1
    spread_at_max, spread_final = 0.0, 0.0
    for i, s in enumerate(snap_steps):
        Efl_max = max(Efl_max, EB[i]) if not math.isnan(EB[i]) else Efl_max
        Efl_final = EB[i]
        if fi_level > 0:
            E = rF["steps"][s]["E"]
            if math.isfinite(E) and E > Efa_max:
                Efa_max, step_max, spread_at_max = E, s, rF["steps"][s]["spread"]
            Efa_final = E
            spread_final = rF["steps"][s]["spread"]
            w = (snap_steps[i + 1] - s) * dt if i + 1 < len(snap_steps) else 0.0
            if math.isfinite(E):
                Efa_int += E * w
    iters_delta_max = 0
    if fi_level > 0:
        iters_delta_max = max([0] + [f["cg_iters"] - a["cg_iters"] for f, a in zip(rF["steps"], rA["steps"])])
    thr = max(thr_user, 10.0 * Efl_max)
    cls = "clean"
    if fi_level > 0:
        if rF["nonfinite"]:
            cls = "detected"
        elif Efa_max <= thr:
            cls = "benign"
        elif Efa_final <= thr:
            cls = "transient"
        else:
            cls = "persistent"
    res = dict(E_floor_max=Efl_max, E_floor_final=Efl_final, E_fault_max=Efa_max, step_at_max=step_max,
               E_fault_int=Efa_int, E_fault_final=Efa_final, thr=thr, iters_delta_max=iters_delta_max,
               cls=cls, spread_at_max=spread_at_max, spread_final=spread_final)
    if detect:
        rX = rF if fi_level > 0 else rA
        first = {"d1": -1, "d2": -1, "d3": -1}
        d1m = d2m = 0.0
        for s, (x, a) in enumerate(zip(rX["steps"], rA["steps"])):
            if not (x["d1"] <= 1e-10) and first["d1"] < 0:
                first["d1"] = s
            if not (x["d2"] <= 1e-6) and first["d2"] < 0:
                first["d2"] = s
            fire = not (math.isfinite(x["tmin"]) and math.isfinite(x["tmax"]))
            if rX is not rA:
                margin = 1e-6 * max(abs(a["tmax"]), 1e-300) + 1e-12
                if x["tmax"] > a["tmax"] + margin or x["tmin"] < a["tmin"] - margin:
                    fire = True
            if fire and first["d3"] < 0:
                first["d3"] = s
            d1m = max(d1m, x["d1"]) if math.isfinite(x["d1"]) else 1e300
            d2m = max(d2m, x["d2"]) if math.isfinite(x["d2"]) else 1e300
        by = "+".join(n for n, k in (("D1", "d1"), ("D2", "d2"), ("D3", "d3")) if first[k] >= 0) or "none"
        res.update(d1_first=first["d1"], d2_first=first["d2"], d3_first=first["d3"], d1_max=d1m, d2_max=d2m,
                   detected_by=by)
    return res
