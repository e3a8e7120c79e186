"""Precision, batching and serving forms of the transient-heat solve.

Each subcommand times the batched mixed-precision solver (FP32 inner PCG,
FP64 defect correction on the true residual, hs_batch_*) beside the plain
FP64 drop-in (hs_solver: FP64 Jacobi-PCG, one solve at a time) on the same
GPU and the same seeded synthetic inputs, and prints one JSON line.

  precision  one N=256 solve: lognormal k (sigma 1.5, correlation 16
             elements), 20 steps to rtol 1e-8; error of both against an
             FP64 solve at rtol 1e-12, ABFT noise floors of both precisions.
  batching   an ensemble of independent solves (default 256, N uniform in
             16..96, lognormal k sigma 1 with correlation N/8 elements),
             20 steps each to rtol 1e-8, all in one batch (one graph launch
             per step); the tile depth is chosen by a short autotuning run.
  coverage   detection coverage of the mixed form under 1000 seeded flips
             into its FP32 inner vectors, beside the FP64 drop-in's campaign
             (p, r, Ap) on the same problem (N=64 by default).
  single     one instance of the batched solver alone (default the N=128
             bench problem, 2 steps to rtol 1e-8): its device time and
             inner/outer iteration counts; the short run profiles are taken on.
  serving    a seeded Poisson stream of requests (N uniform in 16..160, steps
             uniform in 10..100, 30 % with one seeded bit flip of the field),
             served by continuous batching: requests join the running batch
             as they arrive and leave when done; p50 / p99 latency and
             solves/s beside serial plain FP64 serving of the same stream.

Fields are generated before the timed regions (the reference generator's
algorithm, host NumPy); every timed region holds solver work only.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from mnhack8_b200 import _lib  # noqa: E402
from mnhack8_b200.fields import FieldSpec, make_field  # noqa: E402

DT = 1e-4
IC_SIGMA = 0.15


def lognormal(N, sigma, corr_elements, seed):
    k, r, _ = make_field(FieldSpec(n=N, model="lognormal", mu=0.0, sigma=sigma, L=corr_elements / N, seed=seed))
    return k.ravel(), r.ravel()


def _lognormal_job(args):
    return lognormal(*args)


def _lognormal_timed_job(args):
    t0 = time.perf_counter()
    k, r = lognormal(*args)
    return k, r, time.perf_counter() - t0


def lognormal_many(jobs, workers=None):
    """Fields for (N, sigma, corr_elements, seed) jobs, generated in a process pool
    (spawned, so no worker inherits a CUDA context)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_lognormal_job, jobs, chunksize=4))


def batch_bytes(N):
    """Device bytes of one batched instance (the allocation hs_batch_add makes)."""
    Nn, Ne = (N + 1) ** 3, N ** 3
    return 8 * 8 * Nn + 7 * 4 * Nn + 48 * Ne + 17 * 256


def fp64_solve(N, k, r, steps, rtol, device=0):
    """Plain FP64 drop-in: steps implicit-Euler steps from the Gaussian IC;
    returns (field, CG iterations, device ms)."""
    g = _lib.Solver(N, DT, k, r, kernel="wht", scatter="colored", detect=True, no_source=True, ic="gaussian",
                    ic_sigma=IC_SIGMA, rtol=rtol, max_iter=1000, device=device)
    it, ms = g.advance(steps, from_ic=True)
    T = g.get_field()
    g.close()
    return T, it, ms


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ---- config 3 --------------------------------------------------------------------
def precision(N=256, steps=20, rtol=1e-8, inner_tol=1e-4, sigma=1.5, corr=16.0, seed=3, device=0):
    (k, r), = lognormal_many([(N, sigma, corr, seed)], workers=1)
    T0 = _lib.gaussian_ic(N, IC_SIGMA)
    T_ref, it_ref, _ = fp64_solve(N, k, r, steps, 1e-12, device)
    fp64_solve(N, k, r, 2, rtol, device)                     # warm-up
    T64, it64, ms64 = fp64_solve(N, k, r, steps, rtol, device)
    b = _lib.Batch(rtol=rtol, inner_tol=inner_tol, device=device)
    w = b.add(N, DT, k, r, T0=T0, steps=2)                   # warm-up (graph capture)
    while b.step()[0]:
        pass
    b.remove(w)
    s = b.add(N, DT, k, r, T0=T0, steps=steps)
    ms_mixed = 0.0
    while True:
        n, ms = b.step()
        if not n:
            break
        ms_mixed += ms
    Tm, inf = b.field(s), b.info(s)
    b.close()
    nodes = (N + 1) ** 3
    return {
        "form": "precision", "N": N, "nodes": nodes, "steps": steps, "rtol": rtol, "inner_tol": inner_tol,
        "field": f"lognormal sigma {sigma}, correlation {corr:g} elements, seed {seed}",
        "fp64": {"ms": ms64, "cg_iters": it64, "err_vs_fp64_1e-12": rel(T64, T_ref),
                 "solves_per_s": 1e3 / ms64},
        "mixed": {"ms": ms_mixed, "inner_iters": inf["inner_iters"], "outer_iters": inf["outer_iters"],
                  "err_vs_fp64_1e-12": rel(Tm, T_ref), "final_true_rel_residual": inf["rel_residual"],
                  "solves_per_s": 1e3 / ms_mixed},
        "speedup_mixed_vs_fp64": ms64 / ms_mixed,
        "abft_noise_floor": {"fp64_applies_max_d1": inf["d1_max64"], "fp32_applies_max_d1": inf["d1_max32"],
                             "fp64_threshold": 1e-10},
        "reference_cg_iters_at_1e-12": it_ref,
    }


# ---- config 4 --------------------------------------------------------------------
def ensemble_specs(n, nmin, nmax, seed):
    rng = np.random.default_rng(seed)
    Ns = rng.integers(nmin, nmax + 1, size=n)
    return [(int(N), 1000 + i) for i, N in enumerate(Ns)]


def run_batch(fields, steps, rtol, inner_tol, planes, device=0):
    b = _lib.Batch(rtol=rtol, inner_tol=inner_tol, tile_planes=planes, device=device)
    slots = [b.add(N, DT, k, r, T0=T0, steps=steps) for (N, k, r, T0) in fields]
    tot = 0.0
    while True:
        n, ms = b.step()
        if not n:
            break
        tot += ms
    infos = [b.info(s) for s in slots]
    b.close()
    return tot, infos


def batching(n=256, nmin=16, nmax=96, steps=20, rtol=1e-8, inner_tol=1e-4, seed=7, serial_sample=None, device=0):
    specs = ensemble_specs(n, nmin, nmax, seed)
    kr = lognormal_many([(N, 1.0, N / 8.0, sd) for N, sd in specs])
    fields = [(N, k, r, _lib.gaussian_ic(N, IC_SIGMA)) for (N, _), (k, r) in zip(specs, kr)]
    # autotuner: planes per operator tile (0: the per-N default), timed on 2 steps of the first 64 instances
    tune = {}
    for planes in (0, 8, 12, 16, 24, 32):
        run_batch(fields[:64], 1, rtol, inner_tol, planes, device)         # capture / warm
        ms, _ = run_batch(fields[:64], 2, rtol, inner_tol, planes, device)
        tune[planes] = ms
    best = min(tune, key=tune.get)
    ms_b, infos = run_batch(fields, steps, rtol, inner_tol, best, device)
    # serial plain FP64, one solve after another (all, or a sample scaled up)
    idx = range(len(specs)) if not serial_sample else range(min(serial_sample, len(specs)))
    fp64_solve(fields[0][0], fields[0][1], fields[0][2], 2, rtol, device)  # warm-up
    ms_s, n_s = 0.0, 0
    for i in idx:
        N, k, r, _ = fields[i]
        _, _, ms = fp64_solve(N, k, r, steps, rtol, device)
        ms_s += ms
        n_s += 1
    ms_serial = ms_s * len(specs) / n_s
    dof_it = sum((N + 1) ** 3 * inf["inner_iters"] for (N, _, _, _), inf in zip(fields, infos))
    return {
        "form": "batching", "instances": n, "N_range": [nmin, nmax], "steps": steps, "rtol": rtol,
        "inner_tol": inner_tol, "autotune_ms_per_tile_planes": tune, "tile_planes": best,
        "batch_ms": ms_b, "batch_solves_per_s": n / (ms_b * 1e-3),
        "batch_fp32_dof_iters_per_s": dof_it / (ms_b * 1e-3),
        "max_final_true_rel_residual": max(inf["rel_residual"] for inf in infos),
        "serial_fp64_ms": ms_serial, "serial_fp64_solves_per_s": n / (ms_serial * 1e-3),
        "serial_fp64_timed_solves": n_s,
        "speedup_vs_serial_fp64": ms_serial / ms_b,
    }


# ---- config 5 --------------------------------------------------------------------
def request_stream(n, rate, seed, nmin=16, nmax=160, smin=10, smax=100, flip_frac=0.3):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    reqs = []
    for i in range(n):
        N = int(rng.integers(nmin, nmax + 1))
        steps = int(rng.integers(smin, smax + 1))
        flip = None
        if rng.random() < flip_frac:
            flip = (int(rng.integers(0, steps)), int(rng.integers(0, (N + 1) ** 3)), int(rng.integers(0, 64)))
        reqs.append(dict(id=i, t=float(t[i]), N=N, steps=steps, flip=flip, seed=5000 + i))
    return reqs


def serving(n=400, rate=200.0, seed=11, rtol=1e-8, inner_tol=1e-4, max_live=256, hbm_fraction=0.5, device=0,
            gpu_fields=False, serial=True):
    """gpu_fields: the batched server generates each request's field on the
    device when it admits the request (hs_batch_add_lognormal), so the field's
    generation is inside the served latency; the serial FP64 side keeps the
    host fields generated before its timed region.  serial=False times the
    batched server alone."""
    import torch
    import concurrent.futures as cf
    import multiprocessing as mp
    reqs = request_stream(n, rate, seed)
    # fields: the reference generator's algorithm on the host, timed per request
    workers = max(1, min(16, (os.cpu_count() or 2) - 1))
    tg = time.perf_counter()
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        kr = list(ex.map(_lognormal_timed_job, [(q["N"], 1.0, q["N"] / 8.0, q["seed"]) for q in reqs], chunksize=2))
    gen_wall = time.perf_counter() - tg
    gen_each = [t for _, _, t in kr]
    for q, (k, r, _) in zip(reqs, kr):
        q["k"], q["r"] = k, r
        q["T0"] = _lib.gaussian_ic(q["N"], IC_SIGMA)
    # admission by free HBM: the live instances' bytes stay within this budget
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(hbm_fraction * free)
    # continuous batching on a wall clock
    b = _lib.Batch(rtol=rtol, inner_tol=inner_tol, device=device)
    w = b.add(16, DT, np.ones(16 ** 3), np.ones(16 ** 3), steps=1)   # graph capture
    b.step()
    b.remove(w)
    lat, live, queue = {}, {}, list(reqs)
    live_bytes, peak_live = 0, 0
    t0 = time.perf_counter()

    def admit():
        nonlocal live_bytes
        now = time.perf_counter() - t0
        while (queue and queue[0]["t"] <= now and len(live) < max_live and
               live_bytes + batch_bytes(queue[0]["N"]) <= budget):
            q = queue.pop(0)
            live_bytes += batch_bytes(q["N"])
            if gpu_fields:
                s = b.add_lognormal(q["N"], DT, 0.0, 1.0, 1.0 / 8.0, q["seed"], rhoc=1.0, T0=q["T0"], steps=q["steps"])
            else:
                s = b.add(q["N"], DT, q["k"], q["r"], T0=q["T0"], steps=q["steps"])
            if q["flip"]:
                b.arm_flip(s, *q["flip"])
            q["left"] = q["steps"]
            live[s] = q

    while queue or live:
        if not live:
            admit()
            if not live:
                time.sleep(max(0.0, queue[0]["t"] - (time.perf_counter() - t0)))
            continue
        # the live instances step on the GPU while the host sets up arrivals;
        # those join at the next step
        stepping = list(live)
        b.step_begin()
        admit()
        b.step_end()
        peak_live = max(peak_live, len(live))
        done_at = time.perf_counter() - t0
        for s in stepping:
            live[s]["left"] -= 1
        for s in [s for s in stepping if live[s]["left"] == 0]:
            q = live.pop(s)
            live_bytes -= batch_bytes(q["N"])
            lat[q["id"]] = done_at - q["t"]
            b.remove(s)
    wall_b = time.perf_counter() - t0
    b.close()
    if not serial:
        return {"form": "serving", "requests": n, "max_live": max_live, "peak_live": peak_live,
                "batched": {"wall_s": wall_b, "solves_per_s": n / wall_b,
                            "p50_latency_s": float(np.percentile(list(lat.values()), 50)),
                            "p99_latency_s": float(np.percentile(list(lat.values()), 99))}}
    # serial plain FP64: the same stream, one solve at a time
    lat_s = {}
    create_s = 0.0
    t0 = time.perf_counter()
    busy_until = 0.0
    for q in reqs:
        while time.perf_counter() - t0 < q["t"]:
            time.sleep(min(1e-3, q["t"] - (time.perf_counter() - t0)))
        tc = time.perf_counter()
        g = _lib.Solver(q["N"], DT, q["k"], q["r"], kernel="wht", scatter="colored", detect=True, no_source=True,
                        ic="gaussian", ic_sigma=IC_SIGMA, rtol=rtol, max_iter=1000, device=device)
        g.advance(0, from_ic=True)
        create_s += time.perf_counter() - tc
        if q["flip"]:
            fs, fi, fb = q["flip"]
            if fs > 0:
                g.advance(fs, from_ic=False)
            T = g.get_field()
            T.view(np.uint64)[fi] ^= np.uint64(1) << np.uint64(fb)
            g.set_field(T)
            g.advance(q["steps"] - fs, from_ic=False)
        else:
            g.advance(q["steps"], from_ic=False)
        g.close()
        busy_until = time.perf_counter() - t0
        lat_s[q["id"]] = busy_until - q["t"]
    wall_s = time.perf_counter() - t0

    def pct(d, p):
        return float(np.percentile(np.array(list(d.values())), p))

    return {
        "form": "serving", "requests": n, "rate_per_s": rate, "N_range": [16, 160], "steps_range": [10, 100],
        "flip_fraction": 0.3, "rtol": rtol, "max_live": max_live, "hbm_budget_bytes": budget,
        "peak_live": peak_live,
        "batched": {"wall_s": wall_b, "solves_per_s": n / wall_b, "p50_latency_s": pct(lat, 50),
                    "p99_latency_s": pct(lat, 99)},
        "serial_fp64": {"wall_s": wall_s, "solves_per_s": n / wall_s, "p50_latency_s": pct(lat_s, 50),
                        "p99_latency_s": pct(lat_s, 99), "handle_setup_s_total": create_s,
                        "handle_setup_s_per_request": create_s / n},
        "throughput_ratio": (n / wall_b) / (n / wall_s),
        "batched_fields": "device, at admission, inside the timed stream" if gpu_fields else
                          "host, before the stream",
        "field_generation": {"where": "host, the reference generator's FFT algorithm (NumPy), before the stream",
                             "per_request_mean_s": float(np.mean(gen_each)),
                             "per_request_p99_s": float(np.percentile(gen_each, 99)),
                             "pool_wall_s": gen_wall, "pool_workers": workers},
        "stream_span_s": reqs[-1]["t"],
    }


# ---- config 3: detection coverage of the mixed form, beside FP64 ------------------------
FP32_D1_LAMBDA = 6.0        # tail factor of the probabilistic bound (false-alarm odds ~2 exp(-18) per check)
FP32_D1_DEPTH = 16          # roundings on the path of one node output of the FP32 apply


def checksum_weights(N, k, rhoc, dt):
    """w = A 1_int and w_abs = |A| 1_int on the interior rows (the rows the
    checksum 1_int . y sums), from the Q1 cube element matrices
    M^ = m(x)m(x)m and K^ = k(x)m(x)m + m(x)k(x)m + m(x)m(x)k (m = h/6 [2 1; 1 2],
    k = 1/h [1 -1; -1 1]); |A| takes the absolute value of every element
    matrix entry.  Host NumPy, for the threshold below."""
    h = 1.0 / N
    m = h / 6.0 * np.array([[2.0, 1.0], [1.0, 2.0]])
    kk = 1.0 / h * np.array([[1.0, -1.0], [-1.0, 1.0]])
    M = np.kron(m, np.kron(m, m))
    K = np.kron(kk, np.kron(m, m)) + np.kron(m, np.kron(kk, m)) + np.kron(m, np.kron(m, kk))
    k3, r3 = np.asarray(k).reshape(N, N, N), np.asarray(rhoc).reshape(N, N, N)
    inner = np.zeros((N + 1,) * 3)
    inner[1:-1, 1:-1, 1:-1] = 1.0
    corner = [((q >> 2) & 1, (q >> 1) & 1, q & 1) for q in range(8)]
    mask = [inner[ox:ox + N, oy:oy + N, oz:oz + N] for ox, oy, oz in corner]
    w, wabs = np.zeros((N + 1,) * 3), np.zeros((N + 1,) * 3)
    for i, (ox, oy, oz) in enumerate(corner):
        mr = sum(M[i, j] * mask[j] for j in range(8))
        kr = sum(K[i, j] * mask[j] for j in range(8))
        ma = sum(abs(M[i, j]) * mask[j] for j in range(8))
        ka = sum(abs(K[i, j]) * mask[j] for j in range(8))
        w[ox:ox + N, oy:oy + N, oz:oz + N] += r3 * mr + dt * k3 * kr
        wabs[ox:ox + N, oy:oy + N, oz:oz + N] += r3 * ma + dt * k3 * ka
    return w * inner, wabs * inner


def fp32_d1_threshold(N, k, rhoc, dt, lam=FP32_D1_LAMBDA, depth=FP32_D1_DEPTH):
    """D1 threshold of an FP32 apply from a probabilistic rounding-error bound.

    D1 = |1_int . y^ - w . p| / (||w|| ||p||), y^ the FP32 apply of the FP32
    vector p (the checksum sums themselves are FP64).  Each node output
    carries `depth` roundings of unit u = 2^-24 (the WHT butterflies, the
    eigenvalue scaling, the node sum, the coefficients rounded to FP32), each
    at most u times a value bounded by (|A| |p|)_i.  Modelling them as
    independent, mean-zero (Higham and Mary, SIAM J. Sci. Comput. 41 (2019)
    A2815), their sum over the interior nodes stays below
    lam sqrt(depth) u || |A| |p| ||_2 except with probability 2 exp(-lam^2/2).
    For a field p that is smooth on the element scale, (|A| |p|)_i ~
    w_abs,i |p_i|, and with |p| spread over the domain
    || w_abs o p || ~ ||w_abs|| ||p|| / sqrt(n_int), so

        D1 < lam sqrt(depth) u ||w_abs|| / (sqrt(n_int) ||w||).

    The threshold is this bound: a fixed function of the problem (grid,
    field, dt), with no input from a clean run."""
    w, wabs = checksum_weights(N, k, rhoc, dt)
    n_int = (N - 1) ** 3
    return lam * np.sqrt(depth) * 2.0 ** -24 * float(np.linalg.norm(wabs)) / (
        np.sqrt(n_int) * float(np.linalg.norm(w)))


def coverage(N=64, steps=20, flips=1000, seed=21, per_batch=None, rtol=1e-8, inner_tol=1e-4, sigma=1.5,
             corr_frac=1.0 / 16.0, sig_err=1e-6, device=0, rows_out=None, fp64=True):
    """Seeded single-bit flips into the FP32 inner vectors of the mixed form
    (p after formation, r after its update, Ap after projection; bits 0..31,
    step and inner iteration of the first correction uniform), run as batches
    of faulted copies of one problem, beside the FP64 drop-in's campaign
    (p, r, Ap, bits 0..63) on the same problem.  A mixed-form flip counts as
    detected when an FP32 apply's D1 exceeds the threshold of the
    probabilistic rounding bound (fp32_d1_threshold; the clean run's FP32
    noise floor is reported beside it), an FP64 apply's D1 exceeds 1e-10 (the
    reference's rule), or a step ends at the correction
    cap or an inner solve goes non-finite (its correction is then discarded);
    it is significant when its final field error exceeds sig_err (or is not
    finite)."""
    from mnhack8_b200.campaign import coverage as fp64_coverage
    (k, r), = lognormal_many([(N, sigma, corr_frac * N, 3)], workers=1)
    T0 = _lib.gaussian_ic(N, IC_SIGMA)
    Nn = (N + 1) ** 3
    b = _lib.Batch(rtol=rtol, inner_tol=inner_tol, device=device)
    s = b.add(N, DT, k, r, T0=T0, steps=steps)
    while b.step()[0]:
        pass
    T_clean, clean = b.field(s), b.info(s)
    b.close()
    thr32 = fp32_d1_threshold(N, k, r, DT)
    if per_batch is None:
        # faulted copies per batch: at most 125, within 60 % of the free HBM
        import torch
        free, _ = torch.cuda.mem_get_info(device)
        per_batch = int(max(1, min(125, 0.6 * free // batch_bytes(N))))
    per_corr = max(1, int(clean["inner_iters"] / max(1, clean["outer_iters"])))
    rng = np.random.default_rng(seed)
    sites = [dict(level=int(rng.choice([5, 6, 7])), step=int(rng.integers(0, steps)), outer=1,
                  iter=int(rng.integers(0, per_corr)), idx=int(rng.integers(0, Nn)), bit=int(rng.integers(0, 32)))
             for _ in range(flips)]
    t0 = time.perf_counter()
    rows = []
    for c0 in range(0, flips, per_batch):
        chunk = sites[c0:c0 + per_batch]
        b = _lib.Batch(rtol=rtol, inner_tol=inner_tol, device=device)
        slots = []
        for f in chunk:
            sl = b.add(N, DT, k, r, T0=T0, steps=steps)
            b.arm_fault(sl, f["level"], f["step"], f["outer"], f["iter"], f["idx"], f["bit"])
            slots.append(sl)
        while b.step()[0]:
            pass
        for f, sl in zip(chunk, slots):
            inf = b.info(sl)
            T = b.field(sl)
            err = float(np.linalg.norm(T - T_clean) / np.linalg.norm(T_clean)) if np.all(np.isfinite(T)) \
                else float("inf")
            det = (inf["d1_max32"] > thr32 or inf["d1_max64"] > 1e-10 or inf["stalls"] > 0 or
                   inf["inner_faults"] > 0)
            rows.append(dict(f, fired=inf["fault_fired"], err=err, detected=bool(det), stalls=inf["stalls"],
                             inner_faults=inf["inner_faults"],
                             d1_max32=inf["d1_max32"], extra_inner=inf["inner_iters"] - clean["inner_iters"]))
        b.close()
    wall = time.perf_counter() - t0
    fired = [x for x in rows if x["fired"]]
    sig = [x for x in fired if not (x["err"] <= sig_err)]

    def share(sel, pool):
        return (sum(1 for x in pool if sel(x)) / len(pool)) if pool else None

    mixed = {
        "flips": flips, "fired": len(fired), "significant": len(sig),
        "detected_rate_of_fired": share(lambda x: x["detected"], fired),
        "coverage_of_significant": share(lambda x: x["detected"], sig),
        "missed_significant": sum(1 for x in sig if not x["detected"]),
        "silent_corruptions": sum(1 for x in sig if not x["detected"]),
        "abft_d1_rate_of_fired": share(lambda x: x["d1_max32"] > thr32, fired),
        "max_err_of_undetected": max([x["err"] for x in fired if not x["detected"]] or [0.0]),
        "median_extra_inner_iters": float(np.median([x["extra_inner"] for x in fired])) if fired else None,
        "fp32_noise_floor_max_d1": clean["d1_max32"], "fp32_threshold": thr32,
        "fp32_threshold_rule": f"probabilistic rounding bound, lambda {FP32_D1_LAMBDA:g}, depth {FP32_D1_DEPTH}",
        "clean_run_false_alarm": bool(clean["d1_max32"] > thr32), "wall_s": wall,
        "by_vector": {v: {"fired": sum(1 for x in fired if x["level"] == lv),
                          "detected_rate": share(lambda x: x["detected"], [x for x in fired if x["level"] == lv])}
                      for v, lv in (("p", 5), ("r", 6), ("Ap", 7))},
    }
    if rows_out:
        with open(rows_out, "w") as fh:
            json.dump(rows, fh, default=lambda v: None if isinstance(v, float) and not np.isfinite(v) else v)
    if not fp64:
        return {"form": "precision-coverage", "N": N, "mixed": mixed}
    # FP64 drop-in: the same problem through hs_campaign
    g = _lib.Solver(N, DT, k, r, kernel="wht", scatter="colored", detect=True, no_source=True, ic="gaussian",
                    ic_sigma=IC_SIGMA, rtol=rtol, max_iter=1000, device=device)
    t0 = time.perf_counter()
    clean64, recs = g.campaign(steps, 1, flips, seed)
    wall64 = time.perf_counter() - t0
    g.close()
    cov64 = fp64_coverage(recs, clean64, sig_err)
    fp64 = {k2: cov64[k2] for k2 in ("flips", "significant", "any_detector_coverage_of_significant",
                                      "missed_significant", "abft_d1_rate", "any_detector_rate",
                                      "abft_noise_floor_clean_max_d1")}
    fp64["wall_s"] = wall64
    fp64["silent_corruptions"] = cov64["missed_significant"]
    return {"form": "precision-coverage", "N": N, "steps": steps, "rtol": rtol, "significant_error": sig_err,
            "mixed": mixed, "fp64": fp64,
            "abft_d1_rate_difference_points": 100.0 * (mixed["abft_d1_rate_of_fired"] - fp64["abft_d1_rate"]),
            "silent_corruptions": {"mixed": mixed["silent_corruptions"], "fp64": fp64["silent_corruptions"]}}


def single(N=128, steps=2, rtol=1e-8, sigma=1.0, corr=8.0, seed=1, device=0):
    """One instance of the batched mixed-precision solver: lognormal k (sigma,
    correlation corr elements), Gaussian IC sigma 0.15, dt 1e-4, `steps`
    implicit-Euler steps to rtol."""
    k, r = lognormal(N, sigma, corr, seed)
    b = _lib.Batch(rtol=rtol, device=device)
    s = b.add(N, 1e-4, k, r, T0=_lib.gaussian_ic(N, 0.15), steps=steps)
    ms = 0.0
    while True:
        n, t = b.step()
        if not n:
            break
        ms += t
    inf = b.info(s)
    b.close()
    return {"N": N, "steps": steps, "ms": ms, "inner_iters": inf["inner_iters"], "outer_iters": inf["outer_iters"],
            "rel_residual": inf["rel_residual"]}


def _main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("precision")
    p.add_argument("--N", type=int, default=256)
    p.add_argument("--steps", type=int, default=20)
    p = sub.add_parser("batching")
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--serial-sample", type=int, default=None)
    p = sub.add_parser("coverage")
    p.add_argument("--N", type=int, default=64)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--flips", type=int, default=1000)
    p.add_argument("--rows", default=None, help="write the mixed form's per-flip rows (JSON) here")
    p.add_argument("--no-fp64", action="store_true")
    p = sub.add_parser("single")
    p.add_argument("--N", type=int, default=128)
    p.add_argument("--steps", type=int, default=2)
    p = sub.add_parser("serving")
    p.add_argument("--gpu-fields", action="store_true")
    p.add_argument("--n", type=int, default=400)
    p.add_argument("--rate", type=float, default=200.0)
    p.add_argument("--max-live", type=int, default=256)
    a = ap.parse_args(argv)
    if a.cmd == "precision":
        out = precision(N=a.N, steps=a.steps)
    elif a.cmd == "coverage":
        out = coverage(N=a.N, steps=a.steps, flips=a.flips, rows_out=a.rows, fp64=not a.no_fp64)
    elif a.cmd == "batching":
        out = batching(n=a.n, steps=a.steps, serial_sample=a.serial_sample)
    elif a.cmd == "single":
        out = single(N=a.N, steps=a.steps)
    else:
        out = serving(n=a.n, rate=a.rate, max_live=a.max_live, gpu_fields=a.gpu_fields)
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(_main())
