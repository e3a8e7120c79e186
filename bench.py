#!/usr/bin/env python3
"""Throughput of the transient-heat PCG hot path on B200 (one JSON line).

Workload (one "step" of this benchmark): one complete implicit-Euler
trajectory of the FP64 N=128 problem -- 128^3 Q1 elements (129^3 = 2,146,689
nodes) on the unit cube, lognormal conductivity ln k ~ N(0, 1) with Gaussian
correlation length 8 elements (seeded synthetic field, the reference
generator's FFT algorithm), rho*c = 1, Dirichlet T = 0, Gaussian initial bump
(sigma 0.15), source off, dt = 1e-4, 50 steps, each a Jacobi-PCG solve to
relative residual 1e-10 with the ABFT checksum (D1) on every operator apply,
deterministic (colored) scatter.  Metric: DOF-iterations per second =
(N+1)^3 x total CG iterations / time (the reference's solve_ms definition:
build_rhs + PCG).

value: device time (CUDA events) of K trajectories with every input resident
in HBM.  e2e: the same through the public C ABI with host buffers
(hs_solve_host: pinned initial field in, 50 steps, final field out).  The
working set (~170 MB of node and element arrays) exceeds the 126 MB L2.

--impl reference: the reference path on the host cores: the CPU restatement
of the reference solver (its dense `fast` element form, colored order, all
host threads); each of its steps is one whole implicit-Euler step of the same
problem (build_rhs + Jacobi-PCG to rtol 1e-10).

Multi-GPU (torchrun): replicas only -- every rank solves its own seeded
instance, no collective on the data path; value = all ranks' DOF-iterations
/ the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 128
DT = 1e-4
STEPS_PER_TRAJ = 50
RTOL = 1e-10
IC_SIGMA = 0.15
CORR_ELEMENTS = 8.0
METRIC = "DOF-iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10, help="timed trajectories")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=N_DEFAULT)
    ap.add_argument("--kernel", default="wht", choices=["wht", "fast", "gauss"])
    ap.add_argument("--scatter", default="colored", choices=["colored", "atomic"])
    ap.add_argument("--no-detect", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gate", action="store_true",
                    help="skip the supplementary N=256 operator-kernel measurement")
    ap.add_argument("--serving-requests", type=int, default=300,
                    help="requests of the supplementary serving measurement (0: skip)")
    ap.add_argument("--batching-instances", type=int, default=256,
                    help="instances of the supplementary batching measurement (0: skip)")
    ap.add_argument("--profile", action="store_true",
                    help="only the timed trajectories (no e2e, kernel timing or CPU baseline): for ncu captures")
    ap.add_argument("--measure-traffic", action=argparse.BooleanOptionalAction, default=True,
                    help="take roofline.traffic from a one-pass ncu capture of the operator kernel at --N "
                         "(two DRAM counters, run after the same command exited 0 without ncu)")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="only a few launches of the PCG operator kernel at --N (L2 scrubbed before each): "
                         "for one-launch ncu captures")
    return ap.parse_args()


def make_field(N, seed):
    from mnhack8_b200.fields import FieldSpec, make_field as mk
    k, r, _ = mk(FieldSpec(n=N, model="lognormal", mu=0.0, sigma=1.0, L=CORR_ELEMENTS / N, seed=seed))
    return k.ravel(), r.ravel()


def workload_config(args, world):
    return {
        "workload": f"implicit-Euler trajectory, Q1 hex N={args.N}^3 elements ({(args.N + 1) ** 3} nodes), "
                    f"lognormal k sigma=1 corr=8 elements, Gaussian IC sigma=0.15, dt=1e-4, {STEPS_PER_TRAJ} steps, "
                    f"Jacobi-PCG rtol 1e-10, ABFT D1 {'off' if args.no_detect else 'on'}, {args.scatter} scatter",
        "N": args.N, "nodes": (args.N + 1) ** 3, "elements": args.N ** 3, "time_steps_per_step": STEPS_PER_TRAJ,
        "dt": DT, "rtol": RTOL, "element_form": args.kernel, "scatter": args.scatter,
        "abft": not args.no_detect, "precision": "fp64",
        "l2": "inputs larger than L2 (~170 MB working set vs 126 MB L2)",
        "parallelism": f"replicas x{world}",
    }


def reduce_over_ranks(dist, elapsed, iters, device):
    """Replica aggregation: the slowest rank's elapsed time and all ranks' CG
    iterations (every rank calls the same two collectives in the same order)."""
    import torch
    t = torch.tensor([float(elapsed), float(iters)], dtype=torch.float64, device=device)
    if dist is not None:
        tmax, tsum = t[0:1].clone(), t[1:2].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        return float(tmax[0]), float(tsum[0])
    return float(t[0]), float(t[1])


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measure_traffic(N, args):
    """DRAM bytes (read + write) per launch of the PCG operator kernel, from one
    ncu capture of `bench.py --profile-kernel` at this N taken by this run:
    the command first runs without ncu and must exit 0, then ncu collects
    only dram__bytes_read.sum and dram__bytes_write.sum (one pass, no memory
    save/restore, clocks untouched) over the timed launches.  Returns (bytes
    per launch or None, a note saying where the figure came from)."""
    import csv
    import io
    import shutil
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--N", str(N), "--profile-kernel",
           "--kernel", args.kernel, "--scatter", args.scatter] + (["--no-detect"] if args.no_detect else [])
    try:
        plain = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return None, "not measured: the uncaptured kernel run did not finish"
    if plain.returncode != 0:
        return None, "not measured: the uncaptured kernel run failed"
    ncu = shutil.which("ncu") or "/usr/local/cuda/bin/ncu"
    if not os.path.exists(ncu):
        return None, "not measured: ncu not found"
    prof = [ncu, "--metrics", "dram__bytes_read.sum,dram__bytes_write.sum", "--clock-control", "none",
            "-k", "regex:k_apply_slab", "--print-units", "base", "--csv"] + cmd
    try:
        out = subprocess.run(prof, capture_output=True, text=True, timeout=1800)
    except subprocess.TimeoutExpired:
        return None, "not measured: the ncu capture did not finish"
    lines = out.stdout.splitlines()
    head = next((i for i, l in enumerate(lines) if '"Metric Name"' in l), None)
    if out.returncode != 0 or head is None:
        return None, "not measured: " + ((out.stdout + out.stderr).strip().splitlines() or ["ncu failed"])[-1][:200]
    per = {}
    for row in csv.DictReader(io.StringIO("\n".join(lines[head:]))):
        if "k_apply_slab" not in row.get("Kernel Name", ""):
            continue
        try:
            v = float(row["Metric Value"].replace(",", ""))
        except (KeyError, ValueError):
            continue
        per.setdefault(row["ID"], 0.0)
        per[row["ID"]] += v
    if not per:
        return None, "not measured: no k_apply_slab launch in the capture"
    ids = sorted(per, key=int)[-PROFILE_REPS:]          # the timed launches
    vals = sorted(per[i] for i in ids)
    return vals[len(vals) // 2], (f"ncu dram__bytes_read.sum + dram__bytes_write.sum, median of the last "
                                  f"{len(ids)} k_apply_slab launches of `bench.py --N {N} --profile-kernel`, "
                                  f"captured by this run")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def host_cpu():
    """The host's CPU model and logical core count (the CPU baseline's machine)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def reference_problem(N, threads):
    """The CPU restatement of the reference solver on the bench problem: the
    reference's dense element form, colored order, ABFT on, same field, IC,
    dt and tolerance."""
    from oracle import oracle as om
    n = om.set_threads(threads)
    k, r = make_field(N, 1)
    o = om.Oracle(N, DT, k, r, form="fast", colored=True, detect=True, no_source=True, ic="gaussian",
                  ic_sigma=IC_SIGMA)
    return o, n


def reference_step(o, T, cap=500):
    """One whole implicit-Euler step (build_rhs + Jacobi-PCG to rtol 1e-10):
    (CG iterations, seconds)."""
    t0 = time.perf_counter()
    b = o.build_rhs(T)
    it, _, _ = o.pcg(b, T, cap, RTOL)
    return it, time.perf_counter() - t0


def cpu_baseline_sample(N, one_thread_iters=12):
    """The reference algorithm on the host cores: one whole implicit-Euler step
    of the bench problem on all host threads, and a bounded one-thread sample
    (build_rhs + a few CG iterations of the same step)."""
    from oracle import oracle as om
    nproc = os.cpu_count() or 1
    o, om_threads = reference_problem(N, nproc)
    T = o.initial_condition()
    it, dt = reference_step(o, T)
    nodes = (N + 1) ** 3
    om.set_threads(1)
    it1, dt1 = reference_step(o, T, cap=one_thread_iters)
    om.set_threads(nproc)
    return {"value": nodes * it / dt, "unit": METRIC, "cores": om_threads, "kind": "port",
            "sample": f"one whole implicit-Euler step of the same N={N} problem (build_rhs + {it} CG iterations to "
                      f"rtol 1e-10, the reference's dense element form, colored order, ABFT on), {dt:.1f} s on "
                      f"{om_threads} host threads",
            "value_1thread": nodes * it1 / dt1,
            "sample_1thread": f"build_rhs + {it1} CG iterations of the same step on 1 thread, {dt1:.1f} s",
            "host": host_cpu()}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    o, n_threads = reference_problem(args.N, os.cpu_count() or 1)
    T = o.initial_condition()
    for _ in range(args.warmup):
        reference_step(o, T)
    tot_it, tot_s = 0, 0.0
    for _ in range(args.steps):
        it, dt = reference_step(o, T)
        tot_it += it
        tot_s += dt
    nodes = (args.N + 1) ** 3
    v = nodes * tot_it / tot_s
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded lognormal field)",
        "config": dict(workload_config(args, 1), element_form="fast (reference dense 8x8)"),
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": n_threads, "kind": "port",
                         "sample": f"each step: one whole implicit-Euler step of the same problem (build_rhs + "
                                   f"Jacobi-PCG to rtol 1e-10, {tot_it / max(1, args.steps):.0f} CG iterations on "
                                   f"average), the CPU restatement of the reference solver with its dense element "
                                   f"form, on {n_threads} host threads",
                         "host": host_cpu()},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    from mnhack8_b200 import _lib

    if args.profile_kernel:
        return profile_kernel(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(local)

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    N = args.N
    nodes, elems = (N + 1) ** 3, N ** 3
    k, r = make_field(N, 1 + rank)
    g = _lib.Solver(N, DT, k, r, kernel=args.kernel, scatter=args.scatter, detect=not args.no_detect,
                    no_source=True, ic="gaussian", ic_sigma=IC_SIGMA, rtol=RTOL, max_iter=500, device=local)
    # warm-up trajectories (graph instantiation, clocks)
    for _ in range(args.warmup):
        g.advance(STEPS_PER_TRAJ, from_ic=True)
    barrier()
    sampler = ClockSampler(local)
    with sampler:
        barrier()
        tot_it, tot_ms = 0, 0.0
        for _ in range(args.steps):
            it, ms = g.advance(STEPS_PER_TRAJ, from_ic=True)
            tot_it += it
            tot_ms += ms
        barrier()
    clocks = sampler.summary()
    # slowest rank's device time, all ranks' work
    ms_total, it_all = reduce_over_ranks(dist, tot_ms, tot_it, "cuda")
    value = nodes * it_all / (ms_total * 1e-3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "profile_run": True}), flush=True)
        g.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # ---- end to end through the C ABI with pinned host buffers -------------------
    T0 = torch.empty(nodes, dtype=torch.float64, pin_memory=True)
    T0.copy_(torch.from_numpy(_initial(g, N)))
    Tout = torch.empty(nodes, dtype=torch.float64, pin_memory=True)
    g.solve_host_ptr(T0.data_ptr(), Tout.data_ptr(), STEPS_PER_TRAJ)   # warm
    barrier()
    e2e_it, t0 = 0, time.perf_counter()
    for _ in range(args.steps):
        it, _ = g.solve_host_ptr(T0.data_ptr(), Tout.data_ptr(), STEPS_PER_TRAJ)
        e2e_it += it
    e2e_s = time.perf_counter() - t0
    e2e_all_s, e2e_it_all = reduce_over_ranks(dist, e2e_s, e2e_it, "cuda")
    e2e_value = nodes * e2e_it_all / e2e_all_s

    # ---- roofline of the dominant kernel (the fused PCG operator kernel) ----------
    ms_k1 = g.time_kernel(0, reps=20)
    ms_k2 = g.time_kernel(1, reps=20)
    detect = not args.no_detect
    alg_k1 = (40 if detect else 32) * nodes + 16 * elems   # read z, p_old[, w]; write p, Ap; read k, rho*c
    # the update at an odd iteration (timed): read x, p_{k-1}, p_k, Ap, r, d; write x, r, z
    # (an even iteration skips x: read Ap, r, d; write r, z)
    alg_k2 = 72 * nodes
    peak, peak_kind = peaks()
    ach = alg_k1 / (ms_k1 * 1e-3) / 1e9
    traffic, traffic_src = measure_traffic(N, args) if (world == 1 and args.measure_traffic) else \
        (None, "not measured in this run (a 1-GPU bench.py --measure-traffic takes it)")
    iters_per_traj = it_all / max(1, world) / args.steps
    # per time step: step begin/end, RHS and x0 operator (+ their final kernel with
    # ABFT), the PCG prologue's update, the solution update owed after the loop;
    # per CG iteration: operator and update (whose last CTA finishes the
    # reductions); the graph's while body runs 4 iterations per pass, so a step
    # launches whole passes.  The atomic scatter adds p formation, zeroing and
    # the finishing pass to each operator.
    if args.scatter == "colored":
        per_step, per_iter = 2 + 2 * (2 if detect else 1) + 2, 2
    else:
        per_step, per_iter = 2 + 2 * (4 if detect else 3) + 2, 5
    it_step = iters_per_traj / STEPS_PER_TRAJ
    loop_iters = 4 * int(np.ceil(it_step / 4))
    launches = int(round(args.steps * STEPS_PER_TRAJ * (per_step + per_iter * loop_iters)))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded lognormal conductivity, FFT Gaussian-field algorithm of the reference generator)",
        "config": workload_config(args, world),
        "cg_iters_per_trajectory": iters_per_traj,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "traffic": traffic, "traffic_source": traffic_src, "kernel": "k_apply_slab (PCG operator: p = z + beta p, Ap = A p, "
                     "p.Ap and ABFT partials)", "alg_bytes_per_launch": alg_k1, "ms_per_launch": ms_k1,
                     "peak_source": f"{peak_kind} hbm_gbs", "l2": "flushed before each timed launch",
                     "update_kernel": {"ms_per_launch": ms_k2, "alg_bytes_per_launch": alg_k2,
                                       "achieved": alg_k2 / (ms_k2 * 1e-3) / 1e9}},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": nodes * 8, "d2h_bytes_per_step": nodes * 8},
        "gpu_launches": launches,
        "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"]},
    }
    if rank == 0 and not args.no_gate and N != GATE_N:
        line["apply_gate_N256"] = gate_apply(local, detect, args.kernel, args.scatter)
    if rank == 0 and args.scatter == "colored":
        line["scatter_pair"] = scatter_pair(N, local, detect, args.kernel, ms_k1)
    if rank == 0 and world == 1 and args.batching_instances > 0:
        line["batching"] = batching_leg(args.batching_instances, local)
    if rank == 0 and world == 1 and args.serving_requests > 0:
        line["serving"] = serving_leg(args.serving_requests, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(N)
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    return 0


GATE_N = 256
PROFILE_REPS = 3


def profile_kernel(args):
    """Three launches of the PCG operator kernel on the bench's field at --N
    (the L2 scrubbed before each), timed with CUDA events; prints one JSON line."""
    from mnhack8_b200 import _lib
    N = args.N
    k, r = make_field(N, 1)
    g = _lib.Solver(N, DT, k, r, kernel=args.kernel, scatter=args.scatter, detect=not args.no_detect,
                    no_source=True, ic="gaussian", ic_sigma=IC_SIGMA, rtol=RTOL, max_iter=500, device=0)
    ms = g.time_kernel(0, reps=PROFILE_REPS)
    g.close()
    alg = (40 if not args.no_detect else 32) * (N + 1) ** 3 + 16 * N ** 3
    print(json.dumps({"N": N, "ms_per_launch": ms, "alg_bytes_per_launch": alg,
                      "achieved_gbs": alg / (ms * 1e-3) / 1e9}), flush=True)
    return 0


def serving_leg(n, device):
    """Supplementary: served solves/s and p50 / p99 latency of the batched
    mixed-precision server beside serial plain FP64 on this GPU, for the first
    n requests of the seeded serving stream (Poisson 200/s, N 16..160, 10..100
    steps, 30 % flipped, rtol 1e-8); fields are generated before timing (their
    per-request generation time is reported beside the latencies)."""
    from mnhack8_b200 import ensemble
    r = ensemble.serving(n=n, device=device)
    return {"requests": n, "stream": "Poisson 200/s, N 16..160, steps 10..100, 30% one bit flip, rtol 1e-8",
            "stream_span_s": r["stream_span_s"], "max_live": r["max_live"], "peak_live": r["peak_live"],
            "batched": r["batched"], "serial_fp64": r["serial_fp64"], "solves_per_s_ratio": r["throughput_ratio"],
            "field_generation": r["field_generation"]}


def batching_leg(n, device):
    """Supplementary: the ensemble of n independent solves (N uniform in
    16..96, lognormal k sigma 1 with correlation N/8 elements, 20 steps to
    rtol 1e-8) in one batch (one graph launch per step, autotuned tile depth)
    beside the same solves one at a time through the plain FP64 drop-in."""
    from mnhack8_b200 import ensemble
    r = ensemble.batching(n=n, device=device)
    keep = ("instances", "N_range", "steps", "rtol", "tile_planes", "autotune_ms_per_tile_planes", "batch_ms",
            "batch_solves_per_s", "serial_fp64_ms", "serial_fp64_solves_per_s", "serial_fp64_timed_solves",
            "max_final_true_rel_residual")
    out = {k: r[k] for k in keep}
    out["solves_per_s_ratio"] = r["speedup_vs_serial_fp64"]
    return out


def gate_apply(device, detect, kernel, scatter):
    """Supplementary: the PCG operator kernel alone at N=256 (129^3 -> 257^3
    nodes, the apply-roofline configuration), L2 scrubbed before each launch,
    on the same lognormal field family; not part of the headline metric."""
    from mnhack8_b200 import _lib
    N = GATE_N
    nodes, elems = (N + 1) ** 3, N ** 3
    k, r = make_field(N, 1)
    g = _lib.Solver(N, DT, k, r, kernel=kernel, scatter=scatter, detect=detect, no_source=True, ic="gaussian",
                    ic_sigma=IC_SIGMA, rtol=RTOL, max_iter=500, device=device)
    g.time_kernel(0, reps=3)
    ms = min(g.time_kernel(0, reps=20) for _ in range(2))
    g.close()
    alg = (40 if detect else 32) * nodes + 16 * elems
    peak, kind = peaks()
    ach = alg / (ms * 1e-3) / 1e9
    return {"N": N, "ms_per_launch": ms, "alg_bytes_per_launch": alg, "achieved": ach, "peak": peak,
            "unit": "GB/s", "frac": ach / peak, "peak_source": f"{kind} hbm_gbs", "l2": "flushed before each launch"}


def scatter_pair(N, device, detect, kernel, ms_colored):
    """Supplementary (config 2's comparison): the PCG operator per application
    with the atomic scatter (p formation, zeroing, element bricks with shared-
    memory accumulation and global atomics on brick faces, projection and
    partials) beside the colored kernel, same field, L2 scrubbed."""
    from mnhack8_b200 import _lib
    k, r = make_field(N, 1)
    g = _lib.Solver(N, DT, k, r, kernel=kernel, scatter="atomic", detect=detect, no_source=True, ic="gaussian",
                    ic_sigma=IC_SIGMA, rtol=RTOL, max_iter=500, device=device)
    g.time_kernel(0, reps=3)
    ms = g.time_kernel(0, reps=20)
    g.close()
    return {"N": N, "colored_ms_per_apply": ms_colored, "atomic_ms_per_apply": ms,
            "atomic_over_colored": ms / ms_colored}


def _initial(g, N):
    from mnhack8_b200 import _lib  # noqa: F401
    g.advance(0, from_ic=True)           # puts the initial condition into the solver's field
    return g.get_field()


if __name__ == "__main__":
    sys.exit(main())
