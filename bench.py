#!/usr/bin/env python
"""Throughput and accuracy of the D3Q19 TRT + squirmer time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32]
                    [--workload bulk_0] [--impl ours|reference] [--headline-only]

Headline (one JSON line): the precision/roofline sweep lattice -- a fully
periodic 256x128x128 box with one squirmer (a=8, beta=0, B1=1e-3, tau=0.9,
seeded 3-D orientation) -- with FP32-shifted populations, as MLUPS. A "step" is
one time step of the whole hot path (collide-stream + bounce-back + momentum
exchange + rigid body + remap + mass correction every 10 steps), run through
the C ABI's time loop. The populations (319 MB in FP32) are larger than the
126 MB L2, so no flush is needed between steps. MLUPS counts every lattice
node, as the reference does (src/main.cpp:90).

The same line carries the rest of the metric ("MLUPS & %HBM roofline FP64 vs
FP32-shifted at <=1e-5 err; sweep trajectories/hr"), each measured in this run:
  forms     the FP64 and FP16-storage forms of the same lattice: MLUPS, the
            bulk kernel's roofline, the step's roofline;
  accuracy  the lattice at full length (10000 steps) for beta = -3, 0, +3 in
            all three forms: u / rho relative L2 and centre drift of FP32 and
            FP16 against the FP64 run, and of FP64 against the reference's own
            run (committed fixtures, seeded sample + the sphere's shell);
  ensemble  the 256-member slit-channel ensemble (FP32 and FP16, autotuned,
            CUDA graphs): trajectories per hour against sequential solves.
The K-step timed window sits inside a span of at least a second of the same
steps, so the nvidia-smi sampler (200 ms period) sees the clocks it ran at.

One process per GPU (torchrun for N > 1): each rank advances its own replica of
the lattice -- a single lattice is not split across GPUs -- so scaling is weak
and `value` is the sum over ranks (cells x steps / slowest rank's time). With
N > 1 only the headline and e2e are measured.

--impl reference times the reference's own CPU code (compiled from its sources
into oracle/_ref) on the host cores, on the same workload.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS & %HBM roofline FP64 vs FP32-shifted at ≤1e-5 err; sweep trajectories/hr"
BYTES = {"fp64": 8, "fp32": 4, "fp16": 2}
DTYPE = {"fp64": "f64", "fp32": "f32-shifted", "fp16": "f16-storage/f32-math"}
SPAN_S = 0.6          # loaded time before and after the timed window (clock sampling)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc = gpu, [], None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            deadline = time.time() + 5.0      # the timed region starts once sampling runs
            while not self.rows and time.time() < deadline:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), [c.strip() for c in line.split(",")]))

    def start(self):
        self.t0 = time.time()

    def stop(self):
        self.t1 = time.time()

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = self.rows
        if self.t0 is not None and self.t1 is not None:
            inside = [r for t, r in rows if self.t0 <= t <= self.t1]
        else:
            inside = [r for _, r in rows]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside),
                "span_s": round(self.t1 - self.t0, 3) if self.t0 and self.t1 else None}


# ---------------------------------------------------------------------------
#  CPU legs: the reference's own code (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------
def cpu_baseline(p, seconds_target=15.0):
    """The reference's own code (oracle/_ref, compiled from its sources) on the
    host cores: a bounded sample of the same workload."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    if not oracle.ref_available():
        s = oracle.PortSolver(p)
        kind = "port"
    else:
        s = oracle.RefSolver(p, timed=True)
        kind = "reference"
    s.run(1)  # first touch
    steps, t = 1, 0.0
    while True:
        t0 = time.perf_counter()
        s.run(steps)
        t = time.perf_counter() - t0
        if t > 0.25 * seconds_target or steps >= 256:
            break
        steps *= 2
    mlups = p.ncells * steps / t / 1e6
    # the same sample on one thread (a bounded number of steps)
    oracle.set_threads(1)
    steps1 = max(1, min(steps, int(0.2 * seconds_target / max(t / steps * threads, 1e-9))))
    t0 = time.perf_counter()
    s.run(steps1)
    t1 = time.perf_counter() - t0
    oracle.set_threads(threads)
    return {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind, "build": oracle.ref_build(),
            "sample": f"{p.NX}x{p.NY}x{p.NZ} lattice, {steps} time steps after 1 warm-up step, "
                      f"{threads} OpenMP threads, FP64 (the reference's only form)",
            "one_thread": {"value": p.ncells * steps1 / t1 / 1e6, "unit": "MLUPS", "cores": 1,
                           "sample": f"{steps1} further time steps on 1 thread"}}


def run_reference_arm(args, p):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    kind = "reference" if oracle.ref_available() else "port"
    s = oracle.RefSolver(p, timed=True) if kind == "reference" else oracle.PortSolver(p)
    # a bounded sample of the workload: at most K steps and about 90 s of CPU time
    warm = min(args.warmup, 3)
    for _ in range(warm):
        s.run(1)
    times = []
    budget = 90.0
    while len(times) < args.steps and sum(times) < budget:
        t0 = time.perf_counter()
        s.run(1)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    n = len(times)
    mlups = p.ncells * n / tot / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args, p, reference=True),
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind, "build": oracle.ref_build(),
                         "sample": f"{n} of the workload's time steps (bounded to ~{budget:.0f} s) after {warm} "
                                   f"warm-up steps, {threads} OpenMP threads"},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args, p, reference=False):
    if not p.squirmer:
        what = f"{args.workload}: {p.NX}x{p.NY}x{p.NZ} duct, walls in y and z, body force fx={p.Fx:g}"
    elif args.workload == "slit":
        what = (f"slit: {p.NX}x{p.NY}x{p.NZ}, walls in y, one squirmer a={p.R:g} beta={p.beta:g} "
                f"B1={p.B1:g} tau={p.tau:g} angle={p.angle:g}")
    else:
        what = (f"{args.workload}: periodic {p.NX}x{p.NY}x{p.NZ} box, one squirmer a={p.R:g} beta={p.beta:g} "
                f"B1={p.B1:g} tau={p.tau:g}, seeded 3-D orientation")
    prec = "fp64" if reference else args.precision
    return {"workload": what,
            "cells": p.ncells, "precision": prec,
            "mass_correction_every": p.massCorrectionEvery,
            "l2": ("populations larger than L2 (126 MB); no flush"
                   if 38 * BYTES[prec] * p.ncells / 2 > 126e6
                   else "populations fit in L2 (126 MB): L2-resident, the roofline fraction is not an HBM claim"),
            "parallelism": f"replica per GPU x{dist_env()[0]}"}


# ---------------------------------------------------------------------------
#  GPU legs
# ---------------------------------------------------------------------------
def timed_window(run, steps, warm_ms_per_step, stream, dev, pg=None):
    """Time exactly `steps` steps between CUDA events on `stream`, inside a
    span of the same steps of at least SPAN_S seconds before and after, with
    nvidia-smi sampling the clocks over the whole span. Returns (ms of the
    window, clock summary)."""
    import torch
    pre = max(1, int(SPAN_S * 1e3 / max(warm_ms_per_step, 1e-4)))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        clk.start()
        run(pre)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            run(steps)
            ev1.record(stream)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        run(pre)
        torch.cuda.synchronize()
        clk.stop()
    return ev0.elapsed_time(ev1), clk.summary()


def warm_rate(run, warmup, stream):
    """Runs the warm-up steps and returns their ms per step."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    run(1)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        run(max(1, warmup - 1))
        ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / max(1, warmup - 1)


# the bulk kernel of steps without sums, per storage form (nx a multiple of 64)
BULK_KERNEL = {"fp64": "k_bulk_rows", "fp32": "k_bulk_rows", "fp16": "k_bulk_rows2"}


def measure_lattice(p, prec, args, stream, dev, pg=None):
    """MLUPS of K steps and the bulk kernel's roofline for one storage form."""
    from lbm_solver_3d_b200.solver import Solver
    sol = Solver(p)
    sol.set_stream(stream.cuda_stream)
    ms_w = warm_rate(sol.run, args.warmup, stream)
    l0 = sol.launch_count()
    ms, clocks = timed_window(sol.run, args.steps, ms_w, stream, dev, pg)
    pre = max(1, int(SPAN_S * 1e3 / max(ms_w, 1e-4)))
    launches = sol.launch_count() - l0
    kt = sol.time_kernels(reps=20)
    sol.close()
    peak, peak_kind = peaks()
    bytes_per_launch = 2 * 19 * BYTES[prec] * p.ncells
    achieved = bytes_per_launch / (kt["bulk"] * 1e-3) / 1e9
    ms_step = ms / args.steps
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            tr = json.loads(tf.read_text())
            traffic = tr.get(f"{BULK_KERNEL[prec]}:{args.workload}:{prec}")
        except Exception:
            traffic = None
    return {
        "ms": ms, "ms_per_step": ms_step, "value": p.ncells / (ms_step * 1e-3) / 1e6,
        # kernels of the K-step window alone (the span's extra steps excluded)
        "launches": int(round(launches * args.steps / (args.steps + 2 * pre))),
        "clocks": clocks,
        "roofline": {"bound": "hbm", "kernel": f"bulk collide-stream ({BULK_KERNEL[prec]} on steps without sums, "
                                               "k_bulk_rows with sums on the one in ten with sums; averaged)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_launch": bytes_per_launch, "launch_ms": kt["bulk"],
                     "per_unit": f"2 x 19 x {BYTES[prec]} B per lattice node"},
        "step_breakdown_ms": kt,
        "step_roofline_frac": (bytes_per_launch / (ms_step * 1e-3) / 1e9) / peak,
    }


def _rel(a, b, m):
    d = np.linalg.norm(b[m])
    return float(np.linalg.norm((a - b)[m]) / d) if d > 0 else 0.0


def accuracy_record(workloads=("bulk_m3", "bulk_0", "bulk_p3")):
    """Each precision form against the FP64 form at full length, and the FP64
    form against the reference's own run of the same workload (committed
    fixtures: the seeded sample of 4096 nodes and every node of the sphere's
    shell)."""
    from lbm_solver_3d_b200.solver import Solver
    from lbm_solver_3d_b200.workloads import workload_params
    out = {}
    for wl in workloads:
        p64 = workload_params(wl, "fp64")
        steps = p64.steps
        rec = {"steps": steps, "beta": p64.beta}
        s = Solver(p64)
        s.run(steps)
        f64, r64, u64 = s.fields()
        sq64 = s.squirmer()
        s.close()
        g = np.load(ROOT / "tests" / "golden" / f"ref_{wl}.npz")
        vs_ref = {"X_abs": float(np.abs(sq64["X"] - g["sq_X"]).max()),
                  "e_abs": float(np.abs(sq64["e"] - g["sq_e"]).max())}
        for key in ("sample", "shell"):
            if f"{key}_idx" in g.files:
                idx = g[f"{key}_idx"]
                fl = g[f"{key}_flag"] == 0   # rho/u of solid nodes are stale values, not compared
                vs_ref[f"{key}_nodes"] = int(idx.size)
                vs_ref[f"{key}_flags_equal"] = bool(np.array_equal(f64.reshape(-1)[idx], g[f"{key}_flag"]))
                vs_ref[f"{key}_u_rel_l2"] = float(np.linalg.norm(u64.reshape(-1, 3)[idx][fl] - g[f"{key}_u"][fl]) /
                                                  np.linalg.norm(g[f"{key}_u"][fl]))
                vs_ref[f"{key}_rho_rel_l2"] = float(np.linalg.norm(r64.reshape(-1)[idx][fl] - g[f"{key}_rho"][fl]) /
                                                    np.linalg.norm(g[f"{key}_rho"][fl]))
        rec["fp64_vs_reference"] = vs_ref
        for prec in ("fp32", "fp16"):
            s = Solver(workload_params(wl, prec))
            s.run(steps)
            f, r, u = s.fields()
            sq = s.squirmer()
            s.close()
            m = (f64 == 0) & (f == 0)
            rec[prec] = {"u_rel_l2": _rel(u, u64, m[..., None].repeat(3, -1)), "rho_rel_l2": _rel(r, r64, m),
                         "X_abs": float(np.abs(sq["X"] - sq64["X"]).max()),
                         "X_rel": float(np.linalg.norm(sq["X"] - sq64["X"]) /
                                        max(np.linalg.norm(sq64["X"] - np.asarray(g["traj"][0, 1:4])), 1e-30)),
                         "e_abs": float(np.abs(sq["e"] - sq64["e"]).max()),
                         "flag_differences": int((f != f64).sum())}
        out[wl] = rec
    return out


def ensemble_record(args, prec, stream, dev, with_sequential):
    """Trajectories per hour of the 256-member slit-channel ensemble (30000
    steps per trajectory, autotuned bulk tiling, CUDA graphs), and optionally
    the same members solved one after another (a seeded sample of 12, each
    alone, FP64 and FP32, scaled to all 256)."""
    import torch
    from lbm_solver_3d_b200.ensemble import Ensemble
    from lbm_solver_3d_b200.solver import Solver
    from lbm_solver_3d_b200.workloads import ensemble_members
    ps = ensemble_members(256)
    for p in ps:
        p.update(precision=prec, device=dev)
    traj_steps = ps[0].steps
    t0 = time.perf_counter()
    ens = Ensemble(ps)
    ens.set_stream(stream.cuda_stream)
    create_s = time.perf_counter() - t0
    tune = ens.autotune(reps=3)
    ms_w = warm_rate(ens.run, args.warmup, stream)
    l0 = ens.launch_count()
    ms, clocks = timed_window(ens.run, args.steps, ms_w, stream, dev)
    launches = ens.launch_count() - l0
    bulk_ms = ens.time_bulk(reps=5)
    cells = ens.cells
    ens.close()
    ms_step = ms / args.steps
    traj_h = len(ps) * 3600.0 / (traj_steps * ms_step * 1e-3)
    peak, peak_kind = peaks()
    bytes_step = 2 * 19 * BYTES[prec] * cells
    rec = {"dtype": DTYPE[prec], "members": len(ps), "cells": cells, "ms_per_step": ms_step,
           "trajectories_per_hour": traj_h, "tiling": tune, "create_s": create_s, "clocks": clocks,
           "launches_per_step": launches / (args.steps + 2 * max(1, int(SPAN_S * 1e3 / max(ms_w, 1e-4)))),
           "roofline": {"bound": "hbm", "kernel": "ensemble bulk kernel", "launch_ms": bulk_ms,
                        "achieved": bytes_step / (bulk_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": bytes_step / (bulk_ms * 1e-3) / 1e9 / peak, "peak_source": peak_kind,
                        "step_frac": bytes_step / (ms_step * 1e-3) / 1e9 / peak,
                        "per_unit": f"2 x 19 x {BYTES[prec]} B per lattice node"}}
    if with_sequential:
        rng = np.random.default_rng(7)
        sample = sorted(rng.choice(len(ps), size=12, replace=False).tolist())
        seq = {"sample_members": sample}
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for sp in ("fp64", "fp32"):
            per = []
            for i in sample:
                s = Solver(ps[i].copy().update(precision=sp))
                s.set_stream(stream.cuda_stream)
                s.run(args.warmup)
                torch.cuda.synchronize()
                with torch.cuda.stream(stream):
                    ev0.record(stream)
                    s.run(max(args.steps, 50))
                    ev1.record(stream)
                torch.cuda.synchronize()
                per.append(ev0.elapsed_time(ev1) / max(args.steps, 50))
                s.close()
            mean_ms = float(np.mean(per))
            seq[sp] = {"ms_per_step_mean": mean_ms,
                       "trajectories_per_hour": 3600.0 / (traj_steps * mean_ms * 1e-3)}
        rec["sequential"] = seq
    return rec


def e2e_record(p, args):
    """The metric end to end through the C ABI with host buffers, over the
    whole job a user runs: create the lattice from host parameters (flags and
    boundary links built and copied to the device), run the workload's full
    length (or --e2e-steps) in chunks reading the trajectory rows back at the
    driver's cadence, then copy the final node types, density and velocity
    into page-locked host buffers (allocated before the timed region); wall
    clock. The creation alone is also reported."""
    import torch
    from lbm_solver_3d_b200.solver import HostFields, Solver
    steps = args.e2e_steps or p.steps
    out = HostFields(p.ncells, pinned=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = Solver(p)
    t_create = time.perf_counter() - t0
    traj_bytes = 0
    remaining = steps
    chunk = max(p.trajEvery, min(remaining, 1000))
    while remaining > 0:
        k = min(chunk, remaining)
        s2.run(k)
        traj_bytes += s2.traj_rows().nbytes
        remaining -= k
    flag, rho, u = s2.fields_into(out)
    t_e2e = time.perf_counter() - t0
    s2.close()
    out.close()
    h2d = p.ncells * 1 + 4 * (p.ncells if p.squirmer else 0)  # flags + boundary-link set-up
    d2h = traj_bytes + flag.nbytes + rho.nbytes + u.nbytes
    world = dist_env()[0]
    return {"value": world * p.ncells * steps / t_e2e / 1e6, "unit": "MLUPS", "steps": steps,
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "create_s": t_create, "run_and_readback_s": t_e2e - t_create,
            "value_excluding_create": world * p.ncells * steps / (t_e2e - t_create) / 1e6,
            "what": "lbmgpu_create (host parameters -> lattice on the device) + lbmgpu_run in chunks + "
                    "trajectory rows + final flag/rho/u fields to host, wall clock per rank"}


def bench_ensemble(args):
    """--workload ensemble: the ensemble alone as the line (members split
    across ranks with shard_members, no exchange)."""
    import torch
    from lbm_solver_3d_b200.ensemble import Ensemble, shard_members
    from lbm_solver_3d_b200.workloads import ensemble_members

    world, rank, local = dist_env()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs one lattice per "
                              "process; its ensemble is the sequential loop measured by --workload ensemble"}))
        return
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    prec = args.precision if args.precision_set else "fp32"
    if world == 1:
        rec = ensemble_record(args, prec, stream, local, with_sequential=True)
        line = {
            "metric": "ensemble trajectories/hour (256 slit channels, 30000 steps each)",
            "value": rec["trajectories_per_hour"], "unit": "trajectories/h", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[prec], "data": "synthetic",
            "config": {"workload": "ensemble: 256 slit-channel squirmers, Nx 64-160, Ny/Nz 48-96, a 4-8, "
                                   "beta -5..5, angle -30..30 deg, seed 2024", "cells": rec["cells"],
                       "tiling": rec["tiling"], "parallelism": "one GPU",
                       "l2": "populations larger than L2; no flush"},
            "sequential": rec["sequential"],
            "speedup_vs_sequential_fp64": rec["trajectories_per_hour"] /
            rec["sequential"]["fp64"]["trajectories_per_hour"],
            "speedup_vs_sequential_fp32": rec["trajectories_per_hour"] /
            rec["sequential"]["fp32"]["trajectories_per_hour"],
            "roofline": rec["roofline"], "gpu_launches": int(rec["launches_per_step"] * args.steps),
            "clocks": rec["clocks"],
        }
        print(json.dumps(line), flush=True)
        return
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    all_ps = ensemble_members(256)
    for p in all_ps:
        p.update(precision=prec, device=local)
    ps = [all_ps[i] for i in shard_members(all_ps, rank, world)]
    ens = Ensemble(ps)
    ens.set_stream(stream.cuda_stream)
    tune = ens.autotune(reps=3)
    ms_w = warm_rate(ens.run, args.warmup, stream)
    l0 = ens.launch_count()
    ms, clocks = timed_window(ens.run, args.steps, ms_w, stream, local, dist)
    launches = ens.launch_count() - l0
    cells = ens.cells
    ens.close()
    t_max = torch.tensor([ms / args.steps], device=f"cuda:{local}")
    dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_step = float(t_max.item())
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        traj_h = len(all_ps) * 3600.0 / (all_ps[0].steps * ms_step * 1e-3)
        print(json.dumps({
            "metric": "ensemble trajectories/hour (256 slit channels, 30000 steps each)", "value": traj_h,
            "unit": "trajectories/h", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[prec], "data": "synthetic",
            "config": {"workload": "ensemble: 256 slit-channel squirmers (seed 2024)", "cells_on_rank0": cells,
                       "tiling_rank0": tune, "parallelism": f"members split across {world} GPUs"},
            "gpu_launches": launches, "clocks": clocks}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", default=None, choices=list(BYTES))
    ap.add_argument("--workload", default="bulk_0")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end record (default: the workload's full length)")
    ap.add_argument("--headline-only", action="store_true",
                    help="measure the headline line only (no forms/accuracy/ensemble sub-records)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: warm-up and K steps of the workload, then each kernel timed alone; "
                         "a short JSON line, no span, e2e or CPU legs (for a launch list or one ncu capture)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    args.precision_set = args.precision is not None
    if args.precision is None:
        args.precision = "fp32"

    if args.workload == "ensemble":
        bench_ensemble(args)
        return

    from lbm_solver_3d_b200.workloads import workload_params
    p = workload_params(args.workload, "fp64" if args.impl == "reference" else args.precision)

    if args.impl == "reference":
        run_reference_arm(args, p)
        return

    world, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if args.profile:
        from lbm_solver_3d_b200.solver import Solver
        sol = Solver(p.update(device=local))
        sol.run(args.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol.run(args.steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        kt = sol.time_kernels(reps=4)
        sol.close()
        print(json.dumps({"profile": args.workload, "precision": args.precision, "steps": args.steps,
                          "wall_ms_per_step": 1e3 * wall / args.steps, "kernels_ms": kt}), flush=True)
        return
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    p.update(device=local)
    stream = torch.cuda.Stream(device=local)

    # ---- headline: K time steps on the device, inputs resident in HBM ----
    head = measure_lattice(p, args.precision, args, stream, local, pg)
    t_max = torch.tensor([head["ms"]], device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t_max, op=pg.ReduceOp.MAX)
    ms_max = float(t_max.item())
    value = world * p.ncells * args.steps / (ms_max * 1e-3) / 1e6

    # ---- end to end through the C ABI with host buffers ----
    e2e = e2e_record(p, args)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return

    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[args.precision], "data": "synthetic",
        "config": workload_config(args, p),
        "roofline": head["roofline"],
        "step_breakdown_ms": head["step_breakdown_ms"],
        "step_roofline_frac": head["step_roofline_frac"],
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "e2e": e2e,
    }
    full = world == 1 and not args.headline_only and args.workload == "bulk_0"
    if full:
        # the rest of the metric, measured in the same run
        forms = {}
        for prec in ("fp64", "fp16"):
            if prec == args.precision:
                continue
            r = measure_lattice(workload_params(args.workload, prec).update(device=local), prec, args, stream, local)
            forms[prec] = {k: r[k] for k in ("value", "ms_per_step", "roofline", "step_roofline_frac", "clocks",
                                             "step_breakdown_ms")}
            forms[prec]["dtype"] = DTYPE[prec]
            forms[prec]["unit"] = "MLUPS"
        acc = accuracy_record()
        own = acc["bulk_0"].get(args.precision)
        line["error_vs_fp64"] = (dict(own, workload="bulk_0 at full length (10000 steps), the same run's FP64 form "
                                                    "as the oracle (itself matched to the reference's run: see "
                                                    "accuracy)")
                                 if own else None)
        for prec in forms:
            if prec in acc["bulk_0"]:
                forms[prec]["error_vs_fp64"] = acc["bulk_0"][prec]
        line["forms"] = forms
        line["accuracy"] = acc
        line["ensemble"] = {prec: ensemble_record(args, prec, stream, local, with_sequential=(prec == "fp32"))
                            for prec in ("fp32", "fp16")}
        seq = line["ensemble"]["fp32"]["sequential"]
        for prec in ("fp32", "fp16"):
            e = line["ensemble"][prec]
            e["speedup_vs_sequential_fp64"] = e["trajectories_per_hour"] / seq["fp64"]["trajectories_per_hour"]
            e["speedup_vs_sequential_fp32"] = e["trajectories_per_hour"] / seq["fp32"]["trajectories_per_hour"]
    if not args.no_cpu_baseline and world == 1:
        q = workload_params(args.workload, "fp64")
        line["cpu_baseline"] = cpu_baseline(q)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
