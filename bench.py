#!/usr/bin/env python
"""Throughput of the D3Q19 TRT + squirmer time step on B200, as MLUPS.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32]
                    [--workload bulk_0] [--impl ours|reference]

Workload (default): the precision/roofline sweep lattice -- a fully periodic
256x128x128 box with one squirmer (a=8, beta=0, B1=1e-3, tau=0.9, seeded 3-D
orientation), FP32-shifted populations. A "step" is one time step of the whole
hot path (collide-stream + bounce-back + momentum exchange + rigid body +
remap + mass correction every 10 steps), run through the C ABI's time loop.
The populations (319 MB in FP32) are larger than the 126 MB L2, so no flush is
needed between steps. MLUPS counts every lattice node, as the reference does
(src/main.cpp:90).

One process per GPU (torchrun for N > 1): each rank advances its own replica of
the lattice -- a single lattice is not split across GPUs -- so scaling is weak
and `value` is the sum over ranks (cells x steps / slowest rank's time).

--impl reference times the reference's own CPU code (compiled from its sources
into oracle/_ref) on the host cores, on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
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
            inside = [r for t, r in rows if self.t0 <= t <= self.t1 + 0.2]
        else:
            inside = [r for _, r in rows]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside)}


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
        s = oracle.RefSolver(p)
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
    return {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind,
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
    s = oracle.RefSolver(p) if kind == "reference" else oracle.PortSolver(p)
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
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": kind,
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
    return {"workload": what,
            "cells": p.ncells, "precision": "fp64" if reference else args.precision,
            "mass_correction_every": p.massCorrectionEvery,
            "l2": ("populations larger than L2 (126 MB); no flush"
                   if 38 * BYTES["fp64" if reference else args.precision] * p.ncells / 2 > 126e6
                   else "populations fit in L2 (126 MB): L2-resident, the roofline fraction is not an HBM claim"),
            "parallelism": f"replica per GPU x{dist_env()[0]}"}


def bench_ensemble(args):
    """Trajectories per hour: the 256-member slit-channel ensemble (FP32-shifted
    unless --precision says otherwise, 30000 steps per trajectory, autotuned
    bulk tiling, CUDA graphs) against the same members solved one after
    another with the plain FP64 path (and with FP32 alone, for reference). The
    sequential time per step is measured on a seeded sample of members, each
    alone, and scaled to all 256. With N ranks the members are split across
    the GPUs (shard_members, no exchange): weak in the per-GPU work, and the
    whole ensemble's step time is the slowest rank's."""
    import torch
    from lbm_solver_3d_b200.ensemble import Ensemble, shard_members
    from lbm_solver_3d_b200.solver import Solver
    from lbm_solver_3d_b200.workloads import ensemble_members

    world, rank, local = dist_env()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs one lattice per "
                              "process; its ensemble is the sequential loop measured by --workload ensemble"}))
        return
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    all_ps = ensemble_members(256)
    prec = args.precision if args.precision_set else "fp32"
    for p in all_ps:
        p.update(precision=prec, device=local)
    mine = shard_members(all_ps, rank, world)
    ps = [all_ps[i] for i in mine]
    traj_steps = ps[0].steps
    stream = torch.cuda.Stream(device=local)
    ens = Ensemble(ps)
    ens.set_stream(stream.cuda_stream)
    tune = ens.autotune(reps=3)
    ens.run(args.warmup)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ens.launch_count()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.start()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            ens.run(args.steps)
            ev1.record(stream)
        torch.cuda.synchronize()
        clk.stop()
    if pg:
        pg.barrier()
    t_max = torch.tensor([ev0.elapsed_time(ev1) / args.steps], device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t_max, op=pg.ReduceOp.MAX)
    ms_step = float(t_max.item())
    launches = ens.launch_count() - l0
    bulk_ms = ens.time_bulk(reps=5)
    cells = ens.cells
    ens.close()
    traj_h = len(all_ps) * 3600.0 / (traj_steps * ms_step * 1e-3)

    seq = None
    if rank == 0:
        # sequential solves of a seeded sample of members, each alone
        rng = np.random.default_rng(7)
        sample = sorted(rng.choice(len(all_ps), size=12, replace=False).tolist())
        seq = {"sample_members": sample}
        for sp in ("fp64", "fp32"):
            per = []
            for i in sample:
                q = all_ps[i].copy().update(precision=sp)
                s = Solver(q)
                s.set_stream(stream.cuda_stream)
                s.run(args.warmup)
                torch.cuda.synchronize()
                with torch.cuda.stream(stream):
                    ev0.record(stream)
                    s.run(args.steps)
                    ev1.record(stream)
                torch.cuda.synchronize()
                per.append(ev0.elapsed_time(ev1) / args.steps)
                s.close()
            mean_ms = float(np.mean(per))
            seq[sp] = {"ms_per_step_mean": mean_ms,
                       "trajectories_per_hour": 3600.0 / (traj_steps * mean_ms * 1e-3)}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = peaks()
    bytes_step = 2 * 19 * BYTES[prec] * cells
    line = {
        "metric": "ensemble trajectories/hour (256 slit channels, 30000 steps each)",
        "value": traj_h, "unit": "trajectories/h", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE[prec], "data": "synthetic",
        "config": {"workload": "ensemble: 256 slit-channel squirmers, Nx 64-160, Ny/Nz 48-96, a 4-8, "
                               "beta -5..5, angle -30..30 deg, seed 2024",
                   "members_on_rank0": len(ps), "cells_on_rank0": cells, "tiling_rank0": tune,
                   "parallelism": f"members split across {world} GPU(s)",
                   "l2": "populations larger than L2; no flush"},
        "sequential": seq,
        "speedup_vs_sequential_fp64": traj_h / seq["fp64"]["trajectories_per_hour"],
        "speedup_vs_sequential_fp32": traj_h / seq["fp32"]["trajectories_per_hour"],
        "roofline": {"bound": "hbm", "kernel": "ensemble bulk kernel (rank 0)", "launch_ms": bulk_ms,
                     "achieved": bytes_step / (bulk_ms * 1e-3) / 1e9, "peak": peak,
                     "frac": bytes_step / (bulk_ms * 1e-3) / 1e9 / peak, "unit": "GB/s",
                     "peak_source": peak_kind, "step_frac": bytes_step / (ms_step * 1e-3) / 1e9 / peak},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--precision", default=None, choices=list(BYTES))
    ap.add_argument("--workload", default="bulk_0")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    p.update(device=local)
    from lbm_solver_3d_b200.solver import Solver

    stream = torch.cuda.Stream(device=local)
    sol = Solver(p)
    sol.set_stream(stream.cuda_stream)
    sol.run(args.warmup)
    torch.cuda.synchronize()

    # ---- timed region: K time steps on the device, inputs resident in HBM ----
    l0 = sol.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.start()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            sol.run(args.steps)
            ev1.record(stream)
        torch.cuda.synchronize()
        clk.stop()
    if pg:
        pg.barrier()
    ms = ev0.elapsed_time(ev1)
    launches = sol.launch_count() - l0
    t_max = torch.tensor([ms], device=f"cuda:{local}")
    if pg:
        pg.all_reduce(t_max, op=pg.ReduceOp.MAX)
    ms_max = float(t_max.item())
    value = world * p.ncells * args.steps / (ms_max * 1e-3) / 1e6

    # ---- dominant kernel alone (CUDA events on the library's stream) ----
    kt = sol.time_kernels(reps=20)
    sol.close()
    peak, peak_kind = peaks()
    bytes_per_launch = 2 * 19 * BYTES[args.precision] * p.ncells
    achieved = bytes_per_launch / (kt["bulk"] * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(f"k_bulk:{args.workload}:{args.precision}")
        except Exception:
            traffic = None

    # ---- end to end through the C ABI: create from host params, run, read results ----
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = Solver(p)
    traj_bytes = 0
    remaining = args.steps
    chunk = max(p.trajEvery, min(remaining, 1000))
    while remaining > 0:
        k = min(chunk, remaining)
        s2.run(k)
        traj_bytes += s2.traj_rows().nbytes
        remaining -= k
    flag, rho, u = s2.fields()
    t_e2e = time.perf_counter() - t0
    s2.close()
    h2d = p.ncells * 1 + 4 * (p.ncells if p.squirmer else 0)  # flags + boundary-link set-up
    d2h = traj_bytes + flag.nbytes + rho.nbytes + u.nbytes
    e2e_val = p.ncells * args.steps / t_e2e / 1e6
    e2e = {"value": world * e2e_val, "unit": "MLUPS",
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "what": "lbmgpu_create (host set-up and upload) + lbmgpu_run in chunks + trajectory rows "
                   "+ final flag/rho/u fields to host, wall clock per rank"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[args.precision], "data": "synthetic",
            "config": workload_config(args, p),
            "roofline": {"bound": "hbm", "kernel": "k_bulk (collide-stream, AA, bulk nodes)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_kind,
                         "bytes_per_launch": bytes_per_launch, "launch_ms": kt["bulk"],
                         "per_unit": f"2 x 19 x {BYTES[args.precision]} B per lattice node"},
            "step_breakdown_ms": kt,
            "step_roofline_frac": (bytes_per_launch / (ms_max / args.steps * 1e-3) / 1e9) / peak,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "e2e": e2e,
        }
        if not args.no_cpu_baseline and world == 1:
            q = workload_params(args.workload, "fp64")
            line["cpu_baseline"] = cpu_baseline(q)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
