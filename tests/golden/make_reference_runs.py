"""Generate golden fixtures by running the REFERENCE solver (its own sources,
compiled by oracle/Makefile into oracle/_ref/libref_harness.so) on the named
workloads, at full length.

    python tests/golden/make_reference_runs.py CASE [--threads N] [--full-dir DIR]

CASE is one of: duct, slit, bulk_m3, bulk_0, bulk_p3 (see CASES). Each run
writes tests/golden/ref_<case>.npz with
  * the trajectory rows (the columns of the reference's _traj.dat),
  * the final squirmer state and diagnostics (countFluid/meanDensity/...),
  * rho, u and flag at a fixed seeded sample of nodes (4096, rng seed 7),
  * with a squirmer: rho, u and flag at every node of the sphere's shell,
    i.e. within R + SHELL_PAD of the final centre (minimum image), where the
    moving boundary, the refill and any precision effects concentrate,
  * for the duct: the whole x=0 cross-section,
  * wall-clock seconds and the OpenMP thread count used.
With --full-dir the complete final fields are also written there as .npy
(too large to commit; used for one-off full-field comparisons).

This script needs the reference sources (it runs only where oracle/_ref was
built from them); the fixtures it writes are what the tests read.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from lbm_solver_3d_b200.params import Params  # noqa: E402
from lbm_solver_3d_b200.workloads import workload_params  # noqa: E402
from oracle.oracle import RefSolver, set_threads  # noqa: E402

CASES = ("duct", "slit", "bulk_m3", "bulk_0", "bulk_p3")
SAMPLE_SEED = 7
SAMPLE_SIZE = 4096
SHELL_PAD = 3.0


def shell_nodes(p: Params, X: np.ndarray) -> np.ndarray:
    """Node indices (ascending) within R + SHELL_PAD of centre X, with the
    minimum image along every periodic axis."""
    z, y, x = np.meshgrid(np.arange(p.NZ), np.arange(p.NY), np.arange(p.NX), indexing="ij")
    d = []
    for c, n, periodic in ((x, p.NX, True), (y, p.NY, not p.wallsY), (z, p.NZ, not p.wallsZ)):
        r = c - X[len(d)]
        if periodic:
            r = r - n * np.round(r / n)
        d.append(r)
    r2 = d[0] ** 2 + d[1] ** 2 + d[2] ** 2
    return np.flatnonzero((r2 < (p.R + SHELL_PAD) ** 2).reshape(-1))


def sample_nodes(n_cells: int) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    k = min(SAMPLE_SIZE, n_cells)
    return np.sort(rng.choice(n_cells, size=k, replace=False))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=CASES)
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--full-dir", type=Path, default=None)
    ap.add_argument("--steps", type=int, default=None, help="override the step count (testing only)")
    a = ap.parse_args()

    p: Params = workload_params(a.case)
    steps = a.steps or p.steps
    set_threads(a.threads)
    s = RefSolver(p)
    t0 = time.time()
    traj = s.run(steps)
    sec = time.time() - t0
    flag, rho, u = s.fields()
    sq = s.squirmer() if p.squirmer else None
    diag = s.diag()
    idx = sample_nodes(p.ncells)
    out = dict(
        kv=np.array(p.to_kv()), steps=steps, seconds=sec, threads=a.threads,
        mlups=p.ncells * steps / sec / 1e6,
        traj=traj, wall_force=s.wall_force(),
        diag=np.array([diag["n_fluid"], diag["mean_density"], diag["max_speed"], diag["sum_ux"]]),
        sample_idx=idx, sample_flag=flag.reshape(-1)[idx], sample_rho=rho.reshape(-1)[idx],
        sample_u=u.reshape(-1, 3)[idx],
        sum_rho=float(rho[flag == 0].sum()), sum_u=u[flag == 0].sum(axis=0),
        sum_u2=float((u[flag == 0] ** 2).sum()),
    )
    if sq is not None:
        for k in ("X", "e", "U", "W", "Fh", "Th", "Fc", "Tc", "Fw"):
            out["sq_" + k] = sq[k]
        out["sq_contacts"] = sq["contacts"]
        sh = shell_nodes(p, np.asarray(sq["X"]))
        out.update(shell_idx=sh, shell_flag=flag.reshape(-1)[sh], shell_rho=rho.reshape(-1)[sh],
                   shell_u=u.reshape(-1, 3)[sh])
    if a.case == "duct":
        out["x0_rho"] = rho[:, :, 0]
        out["x0_u"] = u[:, :, 0, :]
        out["x0_flag"] = flag[:, :, 0]
        out["l2_error"] = s.poiseuille_error("/tmp/ref_duct_golden")
    dst = Path(__file__).resolve().parent / f"ref_{a.case}.npz"
    np.savez_compressed(dst, **out)
    if a.full_dir is not None:
        a.full_dir.mkdir(parents=True, exist_ok=True)
        np.save(a.full_dir / f"{a.case}_flag.npy", flag)
        np.save(a.full_dir / f"{a.case}_rho.npy", rho)
        np.save(a.full_dir / f"{a.case}_u.npy", u)
    print(f"{a.case}: {steps} steps in {sec:.1f} s ({out['mlups']:.2f} MLUPS, {a.threads} threads) -> {dst}")


if __name__ == "__main__":
    main()
