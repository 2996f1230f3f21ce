"""Training and held-out data for the swimmer surrogate, generated by the
batched LBM itself (Ensemble over slit channels, FP32-shifted).

Each member of an ensemble records trajectory rows every traj_every steps:
t, X, Y, Z, ex, ey, ez, Ux, Uy, Uz, Wx, Wy, Wz, Fwall_y, Fwall_z (the columns
of the reference's <prefix>_traj.dat, src/utils/io.cpp:79-83). A sample pairs
the swimmer's state with its instantaneous velocity:

    inputs   h/a      height of the centre above the lower wall plane
                      (y = 0.5, halfway bounce-back) in radii
             theta    in-plane orientation atan2(ey, ex) (rad)
             beta     squirming parameter of the member
             H/a      channel height H = Ny - 2 in radii
    targets  Ux/U0, Uy/U0, Omega_z a/U0, with U0 = 2 B1 / 3 (the bulk
             swimming speed of a two-mode squirmer)

Rows before `transient` steps are dropped: the swimmer starts at rest and
its velocity is not yet a function of its state.

Run on a GPU:  python -m lbm_solver_3d_b200.surrogate_data --out DIR
"""
from __future__ import annotations

import argparse
import time
from pathlib import Path

import numpy as np

from .params import Params
from .workloads import ensemble_members

TRAJ_COLS = 15


def member_table(ps: list[Params]) -> np.ndarray:
    """Per member: nx, ny, nz, a, beta, angle, y0, B1."""
    return np.array([[p.NX, p.NY, p.NZ, p.R, p.beta, p.angle, p.y0, p.B1] for p in ps], float)


def run_ensemble_rows(ps: list[Params], steps: int, chunk: int = 10000, autotune: bool = True) -> list[np.ndarray]:
    """Advance all members `steps` steps; return each member's trajectory rows."""
    from .ensemble import Ensemble
    rows = [[] for _ in ps]
    with Ensemble(ps, autotune=autotune) as ens:
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            ens.run(k)
            done += k
            for i in range(len(ps)):
                rows[i].append(ens.member(i).traj_rows())
    return [np.concatenate(r, 0) if r else np.zeros((0, TRAJ_COLS)) for r in rows]


def samples(rows: np.ndarray, p: Params, transient: int, window: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(inputs, targets) of one member's trajectory rows.

    window = 0: the instantaneous velocities of the rows. window = k > 0: the
    velocities from central differences of position and orientation angle over
    +-k rows, i.e. the drift over 2k * traj_every steps. These no longer carry
    the step-to-step kicks of nodes being covered and uncovered, which do not
    move the swimmer on average; the first and last k rows are dropped."""
    r = rows[rows[:, 0] >= transient]
    a, H = p.R, p.NY - 2.0
    U0 = 2.0 * p.B1 / 3.0
    th = np.arctan2(r[:, 5], r[:, 4])
    x = np.stack([(r[:, 2] - 0.5) / a, th, np.full(len(r), p.beta), np.full(len(r), H / a)], 1)
    if window <= 0:
        y = np.stack([r[:, 7] / U0, r[:, 8] / U0, r[:, 12] * a / U0], 1)
        return x, y
    k = window
    if len(r) <= 2 * k:
        return x[:0], np.zeros((0, 3))
    dt = r[2 * k:, 0] - r[:-2 * k, 0]
    thu = np.unwrap(th)
    ux = (r[2 * k:, 1] - r[:-2 * k, 1]) / dt
    uy = (r[2 * k:, 2] - r[:-2 * k, 2]) / dt
    wz = (thu[2 * k:] - thu[:-2 * k]) / dt
    y = np.stack([ux / U0, uy / U0, wz * a / U0], 1)
    return x[k:-k], y


def build(ps: list[Params], trajs: list[np.ndarray], transient: int):
    xs, ys, member = [], [], []
    for i, (p, r) in enumerate(zip(ps, trajs)):
        x, y = samples(r, p, transient)
        xs.append(x); ys.append(y); member.append(np.full(len(x), i))
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(member)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--heldout", type=int, default=32)
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for name, n, seed in (("train", args.members, 2024), ("heldout", args.heldout, 7777)):
        ps = ensemble_members(n, seed=seed)
        t0 = time.time()
        trajs = run_ensemble_rows(ps, args.steps)
        dt = time.time() - t0
        np.savez_compressed(out / f"surrogate_{name}.npz", members=member_table(ps),
                            traj=np.concatenate(trajs, 0).astype(np.float64),
                            counts=np.array([len(t) for t in trajs]), seconds=dt, steps=args.steps)
        print(f"{name}: {n} members, {args.steps} steps, {dt:.1f} s, {sum(len(t) for t in trajs)} rows", flush=True)


if __name__ == "__main__":
    main()
