"""Train the swimmer surrogate on LBM ensemble trajectories and evaluate it
against the LBM on held-out members (different seed: new beta, angle, height, sizes).

    python -m lbm_solver_3d_b200.surrogate_eval --data DIR [--out report.json]

DIR holds surrogate_train.npz and surrogate_heldout.npz from surrogate_data.py.
Reported per held-out member, over the window [transient, end] of its run:
  * drift velocity: displacement (x, y) / time of the LBM trajectory against
    that of the surrogate-integrated trajectory started from the LBM state at
    the window's start; relative error |V_s - V_lbm| / |V_lbm|;
  * the same for the method without the network: a swimmer moving at the
    bulk speed U0 = 2 B1 / 3 along its initial orientation;
  * instantaneous velocity errors at the LBM states (no integration);
  * whether the surrogate stayed trusted (training hull, network agreement),
    i.e. whether a sweep would have answered it or fallen back to the LBM.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from .surrogate import Surrogate, dataset_from_npz, member_params


def drift_window(rows: np.ndarray, transient: int):
    r = rows[rows[:, 0] >= transient]
    t = r[-1, 0] - r[0, 0]
    return r[0], r[-1], t


def evaluate(s: Surrogate, table, rows, transient: int, tol: float = 0.05):
    out = []
    starts, ends = [], []
    for i, row in enumerate(table):
        p = member_params(row)
        r0, r1, t = drift_window(rows[i], transient)
        starts.append((r0, p, t))
        ends.append(r1)
    y0 = np.array([r0[2] for r0, _, _ in starts])
    th0 = np.array([np.arctan2(r0[5], r0[4]) for r0, _, _ in starts])
    beta = np.array([p.beta for _, p, _ in starts])
    a = np.array([p.R for _, p, _ in starts])
    H = np.array([p.NY - 2.0 for _, p, _ in starts])
    steps = int(starts[0][2])
    t0 = time.time()
    tt, states, ok = s.integrate(y0, th0, beta, a, H, steps, B1=starts[0][1].B1, tol=tol)
    t_sur = time.time() - t0
    for i, ((r0, p, t), r1) in enumerate(zip(starts, ends)):
        v_lbm = (r1[1:3] - r0[1:3]) / t
        v_sur = (states[-1, i, :2] - states[0, i, :2]) / tt[-1]
        U0 = 2.0 * p.B1 / 3.0
        v_bulk = U0 * np.array([np.cos(th0[i]), np.sin(th0[i])])
        nv = np.linalg.norm(v_lbm)
        out.append(dict(member=i, beta=p.beta, a=p.R, H_over_a=(p.NY - 2) / p.R, h0_over_a=(y0[i] - 0.5) / p.R,
                        nx=p.NX, nz=p.NZ,
                        theta0=float(th0[i]), v_lbm=v_lbm.tolist(), v_surrogate=v_sur.tolist(),
                        err_surrogate=float(np.linalg.norm(v_sur - v_lbm) / nv),
                        err_bulk_speed=float(np.linalg.norm(v_bulk - v_lbm) / nv),
                        speed_err_surrogate=float(abs(np.linalg.norm(v_sur) - nv) / nv),
                        trusted=bool(ok[i])))
    return out, t_sur


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--data", required=True)
    ap.add_argument("--out", default=None)
    ap.add_argument("--transient", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--nets", type=int, default=3)
    ap.add_argument("--fp32", action="store_true", help="FP32 GEMMs instead of BF16")
    ap.add_argument("--window", type=int, default=0,
                    help="train on velocities from central differences over +-window rows (0: instantaneous)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--beta-emphasis", type=float, default=0.0,
                    help="draw training samples with probability 1 + w (|beta|/max)^2 (0: plain permutation)")
    args = ap.parse_args()
    d = Path(args.data)
    table, rows, x, y, mem = dataset_from_npz(d / "surrogate_train.npz", args.transient, args.window)
    # validation: 10% of the training members
    rng = np.random.default_rng(0)
    val_members = rng.choice(len(table), max(1, len(table) // 10), replace=False)
    vmask = np.isin(mem, val_members)
    t0 = time.time()
    s = Surrogate.fit(x[~vmask], y[~vmask], x[vmask], y[vmask], n_nets=args.nets, bf16=not args.fp32,
                      epochs=args.epochs, seed=args.seed, beta_emphasis=args.beta_emphasis)
    t_fit = time.time() - t0
    htable, hrows, hx, hy, hmem = dataset_from_npz(d / "surrogate_heldout.npz", args.transient)
    pred, spread = s.predict(hx)
    inst = np.linalg.norm(pred[:, :2] - hy[:, :2], axis=1) / np.linalg.norm(hy[:, :2], axis=1)
    per_member, t_sur = evaluate(s, htable, hrows, args.transient)
    e_s = np.array([m["err_surrogate"] for m in per_member])
    e_b = np.array([m["err_bulk_speed"] for m in per_member])
    trusted = np.array([m["trusted"] for m in per_member])
    by_tol = {}
    for tol in (0.02, 0.03, 0.05, 0.1):
        pm, _ = evaluate(s, htable, hrows, args.transient, tol=tol)
        tr = np.array([m["trusted"] for m in pm])
        by_tol[str(tol)] = {"trusted_members": int(tr.sum()),
                            "max_err_trusted": float(e_s[tr].max()) if tr.any() else None}
    dgen = np.load(d / "surrogate_heldout.npz")
    # does the error follow what the four inputs leave out, the periodic box
    # length and width (the swimmer's images)? Spearman rank correlations
    def spearman(u, v):
        ru, rv = np.argsort(np.argsort(u)), np.argsort(np.argsort(v))
        return float(np.corrcoef(ru, rv)[0, 1])
    a_nx = np.array([m["a"] / m["nx"] for m in per_member])
    a_nz = np.array([m["a"] / m["nz"] for m in per_member])
    h_a = np.array([m["h0_over_a"] for m in per_member])
    bet = np.array([m["beta"] for m in per_member])
    corr = {"a/Nx": spearman(e_s, a_nx), "a/Nz": spearman(e_s, a_nz), "h0/a": spearman(e_s, h_a),
            "|beta|": spearman(e_s, np.abs(bet))}
    report = {
        "samples_train": int((~vmask).sum()) * 2, "samples_val": int(vmask.sum()),
        "samples_heldout": int(len(hx)), "gemm": "fp32" if args.fp32 else "bf16", "nets": args.nets,
        "window": args.window, "beta_emphasis": args.beta_emphasis,
        "epochs": args.epochs, "fit_seconds": t_fit,
        "val_loss_final": [lg.val_loss[-1] for lg in s.logs],
        "heldout_instantaneous_velocity_rel_err": {"median": float(np.median(inst)), "mean": float(inst.mean()),
                                                   "p95": float(np.percentile(inst, 95))},
        "heldout_drift_rel_err_surrogate": {"median": float(np.median(e_s)), "mean": float(e_s.mean()),
                                            "max": float(e_s.max()), "within_5pct": int((e_s <= 0.05).sum()),
                                            "members": len(e_s)},
        "heldout_drift_rel_err_without_network": {"median": float(np.median(e_b)), "mean": float(e_b.mean()),
                                                  "max": float(e_b.max()),
                                                  "within_5pct": int((e_b <= 0.05).sum())},
        "trusted_members": int(trusted.sum()),
        "trust_tolerance_sweep": by_tol,
        "drift_rel_err_trusted_only": {"max": float(e_s[trusted].max()) if trusted.any() else None,
                                       "median": float(np.median(e_s[trusted])) if trusted.any() else None},
        "err_rank_correlation": corr,
        "time_surrogate_s": t_sur,
        "time_lbm_s": float(dgen["seconds"]),
        "per_member": per_member,
    }
    txt = json.dumps(report, indent=1)
    if args.out:
        Path(args.out).write_text(txt)
    summary = {k: v for k, v in report.items() if k != "per_member"}
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
