"""Swimmer surrogate: an MLP that maps the state of a squirmer in a slit
channel to its instantaneous velocity, trained on trajectories generated by
the batched LBM (surrogate_data.py) with the library's own kernels (mlp.py).

    inputs   h/a, theta, beta, H/a   (see surrogate_data.py)
    outputs  Ux/U0, Uy/U0, Omega_z a/U0

Uses:
  * ``Surrogate.integrate``  planar trajectories (x, y, theta) by RK4 on the
    predicted velocities, thousands of times faster than the LBM;
  * ``Surrogate.sweep``      drift velocities of a parameter sweep. A point is
    answered by the surrogate only while its whole trajectory stays inside the
    training hull and the networks of the ensemble agree; every other point is
    run with the full LBM (an ``Ensemble``), which is the fallback and the
    measure of the surrogate's error;
  * ``Surrogate.warm_start`` the velocities that start an LBM run of the
    near-wall phase at the surrogate's state instead of at rest.

Symmetry: the slit is symmetric about its mid-plane, so every sample (h, theta)
also gives the mirrored sample (H - h, -theta) with (Ux, -Uy, -Omega_z); the
training set holds both.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .mlp import MLP
from .params import Params
from .surrogate_data import samples

FEATURES = ("h/a", "theta", "beta", "H/a")
TARGETS = ("Ux/U0", "Uy/U0", "Omega_z*a/U0")


def mirror(x: np.ndarray, y: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    xm = x.copy()
    xm[:, 0] = x[:, 3] - x[:, 0]
    xm[:, 1] = -x[:, 1]
    ym = y * np.array([1.0, -1.0, -1.0])
    return xm, ym


def dataset_from_npz(path, transient: int = 2000, window: int = 0):
    """Per-member Params-like table, and the (inputs, targets, member) arrays
    (window: see surrogate_data.samples)."""
    d = np.load(path)
    table, traj, counts = d["members"], d["traj"], d["counts"]
    off = np.concatenate([[0], np.cumsum(counts)])
    xs, ys, mem = [], [], []
    for i, row in enumerate(table):
        p = member_params(row)
        x, y = samples(traj[off[i]:off[i + 1]], p, transient, window)
        xs.append(x); ys.append(y); mem.append(np.full(len(x), i))
    rows = [traj[off[i]:off[i + 1]] for i in range(len(table))]
    return table, rows, np.concatenate(xs), np.concatenate(ys), np.concatenate(mem)


def member_params(row) -> Params:
    """Params of a member from its table row (nx, ny, nz, a, beta, angle, y0, B1)."""
    from .workloads import SLIT_DECK
    p = Params()
    p.update(**SLIT_DECK)
    p.update(nx=int(row[0]), ny=int(row[1]), nz=int(row[2]), radius=float(row[3]), beta=float(row[4]),
             angle=float(row[5]), y0=float(row[6]), b1=float(row[7]), tau=1.0, precision="fp32")
    return p


class Hull:
    """Training hull: the per-feature range of the training inputs, and a
    neighbourhood test in standardised input space (a point is inside when a
    training point lies within `radius`, the 99.5th percentile of the training
    points' own nearest-neighbour distances, times `slack`)."""

    def __init__(self, x: np.ndarray, scale: np.ndarray, slack: float = 3.0, max_points: int = 40000, seed: int = 0):
        from scipy.spatial import cKDTree
        rng = np.random.default_rng(seed)
        pts = x if len(x) <= max_points else x[rng.choice(len(x), max_points, replace=False)]
        self.lo, self.hi = x.min(0), x.max(0)
        self.scale = scale
        self.tree = cKDTree(pts / scale)
        dist, _ = self.tree.query(pts / scale, k=2)
        self.radius = float(np.percentile(dist[:, 1], 99.5)) * slack

    def inside(self, x: np.ndarray) -> np.ndarray:
        x = np.atleast_2d(x)
        box = np.all((x >= self.lo) & (x <= self.hi), axis=1)
        dist, _ = self.tree.query(x / self.scale, k=1)
        return box & (dist <= self.radius)


@dataclass
class FitLog:
    epochs: int
    train_loss: list
    val_loss: list
    seconds: float


class Surrogate:
    def __init__(self, nets: list[MLP], xm, xs, ym, ys, hull: Hull):
        self.nets, self.xm, self.xs, self.ym, self.ys, self.hull = nets, xm, xs, ym, ys, hull

    # ---- training ----
    @classmethod
    def fit(cls, x, y, x_val=None, y_val=None, n_nets: int = 3, bf16: bool = True, epochs: int = 40,
            batch: int = 512, lr: float = 2e-3, lr_min: float = 5e-5, seed: int = 0, device: int = 0,
            augment: bool = True, beta_emphasis: float = 0.0):
        """beta_emphasis w > 0 draws each epoch's samples with replacement, with
        probability proportional to 1 + w (|beta| / max |beta|)^2: the strong
        pushers and pullers, whose near-wall dynamics carry most of the
        held-out error, are seen more often."""
        import time
        if augment:
            xa, ya = mirror(x, y)
            x, y = np.concatenate([x, xa]), np.concatenate([y, ya])
        xm, xs = x.mean(0), x.std(0) + 1e-12
        ym, ys = y.mean(0), y.std(0) + 1e-12
        xn, yn = ((x - xm) / xs).astype(np.float32), ((y - ym) / ys).astype(np.float32)
        prob = None
        if beta_emphasis > 0:
            b = np.abs(x[:, 2]) / max(np.abs(x[:, 2]).max(), 1e-12)
            prob = 1.0 + beta_emphasis * b * b
            prob /= prob.sum()
        nets, logs = [], []
        t0 = time.time()
        for k in range(n_nets):
            net = MLP(bf16=bf16, device=device, seed=seed * 100 + k)
            net.set_data(xn, yn)
            rng = np.random.default_rng(seed * 100 + k)
            tl, vl = [], []
            for ep in range(epochs):
                cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * ep / max(1, epochs - 1)))
                order = rng.permutation(len(xn)) if prob is None else rng.choice(len(xn), size=len(xn), p=prob)
                tl.append(net.train_epoch(order, batch=batch, lr=cur))
                if x_val is not None:
                    pv = net.forward((x_val - xm) / xs) * ys + ym
                    vl.append(float(np.mean(((pv - y_val) / ys) ** 2)))
            nets.append(net)
            logs.append(FitLog(epochs, tl, vl, time.time() - t0))
        s = cls(nets, xm, xs, ym, ys, Hull(x, xs))
        s.logs = logs
        return s

    # ---- inference ----
    def predict(self, x) -> tuple[np.ndarray, np.ndarray]:
        """Mean over the networks and the largest deviation from it (both in
        target units)."""
        x = np.atleast_2d(np.asarray(x, float))
        xn = ((x - self.xm) / self.xs).astype(np.float32)
        outs = np.stack([n.forward(xn) * self.ys + self.ym for n in self.nets])
        mean = outs.mean(0)
        spread = np.abs(outs - mean).max(0)
        return mean, spread

    def trusted(self, x, tol: float = 0.05) -> np.ndarray:
        """Inside the training hull and the networks agree within `tol` (in
        units of U0 for the velocities and U0/a for the rotation rate)."""
        _, spread = self.predict(x)
        return self.hull.inside(x) & np.all(spread <= tol, axis=1)

    # ---- trajectories ----
    def integrate(self, y0, theta0, beta, a, H, steps: int, B1: float = 0.015, dt: float = 50.0, tol: float = 0.05):
        """Planar trajectories of many swimmers at once (arrays of equal
        length): RK4 in steps of dt lattice time units. Returns times and
        states (x, y, theta) of shape (k+1, n, 3), and whether each swimmer
        stayed trusted for the whole run."""
        y0, theta0, beta, a, H = (np.broadcast_to(np.asarray(v, float), np.shape(y0)).copy()
                                  for v in (y0, theta0, beta, a, H))
        n = y0.size
        U0 = 2.0 * B1 / 3.0
        state = np.stack([np.zeros(n), y0, theta0], 1)
        ok = np.ones(n, bool)

        def rate(s):
            feats = np.stack([(s[:, 1] - 0.5) / a, s[:, 2], beta, H / a], 1)
            mean, spread = self.predict(feats)
            good = self.hull.inside(feats) & np.all(spread <= tol, axis=1)
            v = np.stack([mean[:, 0] * U0, mean[:, 1] * U0, mean[:, 2] * U0 / a], 1)
            return v, good

        k = int(round(steps / dt))
        out = [state.copy()]
        for _ in range(k):
            k1, g1 = rate(state)
            k2, g2 = rate(state + 0.5 * dt * k1)
            k3, g3 = rate(state + 0.5 * dt * k2)
            k4, g4 = rate(state + dt * k3)
            state = state + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
            ok &= g1 & g2 & g3 & g4
            out.append(state.copy())
        return np.arange(k + 1) * dt, np.stack(out), ok

    def sweep(self, members: list[Params], steps: int, t0: int = 0, tol: float = 0.05, lbm_runner=None):
        """Drift velocities (mean Ux, Uy over steps) of each member, from the
        surrogate where it is trusted along the whole trajectory and from the
        LBM otherwise. `lbm_runner(params_list, steps)` returns the LBM drift
        velocities of the members it is given (default: an Ensemble run)."""
        y0 = np.array([p.y0 for p in members])
        th = np.radians([p.angle for p in members])
        beta = np.array([p.beta for p in members])
        a = np.array([p.R for p in members])
        H = np.array([p.NY - 2.0 for p in members])
        t, states, ok = self.integrate(y0, th, beta, a, H, steps, B1=members[0].B1, tol=tol)
        drift = (states[-1, :, :2] - states[0, :, :2]) / t[-1]
        src = np.where(ok, "surrogate", "lbm")
        if (~ok).any():
            runner = lbm_runner or lbm_drift
            idx = np.flatnonzero(~ok)
            drift[idx] = runner([members[i] for i in idx], steps)
        return drift, src

    def warm_start(self, p: Params) -> tuple[np.ndarray, np.ndarray]:
        """(U, W) predicted at the initial state of p, to start an LBM run of
        that state with the swimmer already moving."""
        a, H = p.R, p.NY - 2.0
        th = math.radians(p.angle)
        mean, _ = self.predict([[(p.y0 - 0.5) / a, th, p.beta, H / a]])
        U0 = 2.0 * p.B1 / 3.0
        U = np.array([mean[0, 0] * U0, mean[0, 1] * U0, 0.0])
        W = np.array([0.0, 0.0, mean[0, 2] * U0 / a])
        return U, W


def lbm_drift(members: list[Params], steps: int) -> np.ndarray:
    """Mean (Ux, Uy) of each member over `steps` LBM steps: its displacement
    divided by the time (the full LBM, all members in one Ensemble)."""
    from .ensemble import Ensemble
    with Ensemble(members, autotune=True) as ens:
        x0 = np.array([ens.member(i).squirmer()["X"][:2] for i in range(len(members))])
        ens.run(steps)
        x1 = np.array([ens.member(i).squirmer()["X"][:2] for i in range(len(members))])
    return (x1 - x0) / steps
