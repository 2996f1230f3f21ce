"""The surrogate end to end on a small sweep: LBM ensemble -> training data ->
networks trained by the library's kernels -> held-out drift velocities checked
against the LBM.

Small configuration (about a minute on one B200): 48 training and 8 held-out
slit channels of reduced size (Nx 48-80, Ny, Nz 32-48, a 3-5), 6000 steps,
2000-step transient. The full-size result (256 members, 30000 steps, 32
held-out draws) is produced by lbm_solver_3d_b200.surrogate_eval.
Checked here:
  * the surrogate's held-out drift error (median) is below 5% and at least
    4x smaller than that of the method without the network (a swimmer moving
    at U0 along its initial orientation);
  * a sweep answers trusted members from the surrogate and sends the others
    to the LBM, whose answers are exact by construction;
  * the surrogate is much faster than the LBM on the same sweep.
"""
import time

import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params
from lbm_solver_3d_b200.workloads import SLIT_DECK

pytestmark = pytest.mark.gpu


def small_members(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ny = int(rng.integers(32, 49))
        a = float(rng.uniform(3.0, 5.0))
        p = Params()
        p.update(**SLIT_DECK)
        p.update(nx=int(rng.integers(48, 81)), ny=ny, nz=int(rng.integers(32, 49)), radius=a,
                 beta=float(rng.uniform(-5, 5)), angle=float(rng.uniform(-30, 30)),
                 y0=0.5 + float(rng.uniform(1.5 * a, ny - 2 - 1.5 * a)), b1=0.015, tau=1.0, traj_every=25,
                 precision="fp32")
        p.validate()
        out.append(p)
    return out


@pytest.fixture(scope="module")
def data():
    from lbm_solver_3d_b200.surrogate_data import run_ensemble_rows, samples
    train, held = small_members(48, 11), small_members(8, 12)
    t0 = time.time()
    rows_t = run_ensemble_rows(train, 6000)
    t_lbm_train = time.time() - t0
    t0 = time.time()
    rows_h = run_ensemble_rows(held, 6000)
    t_lbm_held = time.time() - t0
    xs, ys = zip(*[samples(r, p, 2000) for r, p in zip(rows_t, train)])
    return dict(train=train, held=held, rows_h=rows_h, x=np.concatenate(xs), y=np.concatenate(ys),
                t_lbm_held=t_lbm_held, t_lbm_train=t_lbm_train)


def test_surrogate_beats_the_method_without_it(data):
    from lbm_solver_3d_b200.surrogate import Surrogate
    from lbm_solver_3d_b200.surrogate_eval import evaluate
    from lbm_solver_3d_b200.surrogate_data import member_table
    s = Surrogate.fit(data["x"], data["y"], n_nets=3, bf16=True, epochs=60, batch=256)
    res, t_sur = evaluate(s, member_table(data["held"]), data["rows_h"], 2000)
    e_s = np.array([r["err_surrogate"] for r in res])
    e_b = np.array([r["err_bulk_speed"] for r in res])
    print(f"held-out drift error: surrogate median {np.median(e_s):.3f} max {e_s.max():.3f}; "
          f"without network median {np.median(e_b):.3f}; surrogate {t_sur:.2f} s vs LBM {data['t_lbm_held']:.2f} s")
    assert np.median(e_s) < 0.05
    assert np.median(e_s) * 4 < np.median(e_b)
    assert t_sur < data["t_lbm_held"]


def test_sweep_falls_back_to_the_lbm_outside_the_hull(data):
    from lbm_solver_3d_b200.surrogate import Surrogate
    s = Surrogate.fit(data["x"], data["y"], n_nets=2, bf16=False, epochs=30, batch=256)
    members = data["held"][:3]
    far = Params()
    far.update(**SLIT_DECK)   # H/a = 31 and a = 1.5: far outside the training inputs
    far.update(nx=48, ny=48, nz=32, radius=1.5, beta=0.0, angle=10, y0=24.0, b1=0.015, tau=1.0, precision="fp32")
    far.validate()
    calls = []

    def runner(ps, steps):
        calls.append(len(ps))
        return np.full((len(ps), 2), 123.0)

    drift, src = s.sweep(members + [far], 2000, lbm_runner=runner)
    assert src[-1] == "lbm" and np.all(drift[-1] == 123.0)
    assert calls == [int((src == "lbm").sum())]
    assert np.all(np.isfinite(drift))
