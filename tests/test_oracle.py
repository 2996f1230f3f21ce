"""Pinning the oracle (test infrastructure) before trusting it.

1. The plain-C restatement reproduces the reference compiled from its own
   sources bit for bit (one OpenMP thread, no FMA contraction in either).
2. It reproduces the reference's shipped results (tests/golden/shipped.npz,
   extracted by tests/golden/extract_shipped.py): the trajectory files of the
   channel runs to their printed precision, the duct summary and profiles.
3. It reproduces the full-length duct workload fixture generated by running
   the reference (tests/golden/make_reference_runs.py -> ref_duct.npz).
"""
import numpy as np
import pytest

from conftest import GOLDEN
from lbm_solver_3d_b200.params import Params
from lbm_solver_3d_b200.workloads import workload_params

SHIPPED = np.load(GOLDEN / "shipped.npz")

# The reference's input decks (inputs/*.in), as key = value overrides.
CHANNEL = dict(nx=64, ny=34, nz=32, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4, b1=0.015,
               angle=30, planar=1, eps=0.2, hc=2.0, hmin=0.5, steps=60000, print_every=2000, traj_every=50)
DUCT = dict(nx=4, ny=34, nz=34, tau=0.8, fx=5e-5, walls_y=1, walls_z=1, squirmer=0, steps=100000,
            tol=1e-12, print_every=1000)


def deck(base, **kw):
    return Params().update(**base).update(**kw)


def traj_close(rows, ref):
    """Columns printed with %.6f (t, X, e) and %.6e (U, W, Fwall)."""
    assert rows.shape == ref.shape
    assert np.array_equal(rows[:, 0], ref[:, 0])
    assert np.all(np.abs(rows[:, 1:7] - ref[:, 1:7]) <= 5.1e-7)
    big = np.abs(ref[:, 7:]) > 0
    rel = np.abs(rows[:, 7:] - ref[:, 7:])[big] / np.abs(ref[:, 7:])[big]
    assert np.all(rel <= 5.1e-7)
    assert np.all(np.abs(rows[:, 7:][~big]) < 1e-12)


@pytest.fixture(scope="module")
def port(oracle_mod):
    oracle_mod.set_threads(8)
    return oracle_mod.PortSolver


@pytest.mark.parametrize("kw", [
    dict(base=CHANNEL, steps=120, mass_correction_every=10),
    dict(base=CHANNEL, steps=60, nx=20, ny=16, nz=14, radius=3.0, beta=2.0, angle=-20, z0=6.2, walls_z=1),
    dict(base=DUCT, steps=200, fy=1e-5, fz=-2e-5),
    dict(base=CHANNEL, steps=80, nx=22, ny=20, nz=18, walls_y=0, planar=0, ex=0.2, ey=0.5, ez=-0.8, beta=-3),
])
def test_port_is_bitwise_the_reference(oracle_mod, kw):
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built (needs the reference sources)")
    oracle_mod.set_threads(1)
    kw = dict(kw)
    base, steps = kw.pop("base"), kw.pop("steps")
    p = deck(base, **kw)
    a, b = oracle_mod.PortSolver(p), oracle_mod.RefSolver(p)
    ta, tb = a.run(steps), b.run(steps)
    assert np.array_equal(ta, tb)
    assert np.array_equal(a.get_f(), b.get_f())
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
    if p.squirmer:
        sa, sb = a.squirmer(), b.squirmer()
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(a.wall_force(), b.wall_force())
    oracle_mod.set_threads(8)


@pytest.mark.parametrize("label,kw,key", [
    ("neutral", {}, "example_neutral_traj"),                       # examples/reference_data, 40000-step run
    ("puller", dict(beta=1, ny=24, nz=20), "outputs_channel_puller_traj"),   # inputs/channel_puller.in
    ("puller_ny34", dict(beta=1), "example_puller_traj"),           # an older deck: ny=34, nz=32
    ("pusher_b-3", dict(beta=-3), "example_pusher_traj"),           # the README's beta=-3 run
])
def test_port_reproduces_shipped_trajectories(port, label, kw, key):
    p = deck(CHANNEL, **kw)
    rows = port(p).run(400)
    traj_close(rows, SHIPPED[key][: len(rows)])


def run_duct_to_convergence(solver, p):
    """main.cpp:60-87 for a run without squirmer: tol check at print steps."""
    prev, t = 0.0, 0
    while t < p.steps:
        solver.run(p.printEvery)
        t += p.printEvery
        sx = solver.diag()["sum_ux"]
        change = abs(sx - prev) / (abs(sx) + 1e-30)
        prev = sx
        if p.tol > 0 and change < p.tol:
            return t, True
    return t, False


@pytest.mark.slow
def test_port_reproduces_shipped_duct_summary(port):
    p = deck(DUCT)
    s = port(p)
    t, conv = run_duct_to_convergence(s, p)
    assert conv and t == int(SHIPPED["duct_summary_steps"][0])
    assert abs(s.poiseuille_error() - SHIPPED["duct_summary_l2_error"][0]) < 5e-14
    d = s.diag()
    assert abs(d["max_speed"] - SHIPPED["duct_summary_max_speed"][0]) < 1e-12
    assert abs(d["mean_density"] - 1.0) < 1e-10
    assert np.allclose(s.wall_force(), SHIPPED["duct_summary_wall_force"], rtol=1e-9, atol=1e-12)
    _, _, u = s.fields()
    prof = SHIPPED["duct_profile_y"]          # y - yc, ux_lbm, ux_exact at z = nz/2, x = 0
    ux = u[p.NZ // 2, 1:-1, 0, 0]
    assert np.allclose(ux, prof[:, 1], rtol=1e-9)
    from oracle.oracle import port_lib
    a, b = 0.5 * (p.NY - 2), 0.5 * (p.NZ - 2)
    exact = [port_lib().lbo_duct_velocity(yy, p.NZ // 2 - 0.5 * (p.NZ - 1), a, b, p.Fx, p.nu) for yy in prof[:, 0]]
    assert np.allclose(exact, prof[:, 2], rtol=1e-9)


@pytest.mark.slow
def test_port_matches_full_duct_fixture(port):
    """The duct workload (16x32x32, 20000 steps) against the reference's own run."""
    g = np.load(GOLDEN / "ref_duct.npz")
    p = workload_params("duct")
    s = port(p)
    s.run(int(g["steps"]))
    flag, rho, u = s.fields()
    assert np.array_equal(flag[:, :, 0], g["x0_flag"])
    assert np.allclose(rho[:, :, 0], g["x0_rho"], rtol=1e-13, atol=0)
    assert np.allclose(u[:, :, 0], g["x0_u"], rtol=1e-9, atol=1e-18)
    assert abs(s.poiseuille_error() - float(g["l2_error"])) < 1e-12


def test_timed_reference_build_computes_the_parity_build(oracle_mod):
    """The CPU baseline loads the reference compiled with its Makefile's own
    flags at this CPU's x86-64 level. GCC contracts multiply-adds there (its
    C++ default), so it matches the parity build to rounding: the same
    solver, timed as its author builds it."""
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built (needs the reference sources)")
    oracle_mod.set_threads(1)
    p = deck(CHANNEL, nx=24, ny=18, nz=16, radius=3.5, beta=1.5, angle=10, traj_every=10)
    a, b = oracle_mod.RefSolver(p), oracle_mod.RefSolver(p, timed=True)
    ra, rb = a.run(60), b.run(60)
    assert ra.shape == rb.shape == (6, 15)
    assert np.allclose(ra, rb, rtol=1e-10, atol=1e-14)
    fa, fb = a.get_f(), b.get_f()
    assert np.abs(fa - fb).max() <= 1e-13
    assert "reference sources" in oracle_mod.ref_build()
    a.close(); b.close()
