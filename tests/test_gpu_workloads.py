"""Full-length workloads on the GPU against the reference's own runs.

Fixtures (tests/golden/ref_*.npz) were produced by running the reference
compiled from its sources (tests/golden/make_reference_runs.py) for the full
step count: trajectories, final squirmer state and rho/u at a seeded sample of
4096 nodes. Tolerances: FP64 relative L2 <= 1e-10 (rho, u, X, e); FP32-shifted:
squirmer drift <= 1e-4 relative over the full run, relative L2 of u <= 1e-5
without moving boundaries (full run) and with them until remap events start
to differ in timing (see test_squirmer_workload_fp32_error).

The shipped results of the reference (tests/golden/shipped.npz) are checked
through the drop-in driver binary at their printed precision.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from lbm_solver_3d_b200.workloads import workload_params

pytestmark = pytest.mark.gpu
DRIVER = ROOT / "lbm_solver_3d_b200" / "bin" / "lbm_squirmer_gpu"


def rel_l2(a, b):
    a = np.asarray(a, float).ravel()
    b = np.asarray(b, float).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def Solver():
    from lbm_solver_3d_b200.solver import Solver
    return Solver


def fixture(name):
    path = GOLDEN / f"ref_{name}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    return np.load(path)


def sampled(solver, g):
    flag, rho, u = solver.fields()
    idx = g["sample_idx"]
    fl = flag.reshape(-1)[idx]
    fluid = (fl == 0) & (g["sample_flag"] == 0)
    return fl, rho.reshape(-1)[idx], u.reshape(-1, 3)[idx], fluid


def test_duct_workload_fp64(Solver):
    """16x32x32 duct, 20000 steps: the x = 0 cross-section against the reference."""
    g = fixture("duct")
    s = Solver(workload_params("duct"))
    s.run(int(g["steps"]))
    flag, rho, u = s.fields()
    assert np.array_equal(flag[:, :, 0], g["x0_flag"])
    fl = g["x0_flag"] == 0
    assert rel_l2(rho[:, :, 0][fl], g["x0_rho"][fl]) < 1e-10
    assert rel_l2(u[:, :, 0][fl], g["x0_u"][fl]) < 1e-10
    d = s.diag()
    assert abs(d["mean_density"] - 1.0) < 1e-10
    body = 1e-6 * d["n_fluid"]
    assert abs(d["wall_force"][0] - body) / body < 1e-6   # momentum balance


@pytest.mark.parametrize("name", ["slit", "bulk_0", "bulk_m3", "bulk_p3"])
def test_squirmer_workload_fp64(Solver, name):
    g = fixture(name)
    p = workload_params(name)
    s = Solver(p)
    steps = int(g["steps"])
    s.run(steps)
    tr = s.traj_rows()
    ref = g["traj"]
    assert tr.shape == ref.shape and np.array_equal(tr[:, 0], ref[:, 0])
    print(f"{name}: X {rel_l2(tr[:, 1:4], ref[:, 1:4]):.2e} e {rel_l2(tr[:, 4:7], ref[:, 4:7]):.2e} "
          f"U {rel_l2(tr[:, 7:10], ref[:, 7:10]):.2e}")
    assert rel_l2(tr[:, 1:4], ref[:, 1:4]) < 1e-10
    assert rel_l2(tr[:, 4:7], ref[:, 4:7]) < 1e-10
    sq = s.squirmer()
    assert np.allclose(sq["X"], g["sq_X"], rtol=1e-10)
    assert sq["contacts"] == int(g["sq_contacts"])
    fl, rho, u, fluid = sampled(s, g)
    assert rel_l2(rho[fluid], g["sample_rho"][fluid]) < 1e-10
    assert rel_l2(u[fluid], g["sample_u"][fluid]) < 1e-10
    if "shell_idx" in g.files:   # every node within R + 3 of the final centre
        flag, rho_all, u_all = s.fields()
        idx = g["shell_idx"]
        assert np.array_equal(flag.reshape(-1)[idx], g["shell_flag"])
        sh = g["shell_flag"] == 0
        assert rel_l2(rho_all.reshape(-1)[idx][sh], g["shell_rho"][sh]) < 1e-10
        assert rel_l2(u_all.reshape(-1, 3)[idx][sh], g["shell_u"][sh]) < 1e-10


@pytest.mark.parametrize("name", ["slit", "bulk_0"])
def test_squirmer_workload_fp32_error(Solver, name):
    """FP32-shifted storage on the full-length squirmer workloads.

    Drift of the squirmer's position stays within 1e-4 of its displacement for
    the whole run. The velocity field stays within 1e-5 relative L2 of the FP64
    path until the first cover/uncover event falls on a different step: the
    remap is a discrete function of the sphere's position, FP32 rounding moves
    the sphere by ~1e-6 cells, and after a few thousand steps a handful of
    surface nodes change type one step apart. Those events, not the storage
    precision of the bulk, set the late-time field difference; it is reported
    here, not bounded."""
    g = fixture(name)
    p32, p64 = workload_params(name, "fp32"), workload_params(name)
    early = 1000
    s32, s64 = Solver(p32), Solver(p64)
    s32.run(early); s64.run(early)
    f32, _, u32 = s32.fields()
    f64, _, u64 = s64.fields()
    fluid = (f32 == 0) & (f64 == 0)
    err_early = rel_l2(u32[fluid], u64[fluid])
    s32.run(int(g["steps"]) - early)
    fl, rho, u, fl_ok = sampled(s32, g)
    err_u = rel_l2(u[fl_ok], g["sample_u"][fl_ok])
    X0 = g["traj"][0, 1:4] - g["traj"][0, 7:10]          # position before the first step
    disp_ref = g["sq_X"] - X0
    drift = np.linalg.norm(s32.squirmer()["X"] - g["sq_X"]) / np.linalg.norm(disp_ref)
    print(f"{name} fp32: rel L2 u at {early} steps {err_early:.2e}; at {int(g['steps'])} steps {err_u:.2e} "
          f"(sampled nodes); drift {drift:.2e}")
    assert err_early < 1e-5
    assert drift < 1e-4


def test_duct_workload_fp32_error(Solver):
    """Without moving boundaries the FP32-shifted form holds 1e-5 relative L2 in
    u for the full 20000 steps of the duct workload."""
    g = fixture("duct")
    s = Solver(workload_params("duct", "fp32"))
    s.run(int(g["steps"]))
    flag, rho, u = s.fields()
    fl = g["x0_flag"] == 0
    err = rel_l2(u[:, :, 0][fl], g["x0_u"][fl])
    print(f"duct fp32: rel L2 u {err:.2e}")
    assert err < 1e-5


def run_driver(tmp_path, deck_kv, **kw):
    args = [str(DRIVER), "/dev/null"] + [f"{k}={v}" for k, v in {**deck_kv, **kw}.items()]
    args.append(f"output_dir={tmp_path}")
    res = subprocess.run(args, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout


def keyvalue(path):
    out = {}
    for line in Path(path).read_text().splitlines():
        tok = line.split()
        if tok:
            out[tok[0]] = np.array([float(v) for v in tok[1:]])
    return out


def test_driver_reproduces_shipped_duct(tmp_path):
    """inputs/duct.in through the drop-in driver: converges at the same print
    step with the same L2 error as the reference's shipped duct_summary.txt."""
    shipped = np.load(GOLDEN / "shipped.npz")
    deck = dict(nx=4, ny=34, nz=34, tau=0.8, fx=5e-5, walls_y=1, walls_z=1, squirmer=0, steps=100000,
                tol=1e-12, print_every=1000, prefix="duct")
    out = run_driver(tmp_path, deck)
    s = keyvalue(tmp_path / "duct_summary.txt")
    assert int(s["steps"][0]) == int(shipped["duct_summary_steps"][0]) and int(s["converged"][0]) == 1
    assert abs(s["l2_error"][0] - shipped["duct_summary_l2_error"][0]) < 1e-12
    assert abs(s["max_speed"][0] - shipped["duct_summary_max_speed"][0]) < 1e-12
    assert np.allclose(s["wall_force"], shipped["duct_summary_wall_force"], rtol=1e-8, atol=1e-12)
    prof = np.loadtxt(tmp_path / "duct_profile_y.dat")
    assert np.allclose(prof, shipped["duct_profile_y"], rtol=1e-9, atol=1e-12)
    assert "relative L2 error vs exact Poiseuille solution" in out


def test_driver_reproduces_shipped_channel_trajectory(tmp_path):
    """inputs/channel_neutral.in for 2000 steps: the trajectory file equals the
    reference's shipped examples/reference_data/channel_neutral_traj.dat rows to
    the printed precision."""
    shipped = np.load(GOLDEN / "shipped.npz")
    deck = dict(nx=64, ny=34, nz=32, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4, b1=0.015, beta=0,
                angle=30, planar=1, eps=0.2, hc=2.0, hmin=0.5, steps=2000, print_every=500, traj_every=50,
                prefix="channel_neutral")
    run_driver(tmp_path, deck)
    rows = np.loadtxt(tmp_path / "channel_neutral_traj.dat")
    ref = shipped["example_neutral_traj"][: len(rows)]
    assert rows.shape == ref.shape
    assert np.all(np.abs(rows[:, 1:7] - ref[:, 1:7]) <= 5.1e-7)
    big = np.abs(ref[:, 7:]) > 0
    assert np.all(np.abs(rows[:, 7:] - ref[:, 7:])[big] / np.abs(ref[:, 7:])[big] <= 5.1e-7)
    assert (tmp_path / "channel_neutral_final.vtk").exists()
    assert (tmp_path / "channel_neutral_squirmer.dat").exists()


def test_driver_checkpoint_and_restart(tmp_path):
    """The drop-in driver with checkpoint_every writes <prefix>_checkpoint.bin;
    a second run with restart= continues from it and writes the same
    trajectory rows and final squirmer state as one uninterrupted run."""
    deck = dict(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015, beta=-2,
                angle=20, planar=1, print_every=100, traj_every=20)
    full = tmp_path / "full"; full.mkdir()
    run_driver(full, deck, steps=400, prefix="run")
    part = tmp_path / "part"; part.mkdir()
    run_driver(part, deck, steps=200, prefix="run", checkpoint_every=200)
    ck = part / "run_checkpoint.bin"
    assert ck.exists()
    out = run_driver(part, deck, steps=400, prefix="run", restart=str(ck))
    assert "restarted from" in out and "t=200" in out
    a = np.loadtxt(full / "run_traj.dat")
    b = np.loadtxt(part / "run_traj.dat")
    assert a.shape == b.shape and np.array_equal(a, b)
    assert (full / "run_squirmer.dat").read_text() == (part / "run_squirmer.dat").read_text()
