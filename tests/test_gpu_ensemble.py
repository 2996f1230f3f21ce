"""Ensembles (lbmgpu_batch_*) against the same lattices run alone.

A member of an ensemble runs the per-node arithmetic of a lattice created
alone and forms its row, zone and mass sums in the same order (rows of at most
256 nodes), so after the same number of steps its populations, squirmer state
and trajectory rows equal those of Solver(params).run(n) bit for bit. The
lattice run alone is itself pinned to the oracle (test_gpu_parity.py) and to
the reference's own runs (test_gpu_workloads.py).
"""
import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params

pytestmark = pytest.mark.gpu

SLIT = dict(walls_y=1, walls_z=0, squirmer=1, planar=1, eps=0.2, hc=2.0, hmin=0.5, tau=1.0, b1=0.015,
            traj_every=10, mass_correction_every=7)

MEMBERS = [
    dict(nx=40, ny=26, nz=22, radius=4.5, beta=-2.0, angle=20, y0=12.0),
    dict(nx=33, ny=30, nz=24, radius=3.6, beta=3.5, angle=-25, y0=14.5),
    dict(nx=64, ny=22, nz=30, radius=5.2, beta=0.0, angle=5, y0=10.2),
    dict(nx=47, ny=34, nz=20, radius=4.0, beta=-4.5, angle=-12, y0=20.0),
    dict(nx=71, ny=28, nz=26, radius=3.1, beta=1.5, angle=28, y0=9.0),
]


def members(precision="fp64", **extra):
    out = []
    for m in MEMBERS:
        p = Params()
        p.update(**SLIT)
        p.update(**m)
        p.update(precision=precision, **extra)
        p.validate()
        out.append(p)
    return out


@pytest.fixture(scope="module")
def api():
    from lbm_solver_3d_b200.ensemble import Ensemble
    from lbm_solver_3d_b200.solver import Solver
    return Ensemble, Solver


def assert_member_equals_alone(ens, i, p, Solver, chunks):
    """The lattice alone runs the same sequence of run() calls: rho/u are
    stored on the last step of each call, so covered nodes keep the values of
    the last such step while they were fluid."""
    s = Solver(p)
    for c in chunks:
        s.run(c)
    m = ens.member(i)
    assert m.t == s.t == sum(chunks)
    a, b = m.squirmer(), s.squirmer()
    for k in ("X", "e", "U", "W", "Fh", "Th"):
        assert np.array_equal(a[k], b[k]), (i, k, a[k], b[k])
    assert a["contacts"] == b["contacts"]
    assert np.array_equal(m.traj_rows(), s.traj_rows())
    assert np.array_equal(m.get_f(), s.get_f())
    fa, ra, ua = m.fields()
    fb, rb, ub = s.fields()
    assert np.array_equal(fa, fb) and np.array_equal(ra, rb) and np.array_equal(ua, ub)
    da, db = m.diag(), s.diag()
    assert da["n_fluid"] == db["n_fluid"] and np.array_equal(da["wall_force"], db["wall_force"])
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
def test_ensemble_equals_members_alone(api, precision):
    """230 steps: graph chunks of 48 steps plus single steps, mass corrections
    every 7 steps (inside and outside the captured pattern)."""
    Ensemble, Solver = api
    ps = members(precision)
    with Ensemble(ps) as ens:
        assert len(ens) == len(ps)
        assert ens.cells == sum(p.ncells for p in ps)
        ens.run(101)
        ens.run(129)
        for i, p in enumerate(ps):
            assert_member_equals_alone(ens, i, p, Solver, [101, 129])


@pytest.mark.parametrize("tiling", [(32, 1), (64, 3), (128, 8), (1, 1), (2, 1), (3, 4), (3, 7), (-3, 4), (-4, 2), (-3, 16),
                                    (4, 1), (4, 2)])
def test_ensemble_tiling_does_not_change_results(api, tiling):
    """Row kernel (tile > 0 threads per row) and staged kernel (tile = -2, -3
    stages), with few or many CTAs per SM: bit-identical to the lattices run
    alone, in FP32 and FP64."""
    Ensemble, Solver = api
    for prec in ("fp32", "fp64"):
        ps = members(prec)
        with Ensemble(ps) as ens:
            ens.set_tiling(*tiling)
            ens.run(60)
            for i in (0, 2, 4):
                assert_member_equals_alone(ens, i, ps[i], Solver, [60])


def test_ensemble_autotune_restores_state(api):
    Ensemble, Solver = api
    ps = members("fp32")
    with Ensemble(ps) as ens:
        ens.run(30)
        tuned = ens.autotune(reps=2)
        assert tuned["tile"] in (1, 2, 3, 4, 32, 64, 128, -3, -4) and 1 <= tuned["ctas_per_sm"] <= 16
        assert tuned["ms"] > 0
        ens.run(40)
        for i in range(len(ps)):
            assert_member_equals_alone(ens, i, ps[i], Solver, [30, 40])


def test_ensemble_without_squirmer(api):
    """Duct members (walls in y and z, body force): no zone, no squirmer launch."""
    Ensemble, Solver = api
    ps = []
    for nx, ny, nz in ((12, 14, 10), (20, 9, 17), (7, 16, 16)):
        p = Params()
        p.update(nx=nx, ny=ny, nz=nz, tau=0.8, fx=1e-5, fy=2e-6, fz=-3e-6, walls_y=1, walls_z=1, squirmer=0)
        p.validate()
        ps.append(p)
    with Ensemble(ps) as ens:
        ens.run(75)
        for i, p in enumerate(ps):
            s = Solver(p)
            s.run(75)
            m = ens.member(i)
            assert np.array_equal(m.get_f(), s.get_f())
            assert np.array_equal(m.diag()["wall_force"], s.diag()["wall_force"])
            s.close()


def test_member_handles_are_read_only(api):
    Ensemble, _ = api
    from lbm_solver_3d_b200._lib import LbmgpuError
    with Ensemble(members("fp32")[:2]) as ens:
        m = ens.member(1)
        with pytest.raises(LbmgpuError, match="ensemble"):
            m.run(1)
        with pytest.raises(LbmgpuError, match="ensemble"):
            m.step()
        with pytest.raises(LbmgpuError, match="ensemble"):
            m.set_f(m.get_f())
        ens.run(3)
        assert m.t == 3


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_config4_ensemble_members_equal_alone(api, precision):
    """The 256-member slit-channel ensemble of the benchmark (Nx 64-160, Ny/Nz
    48-96, a 4-8, beta -5..5, seed 2024; 153 M nodes) with the autotuned bulk
    tiling: after 60 steps (a graph chunk and single steps, six mass
    corrections), five seeded members -- the smallest, the largest and three
    drawn at random -- equal the same lattices run alone, bit for bit."""
    from lbm_solver_3d_b200.workloads import ensemble_members
    Ensemble, Solver = api
    ps = ensemble_members(256)
    for p in ps:
        p.update(precision=precision)
    sizes = [p.ncells for p in ps]
    pick = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    pick |= set(np.random.default_rng(11).choice(256, 3, replace=False).tolist())
    with Ensemble(ps) as ens:
        assert ens.cells == sum(sizes)
        tune = ens.autotune(reps=2)
        print(f"{precision}: tiling {tune}")
        ens.run(60)
        for i in sorted(pick):
            assert_member_equals_alone(ens, i, ps[i], Solver, [60])
