"""Checkpoint / restart: a lattice created with the same parameters and loaded
from a checkpoint continues bit for bit as the saved one (populations,
squirmer state, trajectory rows, fields), in every storage form; loading
into another lattice is rejected."""
import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params

pytestmark = pytest.mark.gpu

SLIT = dict(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015, beta=-2.0,
            angle=20, planar=1, traj_every=10, mass_correction_every=7)


def params(**kw):
    p = Params().update(**{**SLIT, **kw})
    p.validate()
    return p


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
def test_restart_continues_bit_for_bit(precision, tmp_path):
    from lbm_solver_3d_b200.solver import Solver
    p = params(precision=precision)
    a = Solver(p)
    a.run(137)            # odd step count: the checkpoint holds the swapped AA parity
    path = tmp_path / "ck.bin"
    a.save(path)
    a.run(113)
    b = Solver(p)
    b.load(path)
    assert b.t == 137
    b.run(113)
    assert a.t == b.t == 250
    sa, sb = a.squirmer(), b.squirmer()
    for k in ("X", "e", "U", "W", "Fh", "Th", "Fc", "Tc"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(a.traj_rows(), b.traj_rows())
    assert np.array_equal(a.get_f(), b.get_f())
    fa, ra, ua = a.fields()
    fb, rb, ub = b.fields()
    assert np.array_equal(fa, fb) and np.array_equal(ra, rb) and np.array_equal(ua, ub)
    a.close(); b.close()


def test_load_rejects_another_lattice():
    from lbm_solver_3d_b200._lib import LbmgpuError
    from lbm_solver_3d_b200.solver import Solver
    a = Solver(params())
    a.run(5)
    data = a.checkpoint()
    for other in (params(nx=41), params(precision="fp32")):
        with pytest.raises(LbmgpuError, match="another lattice"):
            Solver(other).restore(data)
    with pytest.raises(LbmgpuError, match="not a checkpoint"):
        Solver(params()).restore(b"x" * 200)
    with pytest.raises(LbmgpuError, match="truncated"):
        Solver(params()).restore(data[: len(data) // 2])
    a.close()
