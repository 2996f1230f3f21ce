"""The bulk kernels are interchangeable bit for bit.

Where a lattice allows several bulk kernels for its rows away from walls --
rows staged in shared memory (the default; two nodes per update thread and
whole-row bulk stores in FP16 storage), rows staged with one node per thread,
two nodes per thread loaded from global memory, one node per thread -- the
choice (LBMGPU_BULK, read when a lattice is created) changes the speed, not
the numbers: the populations and the squirmer state after steps that include
mass-correction steps (every 10) and the last step of a call are identical.
The lattices mix rows that the bulk updates whole with rows that cross the
zone around a moving squirmer, and nx = 64 gives the two-node kernel a single
update warp.
"""
import os

import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params

pytestmark = pytest.mark.gpu

KINDS = ("rows", "rows1", "pair", "node")
CASES = {
    # periodic box, a squirmer that moves (beta = 3) through rows of all kinds
    "box": dict(nx=128, ny=40, nz=36, tau=0.9, walls_y=0, walls_z=0, squirmer=1, radius=6.0, b1=0.02,
                beta=3.0, planar=0, ex=0.6, ey=0.64, ez=0.48),
    # slit channel (walls in y), nx = 64
    "slit64": dict(nx=64, ny=30, nz=28, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015,
                   beta=-2.0, angle=20, planar=1),
}


def run_with(kind, case, precision, steps):
    from lbm_solver_3d_b200.solver import Solver
    old = os.environ.get("LBMGPU_BULK")
    os.environ["LBMGPU_BULK"] = kind
    try:
        p = Params().update(**CASES[case], precision=precision)
        s = Solver(p)
    finally:
        if old is None:
            os.environ.pop("LBMGPU_BULK", None)
        else:
            os.environ["LBMGPU_BULK"] = old
    s.run(steps - 7)
    s.run(7)
    f = s.get_f()
    sq = s.squirmer()
    s.close()
    return f, sq


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp16", "fp32", "fp64"])
def test_bulk_kernels_bit_identical(case, precision):
    steps = 43
    ref_f, ref_sq = run_with("node", case, precision, steps)
    for kind in KINDS[:-1]:
        f, sq = run_with(kind, case, precision, steps)
        assert f.dtype == ref_f.dtype
        assert np.array_equal(f.view(np.uint8), ref_f.view(np.uint8)), f"{kind} differs from node ({precision})"
        for k in ("X", "e", "U", "W"):
            assert np.array_equal(np.asarray(sq[k]), np.asarray(ref_sq[k])), f"{kind}: squirmer {k} differs"
