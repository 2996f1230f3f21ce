"""Failure detection, exercised without a GPU fault.

The reference reports failures as exceptions caught once in main, printed as
"error: ..." with exit status 1 (src/main.cpp:38-45 in the reference). Here
every failure becomes a status code of the C ABI (lbmgpu_last_error gives the
message) and the drop-in driver turns it into the same "error:" line and exit
status. Each failure is made on the host:
  * non-finite populations written through lbmgpu_set_populations -> the
    device sets ST_NAN when the sphere's force becomes non-finite, and
    lbmgpu_run returns LBMGPU_ERR_NAN;
  * a squirmer velocity of more than one cell per step written through
    lbmgpu_set_squirmer_state -> ST_REMAP_RANGE, LBMGPU_ERR_DEVICE;
  * a bounded device wait on an mbarrier that nothing arrives at (no copy
    issued), with a short limit -> ST_WATCHDOG, LBMGPU_ERR_WATCHDOG.
After each, the device stays usable: a new lattice runs and matches the
oracle's first steps. Nothing here traps, asserts on the device or reads a
bad address.
"""
import ctypes
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from lbm_solver_3d_b200.params import Params

DRIVER = ROOT / "lbm_solver_3d_b200" / "bin" / "lbm_squirmer_gpu"
SLIT = dict(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015, beta=-2.0,
            angle=20, planar=1, traj_every=10)


def params(**kw):
    p = Params().update(**{**SLIT, **kw})
    p.validate()
    return p


def device_still_usable():
    """A fresh lattice runs 20 steps and equals the oracle's (FP64)."""
    from lbm_solver_3d_b200.solver import Solver
    from oracle.oracle import PortSolver
    p = params()
    g = Solver(p)
    g.run(20)
    o = PortSolver(p)
    o.run(20)
    fl, rg, ug = g.fields()
    flo, ro, uo = o.fields()
    assert np.array_equal(fl, flo)
    f = flo == 0
    assert np.linalg.norm(ug[f] - uo[f]) <= 1e-10 * np.linalg.norm(uo[f])
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nan_populations_are_reported(precision):
    from lbm_solver_3d_b200._lib import LBMGPU_ERR_NAN, LbmgpuError
    from lbm_solver_3d_b200.solver import Solver
    s = Solver(params(precision=precision))
    s.run(12)
    f = s.get_f()
    X = s.squirmer()["X"]
    x, y, z = (int(round(c)) for c in X)
    f[:, z - 6:z + 7, y - 6:y + 7, x - 6:x + 7] = np.nan   # every population around the sphere
    s.set_f(f)
    with pytest.raises(LbmgpuError, match="non-finite") as ei:
        s.run(5)
    assert ei.value.code == LBMGPU_ERR_NAN
    with pytest.raises(LbmgpuError) as ei:   # the status stays set: the lattice is not advanced further
        s.run(3)
    assert ei.value.code == LBMGPU_ERR_NAN
    s.close()
    device_still_usable()


@pytest.mark.gpu
def test_squirmer_faster_than_a_cell_per_step_is_reported():
    from lbm_solver_3d_b200._lib import LBMGPU_ERR_DEVICE, LbmgpuError
    from lbm_solver_3d_b200.solver import Solver
    s = Solver(params())
    s.run(8)
    st = s.squirmer()
    s.set_squirmer(st["X"], st["e"], [1.5, 0.0, 0.0], st["W"])
    with pytest.raises(LbmgpuError, match="one lattice cell or more") as ei:
        s.run(2)
    assert ei.value.code == LBMGPU_ERR_DEVICE
    s.close()
    device_still_usable()


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_reports_watchdog():
    from lbm_solver_3d_b200 import _lib
    lib = _lib.load()
    st = ctypes.c_int(-1)
    rc = lib.lbmgpu_watchdog_selftest(0, 2000, ctypes.byref(st))
    assert rc == _lib.LBMGPU_ERR_WATCHDOG
    assert st.value == 16
    assert b"bounded device wait" in lib.lbmgpu_last_error(None)
    assert lib.lbmgpu_watchdog_selftest(0, 0, ctypes.byref(st)) == _lib.LBMGPU_ERR_INVALID
    device_still_usable()


@pytest.mark.gpu
def test_driver_reports_a_rejected_restart_as_error_exit_1(tmp_path):
    """A restart file of another deck: the driver prints "error: ..." and
    exits 1, as the reference does for any failure."""
    deck = dict(SLIT, steps=40, print_every=20)
    args = [str(DRIVER), "/dev/null"] + [f"{k}={v}" for k, v in deck.items()]
    res = subprocess.run(args + [f"output_dir={tmp_path}", "checkpoint_every=40", "prefix=a"],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    res = subprocess.run(args + [f"output_dir={tmp_path}", "tau=0.9", f"restart={tmp_path / 'a_checkpoint.bin'}",
                                 "prefix=b"], capture_output=True, text=True, timeout=300)
    assert res.returncode == 1
    assert res.stderr.startswith("error: device: checkpoint of another deck")


@pytest.mark.parametrize("kv,msg", [
    (["tau=0.4"], "error: tau must be > 0.5"),
    (["foo=1"], "error: unknown parameter 'foo'"),
    (["squirmer=1", "angle=50"], "error: initial angle must satisfy |angle| < 45 deg from the x-axis"),
])
def test_driver_rejects_bad_parameters_like_the_reference(kv, msg):
    """Parameter errors are caught before any device call (no GPU needed):
    "error: <message>" on stderr and exit status 1 (main.cpp:38-45)."""
    if not DRIVER.exists():
        pytest.skip("driver not built")
    res = subprocess.run([str(DRIVER), "/dev/null", *kv], capture_output=True, text=True, timeout=60)
    assert res.returncode == 1
    assert res.stderr.strip() == msg
