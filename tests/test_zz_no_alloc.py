"""lbmgpu_field_stats_static (allocation-free diagnostics over the caller's
device fields) against lbmgpu_diag on the same lattice.

The fields come from a solver run: lbmgpu_fields copies them to the host, the
test puts them in device memory of its own (torch) and calls the static entry
point through the C ABI twice in a row, after the solver's own lbmgpu_diag.
Counts and max |u| are exact; the sums are added in a different order than
lbmgpu_diag's grid-stride reduction, so they agree to 1e-12 relative.
This file is collected last so that it also runs after every other test.
"""
import ctypes

import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params

pytestmark = pytest.mark.gpu


def stats_static(lib, dev_arrays, n, stream=None):
    from lbm_solver_3d_b200._lib import LbmgpuDiagnostics, check
    d = LbmgpuDiagnostics()
    flag, rho, ux, uy, uz = (ctypes.c_void_p(a.data_ptr()) for a in dev_arrays)
    check(lib.lbmgpu_field_stats_static(flag, rho, ux, uy, uz, n, ctypes.c_void_p(stream or 0), ctypes.byref(d)))
    return dict(n_fluid=d.n_fluid, mean_density=d.mean_density, max_speed=d.max_speed, sum_ux=d.sum_ux,
                wall_force=np.array(d.wall_force[:]))


def device_fields(solver):
    import torch
    flag, rho, u = solver.fields()
    t = [torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
         for a in (flag, rho, u[..., 0], u[..., 1], u[..., 2])]
    torch.cuda.synchronize()
    fluid = flag == 0
    return t, float(np.abs(u[..., 0][fluid]).sum())


def close(a, b, rel):  # relative closeness
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("deck", [
    dict(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015, beta=-2.0,
         angle=20, planar=1),
    dict(nx=16, ny=32, nz=32, tau=0.8, fx=1e-6, walls_y=1, walls_z=1, squirmer=0),
])
def test_static_stats_match_diag_two_calls_in_a_row(deck):
    import torch
    from lbm_solver_3d_b200 import _lib
    from lbm_solver_3d_b200.solver import Solver
    lib = _lib.load()
    p = Params().update(**deck)
    p.validate()
    s = Solver(p)
    for steps in (57, 40):
        s.run(steps)
        ref = s.diag()
        dev, sum_abs_ux = device_fields(s)
        stream = torch.cuda.Stream()
        a = stats_static(lib, dev, p.ncells, stream.cuda_stream)
        b = stats_static(lib, dev, p.ncells, stream.cuda_stream)
        for r in (a, b):
            assert r["n_fluid"] == ref["n_fluid"]
            assert r["max_speed"] == ref["max_speed"]
            assert close(r["mean_density"], ref["mean_density"], 1e-12)
            assert abs(r["sum_ux"] - ref["sum_ux"]) <= 1e-12 * sum_abs_ux
            assert np.all(r["wall_force"] == 0)
        for k in ("n_fluid", "mean_density", "max_speed", "sum_ux"):
            assert a[k] == b[k]   # the reduction order is fixed: repeated calls agree bit for bit
    s.close()


def test_static_stats_allocates_no_device_memory():
    """The property the entry point exists for: after one warm-up call (which
    may load the kernel's module and look up the scratch's address), further
    calls leave the device's free memory (cudaMemGetInfo) unchanged."""
    import torch
    from lbm_solver_3d_b200 import _lib
    from lbm_solver_3d_b200.solver import Solver
    lib = _lib.load()
    p = Params().update(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, squirmer=1, radius=4.5, b1=0.015, angle=20)
    p.validate()
    s = Solver(p)
    s.run(30)
    dev, _ = device_fields(s)
    stream = torch.cuda.Stream()
    first = stats_static(lib, dev, p.ncells, stream.cuda_stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        r = stats_static(lib, dev, p.ncells, stream.cuda_stream)
        assert r["n_fluid"] == first["n_fluid"] and r["sum_ux"] == first["sum_ux"]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes across 5 calls"
    s.close()


def test_static_stats_rejects_sizes_beyond_its_scratch():
    from lbm_solver_3d_b200 import _lib
    from lbm_solver_3d_b200._lib import LbmgpuDiagnostics
    lib = _lib.load()
    d = LbmgpuDiagnostics()
    fake = ctypes.c_void_p(256)   # never dereferenced: the size is checked first
    for n in (0, (1 << 25) + 1):
        rc = lib.lbmgpu_field_stats_static(fake, fake, fake, fake, fake, n, None, ctypes.byref(d))
        assert rc == -1
        assert b"static scratch" in lib.lbmgpu_last_error(None)
