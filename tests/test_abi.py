"""The C ABI library loads, exports every symbol include/lbmgpu.h declares, and
its host-side entry points behave like the reference's Params (no GPU needed:
nothing here launches a kernel)."""
import ctypes
import re
from pathlib import Path

import pytest

from lbm_solver_3d_b200 import _lib
from lbm_solver_3d_b200.params import ParamError, Params

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "lbmgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbmgpu_[a-z_0-9]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/lbmgpu.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.lbmgpu_abi_version() == 1


def test_defaults_are_the_reference_defaults():
    lib = _lib.load()
    c = _lib.LbmgpuParams()
    lib.lbmgpu_params_default(ctypes.byref(c))
    ref = Params().to_c()
    for name, _ in _lib.LbmgpuParams._fields_:
        assert getattr(c, name) == getattr(ref, name), name


INVALID = [
    (dict(nx=0), "grid dimensions must be positive"),
    (dict(ny=3, walls_y=1), "ny must be >= 4 with walls in y"),
    (dict(nz=3, walls_z=1), "nz must be >= 4 with walls in z"),
    (dict(tau=0.5), "tau must be > 0.5"),
    (dict(**{"lambda": 0}), "lambda must be > 0"),
    (dict(traj_every=0), "print_every and traj_every must be >= 1"),
    (dict(squirmer=1, radius=1.0), "squirmer radius must be > 1 lattice unit"),
    (dict(squirmer=1, angle=45), "initial angle must satisfy |angle| < 45 deg from the x-axis"),
    (dict(squirmer=1, rho_p=0), "rho_p must be > 0"),
    (dict(squirmer=1, hc=0), "eps >= 0, hc > 0, hmin >= 0 required"),
    (dict(squirmer=1, y0=4.0), "squirmer initially overlaps (or is too close to) a y-wall"),
    (dict(squirmer=1, nx=9), "domain too small for the squirmer"),
    (dict(squirmer=1, b1=0.08), "swimming speed U0 = 2 B1 / 3 too large (Mach number); keep U0 < 0.05"),
]


@pytest.mark.parametrize("kw,msg", INVALID)
def test_validate_messages_match_reference_rules(kw, msg):
    """lbmgpu_validate (C) and Params.validate (Python) both apply
    params.cpp:120-140 with its messages."""
    p = Params().update(**kw)
    with pytest.raises(ParamError, match=re.escape(msg)):
        p.validate()
    lib = _lib.load()
    buf = ctypes.create_string_buffer(256)
    rc = lib.lbmgpu_validate(ctypes.byref(p.to_c()), buf, 256)
    assert rc == -1 and buf.value.decode() == msg


def test_create_fails_loudly_without_a_device_or_with_bad_params():
    lib = _lib.load()
    h = ctypes.c_void_p()
    bad = Params().update(tau=0.4).to_c()
    assert lib.lbmgpu_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert b"tau must be > 0.5" in lib.lbmgpu_last_error(None)
    assert not h.value


def test_null_handles_are_rejected():
    lib = _lib.load()
    assert lib.lbmgpu_run(None, 1) == -1
    assert lib.lbmgpu_step(None) == -1
    assert lib.lbmgpu_destroy(None) == 0


def test_ensemble_create_rejects_mixed_or_bad_members():
    """lbmgpu_batch_create checks every member before touching the device."""
    lib = _lib.load()
    b = ctypes.c_void_p()
    base = dict(nx=40, ny=26, nz=22, squirmer=1, radius=4.0)
    cases = [
        ([dict(base), dict(base, tau=0.9)], "members must share tau"),
        ([dict(base), dict(base, nx=300)], "nx must be <= 256"),
        ([dict(base), dict(base, tau=0.4)], "member 1: tau must be > 0.5"),
    ]
    for members, msg in cases:
        arr = (_lib.LbmgpuParams * len(members))(*[Params().update(**m).to_c() for m in members])
        assert lib.lbmgpu_batch_create(arr, len(members), ctypes.byref(b)) == -1
        assert msg in lib.lbmgpu_batch_last_error(None).decode()
        assert not b.value
    assert lib.lbmgpu_batch_create(None, 0, ctypes.byref(b)) == -1
    assert lib.lbmgpu_batch_run(None, 1) == -1
    assert lib.lbmgpu_batch_destroy(None) == 0


def test_static_stats_checks_arguments_before_touching_the_device():
    """lbmgpu_field_stats_static rejects null pointers and sizes beyond its
    static scratch (2^25 nodes) with a message, before any CUDA call."""
    lib = _lib.load()
    d = _lib.LbmgpuDiagnostics()
    fake = ctypes.c_void_p(256)   # never dereferenced
    assert lib.lbmgpu_field_stats_static(None, fake, fake, fake, fake, 10, None, ctypes.byref(d)) == -1
    assert b"null pointer" in lib.lbmgpu_last_error(None)
    for n in (0, -5, (1 << 25) + 1):
        assert lib.lbmgpu_field_stats_static(fake, fake, fake, fake, fake, n, None, ctypes.byref(d)) == -1
        assert b"33554432, the capacity of its static scratch" in lib.lbmgpu_last_error(None)


def test_checkpoint_check_rejects_garbage_without_a_device():
    """lbmgpu_checkpoint_check validates a restart buffer against parameters on
    the host alone: no handle, no device."""
    from lbm_solver_3d_b200.solver import Solver
    p = Params().update(nx=40, ny=26, nz=22, squirmer=1, radius=4.5)
    assert "not a checkpoint" in Solver.check_checkpoint(p, b"x" * 400)
    assert "too short" in Solver.check_checkpoint(p, b"LBMGPUCK")
    bad = Params().update(nx=0)
    assert "grid dimensions" in Solver.check_checkpoint(bad, b"x" * 400)
