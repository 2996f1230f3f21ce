"""Python face of the CUDA library: the reference's ``lbm::LBM`` interface.

``Solver(params)`` mirrors ``LBM::LBM(const Params&)`` (src/utils/lbm.cpp:60-94)
and exposes ``step()``, ``advance_squirmer()``, ``correct_mass()`` (lbm.cpp:128,
:257, :324), the diagnostics (lbm.cpp:342-364) and the fields the output
writers read, plus ``run(n)``: n iterations of the time-loop body of
src/main.cpp:60-64 executed on the device in CUDA graphs. Every call goes
through the C ABI of include/lbmgpu.h; there is no CPU implementation.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import LBMGPU_OK, LbmgpuDiagnostics, LbmgpuSquirmer, check, dptr, load, u8ptr
from .params import Params

Q = 19


class Solver:
    def __init__(self, params: Params):
        params.validate()
        self.params = params
        self.lib = _lib.load()
        self.N = params.ncells
        self.shape = (params.NZ, params.NY, params.NX)
        c = params.to_c()
        h = ctypes.c_void_p()
        check(self.lib.lbmgpu_create(ctypes.byref(c), ctypes.byref(h)), None)
        self.h = h
        self._owned = True

    @classmethod
    def _member(cls, params: Params, handle: ctypes.c_void_p, owner) -> "Solver":
        """View of a lattice owned by an ensemble (lbmgpu_batch_member): the
        read-only calls work, the ensemble advances it and frees it."""
        s = cls.__new__(cls)
        s.params = params
        s.lib = _lib.load()
        s.N = params.ncells
        s.shape = (params.NZ, params.NY, params.NX)
        s.h = handle
        s._owned = False
        s._owner = owner
        return s

    # ---- the reference's three per-step calls ----
    def step(self) -> None:
        check(self.lib.lbmgpu_step(self.h), self.h)

    def advance_squirmer(self) -> None:
        check(self.lib.lbmgpu_advance_squirmer(self.h), self.h)

    def correct_mass(self) -> None:
        check(self.lib.lbmgpu_correct_mass(self.h), self.h)

    # ---- the fused time loop ----
    def run(self, nsteps: int) -> None:
        check(self.lib.lbmgpu_run(self.h, int(nsteps)), self.h)

    @property
    def t(self) -> int:
        v = ctypes.c_longlong()
        check(self.lib.lbmgpu_time(self.h, ctypes.byref(v)), self.h)
        return v.value

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        check(self.lib.lbmgpu_launch_count(self.h, ctypes.byref(v)), self.h)
        return v.value

    def time_kernels(self, reps: int = 20) -> dict:
        """Per-launch milliseconds of the bulk, zone and squirmer kernels,
        each timed alone with CUDA events (advances the populations without
        the sphere update: use on a handle kept for measurement)."""
        ms = np.zeros(3)
        check(self.lib.lbmgpu_time_kernels(self.h, int(reps), dptr(ms)), self.h)
        return dict(bulk=ms[0], zone=ms[1], squirmer=ms[2])

    def set_stream(self, stream_handle: int | None) -> None:
        check(self.lib.lbmgpu_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)), self.h)

    # ---- state ----
    def squirmer(self) -> dict:
        s = LbmgpuSquirmer()
        check(self.lib.lbmgpu_squirmer_state(self.h, ctypes.byref(s)), self.h)
        out = {k: np.array(getattr(s, k)[:]) for k in ("X", "e", "U", "W", "Fh", "Th", "Fc", "Tc", "Fw")}
        out.update(R=s.R, B1=s.B1, beta=s.beta, M=s.M, I=s.I, FS=s.FS, U0=s.U0, contacts=int(s.contacts))
        return out

    def set_squirmer(self, X, e, U, W) -> None:
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (X, e, U, W)]
        check(self.lib.lbmgpu_set_squirmer_state(self.h, *[dptr(v) for v in a]), self.h)

    def fields(self):
        """(flag, rho, u) as arrays indexed [z, y, x] and [z, y, x, 3]."""
        flag = np.empty(self.N, np.uint8)
        rho = np.empty(self.N)
        u = np.empty(3 * self.N)
        check(self.lib.lbmgpu_fields(self.h, u8ptr(flag), dptr(rho), dptr(u)), self.h)
        return flag.reshape(self.shape), rho.reshape(self.shape), u.reshape(self.shape + (3,))

    def snapshot_begin(self) -> None:
        """Queue a device-side copy of the last step's fields (lbmgpu_snapshot_begin);
        the time loop may continue before it is read."""
        check(self.lib.lbmgpu_snapshot_begin(self.h), self.h)

    def snapshot_read(self, out: "HostFields | None" = None):
        """The fields of the last snapshot (lbmgpu_snapshot_read), as fields() returns them."""
        out = out or HostFields(self.N)
        rc = self.lib.lbmgpu_snapshot_read(self.h, u8ptr(out.flag), dptr(out.rho), dptr(out.u))
        if rc != LBMGPU_OK:
            raise _lib.LbmgpuError(rc, self.lib.lbmgpu_snapshot_last_error(self.h).decode())
        return out.shaped(self.shape)

    def fields_into(self, out: "HostFields"):
        """fields() into caller-owned (e.g. page-locked) host buffers."""
        check(self.lib.lbmgpu_fields(self.h, u8ptr(out.flag), dptr(out.rho), dptr(out.u)), self.h)
        return out.shaped(self.shape)

    def diag(self) -> dict:
        d = LbmgpuDiagnostics()
        check(self.lib.lbmgpu_diag(self.h, ctypes.byref(d)), self.h)
        return dict(n_fluid=int(d.n_fluid), mean_density=d.mean_density, max_speed=d.max_speed,
                    sum_ux=d.sum_ux, wall_force=np.array(d.wall_force[:]))

    def wall_force(self) -> np.ndarray:
        return self.diag()["wall_force"]

    def traj_rows(self, max_rows: int = 1 << 16) -> np.ndarray:
        buf = np.empty((max_rows, 15))
        n = ctypes.c_int()
        dropped = ctypes.c_longlong()
        check(self.lib.lbmgpu_traj_rows(self.h, dptr(buf), max_rows, ctypes.byref(n), ctypes.byref(dropped)), self.h)
        if dropped.value:
            raise RuntimeError(f"{dropped.value} trajectory rows were overwritten before being read")
        return buf[: n.value].copy()

    def get_f(self) -> np.ndarray:
        f = np.empty(Q * self.N)
        check(self.lib.lbmgpu_get_populations(self.h, dptr(f)), self.h)
        return f.reshape((Q,) + self.shape)

    def set_f(self, f) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        assert f.size == Q * self.N
        check(self.lib.lbmgpu_set_populations(self.h, dptr(f)), self.h)

    # ---- checkpoint / restart ----
    def checkpoint(self) -> bytes:
        """The complete device state of the lattice (lbmgpu_checkpoint_save)."""
        n = ctypes.c_size_t()
        check(self.lib.lbmgpu_checkpoint_size(self.h, ctypes.byref(n)), self.h)
        buf = ctypes.create_string_buffer(n.value)
        check(self.lib.lbmgpu_checkpoint_save(self.h, buf, n.value), self.h)
        return buf.raw

    def restore(self, data: bytes) -> None:
        """Continue from a checkpoint of a lattice with the same parameters."""
        check(self.lib.lbmgpu_checkpoint_load(self.h, data, len(data)), self.h)

    @staticmethod
    def check_checkpoint(p, data: bytes):
        """None if `data` may be loaded into a lattice with parameters `p`, else
        the reason (lbmgpu_checkpoint_check: host only, no device, no handle)."""
        lib = load()
        msg = ctypes.create_string_buffer(256)
        c = p.to_c()
        rc = lib.lbmgpu_checkpoint_check(ctypes.byref(c), data, len(data), msg, 256)
        return None if rc == LBMGPU_OK else msg.value.decode()

    def save(self, path) -> None:
        with open(path, "wb") as fh:
            fh.write(self.checkpoint())

    def load(self, path) -> None:
        with open(path, "rb") as fh:
            self.restore(fh.read())

    def close(self) -> None:
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.lbmgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class HostFields:
    """Host buffers for the fields of an N-node lattice (node types, rho, u
    interleaved). pinned=True places them in page-locked memory
    (lbmgpu_host_alloc), which the device copies into directly."""

    def __init__(self, n: int, pinned: bool = False):
        self.n = n
        self._ptrs = []
        if pinned:
            lib = load()

            def alloc(count, ctype):
                p = lib.lbmgpu_host_alloc(count * ctypes.sizeof(ctype))
                if not p:
                    raise MemoryError("lbmgpu_host_alloc failed")
                self._ptrs.append(p)
                return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctype)), shape=(count,))
            self.flag = alloc(n, ctypes.c_uint8)
            self.rho = alloc(n, ctypes.c_double)
            self.u = alloc(3 * n, ctypes.c_double)
        else:
            self.flag = np.empty(n, np.uint8)
            self.rho = np.empty(n)
            self.u = np.empty(3 * n)

    def shaped(self, shape):
        return self.flag.reshape(shape), self.rho.reshape(shape), self.u.reshape(shape + (3,))

    def close(self) -> None:
        lib = load() if self._ptrs else None
        for p in self._ptrs:
            lib.lbmgpu_host_free(p)
        self._ptrs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
