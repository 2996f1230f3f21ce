"""TEST INFRASTRUCTURE ONLY -- Python handles on the oracle.

Two CPU solvers with one interface:
  * ``PortSolver``: the plain-C restatement in oracle/lbm_oracle.c
    (oracle/_ref/liblbm_oracle.so);
  * ``RefSolver``: the reference's own sources compiled with a C harness
    (oracle/_ref/libref_harness.so, recipe oracle/Makefile).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, as the checker; the product path never does.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
Q = 19

_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_P = ctypes.c_void_p


def _dp(a):
    return a.ctypes.data_as(_DP)


def _u8(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


_port = None
_ref = None


def port_lib():
    global _port
    if _port is None:
        path = REF_DIR / "liblbm_oracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run make -C oracle")
        lib = ctypes.CDLL(str(path))
        from lbm_solver_3d_b200._lib import LbmgpuParams
        lib.lbo_create.restype = _P
        lib.lbo_create.argtypes = [ctypes.POINTER(LbmgpuParams)]
        for name in ("lbo_destroy", "lbo_step", "lbo_advance_squirmer", "lbo_correct_mass"):
            getattr(lib, name).argtypes = [_P]
            getattr(lib, name).restype = None
        lib.lbo_run.argtypes = [_P, ctypes.c_int, _DP, ctypes.c_int]
        lib.lbo_run.restype = ctypes.c_int
        lib.lbo_ncells.argtypes = [_P]; lib.lbo_ncells.restype = ctypes.c_long
        lib.lbo_time.argtypes = [_P]; lib.lbo_time.restype = ctypes.c_long
        for name in ("lbo_get_f", "lbo_set_f", "lbo_squirmer_state", "lbo_wall_force", "lbo_diag"):
            getattr(lib, name).argtypes = [_P, _DP]
            getattr(lib, name).restype = None
        lib.lbo_set_flags.argtypes = [_P, ctypes.POINTER(ctypes.c_uint8)]
        lib.lbo_get_fields.argtypes = [_P, ctypes.POINTER(ctypes.c_uint8), _DP, _DP]
        lib.lbo_set_squirmer_state.argtypes = [_P, _DP, _DP, _DP, _DP]
        lib.lbo_duct_velocity.argtypes = [_D] * 6; lib.lbo_duct_velocity.restype = _D
        lib.lbo_poiseuille_error.argtypes = [_P]; lib.lbo_poiseuille_error.restype = _D
        _port = lib
    return _port


def ref_available() -> bool:
    return (REF_DIR / "libref_harness.so").exists()


def _cpu_has_avx512() -> bool:
    try:
        flags = set()
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
        return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    except OSError:
        return False


def timed_build() -> Path:
    """The build of the reference used for timing: the reference Makefile's
    flags (-O3 -std=c++17 -fopenmp) at the highest x86-64 level this CPU runs
    (what -march=native would choose among the levels built), else the parity
    build."""
    for name, ok in (("libref_harness_timed_v4.so", _cpu_has_avx512()), ("libref_harness_timed_v3.so", True)):
        if ok and (REF_DIR / name).exists():
            return REF_DIR / name
    return REF_DIR / "libref_harness.so"


def ref_build() -> str:
    """Which compiled reference the timed CPU legs load."""
    name = timed_build().name
    return {"libref_harness_timed_v4.so": "reference sources, -O3 -march=x86-64-v4 -std=c++17 -fopenmp",
            "libref_harness_timed_v3.so": "reference sources, -O3 -march=x86-64-v3 -std=c++17 -fopenmp",
            }.get(name, "reference sources, parity build -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp")


_ref_timed = None


def ref_lib(timed: bool = False):
    global _ref, _ref_timed
    if (_ref_timed if timed else _ref) is None:
        path = timed_build() if timed else REF_DIR / "libref_harness.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run make -C oracle (needs the reference sources)")
        lib = ctypes.CDLL(str(path))
        lib.ref_create.restype = _P
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_char_p, ctypes.c_int]
        for name in ("ref_destroy", "ref_step", "ref_advance_squirmer", "ref_correct_mass"):
            getattr(lib, name).argtypes = [_P]
            getattr(lib, name).restype = None
        lib.ref_set_orientation.argtypes = [_P, _D, _D, _D]
        lib.ref_run.argtypes = [_P, ctypes.c_int, _DP, ctypes.c_int]
        lib.ref_run.restype = ctypes.c_int
        lib.ref_ncells.argtypes = [_P]; lib.ref_ncells.restype = ctypes.c_long
        lib.ref_time.argtypes = [_P]; lib.ref_time.restype = ctypes.c_long
        for name in ("ref_get_f", "ref_set_f", "ref_squirmer_state", "ref_wall_force", "ref_diag"):
            getattr(lib, name).argtypes = [_P, _DP]
            getattr(lib, name).restype = None
        lib.ref_get_fields.argtypes = [_P, ctypes.POINTER(ctypes.c_uint8), _DP, _DP]
        lib.ref_set_squirmer_state.argtypes = [_P, _DP, _DP, _DP, _DP]
        lib.ref_poiseuille_error.argtypes = [_P, ctypes.c_char_p]; lib.ref_poiseuille_error.restype = _D
        lib.ref_duct_velocity.argtypes = [_D] * 6; lib.ref_duct_velocity.restype = _D
        lib.ref_write_vtk.argtypes = [_P, ctypes.c_char_p]
        if timed:
            _ref_timed = lib
        else:
            _ref = lib
    return _ref_timed if timed else _ref


class _Solver:
    """Common interface: run/step/advance/correct, f, fields, squirmer state."""

    def __init__(self, params):
        self.params = params
        self.N = params.NX * params.NY * params.NZ
        self.shape = (params.NZ, params.NY, params.NX)

    # populations in the reference layout f[i*N + n], returned as (19, nz, ny, nx)
    def get_f(self):
        f = np.empty(Q * self.N)
        self._get_f(_dp(f))
        return f.reshape((Q,) + self.shape)

    def set_f(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        assert f.size == Q * self.N
        self._set_f(_dp(f))

    def fields(self):
        flag = np.empty(self.N, np.uint8)
        rho = np.empty(self.N)
        u = np.empty(3 * self.N)
        self._get_fields(_u8(flag), _dp(rho), _dp(u))
        return flag.reshape(self.shape), rho.reshape(self.shape), u.reshape(self.shape + (3,))

    def squirmer(self):
        o = np.empty(31)
        self._sq(_dp(o))
        return dict(X=o[0:3].copy(), e=o[3:6].copy(), U=o[6:9].copy(), W=o[9:12].copy(),
                    Fh=o[12:15].copy(), Th=o[15:18].copy(), Fc=o[18:21].copy(), Tc=o[21:24].copy(),
                    Fw=o[24:27].copy(), contacts=int(o[27]), M=o[28], I=o[29], FS=o[30])

    def set_squirmer(self, X, e, U, W):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (X, e, U, W)]
        self._set_sq(*[_dp(v) for v in a])

    def wall_force(self):
        o = np.empty(3)
        self._wf(_dp(o))
        return o

    def diag(self):
        o = np.empty(4)
        self._diag(_dp(o))
        return dict(n_fluid=int(o[0]), mean_density=o[1], max_speed=o[2], sum_ux=o[3])

    def run(self, nsteps, max_rows=None):
        """nsteps of the time-loop body; returns the trajectory rows (k, 15)."""
        if max_rows is None:
            max_rows = nsteps // max(1, self.params.trajEvery) + 1
        buf = np.zeros((max(1, max_rows), 15))
        rows = self._run(nsteps, _dp(buf), max_rows)
        return buf[:rows].copy()


class PortSolver(_Solver):
    """The plain-C restatement (oracle/lbm_oracle.c)."""

    def __init__(self, params):
        super().__init__(params)
        lib = self.lib = port_lib()
        c = params.to_c()
        self.h = lib.lbo_create(ctypes.byref(c))
        self._get_f = lambda p: lib.lbo_get_f(self.h, p)
        self._set_f = lambda p: lib.lbo_set_f(self.h, p)
        self._get_fields = lambda a, b, c_: lib.lbo_get_fields(self.h, a, b, c_)
        self._sq = lambda p: lib.lbo_squirmer_state(self.h, p)
        self._set_sq = lambda *a: lib.lbo_set_squirmer_state(self.h, *a)
        self._wf = lambda p: lib.lbo_wall_force(self.h, p)
        self._diag = lambda p: lib.lbo_diag(self.h, p)
        self._run = lambda n, p, m: lib.lbo_run(self.h, n, p, m)

    def step(self): self.lib.lbo_step(self.h)
    def advance_squirmer(self): self.lib.lbo_advance_squirmer(self.h)
    def correct_mass(self): self.lib.lbo_correct_mass(self.h)
    def poiseuille_error(self): return self.lib.lbo_poiseuille_error(self.h)

    def set_flags(self, flag):
        flag = np.ascontiguousarray(flag, dtype=np.uint8).reshape(-1)
        self.lib.lbo_set_flags(self.h, _u8(flag))

    @property
    def t(self): return self.lib.lbo_time(self.h)

    def close(self):
        if self.h:
            self.lib.lbo_destroy(self.h)
            self.h = None

    __del__ = close


class RefSolver(_Solver):
    """The reference's own code (compiled from its sources by oracle/Makefile).
    timed=True loads the build with the reference Makefile's own flags (for
    the CPU baseline); the default is the parity build."""

    def __init__(self, params, timed: bool = False):
        super().__init__(params)
        lib = self.lib = ref_lib(timed)
        kv = [s.encode() for s in params.to_kv(reference_only=True)]
        arr = (ctypes.c_char_p * len(kv))(*kv)
        err = ctypes.create_string_buffer(512)
        self.h = lib.ref_create(len(kv), arr, err, 512)
        if not self.h:
            raise RuntimeError("reference rejected parameters: " + err.value.decode())
        if params.orientation is not None:
            lib.ref_set_orientation(self.h, *params.orientation)
        self._get_f = lambda p: lib.ref_get_f(self.h, p)
        self._set_f = lambda p: lib.ref_set_f(self.h, p)
        self._get_fields = lambda a, b, c_: lib.ref_get_fields(self.h, a, b, c_)
        self._sq = lambda p: lib.ref_squirmer_state(self.h, p)
        self._set_sq = lambda *a: lib.ref_set_squirmer_state(self.h, *a)
        self._wf = lambda p: lib.ref_wall_force(self.h, p)
        self._diag = lambda p: lib.ref_diag(self.h, p)
        self._run = lambda n, p, m: lib.ref_run(self.h, n, p, m)

    def step(self): self.lib.ref_step(self.h)
    def advance_squirmer(self): self.lib.ref_advance_squirmer(self.h)
    def correct_mass(self): self.lib.ref_correct_mass(self.h)

    def poiseuille_error(self, base="/tmp/ref_poiseuille"):
        return self.lib.ref_poiseuille_error(self.h, base.encode())

    def write_vtk(self, path):
        self.lib.ref_write_vtk(self.h, str(path).encode())

    @property
    def t(self): return self.lib.ref_time(self.h)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    __del__ = close


def set_threads(n: int) -> None:
    """OpenMP thread count for both CPU solvers (takes effect for new parallel regions)."""
    os.environ["OMP_NUM_THREADS"] = str(n)
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass
