"""ctypes binding of the C ABI in include/lbmgpu.h (liblbmgpu.so, built in-tree).

There is no fallback: if the CUDA library is missing or fails to load, every
entry point raises. Build it with ``python -c "import __graft_entry__ as g; g.build()"``
or ``make -C lbm_solver_3d_b200/csrc``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "liblbmgpu.so"

LBMGPU_OK = 0
LBMGPU_ERR_INVALID, LBMGPU_ERR_CUDA, LBMGPU_ERR_NAN, LBMGPU_ERR_DEVICE = -1, -2, -3, -4
LBMGPU_ERR_NOMEM, LBMGPU_ERR_WATCHDOG = -5, -6
STATUS = {0: "OK", -1: "INVALID", -2: "CUDA", -3: "NAN", -4: "DEVICE", -5: "NOMEM", -6: "WATCHDOG"}


class LbmgpuParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("tau", ctypes.c_double), ("lambda_", ctypes.c_double),
        ("fx", ctypes.c_double), ("fy", ctypes.c_double), ("fz", ctypes.c_double),
        ("walls_y", ctypes.c_int), ("walls_z", ctypes.c_int),
        ("traj_every", ctypes.c_int), ("mass_correction_every", ctypes.c_int),
        ("squirmer", ctypes.c_int),
        ("radius", ctypes.c_double), ("b1", ctypes.c_double), ("beta", ctypes.c_double),
        ("rho_p", ctypes.c_double), ("x0", ctypes.c_double), ("y0", ctypes.c_double),
        ("z0", ctypes.c_double), ("angle", ctypes.c_double),
        ("planar", ctypes.c_int),
        ("eps", ctypes.c_double), ("hc", ctypes.c_double), ("hmin", ctypes.c_double),
        ("use_orientation", ctypes.c_int),
        ("ex", ctypes.c_double), ("ey", ctypes.c_double), ("ez", ctypes.c_double),
        ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class LbmgpuSquirmer(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 3) for n in ("X", "e", "U", "W", "Fh", "Th", "Fc", "Tc", "Fw")] + [
        ("R", ctypes.c_double), ("B1", ctypes.c_double), ("beta", ctypes.c_double),
        ("M", ctypes.c_double), ("I", ctypes.c_double), ("FS", ctypes.c_double),
        ("U0", ctypes.c_double), ("contacts", ctypes.c_longlong)]


class LbmgpuDiagnostics(ctypes.Structure):
    _fields_ = [("n_fluid", ctypes.c_longlong), ("mean_density", ctypes.c_double),
                ("max_speed", ctypes.c_double), ("sum_ux", ctypes.c_double),
                ("wall_force", ctypes.c_double * 3)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_DP = ctypes.POINTER(ctypes.c_double)
_U8P = ctypes.POINTER(ctypes.c_uint8)

# name -> (restype, argtypes); every symbol declared in include/lbmgpu.h
SIGNATURES = {
    "lbmgpu_params_default": (None, [ctypes.POINTER(LbmgpuParams)]),
    "lbmgpu_validate": (_I, [ctypes.POINTER(LbmgpuParams), ctypes.c_char_p, ctypes.c_size_t]),
    "lbmgpu_create": (_I, [ctypes.POINTER(LbmgpuParams), ctypes.POINTER(_P)]),
    "lbmgpu_destroy": (_I, [_P]),
    "lbmgpu_run": (_I, [_P, _I]),
    "lbmgpu_step": (_I, [_P]),
    "lbmgpu_advance_squirmer": (_I, [_P]),
    "lbmgpu_correct_mass": (_I, [_P]),
    "lbmgpu_time": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "lbmgpu_squirmer_state": (_I, [_P, ctypes.POINTER(LbmgpuSquirmer)]),
    "lbmgpu_fields": (_I, [_P, _U8P, _DP, _DP]),
    "lbmgpu_diag": (_I, [_P, ctypes.POINTER(LbmgpuDiagnostics)]),
    "lbmgpu_traj_rows": (_I, [_P, _DP, _I, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong)]),
    "lbmgpu_get_populations": (_I, [_P, _DP]),
    "lbmgpu_set_populations": (_I, [_P, _DP]),
    "lbmgpu_set_squirmer_state": (_I, [_P, _DP, _DP, _DP, _DP]),
    "lbmgpu_set_stream": (_I, [_P, _P]),
    "lbmgpu_launch_count": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "lbmgpu_time_kernels": (_I, [_P, _I, _DP]),
    "lbmgpu_last_error": (ctypes.c_char_p, [_P]),
    "lbmgpu_abi_version": (_I, []),
    "lbmgpu_field_stats_static": (_I, [_P, _P, _P, _P, _P, ctypes.c_longlong, _P,
                                       ctypes.POINTER(LbmgpuDiagnostics)]),
    "lbmgpu_mlp_create": (_I, [_I, _I, ctypes.POINTER(_P)]),
    "lbmgpu_mlp_destroy": (_I, [_P]),
    "lbmgpu_mlp_set_params": (_I, [_P, ctypes.POINTER(ctypes.c_float), _I]),
    "lbmgpu_mlp_get_params": (_I, [_P, ctypes.POINTER(ctypes.c_float)]),
    "lbmgpu_mlp_set_adam": (_I, [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "lbmgpu_mlp_set_data": (_I, [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), _I]),
    "lbmgpu_mlp_train_epoch": (_I, [_P, ctypes.POINTER(ctypes.c_int), _I, _I, ctypes.c_float,
                                    ctypes.POINTER(ctypes.c_float)]),
    "lbmgpu_mlp_loss_grad": (_I, [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "lbmgpu_mlp_forward": (_I, [_P, ctypes.POINTER(ctypes.c_float), _I, ctypes.POINTER(ctypes.c_float)]),
    "lbmgpu_mlp_forward_ex": (_I, [_P, ctypes.POINTER(ctypes.c_float), _I, ctypes.POINTER(ctypes.c_float), _I]),
    "lbmgpu_mlp_last_error": (ctypes.c_char_p, [_P]),
    "lbmgpu_watchdog_selftest": (_I, [_I, ctypes.c_longlong, ctypes.POINTER(_I)]),
    "lbmgpu_snapshot_begin": (_I, [_P]),
    "lbmgpu_snapshot_read": (_I, [_P, _U8P, _DP, _DP]),
    "lbmgpu_snapshot_last_error": (ctypes.c_char_p, [_P]),
    "lbmgpu_host_alloc": (_P, [ctypes.c_size_t]),
    "lbmgpu_host_free": (_I, [_P]),
    "lbmgpu_checkpoint_size": (_I, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    "lbmgpu_checkpoint_save": (_I, [_P, _P, ctypes.c_size_t]),
    "lbmgpu_checkpoint_load": (_I, [_P, _P, ctypes.c_size_t]),
    "lbmgpu_checkpoint_check": (_I, [ctypes.POINTER(LbmgpuParams), _P, ctypes.c_size_t, ctypes.c_char_p,
                                     ctypes.c_size_t]),
    "lbmgpu_batch_create": (_I, [ctypes.POINTER(LbmgpuParams), _I, ctypes.POINTER(_P)]),
    "lbmgpu_batch_destroy": (_I, [_P]),
    "lbmgpu_batch_run": (_I, [_P, _I]),
    "lbmgpu_batch_member": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "lbmgpu_batch_size": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong)]),
    "lbmgpu_batch_set_tiling": (_I, [_P, _I, _I]),
    "lbmgpu_batch_autotune": (_I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), _DP]),
    "lbmgpu_batch_time_bulk": (_I, [_P, _I, _DP]),
    "lbmgpu_batch_set_stream": (_I, [_P, _P]),
    "lbmgpu_batch_launch_count": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "lbmgpu_batch_last_error": (ctypes.c_char_p, [_P]),
}

_lib = None


class LbmgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lbmgpu error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


def load():
    """Load liblbmgpu.so (in-tree). Raises if it is absent: there is no CPU path."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("LBMGPU_LIB", LIB_PATH))
    if not path.exists():
        raise RuntimeError(f"CUDA library {path} is not built; run __graft_entry__.build() "
                           "or make -C lbm_solver_3d_b200/csrc")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int, handle=None) -> None:
    if code != LBMGPU_OK:
        msg = load().lbmgpu_last_error(handle)
        raise LbmgpuError(code, msg.decode() if msg else "")


def check_batch(code: int, batch=None) -> None:
    if code != LBMGPU_OK:
        msg = load().lbmgpu_batch_last_error(batch)
        raise LbmgpuError(code, msg.decode() if msg else "")


def dptr(a):
    return a.ctypes.data_as(_DP)


def u8ptr(a):
    return a.ctypes.data_as(_U8P)
