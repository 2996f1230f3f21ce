"""Python face of the surrogate network kernels (lbmgpu_mlp_* of
include/lbmgpu.h): a 4 -> 64 -> 64 -> 64 -> 3 SiLU perceptron trained with
Adam by the library's own forward/backward kernels on the GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

NPARAMS = 64 * 4 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 3 * 64 + 3
SHAPES = [("W1", (64, 4)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
          ("W3", (64, 64)), ("b3", (64,)), ("W4", (3, 64)), ("b4", (3,))]
_FP = ctypes.POINTER(ctypes.c_float)


def _fp(a):
    return a.ctypes.data_as(_FP)


def init_params(seed: int) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases (FP32)."""
    rng = np.random.default_rng(seed)
    out = []
    for name, shape in SHAPES:
        fan_in = shape[1] if len(shape) == 2 else (4 if name == "b1" else 64)
        b = 1.0 / np.sqrt(fan_in)
        out.append(rng.uniform(-b, b, size=shape).reshape(-1))
    return np.concatenate(out).astype(np.float32)


class MLP:
    def __init__(self, bf16: bool = False, device: int = 0, params: np.ndarray | None = None, seed: int = 0):
        self.lib = _lib.load()
        self.bf16 = bool(bf16)
        h = ctypes.c_void_p()
        self._check(self.lib.lbmgpu_mlp_create(int(device), int(self.bf16), ctypes.byref(h)), None)
        self.h = h
        self.set_params(init_params(seed) if params is None else params)

    def _check(self, rc, h):
        if rc != 0:
            msg = self.lib.lbmgpu_mlp_last_error(h)
            raise _lib.LbmgpuError(rc, msg.decode() if msg else "")

    def set_params(self, params, reset_optimizer: bool = True) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        assert p.size == NPARAMS
        self._check(self.lib.lbmgpu_mlp_set_params(self.h, _fp(p), int(reset_optimizer)), self.h)

    def params(self) -> np.ndarray:
        p = np.empty(NPARAMS, np.float32)
        self._check(self.lib.lbmgpu_mlp_get_params(self.h, _fp(p)), self.h)
        return p

    def set_data(self, x, y) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        assert x.ndim == 2 and x.shape[1] == 4 and y.shape == (x.shape[0], 3)
        self._check(self.lib.lbmgpu_mlp_set_data(self.h, _fp(x), _fp(y), x.shape[0]), self.h)
        self.n = x.shape[0]

    def train_epoch(self, order, batch: int, lr: float) -> float:
        order = np.ascontiguousarray(order, dtype=np.int32)
        loss = ctypes.c_float()
        self._check(self.lib.lbmgpu_mlp_train_epoch(self.h, order.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                    order.size, int(batch), float(lr), ctypes.byref(loss)), self.h)
        return loss.value

    def loss_grad(self):
        loss = ctypes.c_float()
        g = np.empty(NPARAMS, np.float32)
        self._check(self.lib.lbmgpu_mlp_loss_grad(self.h, ctypes.byref(loss), _fp(g)), self.h)
        return loss.value, g

    PATH_AUTO, PATH_WARP, PATH_TCGEN05 = 0, 1, 2

    def forward(self, x, path: int = 0) -> np.ndarray:
        """Inference. path: PATH_AUTO (tensor memory for BF16 networks, FP32
        FMA otherwise), PATH_WARP (the warp-tiled kernel), PATH_TCGEN05."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 4)
        y = np.empty((x.shape[0], 3), np.float32)
        self._check(self.lib.lbmgpu_mlp_forward_ex(self.h, _fp(x), x.shape[0], _fp(y), int(path)), self.h)
        return y

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.lbmgpu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
