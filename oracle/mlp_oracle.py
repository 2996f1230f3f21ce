"""TEST INFRASTRUCTURE ONLY -- float64 restatement of the surrogate network
and its gradients, the checker of the CUDA kernels in
lbm_solver_3d_b200/csrc/k_mlp.cu.

Network: 4 -> 64 -> 64 -> 64 -> 3, SiLU after each hidden layer.
Loss: mean over samples and outputs of the squared error.
Parameter layout (flat): W1[64][4] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
W4[3][64] b4[3], W[out][in] (the layout of include/lbmgpu.h).

The surrogate has no counterpart in the reference (it is one of the forms
built beside the plain method), so there is no reference code to pin this
restatement to; it is pinned to central finite differences of its own loss
(tests/test_mlp.py) and is what the GPU gradients are checked against.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 4, 64, 3
SHAPES = [("W1", (NH, NI)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
          ("W3", (NH, NH)), ("b3", (NH,)), ("W4", (NO, NH)), ("b4", (NO,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    theta = np.asarray(theta, np.float64)
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = theta[k:k + n].reshape(shape)
        k += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], np.float64).reshape(-1) for name, _ in SHAPES])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(theta, x, keep=False):
    p = unpack(theta)
    h = np.asarray(x, np.float64)
    cache = [(None, h)]
    for l in (1, 2, 3):
        z = h @ p[f"W{l}"].T + p[f"b{l}"]
        h = z * _sig(z)
        cache.append((z, h))
    y = h @ p["W4"].T + p["b4"]
    return (y, cache) if keep else y


def loss_grad(theta, x, y_target):
    """Mean squared error and its gradient with respect to theta."""
    p = unpack(theta)
    y, cache = forward(theta, x, keep=True)
    r = y - np.asarray(y_target, np.float64)
    cnt = r.size
    loss = float((r * r).sum() / cnt)
    d = 2.0 * r / cnt
    g = {}
    g["W4"] = d.T @ cache[3][1]
    g["b4"] = d.sum(0)
    dh = d @ p["W4"]
    for l in (3, 2, 1):
        z, _ = cache[l]
        s = _sig(z)
        dz = dh * s * (1.0 + z * (1.0 - s))
        g[f"W{l}"] = dz.T @ cache[l - 1][1]
        g[f"b{l}"] = dz.sum(0)
        dh = dz @ p[f"W{l}"]
    return loss, pack(g)


def init_params(seed: int) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape in SHAPES:
        fan_in = shape[1] if len(shape) == 2 else {"b1": NI, "b2": NH, "b3": NH, "b4": NH}[name]
        bound = 1.0 / np.sqrt(fan_in)
        parts[name] = rng.uniform(-bound, bound, size=shape)
    return pack(parts)
