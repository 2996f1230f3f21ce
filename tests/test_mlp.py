"""The surrogate network's hand-written CUDA kernels (lbmgpu_mlp_*) against
the float64 oracle (oracle/mlp_oracle.py).

Tolerances: FP32 kernels -- outputs within 1e-5 relative, loss within 1e-5
relative, gradient within 1e-4 relative L2 of the float64 gradient; BF16
GEMMs -- outputs within 2e-2, gradient within 5e-2 relative L2 and cosine
similarity above 0.998 (BF16 keeps 8 bits of mantissa). The oracle itself is
checked against central finite differences of its own loss.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as O


def problem(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.5, 1.5, size=(n, 4))
    y = np.stack([np.sin(2 * x[:, 0]) + 0.3 * x[:, 1] * x[:, 2], np.cos(x[:, 3]) * x[:, 0],
                  np.tanh(x[:, 1] - x[:, 2])], 1)
    return x, y


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a, float) - b) / np.linalg.norm(b)


def test_oracle_gradient_matches_finite_differences():
    x, y = problem(37, 1)
    th = O.init_params(3)
    loss, g = O.loss_grad(th, x, y)
    rng = np.random.default_rng(5)
    pick = rng.choice(O.NPARAMS, 150, replace=False)
    h = 1e-6
    for k in pick:
        e = np.zeros_like(th); e[k] = h
        fd = (O.loss_grad(th + e, x, y)[0] - O.loss_grad(th - e, x, y)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 * max(1.0, abs(g[k])) + 1e-9, k


def test_oracle_layout_and_size():
    assert O.NPARAMS == 64 * 4 + 64 + 2 * (64 * 64 + 64) + 3 * 64 + 3 == 8835
    th = np.arange(O.NPARAMS, dtype=float)
    assert np.array_equal(O.pack(O.unpack(th)), th)


@pytest.mark.gpu
@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("n", [5, 32, 1001])
def test_forward_and_gradient_against_oracle(bf16, n):
    from lbm_solver_3d_b200.mlp import MLP
    x, y = problem(n, 10 + n)
    th = O.init_params(7).astype(np.float32)
    net = MLP(bf16=bf16, params=th)
    out = net.forward(x)
    ref = O.forward(th.astype(np.float64), x)
    net.set_data(x, y)
    loss, g = net.loss_grad()
    rloss, rg = O.loss_grad(th.astype(np.float64), x.astype(np.float32).astype(np.float64),
                            y.astype(np.float32).astype(np.float64))
    cos = float(g @ rg / (np.linalg.norm(g) * np.linalg.norm(rg)))
    print(f"bf16={bf16} n={n}: out {rel_l2(out, ref):.2e} loss {abs(loss - rloss) / rloss:.2e} "
          f"grad {rel_l2(g, rg):.2e} cos {cos:.6f}")
    if bf16:
        assert rel_l2(out, ref) < 2e-2
        assert abs(loss - rloss) / rloss < 2e-2
        assert rel_l2(g, rg) < 5e-2 and cos > 0.998
    else:
        assert rel_l2(out, ref) < 1e-5
        assert abs(loss - rloss) / rloss < 1e-5
        assert rel_l2(g, rg) < 1e-4
    net.close()


@pytest.mark.gpu
def test_one_adam_step_matches_the_update_rule():
    from lbm_solver_3d_b200.mlp import MLP
    x, y = problem(300, 4)
    th = O.init_params(9).astype(np.float32)
    net = MLP(bf16=False, params=th)
    net.set_data(x, y)
    lr = 1e-3
    net.train_epoch(np.arange(300), batch=300, lr=lr)
    new = net.params().astype(np.float64)
    _, g = O.loss_grad(th.astype(np.float64), x.astype(np.float32), y.astype(np.float32))
    # first Adam step: m = 0.1 g, v = 0.001 g^2, bias-corrected -> lr * g / (|g| + eps)
    want = th - lr * g / (np.abs(g) + 1e-8)
    big = np.abs(g) > 1e-5
    assert np.allclose(new[big], want[big], rtol=0, atol=lr * 1e-2)
    assert np.all(np.abs(new - th) <= lr * 1.0001)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("bf16", [False, True])
def test_training_fits_a_smooth_map(bf16):
    from lbm_solver_3d_b200.mlp import MLP
    x, y = problem(4096, 2)
    xt, yt = problem(1024, 3)
    net = MLP(bf16=bf16, seed=1)
    net.set_data(x, y)
    rng = np.random.default_rng(0)
    l0 = net.loss_grad()[0]
    for ep in range(150):
        net.train_epoch(rng.permutation(len(x)), batch=256, lr=3e-3 if ep < 100 else 1e-3)
    l1 = net.loss_grad()[0]
    test = float(np.mean((net.forward(xt) - yt) ** 2))
    print(f"bf16={bf16}: loss {l0:.3e} -> {l1:.3e}, held-out {test:.3e}")
    assert l1 < 2e-3 * l0 and test < 5e-3
    net.close()


@pytest.mark.gpu
def test_training_is_deterministic():
    from lbm_solver_3d_b200.mlp import MLP
    x, y = problem(777, 8)
    outs = []
    for _ in range(2):
        net = MLP(bf16=True, seed=4)
        net.set_data(x, y)
        for ep in range(3):
            net.train_epoch(np.random.default_rng(ep).permutation(777), batch=100, lr=1e-3)
        outs.append(net.params())
        net.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 128, 1001])
def test_tensor_memory_forward(n):
    """BF16 inference through tcgen05.mma / tensor memory (128 samples per CTA)
    against the warp-tiled mma.sync path (same BF16 rounding points, FP32
    accumulation in another order: within 1e-3) and the float64 oracle
    (within the BF16 tolerance, 2e-2)."""
    from lbm_solver_3d_b200.mlp import MLP
    from lbm_solver_3d_b200._lib import LbmgpuError
    x, _ = problem(n, 30 + n)
    th = O.init_params(11).astype(np.float32)
    net = MLP(bf16=True, params=th)
    tc = net.forward(x, path=MLP.PATH_TCGEN05)
    warp = net.forward(x, path=MLP.PATH_WARP)
    auto = net.forward(x)
    ref = O.forward(th.astype(np.float64), x)
    print(f"n={n}: tcgen05 vs warp {rel_l2(tc, warp):.2e}, vs oracle {rel_l2(tc, ref):.2e}")
    assert np.array_equal(auto, tc)
    assert rel_l2(tc, warp) < 1e-3
    assert rel_l2(tc, ref) < 2e-2
    net.close()
    f32 = MLP(bf16=False, params=th)
    with pytest.raises(LbmgpuError, match="BF16"):
        f32.forward(x, path=MLP.PATH_TCGEN05)
    f32.close()
