"""Learned-predictor network on the tensor cores vs the CPU oracle (oracle/mlp_ref.py)."""
import numpy as np
import pytest

from oracle import mlp_ref


def random_params(n_in, n_out, seed=0):
    rng = np.random.default_rng(seed)
    return {
        "W1": (rng.standard_normal((n_in, 128)) / np.sqrt(n_in)).astype(np.float32),
        "b1": (0.1 * rng.standard_normal(128)).astype(np.float32),
        "W2": (rng.standard_normal((128, 128)) / np.sqrt(128)).astype(np.float32),
        "b2": (0.1 * rng.standard_normal(128)).astype(np.float32),
        "W3": (rng.standard_normal((128, n_out)) / np.sqrt(128)).astype(np.float32),
        "b3": (0.1 * rng.standard_normal(n_out)).astype(np.float32),
    }


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.14159, 1.001953125], dtype=np.float32)
    b = mlp_ref.bf16(x)
    # halfway cases go to the even mantissa: 1 + 2^-8 -> 1, 1 + 3 * 2^-8 -> 1 + 2^-6
    assert b[0] == 1.0 and b[1] == 1.0 and b[2] == 1.015625 and b[4] == 1.0
    assert abs(b[3] + 3.140625) < 1e-6


def test_oracle_gradients_match_finite_differences():
    """The oracle's backward pass is the derivative of its forward pass (without the bf16
    roundings, which a finite difference cannot see, the two agree closely)."""
    rng = np.random.default_rng(1)
    p = random_params(7, 3, seed=2)
    x = rng.standard_normal((64, 7)).astype(np.float32)
    t = rng.standard_normal((64, 3)).astype(np.float32)
    orig = mlp_ref.bf16
    try:
        mlp_ref.bf16 = lambda a: np.asarray(a, dtype=np.float32)
        _, g = mlp_ref.loss_and_grads(p, x, t)
        for k, idx in (("W1", (2, 5)), ("W2", (7, 9)), ("W3", (4, 1)), ("b1", (3,)), ("b3", (2,))):
            q = {kk: v.astype(np.float64) for kk, v in p.items()}
            h = 1e-3
            q[k] = q[k].copy()
            q[k][idx] += h
            lp, _ = mlp_ref.loss_and_grads({kk: v.astype(np.float32) for kk, v in q.items()}, x, t)
            q[k][idx] -= 2 * h
            lm, _ = mlp_ref.loss_and_grads({kk: v.astype(np.float32) for kk, v in q.items()}, x, t)
            fd = (lp - lm) / (2 * h)
            # float32 forward passes: the central difference carries ~1e-5 of rounding noise
            assert abs(fd - g[k][idx]) <= 2e-3 * abs(fd) + 5e-5
    finally:
        mlp_ref.bf16 = orig


@pytest.mark.gpu
@pytest.mark.parametrize("n_in,n_out,n", [(29, 3, 300), (41, 6, 300), (48, 16, 128), (5, 1, 1000)])
def test_forward_matches_oracle(gpu_lib, n_in, n_out, n):
    rng = np.random.default_rng(n)
    p = random_params(n_in, n_out, seed=n_in)
    x = rng.standard_normal((n, n_in)).astype(np.float32)
    net = gpu_lib.Mlp(n_in, n_out)
    net.set_params(p)
    y = net.forward(x)
    y_ref, _ = mlp_ref.forward(p, x)
    # bf16 operands, fp32 accumulation in a different order: a few bf16 ulps of the layer inputs
    scale = np.abs(y_ref).max()
    assert np.abs(y - y_ref).max() <= 2e-2 * scale
    assert np.median(np.abs(y - y_ref)) <= 2e-3 * scale
    back = net.get_params()
    for k in p:
        assert np.array_equal(back[k], p[k])
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n_in,n_out,n", [(29, 3, 500), (41, 6, 300), (48, 16, 256)])
def test_gradients_match_oracle(gpu_lib, n_in, n_out, n):
    """The tensor-core backward pass against the oracle's (same bf16 operand roundings): the
    loss and every parameter gradient."""
    rng = np.random.default_rng(7 + n)
    p = random_params(n_in, n_out, seed=3)
    x = rng.standard_normal((n, n_in)).astype(np.float32)
    t = rng.standard_normal((n, n_out)).astype(np.float32)
    net = gpu_lib.Mlp(n_in, n_out)
    net.set_params(p)
    loss, g = net.loss_grad(x, t)
    loss_ref, g_ref = mlp_ref.loss_and_grads(p, x, t)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    for k in g_ref:
        scale = np.abs(g_ref[k]).max()
        err = np.abs(g[k] - g_ref[k])
        assert err.max() <= 5e-2 * scale, k
        assert np.median(err) <= 5e-3 * scale, k
    net.close()


@pytest.mark.gpu
def test_adam_step_matches_oracle(gpu_lib):
    """One full-batch Adam step on the GPU against the oracle's step from the GPU gradient."""
    rng = np.random.default_rng(5)
    p = random_params(9, 3, seed=4)
    x = rng.standard_normal((200, 9)).astype(np.float32)
    t = rng.standard_normal((200, 3)).astype(np.float32)
    net = gpu_lib.Mlp(9, 3)
    net.set_params(p)
    _loss, g = net.loss_grad(x, t)
    net.train(x, t, epochs=1, batch=200, lr=1e-3, seed=1)
    after = net.get_params()
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(v) for k, v in p.items()}
    ref, _, _ = mlp_ref.adam_step({k: val.copy() for k, val in p.items()}, g, m, v, 1)
    for k in p:
        assert np.abs(after[k] - ref[k]).max() <= 1e-6 + 1e-5 * np.abs(ref[k]).max(), k
    net.close()


@pytest.mark.gpu
def test_training_fits_a_smooth_map(gpu_lib):
    """Training on the GPU lowers the error of a smooth nonlinear map by a large factor."""
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (8192, 6)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2], np.tanh(x[:, 3] - x[:, 4])], 1).astype(np.float32)
    net = gpu_lib.Mlp(6, 2)
    net.set_params(random_params(6, 2, seed=12))
    loss0, _ = net.loss_grad(x, t)
    loss = net.train(x, t, epochs=40, batch=1024, lr=3e-3, seed=2)
    loss1, _ = net.loss_grad(x, t)
    assert loss1 < 0.05 * loss0
    net.close()
