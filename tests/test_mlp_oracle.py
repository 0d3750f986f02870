"""The warm-start network's CPU oracle (oracle/mlp.py): BF16 rounding pinned to torch's
bfloat16 conversion, backpropagation pinned to finite differences.  No GPU."""

import numpy as np


def test_bf16_rounding_matches_torch():
    import torch

    from oracle.mlp import bf16

    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(5000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 5000),
                        np.array([0.0, -0.0, 1.0, 65504.0, 1e-38, 3.0e38], np.float32)]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(bf16(x), want)


def test_backprop_matches_finite_differences():
    from oracle.mlp import N_IN, N_PARAMS, init_params, loss_and_grad_exact

    rng = np.random.default_rng(1)
    p = init_params(3).astype(np.float64) + 0.01 * rng.standard_normal(N_PARAMS)
    x = rng.standard_normal((64, N_IN))
    t = rng.standard_normal(64)
    _, g = loss_and_grad_exact(p, x, t)
    idx = rng.choice(N_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(N_PARAMS)
        e[i] = h
        fd = (loss_and_grad_exact(p + e, x, t)[0] - loss_and_grad_exact(p - e, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_network_gradient_close_to_exact():
    """The BF16 forward/backward of the oracle stays within BF16 rounding of the exact one."""
    from oracle.mlp import N_IN, init_params, loss_and_grad, loss_and_grad_exact

    rng = np.random.default_rng(2)
    p = init_params(4)
    x = rng.standard_normal((512, N_IN)).astype(np.float32)
    t = rng.standard_normal(512)
    l1, g1 = loss_and_grad(p, x, t)
    l2, g2 = loss_and_grad_exact(p.astype(np.float64), x.astype(np.float64), t)
    assert abs(l1 - l2) <= 2e-2 * l2
    assert np.linalg.norm(g1 - g2) <= 3e-2 * np.linalg.norm(g2)


def test_product_init_matches_oracle_init():
    from oracle.mlp import init_params as oracle_init
    from pyvl_b200.learned import init_params

    assert np.array_equal(init_params(5), oracle_init(5))
