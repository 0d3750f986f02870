"""The learned warm start on the GPU: its hand-written BF16 kernels against the numpy oracle
(oracle/mlp.py), training, and what the trained network gains in the mixed solve."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand_problem(n, seed):
    from oracle.mlp import N_IN, N_PARAMS, init_params

    rng = np.random.default_rng(seed)
    p = (init_params(seed) + 0.05 * rng.standard_normal(N_PARAMS)).astype(np.float32)
    x = rng.standard_normal((n, N_IN)).astype(np.float32)
    t = rng.standard_normal(n).astype(np.float32)
    return p, x, t


def _device_mlp(p):
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.learned import WarmStartMLP

    mlp = WarmStartMLP(torch.device("cuda"))
    mlp.params.copy_(torch.as_tensor(p))
    _lib.call("pvl_mlp_to_bf16", ptr(mlp.params), ptr(mlp.params_bf16), stream_ptr())
    return mlp


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, float) - np.asarray(b, float)) / np.linalg.norm(np.asarray(b, float)))


@pytest.mark.parametrize("n", [1, 31, 1000, 4096])
def test_forward_matches_oracle(n):
    import torch

    from oracle.mlp import forward

    p, x, _ = _rand_problem(n, 1)
    mlp = _device_mlp(p)
    X = torch.as_tensor(x, device="cuda")
    base = torch.full((n,), 0.5, dtype=torch.float64, device="cuda")
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    mlp.out_scale = 2.0
    mlp.predict(X, base, out)
    y, _ = forward(p, x)
    # FP32 sums on the device vs float64 in the oracle, identical BF16 operands
    assert rel(out.cpu().numpy(), 0.5 + 2.0 * y) <= 2e-3


@pytest.mark.parametrize("n", [100, 8192])
def test_gradient_matches_oracle(n):
    import torch

    from oracle.mlp import SIZES, loss_and_grad, unpack

    p, x, t = _rand_problem(n, 2)
    mlp = _device_mlp(p)
    mlp.gradient(torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda"))
    torch.cuda.synchronize()
    loss, g = loss_and_grad(p, x, t)
    gd = mlp.grad.cpu().numpy().astype(np.float64)
    assert abs(float(mlp.loss.item()) - loss) <= 1e-3 * loss
    gu, du = unpack(g, np.float64), unpack(gd, np.float64)
    for k in SIZES:
        assert rel(du[k], gu[k]) <= 1e-2, (k, rel(du[k], gu[k]))
    assert rel(gd, g) <= 3e-3


def test_adam_matches_oracle():
    import torch

    from oracle.mlp import adam

    p, x, t = _rand_problem(512, 3)
    mlp = _device_mlp(p)
    X, T = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    m = np.zeros(p.size)
    v = np.zeros(p.size)
    w = p.copy()
    for step in range(1, 4):
        mlp.gradient(X, T)
        g = mlp.grad.cpu().numpy().astype(np.float64)
        mlp.step_count = step
        from pyvl_b200 import _lib
        from pyvl_b200.device import ptr, stream_ptr

        _lib.call("pvl_mlp_adam", ptr(mlp.params), ptr(mlp.params_bf16), ptr(mlp.grad), ptr(mlp.m), ptr(mlp.v), step,
                  1e-3, 0.9, 0.999, 1e-8, stream_ptr())
        w, m, v = adam(w, g, m, v, step, 1e-3)
        torch.cuda.synchronize()
        assert np.allclose(mlp.params.cpu().numpy(), w, rtol=1e-5, atol=1e-7)


def test_training_fits_a_smooth_target():
    import torch

    from pyvl_b200.learned import WarmStartMLP

    rng = np.random.default_rng(4)
    x = rng.standard_normal((65536, 12)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * np.abs(x[:, 3])).astype(np.float32)
    mlp = WarmStartMLP(torch.device("cuda"), seed=1)
    X, T = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    losses = mlp.train(X, T, iters=600, batch=8192, lr=3e-3)
    assert losses[-1] < 0.05 * losses[0], losses


def test_warm_start_gain_in_mixed_solve():
    """Trained on plain-engine steps, the network's seed starts GMRES closer to the answer than
    the previous circulation and than one Jacobi correction (the methods without it), and needs
    no more Krylov iterations than either."""
    import torch

    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200.learned import WarmStart, WarmStartMLP, collect, drive_step
    from pyvl_b200.workloads import flapping

    case = flapping(ns=64, nc=16, line_rows=40)
    mesh = Mesh(case.n_points, case.elements)

    def spec():
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    train_t = [i * case.dt for i in range(120)]
    X, T = collect(SolverEngine(mesh, case.freestream, case.tol, spec()), case, train_t)
    mlp = WarmStartMLP(torch.device("cuda"), seed=0)
    Xn, Tn = mlp.fit_statistics(X, T)
    losses = mlp.train(Xn, Tn, iters=800, batch=16384, lr=2e-3)
    assert losses[-1] < 0.2 * losses[0], losses

    test_t = [i * case.dt for i in range(160)]
    results = {}
    for mode in ("previous", "jacobi", "learned"):
        eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec(), refresh=25)
        warm = None
        if mode == "learned":
            warm = WarmStart(eng, mlp)
        elif mode == "jacobi":  # the same seed without the network
            warm = WarmStart(eng, jacobi=True)
        for t in test_t:
            drive_step(eng, warm, t, case.positions_at(t), case.velocities_at(t))
        st = eng.stats
        results[mode] = (float(np.median(st["initial_rel_residual"][125:])), int(np.sum(st["gmres_iters"][125:])),
                         st["fallbacks"])
    print("warm start (median initial residual, GMRES iterations, fallbacks) over steps 125-159:", results)
    assert all(r[2] == 0 for r in results.values())
    assert results["learned"][0] < 0.5 * results["previous"][0]
    assert results["learned"][0] < results["jacobi"][0]
    assert results["learned"][1] <= results["previous"][1]
    assert results["learned"][1] <= results["jacobi"][1]
