"""CPU oracle of the learned warm start's network (test infrastructure only).

The network is the per-panel MLP of the mixed path: 12 inputs -> 128 (ReLU) -> 128 (ReLU) -> 1,
with BF16 weights and BF16 activations and FP32 accumulation, trained by mean squared error.
The reference has no learned component (its solver factorises every step,
python/pyvl/solver.py:223-227); this file restates the numerics of the device kernels in
numpy so that their forward pass and gradients can be checked:

* weights and inputs are rounded to BF16 (round to nearest even) before use;
* h1 = bf16(relu(W1 x + b1)), h2 = bf16(relu(W2 h1 + b2)), y = w3 . h2 + b3 (FP32 sums);
* loss = mean((y - t)^2); backward in FP32 from the BF16 activations and weights.

Parameters are one flat vector: W1 (128 x 12), b1 (128), W2 (128 x 128), b2 (128), w3 (128), b3.
"""

from __future__ import annotations

import numpy as np

N_IN, N_H = 12, 128
SIZES = {"W1": (N_H, N_IN), "b1": (N_H,), "W2": (N_H, N_H), "b2": (N_H,), "w3": (N_H,), "b3": (1,)}
N_PARAMS = sum(int(np.prod(s)) for s in SIZES.values())


def bf16(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(a, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    out = rounded.astype(np.uint32).view(np.float32)
    nan = np.isnan(x)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def unpack(params: np.ndarray, dtype=np.float32) -> dict:
    out, o = {}, 0
    for k, s in SIZES.items():
        n = int(np.prod(s))
        out[k] = np.asarray(params[o:o + n], dtype).reshape(s)
        o += n
    return out


def pack(parts: dict) -> np.ndarray:
    return np.concatenate([np.asarray(parts[k], np.float32).reshape(-1) for k in SIZES])


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases (the device's initialisation uses these values)."""
    rng = np.random.default_rng(seed)
    p = {
        "W1": rng.uniform(-1, 1, SIZES["W1"]) * np.sqrt(6.0 / N_IN),
        "b1": np.zeros(N_H),
        "W2": rng.uniform(-1, 1, SIZES["W2"]) * np.sqrt(6.0 / N_H),
        "b2": np.zeros(N_H),
        "w3": rng.uniform(-1, 1, SIZES["w3"]) * np.sqrt(3.0 / N_H),
        "b3": np.zeros(1),
    }
    return pack(p)


def forward(params: np.ndarray, x: np.ndarray):
    """Returns y and the activations (BF16-rounded, as the device keeps them)."""
    p = {k: bf16(v) for k, v in unpack(params).items()}
    xb = bf16(x).astype(np.float64)
    a1 = xb @ p["W1"].T.astype(np.float64) + p["b1"]
    h1 = bf16(np.maximum(a1, 0.0).astype(np.float32)).astype(np.float64)
    a2 = h1 @ p["W2"].T.astype(np.float64) + p["b2"]
    h2 = bf16(np.maximum(a2, 0.0).astype(np.float32)).astype(np.float64)
    y = h2 @ p["w3"].astype(np.float64) + float(p["b3"][0])
    return y, (xb, h1, h2, p)


def loss_and_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray):
    """Mean squared error and its gradient with respect to the flat parameters."""
    y, (xb, h1, h2, p) = forward(params, x)
    n = x.shape[0]
    r = y - np.asarray(t, np.float64)
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    g = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
    dh2 = np.outer(dy, p["w3"].astype(np.float64)) * (h2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ p["W2"].astype(np.float64)) * (h1 > 0)
    g["W1"] = dh1.T @ xb
    g["b1"] = dh1.sum(axis=0)
    return loss, pack({k: g[k] for k in SIZES}).astype(np.float64)


def loss_and_grad_exact(params: np.ndarray, x: np.ndarray, t: np.ndarray):
    """The same network in float64 without BF16 rounding (for finite-difference checks)."""
    p = unpack(np.asarray(params, np.float64), np.float64)
    a1 = x @ p["W1"].T + p["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(a2, 0.0)
    y = h2 @ p["w3"] + p["b3"][0]
    n = x.shape[0]
    r = y - t
    dy = 2.0 * r / n
    g = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
    dh2 = np.outer(dy, p["w3"]) * (a2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ p["W2"]) * (a1 > 0)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(axis=0)
    return float(np.mean(r * r)), np.concatenate([g[k].reshape(-1) for k in SIZES])


def adam(params, grad, m, v, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One Adam step (Kingma & Ba, 2015) on float32 master parameters."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return (params - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32), m, v
