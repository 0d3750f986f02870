"""Learned warm start for the mixed solve of deforming meshes.

A per-panel MLP (12 -> 128 -> 128 -> 1, BF16 weights and activations, FP32 accumulation; kernels
in csrc/mlp.cu) predicts this step's circulation from local inputs of the new system and the
circulation history.  Its prediction seeds GMRES (MixedSolverEngine.solve_mixed, x0); GMRES and,
when it misses its tolerance, the FP64 factorisation still decide the answer, so the network
changes the cost of a step, never its result beyond the solver tolerance.

What the network predicts: with g0 the previous circulation and r = b - A g0 the residual of
the new system, base = g0 + r / diag(A) is one Jacobi correction; the network predicts
(gamma_new - base) / (out_scale s) with s = ||r|| / sqrt(n) the step's own scale.  Training pairs come from steps of the plain FP64 engine
(``collect``); training runs on the GPU with the hand-written gradient and Adam kernels
(``train``).  Nothing here has a counterpart in the reference, which solves every step from
scratch (python/pyvl/solver.py:223-227).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import ptr, stream_ptr

N_IN = 12
N_H = 128


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights and zero biases, flat in the device layout (W1, b1, W2, b2, w3, b3)."""
    rng = np.random.default_rng(seed)
    parts = [
        rng.uniform(-1, 1, (N_H, N_IN)) * np.sqrt(6.0 / N_IN), np.zeros(N_H),
        rng.uniform(-1, 1, (N_H, N_H)) * np.sqrt(6.0 / N_H), np.zeros(N_H),
        rng.uniform(-1, 1, N_H) * np.sqrt(3.0 / N_H), np.zeros(1),
    ]
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


class WarmStartMLP:
    """Parameters, input statistics and the device kernels of the warm-start network."""

    def __init__(self, device, seed: int = 0):
        self.dev = device
        n = int(_lib.lib().pvl_mlp_param_count())
        assert int(_lib.lib().pvl_mlp_input_count()) == N_IN
        self.n_params = n
        p0 = init_params(seed)
        assert p0.size == n
        self.params = torch.as_tensor(p0, device=device)
        self.params_bf16 = torch.empty(n, dtype=torch.bfloat16, device=device)
        self.m = torch.zeros(n, dtype=torch.float32, device=device)
        self.v = torch.zeros(n, dtype=torch.float32, device=device)
        self.grad = torch.zeros(n, dtype=torch.float32, device=device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step_count = 0
        self.mean = torch.zeros(N_IN, dtype=torch.float32, device=device)
        self.inv_std = torch.ones(N_IN, dtype=torch.float32, device=device)
        self.out_scale = 1.0
        self.n_ctas = 148
        nb = int(_lib.query("pvl_mlp_train_workspace", self.n_ctas))
        self.ws = torch.empty(nb, dtype=torch.uint8, device=device)
        _lib.call("pvl_mlp_to_bf16", ptr(self.params), ptr(self.params_bf16), stream_ptr())
        self.history: list[float] = []

    # ------------------------------------------------------------------ statistics
    def fit_statistics(self, X_raw: torch.Tensor, targets_raw: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """Input mean / inverse std and the output scale from raw training data; returns the
        normalised inputs and targets."""
        Xh = X_raw.double().cpu().numpy()
        mu = Xh.mean(axis=0)
        sd = Xh.std(axis=0)
        inv = np.where(sd > 1e-30, 1.0 / np.maximum(sd, 1e-30), 1.0)
        self.mean.copy_(torch.as_tensor(mu.astype(np.float32)))
        self.inv_std.copy_(torch.as_tensor(inv.astype(np.float32)))
        th = targets_raw.double().cpu().numpy()
        self.out_scale = float(max(th.std(), 1e-300))
        X = torch.as_tensor(((Xh - mu) * inv).astype(np.float32), device=self.dev)
        T = torch.as_tensor((th / self.out_scale).astype(np.float32), device=self.dev)
        return X, T

    # ------------------------------------------------------------------ training
    def gradient(self, X: torch.Tensor, T: torch.Tensor) -> None:
        n = int(X.shape[0])
        _lib.call("pvl_mlp_gradient", n, ptr(X), ptr(T), ptr(self.params_bf16), self.n_ctas, ptr(self.grad),
                  ptr(self.loss), ptr(self.ws), self.ws.numel(), stream_ptr())

    def train(self, X: torch.Tensor, T: torch.Tensor, iters: int = 400, batch: int = 16384, lr: float = 2e-3,
              seed: int = 0) -> list[float]:
        """Adam on mini-batches (contiguous windows at seeded offsets of the shuffled data)."""
        n = int(X.shape[0])
        rng = np.random.default_rng(seed)
        perm = torch.as_tensor(rng.permutation(n), device=self.dev)
        Xs, Ts = X[perm].contiguous(), T[perm].contiguous()
        batch = min(batch, n)
        losses = []
        for it in range(iters):
            o = int(rng.integers(0, n - batch + 1))
            xb, tb = Xs[o:o + batch], Ts[o:o + batch]
            self.gradient(xb, tb)
            self.step_count += 1
            lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * it / iters))  # cosine decay
            _lib.call("pvl_mlp_adam", ptr(self.params), ptr(self.params_bf16), ptr(self.grad), ptr(self.m),
                      ptr(self.v), self.step_count, float(lr_t), 0.9, 0.999, 1e-8, stream_ptr())
            if it % 50 == 0 or it == iters - 1:
                losses.append(float(self.loss.item()))
        self.history += losses
        return losses

    # ------------------------------------------------------------------ inference
    def predict(self, X: torch.Tensor, base: torch.Tensor, out: torch.Tensor, step_scale=None) -> None:
        """out = base + out_scale * s * mlp(X), s = step_scale[0] (device) or 1."""
        _lib.call("pvl_mlp_forward", int(X.shape[0]), ptr(X), ptr(self.params_bf16), float(self.out_scale),
                  ptr(step_scale) if step_scale is not None else None, ptr(base), ptr(out), stream_ptr())


class WarmStart:
    """Per-engine state of the learned warm start: circulation and RHS history, inputs, seed.

    ``prepare()`` runs after the step's assembly and before its solve and returns the seed
    (``None`` until three steps of history exist, or when no network is attached);
    ``finish()`` runs after the solve and rotates the history.  With ``record=True`` the raw
    inputs and targets of every step are kept for training (``training_data``).  Open meshes
    only (the inputs are per panel; a bordered closed-body system keeps its multipliers).

    The base the network corrects is one Jacobi correction of the circulation extrapolated
    from the last steps by the polynomial of degree ``extrapolate`` (at most 4, and at most
    the history there is; 0: the last circulation), which assumes equal time steps: on the
    flapping wing (32 steps per chord) the cubic gives a relative residual of ~1e-8 and, after
    the Jacobi correction, ~2e-12, the quartic ~1e-10 and ~4e-14, against 2.7e-3 and 1.4e-6
    from the last circulation (higher degrees amplify the solves' own 1e-12 residuals).  The
    default is the cubic: the network then still has a remainder worth predicting (7e-13 after
    it); on the quartic base its correction no longer helps (2e-14 against 3.5e-14 at the
    benchmark, worse than the Jacobi seed alone on a short 64 x 16 run).
    """

    _EXTRAPOLATION = {0: (1.0,), 1: (2.0, -1.0), 2: (3.0, -3.0, 1.0), 3: (4.0, -6.0, 4.0, -1.0),
                      4: (5.0, -10.0, 10.0, -5.0, 1.0)}

    def __init__(self, engine, mlp: WarmStartMLP | None = None, record: bool = False, jacobi: bool = False,
                 extrapolate: int = 3):
        if getattr(engine, "m", 0):
            raise ValueError("the learned warm start is for open meshes")
        if jacobi and (mlp is not None or record):
            raise ValueError("jacobi=True is the seed without a network")
        self.eng = engine
        self.mlp = mlp
        self.jacobi = bool(jacobi)  # seed with the Jacobi correction alone (the method without the network)
        if int(extrapolate) not in self._EXTRAPOLATION:
            raise ValueError("extrapolate must be 0, 1, 2, 3 or 4")
        self.order = int(extrapolate)
        P, dev = engine.P, engine.dev
        f64 = dict(dtype=torch.float64, device=dev)
        self.hist = [torch.zeros(P, **f64) for _ in range(5)]  # g0 (last step), g1, ..., g4
        self.gext = torch.zeros(P, **f64)  # the extrapolated circulation
        self.rem = [torch.zeros(P, **f64) for _ in range(2)]   # gamma - base of the last two steps
        self.rhs_prev = torch.zeros(P, **f64)
        self.rhs_cur = torch.zeros(P, **f64)
        self.resid = torch.zeros(P, **f64)
        self.rnorm = torch.zeros(1, **f64)
        self.step_scale = torch.zeros(1, **f64)
        self.X = torch.zeros((P, N_IN), dtype=torch.float32, device=dev)
        self.base = torch.zeros(P, **f64)
        self.seed = torch.zeros(P, **f64)
        self.raw_mean = torch.zeros(N_IN, dtype=torch.float32, device=dev)
        self.raw_inv = torch.ones(N_IN, dtype=torch.float32, device=dev)
        self.n_hist = 0
        self.ready = False
        self.have_base = False
        self.record = record
        self._graphs: dict = {}  # captured prepare / finish pieces (SolverEngine.captured)
        self.rec_X: list[torch.Tensor] = []
        self.rec_target: list[torch.Tensor] = []
        if mlp is not None and not record:
            # One inference on the (zero) buffers now: the forward kernel and the scaling are first
            # needed only once three steps of history exist, and a kernel's first launch in a
            # process loads its code (milliseconds) -- that belongs to the set-up, not to a step.
            torch.mul(self.rnorm, 1.0, out=self.step_scale)
            self.mlp.predict(self.X, self.base, self.seed, self.step_scale)

    def prepare(self) -> torch.Tensor | None:
        eng = self.eng
        self.have_base = self.n_hist >= 1
        self.ready = self.n_hist >= 3  # g1, rem0 and rem1 hold real history
        infer = self.have_base and self.mlp is not None and not self.record and self.ready
        order = min(self.order, self.n_hist - 1) if self.have_base else 0
        run = lambda: self._prepare_ops(self.have_base, infer, order)
        if self.record:
            run()
        else:  # fixed buffers: one captured graph per state (engine.captured)
            scale = self.mlp.out_scale if infer else 0.0  # a host value the graph keeps
            eng.captured(("prepare", self.have_base, infer, scale, order), run, self._graphs)
        if self.jacobi and self.have_base:
            return self.base
        return self.seed if infer else None

    def _prepare_ops(self, have_base: bool, infer: bool, order: int) -> None:
        eng = self.eng
        P = eng.P
        self.rhs_cur.copy_(eng.rhs[:P])
        if not have_base:
            return
        s = stream_ptr()
        g1 = self.hist[1]
        g0 = self.hist[0]
        if order:
            w = self._EXTRAPOLATION[order]
            torch.mul(self.hist[0], w[0], out=self.gext)
            for c, g in zip(w[1:], self.hist[1:]):
                self.gext.add_(g, alpha=c)
            g0 = self.gext
        self.resid.copy_(self.rhs_cur)
        _lib.call("pvl_gemv_f64", P, P, -1.0, ptr(eng.A), eng.N, ptr(g0), 1.0, ptr(self.resid), s)
        _lib.call("pvl_normalize", P, ptr(self.resid), None, ptr(self.rnorm), s)
        mean, inv = (self.mlp.mean, self.mlp.inv_std) if self.mlp is not None and not self.record else \
            (self.raw_mean, self.raw_inv)  # (the Jacobi seed uses base only; X is not read)
        _lib.call("pvl_mlp_features", P, ptr(g0), ptr(g1), ptr(self.rem[0]), ptr(self.rem[1]), ptr(self.resid),
                  ptr(self.rnorm), ptr(eng.A), eng.N, ptr(self.rhs_cur), ptr(self.rhs_prev), ptr(eng.nrm), ptr(eng.cpv),
                  ptr(mean), ptr(inv), ptr(self.X), ptr(self.base), s)
        if infer:
            torch.mul(self.rnorm, 1.0 / float(np.sqrt(P)), out=self.step_scale)
            self.mlp.predict(self.X, self.base, self.seed, self.step_scale)

    def finish(self) -> None:
        eng = self.eng
        if self.record and self.ready:
            s = torch.clamp(self.rnorm / float(np.sqrt(eng.P)), min=1e-300)
            self.rec_X.append(self.X.clone())
            self.rec_target.append((eng.gamma - self.base) / s)
        have_base = self.have_base
        run = lambda: self._finish_ops(have_base)
        if self.record:
            run()
        else:
            eng.captured(("finish", have_base), run, self._graphs)
        self.n_hist += 1

    def _finish_ops(self, have_base: bool) -> None:
        eng = self.eng
        r0, r1 = self.rem
        r1.copy_(r0)
        if have_base:
            torch.sub(eng.gamma, self.base, out=r0)
        else:
            r0.zero_()
        for older, newer in zip(self.hist[:0:-1], self.hist[-2::-1]):  # g4 <- g3, ..., g1 <- g0
            older.copy_(newer)
        self.hist[0].copy_(eng.gamma)
        self.rhs_prev.copy_(self.rhs_cur)

    def training_data(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Raw inputs (n, 12) and raw targets gamma - base (n,) of the recorded steps."""
        return torch.cat(self.rec_X), torch.cat(self.rec_target)


def drive_step(engine, warm: WarmStart | None, time: float, positions, velocities) -> None:
    """One step of a SolverEngine / MixedSolverEngine with the warm start around its solve."""
    engine.load_inputs(positions, velocities)
    engine.assemble()
    x0 = warm.prepare() if warm is not None else None
    if x0 is not None and hasattr(engine, "solve_mixed"):
        engine.solve(x0)
    else:
        engine.solve()
    if warm is not None:
        warm.finish()
    if engine.wake is not None:
        engine.wake_update(time)
    engine.iteration += 1


def collect(engine, case, times) -> tuple[torch.Tensor, torch.Tensor]:
    """Run ``engine`` (normally the plain FP64 SolverEngine) over ``times`` of a workload and
    return the raw inputs and targets of every step with three steps of history."""
    warm = WarmStart(engine, None, record=True)
    for t in times:
        drive_step(engine, warm, t, case.positions_at(t), case.velocities_at(t))
    return warm.training_data()
