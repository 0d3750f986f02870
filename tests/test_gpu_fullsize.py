"""Full-size checks on the benchmark workload (flapping 128x32 wing, 4096 rings, a seeded
400-row wake of 51,200 rings): the two segment sweeps against the CPU oracle on seeded samples
of their points, a size-independent property of the sweeps, and judged mixed steps.  Needs a
B200.

The oracle evaluates the reference's ring formulation (wake_models.py:199-223, explicit term =
sum over rows >= 1 of ring induction x ring circulation; wake_models.py:121-126, node velocity
= freestream + body rings' induction x circulation) on the strip-major wake mesh, while the
GPU sweeps run over merged line tables in row-major order: a different summation, the same
sums to <= 1e-12.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def state():
    import torch

    import bench
    from pyvl_b200.engine import SolverEngine

    case = bench.workload()
    mesh, spec, wpos, wcirc, t0 = bench.wake_setup(case)
    eng = SolverEngine(mesh, case.freestream, case.tol, spec)
    eng.set_wake_state(wpos, wcirc, step_count=case.line_rows + 1, time=t0 - case.dt)
    eng.load_inputs(case.positions_at(t0), case.velocities_at(t0))
    eng.assemble_body_only()
    torch.cuda.synchronize()
    return case, mesh, spec, eng


def _wake_term(eng, scale=1.0):
    """Explicit wake term n . v at every control point (FP64 sweep over the merged lines)."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    w = eng.wake
    rm, d = w["rm"], w["rm_d"]
    crs = w["circ_rs"]
    crs.copy_(eng.wake_circulation.t() * scale)
    crs[0].zero_()  # row 0 is the implicit block
    lg = w["rm_line_gamma"]
    s = stream_ptr()
    _lib.call("pvl_line_circulation", rm.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(crs), 0, ptr(lg),
              s)
    out = torch.zeros(eng.P, dtype=torch.float64, device="cuda")
    _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, rm.n_lines, ptr(d["lines"]),
              ptr(eng.wake_positions.reshape(-1, 3)), ptr(lg), eng.P, ptr(eng.cps), ptr(eng.nrm), eng.tol, 1.0, 0.0,
              ptr(out), ptr(eng.ws), eng._ws_bytes, s)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_full_size_wake_term_vs_oracle_sample(state):
    from oracle.kernels import OracleMesh
    from pyvl_b200.engine import wake_ring_connectivity

    case, mesh, spec, eng = state
    got = _wake_term(eng)
    S, R = eng.wake["S"], eng.wake["R"]
    bn = np.asarray(spec.bordering_nodes, np.int64).reshape(S, 2)
    om = OracleMesh(2 * (R + 1) * S, wake_ring_connectivity(R, S, bn))
    sample = np.sort(np.random.default_rng(11).choice(eng.P, 48, replace=False))
    sample[:4] = [0, 31, eng.P - 32, eng.P - 1]  # trailing-edge and tip panels among them
    cps = eng.cps.cpu().numpy()[sample]
    nrm = eng.nrm.cpu().numpy()[sample]
    ind = om.induction_matrix(eng.tol, eng.wake_positions.cpu().numpy().reshape(-1, 3), cps)  # (n, S*R, 3)
    circ = eng.wake_circulation.cpu().numpy().copy()  # (S, R), ring s*R + r
    circ[:, 0] = 0.0
    v = np.einsum("prc,r->pc", ind, circ.reshape(-1))
    want = np.einsum("pc,pc->p", v, nrm)
    assert rel(got[sample], want) <= PARITY
    assert np.abs(got).max() > 0.0


def test_full_size_wake_term_is_linear_in_circulation(state):
    """Doubling every wake circulation doubles the term exactly (powers of two scale every
    product and sum without rounding)."""
    case, mesh, spec, eng = state
    a = _wake_term(eng)
    b = _wake_term(eng, 2.0)
    assert np.array_equal(b, 2.0 * a)


def test_full_size_node_velocity_vs_oracle_sample(state):
    """Wake node velocities (freestream + body induction, FP64 sweep over the distinct node
    columns, every row) against the oracle's ring formulation on a sample of nodes."""
    import torch

    from oracle.kernels import OracleMesh
    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    case, mesh, spec, eng = state
    w = eng.wake
    S, R = w["S"], w["R"]
    gam = np.random.default_rng(5).normal(size=eng.P)
    eng.gamma.copy_(torch.as_tensor(gam, device="cuda"))
    d = eng.d_body
    s = stream_ptr()
    _lib.call("pvl_line_circulation", mesh.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(eng.gamma), 0,
              ptr(eng.body_line_gamma), s)
    u = np.asarray(case.freestream, np.float64)
    _lib.call("pvl_wake_node_velocity_cols", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]),
              ptr(eng.pos), ptr(eng.body_line_gamma), S, R, R, 0, R, w["n_cols"], ptr(w["cols"]),
              ptr(eng.wake_positions), float(u[0]), float(u[1]), float(u[2]), eng.tol, ptr(w["node_vel"]), ptr(eng.ws),
              eng._ws_bytes, s)
    torch.cuda.synchronize()
    vel = w["node_vel"].cpu().numpy()  # (n_cols, R, 3)
    cols = w["cols"].cpu().numpy().view(np.uint32).astype(np.int64)
    wp = eng.wake_positions.cpu().numpy()  # (S, 2, R + 1, 3)
    rng = np.random.default_rng(7)
    ci = rng.integers(0, cols.size, 64)
    ri = rng.integers(0, R, 64)
    ri[:8] = np.arange(8)  # the rows just behind the trailing edge
    nodes = np.array([wp[c // 2, c % 2, r] for c, r in zip(cols[ci], ri)])
    om = OracleMesh(case.n_points, case.elements)
    ind = om.induction_matrix(eng.tol, eng.pos.cpu().numpy(), nodes)  # (n, P, 3)
    want = np.einsum("prc,r->pc", ind, gam) + u
    assert rel(vel[ci, ri], want) <= PARITY


def test_full_size_mixed_steps_judged(state):
    """Four steps of the mixed path (no learned seed) on the benchmark state, each judged
    against the all-FP64 step of the same state."""
    import bench
    from pyvl_b200.engine import MixedSolverEngine

    case, mesh, spec, _ = state
    _, _, wpos, wcirc, t0 = bench.wake_setup(case)
    eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec)
    eng.set_wake_state(wpos, wcirc, step_count=case.line_rows + 1, time=t0 - case.dt)
    eng.iteration = 1
    errs = []
    for k in range(4):
        t = t0 + k * case.dt
        errs.append(eng.step_judged(t, case.positions_at(t), case.velocities_at(t)))
    st = eng.stats
    assert max(errs) <= 1e-10, errs
    assert st["fallbacks"] == 0
