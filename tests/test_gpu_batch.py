"""Batched stepping (pyvl_b200/batch.py, csrc/batch.cu) against a per-case loop of the
single-case FP64 engine.  Needs a B200."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _per_case(case, steps):
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import SolverEngine, wake_spec_from_te

    mesh = Mesh(case.n_points, case.elements)
    eng = SolverEngine(mesh, case.freestream, case.tol, wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows,
                                                                          case.t0))
    out = []
    for it in range(steps):
        t = it * case.dt
        eng.step(t, case.positions_at(t), case.velocities_at(t))
        out.append(eng.gamma_host())
    eng.check_status()
    return np.array(out), eng.wake_positions.cpu().numpy()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("capture", [False, True])
def test_batch_matches_per_case_loop(capture):
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.workloads import batch_wings

    steps = 8
    cases = batch_wings(n_cases=6, seed=5, steps=steps, p_min=64, p_max=400)
    eng = BatchEngine(cases, solve_tol=1e-13, max_iter=10)
    eng.start(0.0)
    hist = []
    for it in range(steps):
        eng.step()
        if capture and it == 1:
            eng.capture()
        hist.append([eng.gamma_of(k) for k in range(len(cases))])
    assert eng.failures() == 0
    for k, case in enumerate(cases):
        ref, ref_wake = _per_case(case, steps)
        for it in range(steps):
            assert rel(hist[it][k], ref[it]) <= 1e-11, (k, it, rel(hist[it][k], ref[it]))
        w = eng.wake_positions_of(k)
        assert np.abs(w - ref_wake).max() <= 1e-11 * max(1.0, np.abs(ref_wake).max())


def test_batch_graph_replay_is_bitwise_identical_and_tuning_keeps_results():
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.workloads import batch_wings

    steps = 6
    cases = batch_wings(n_cases=5, seed=9, steps=steps, p_min=100, p_max=700)
    a = BatchEngine(cases, solve_tol=1e-13, max_iter=10)
    b = BatchEngine(cases, solve_tol=1e-13, max_iter=10)
    c = BatchEngine(cases, solve_tol=1e-13, max_iter=10, reuse_static_bodies=True)
    for e in (a, b, c):
        e.start(0.0)
    for it in range(steps):
        a.step()
        b.step()
        c.step()
        if it == 0:
            b.capture()
            c.capture()
    for k in range(len(cases)):
        assert np.array_equal(a.gamma_of(k), b.gamma_of(k))
        assert np.array_equal(a.gamma_of(k), c.gamma_of(k))  # the reused matrix is the same matrix
    rep = a.tune(reps=1)
    assert rep["chosen"]["ring"] in (4, 8, 16)
    assert a.failures() == 0 and b.failures() == 0 and c.failures() == 0
