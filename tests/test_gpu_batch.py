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


@pytest.mark.parametrize("cpb", [8, 16, 32])
def test_tiled_ring_blocks_match_per_ring_kernel(cpb):
    """The tiled batched ring kernel (each line once per control point and 128-ring tile) gives
    the body matrices and implicit blocks of the per-ring kernel (each ring's own segments) to
    rounding; two calls in a row agree bit for bit."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.workloads import batch_wings

    cases = batch_wings(n_cases=9, seed=2, steps=6, p_min=64, p_max=1500)
    eng = BatchEngine(cases, solve_tol=1e-13, max_iter=10, tile={"sweep": (128, 1), "ring": cpb})
    eng.start(0.0)
    for _ in range(3):
        eng.step()
    torch.cuda.synchronize()
    d = eng.d_body
    for which, segs, off, sl, n_lines, out in (
            ("body", eng.seg_body, d["offsets"], d["surface_lines"], eng.body.n_lines, eng.A),
            ("implicit", eng.seg_wake, eng.d_row0["offsets"], eng.d_row0["lines"], eng.wake_mesh.n_lines,
             eng.implicit)):
        eng._ring(which, segs, off, sl, n_lines, out)
        tiled = out.clone()
        eng._ring(which, segs, off, sl, n_lines, out)
        assert torch.equal(out, tiled)
        jobs, items, n_items = eng.ring_tables[which]
        ref = torch.full_like(out, float("nan"))
        if cpb in (8, 16):  # the per-ring kernel's tiles use the same item layout
            _lib.call("pvl_batch_ring_matrix", cpb, ptr(jobs), ptr(items), eng.B, n_items, ptr(eng.counter),
                      ptr(off), ptr(sl), n_lines, ptr(segs), ptr(eng.cps), ptr(eng.nrm), eng.tol, ptr(ref), 0,
                      stream_ptr())
            torch.cuda.synchronize()
            scale = float(ref.abs().max())
            err = float((tiled - ref).abs().max()) / scale
            assert err <= 1e-13, (which, err)


def test_implicit_fold_in_ring_kernel_matches_fold_kernel():
    """Folding the implicit wake blocks inside the tiled ring kernel gives, bit for bit, the
    matrices of the implicit block stored first and folded by pvl_batch_fold_implicit."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.workloads import batch_wings

    cases = batch_wings(n_cases=9, seed=4, steps=6, p_min=64, p_max=1500)
    eng = BatchEngine(cases, solve_tol=1e-13, max_iter=10)
    assert eng.fold_in_ring
    eng.start(0.0)
    for _ in range(3):
        eng.step()
    torch.cuda.synchronize()
    d = eng.d_body
    body = lambda: eng._ring("body", eng.seg_body, d["offsets"], d["surface_lines"], eng.body.n_lines, eng.A)
    row0 = (eng.d_row0["offsets"], eng.d_row0["lines"], eng.wake_mesh.n_lines)
    body()
    eng._ring("implicit_fold", eng.seg_wake, *row0, eng.A)
    fused = eng.A.clone()
    body()
    eng._ring("implicit", eng.seg_wake, *row0, eng.implicit)
    _lib.call("pvl_batch_fold_implicit", ptr(eng.wake_cases), ptr(eng.row_case), eng.n_rings, ptr(eng.implicit),
              ptr(eng.adj), ptr(eng.A), stream_ptr())
    torch.cuda.synchronize()
    assert torch.equal(fused, eng.A)
    assert float(eng.implicit.abs().max()) > 0.0
