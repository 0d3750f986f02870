"""Failure reporting on the device, without a GPU fault: a bounded wait that runs out.

The wavefront triangular solve of pvl_lu_solve waits for earlier row blocks through flags in
global memory; every wait has a poll limit after which the block sets an error word,
publishes its own flag and returns.  The probe library launches the same kernel with a short
limit and one block that never publishes, so every later block's wait runs out: the launch
must return, the error word must be set, and the engine must turn it into PVL_ERR_TIMEOUT.
No kernel is left running and the context stays usable (a normal solve follows)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        raise AssertionError("GPU tests need CUDA")
    return torch


def _identity_system(torch, n):
    nblk = (n + 63) // 64
    LU = torch.eye(n, dtype=torch.float64, device="cuda")
    inv = torch.eye(64, dtype=torch.float64, device="cuda").repeat(nblk * 2, 1, 1).contiguous()
    flags = torch.zeros(nblk + 1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    return LU, inv, flags, err


@pytest.mark.parametrize("lower", [1, 0])
def test_wavefront_wait_runs_out_and_sets_the_error_word(torch_cuda, lower):
    torch = torch_cuda
    from pyvl_b200 import _probe
    from pyvl_b200.device import ptr, stream_ptr

    n, skip = 512, 3  # 8 row blocks; block 3 never publishes
    LU, inv, flags, err = _identity_system(torch, n)
    x = torch.arange(1, n + 1, dtype=torch.float64, device="cuda")
    _probe.call("pvl_probe_trsv_timeout", n, ptr(LU), n, ptr(inv), ptr(x), ptr(flags), ptr(err), 2000, skip, lower,
                stream_ptr())
    torch.cuda.synchronize()  # returns: every wait is bounded
    assert int(err.item()) == 1
    # the blocks solved before the missing one (identity factors: x unchanged) published
    done = range(skip) if lower else range(skip + 1, n // 64)
    assert all(int(flags[b].item()) == 1 for b in done)
    assert int(flags[skip].item()) == 0
    # the same kernel with nothing skipped: no error, identity factors leave x as it was
    x.copy_(torch.arange(1, n + 1, dtype=torch.float64, device="cuda"))
    _probe.call("pvl_probe_trsv_timeout", n, ptr(LU), n, ptr(inv), ptr(x), ptr(flags), ptr(err), 2000, -1, lower,
                stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(x, torch.arange(1, n + 1, dtype=torch.float64, device="cuda"))


def test_timed_out_solve_surfaces_as_pvl_err_timeout(torch_cuda):
    """The engine's solve status word, written by a timed-out wavefront pass, raises
    PVL_ERR_TIMEOUT from check_status; the next regular step clears it."""
    torch = torch_cuda
    from pyvl_b200 import _lib, _probe
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.engine import SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flat_wing

    case = flat_wing(nt=3, line_rows=3)
    mesh = Mesh(case.n_points, case.elements)
    eng = SolverEngine(mesh, case.freestream, case.tol, wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows,
                                                                          case.t0))
    eng.step(0.0, case.positions_at(0.0), case.velocities_at(0.0))
    eng.check_status()
    n = 128
    LU, inv, flags, _ = _identity_system(torch, n)
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    _probe.call("pvl_probe_trsv_timeout", n, ptr(LU), n, ptr(inv), ptr(x), ptr(flags), ptr(eng.err), 1000, 0, 1,
                stream_ptr())
    with pytest.raises(_lib.PvlError) as e:
        eng.check_status()
    assert e.value.code == _lib.PVL_ERR_TIMEOUT
    t = case.dt
    eng.step(t, case.positions_at(t), case.velocities_at(t))  # the context is still usable
    eng.check_status()
    assert np.all(np.isfinite(eng.gamma_host()))


def _flat_engine(kind="plain"):
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flat_wing

    case = flat_wing(nt=4, line_rows=4)
    mesh = Mesh(case.n_points, case.elements)
    spec = wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)
    cls = SolverEngine if kind == "plain" else MixedSolverEngine
    return case, cls(mesh, case.freestream, case.tol, spec)


@pytest.mark.parametrize("kind", ["plain", "mixed"])
def test_nan_input_surfaces_as_an_error_status(torch_cuda, kind):
    """A NaN in a node position or velocity reaches the right-hand side, whose kernel sets the
    engine's sticky status word; check_status raises PVL_ERR_NONFINITE and clears it."""
    from pyvl_b200 import _lib

    case, eng = _flat_engine(kind)
    eng.step(0.0, case.positions_at(0.0), case.velocities_at(0.0))
    eng.check_status()
    t = case.dt
    vel = case.velocities_at(t)
    vel[7, 2] = np.nan
    eng.step(t, case.positions_at(t), vel)
    with pytest.raises(_lib.PvlError) as e:
        eng.check_status()
    assert e.value.code == _lib.PVL_ERR_NONFINITE
    eng.check_status()  # read and cleared
    case, eng = _flat_engine(kind)
    pos = case.positions_at(0.0)
    pos[3, 0] = np.inf
    eng.step(0.0, pos, case.velocities_at(0.0))
    with pytest.raises(_lib.PvlError):
        eng.check_status()


def test_failed_preconditioner_rebuild_is_not_adopted(torch_cuda):
    """A rebuild whose FP32 factorisation meets an exactly zero pivot (a system that is
    singular only after rounding to FP32) is counted and dropped: synchronously, the step
    solves by the FP64 LU; on the side stream, the previous inverse stays in use."""
    torch = torch_cuda
    case, eng = _flat_engine("mixed")
    eng.step(0.0, case.positions_at(0.0), case.velocities_at(0.0))
    good = eng.Xinv.clone()
    n = eng.N
    bad = torch.eye(n, dtype=torch.float64, device="cuda")
    bad[0, 1], bad[1, 0], bad[1, 1] = 1.0, 1.0, 1.0 + 1e-9  # rounds to a singular 2 x 2 block in FP32
    # on the side stream: the failed rebuild is dropped when adopted
    eng.A.copy_(bad)
    eng.refresh_preconditioner(wait=False)
    eng.wait_refresh()
    assert eng.stats["refresh_failures"] == 1
    assert torch.equal(eng.Xinv, good)
    # synchronously: no usable preconditioner, the next solve takes the FP64 LU
    eng.A.copy_(bad)
    eng.refresh_preconditioner(wait=True)
    assert eng.stats["refresh_failures"] == 2 and not eng.have_precond
    f0 = eng.stats["fallbacks"]
    t = case.dt
    eng.step(t, case.positions_at(t), case.velocities_at(t))
    assert eng.stats["fallbacks"] == f0 + 1
    eng.check_status()
    ref_case, ref = _flat_engine("plain")
    ref.step(0.0, case.positions_at(0.0), case.velocities_at(0.0))
    ref.step(t, case.positions_at(t), case.velocities_at(t))
    g, r = eng.gamma_host(), ref.gamma_host()
    assert np.linalg.norm(g - r) <= 1e-12 * np.linalg.norm(r)
