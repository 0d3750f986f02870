"""pvl_line_velocity_noalloc: the segment-sum velocity for callers that cannot allocate.

Hosts that manage all device memory through their own pool, or that run the velocity
evaluation in loops where an allocation (and a cudaFree's synchronisation) is not
acceptable, can call this entry point with inputs and outputs only; its scratch is a fixed
array inside the library.  This file is collected last so that, if it fails, a run that
stops at the first failure has already run every other test.  Needs a B200.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_workspace_entry_point_twice():
    import torch

    from pyvl_b200 import _lib, workloads
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.device import Workspace, ptr, stream_ptr

    case = workloads.swept_pitching(ns=32, nc=8)
    mesh = Mesh(case.n_points, case.elements)
    d = mesh.device_arrays()
    rng = np.random.default_rng(12)
    pos = torch.tensor(case.positions_at(0.3), device="cuda")
    lg = torch.tensor(rng.normal(size=mesh.n_lines), device="cuda")
    pts_h = rng.normal(size=(5000, 3)) * 2.0
    pts_h[:7] = case.positions_at(0.3)[:7]  # points on segment ends: cut-off
    pts = torch.tensor(pts_h, device="cuda")
    nrm = torch.nn.functional.normalize(torch.tensor(rng.normal(size=(5000, 3)), device="cuda"), dim=1)
    for normals in (None, nrm):
        shape = (5000,) if normals is not None else (5000, 3)
        ref = torch.empty(shape, dtype=torch.float64, device="cuda")
        ws, nb = Workspace.get(_lib.query("pvl_line_velocity_workspace", mesh.n_lines, 5000, _lib.PVL_F64))
        _lib.call("pvl_line_velocity", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos), ptr(lg),
                  5000, ptr(pts), ptr(normals), 1e-6, 1.0, 0.0, ptr(ref), ws, nb, stream_ptr())
        side = torch.cuda.Stream()
        for call in range(2):  # two calls in a row share (and reuse) the static scratch
            got = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            free0, used0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
            # the second call on a stream of the caller's own, not the default one
            stream = stream_ptr() if call == 0 else side.cuda_stream
            _lib.call("pvl_line_velocity_noalloc", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]),
                      ptr(pos), ptr(lg), 5000, ptr(pts), ptr(normals), 1e-6, 1.0, 0.0, ptr(got), stream)
            torch.cuda.synchronize()
            if call:  # after the first call (its one-time set-up), a call allocates no device memory
                assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == used0
            err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
            assert err <= 1e-12


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch

    from pyvl_b200 import _lib

    n_lines, n_pts = 2_000_000, 2_000_000
    assert _lib.query("pvl_line_velocity_workspace", n_lines, n_pts, _lib.PVL_F64) > (32 << 20)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="static array"):
        # rejected before any pointer is touched
        _lib.call("pvl_line_velocity_noalloc", _lib.PVL_F64, 1, n_lines, out.data_ptr(), out.data_ptr(),
                  out.data_ptr(), n_pts, out.data_ptr(), None, 1e-6, 1.0, 0.0, out.data_ptr(), None)
