"""CUDA kernels vs the reference (golden vectors) and the CPU oracle.  Needs a B200.

Tolerances: the plain path must match the reference's FP64 kernels to <= 1e-12 relative
Frobenius error; cut-off zeros must be exact zeros.
"""

from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as la

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
TOL = 1e-6
PARITY = 1e-12


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def _names():
    d = np.load(GOLD / "kernels.npz")
    return sorted({k.split("/")[0] for k in d.files})


@pytest.mark.parametrize("name", _names())
def test_kernels_match_reference(torch_cuda, name):
    from pyvl_b200.cvl import Mesh

    d = np.load(GOLD / "kernels.npz")
    g = lambda k: d[f"{name}/{k}"]  # noqa: E731
    elems = np.split(g("elements_flat"), np.cumsum(g("elements_counts"))[:-1])
    pos, cps, nrm = g("positions"), g("cps"), g("normals")
    m = Mesh(pos.shape[0], elems)
    li = m.line_induction_matrix(TOL, pos, cps)
    assert rel(li, g("line_ind")) <= PARITY
    # the cut-off zeroes whole pairs (flow_solver.c:107-130): same pairs as the reference.
    # Single components may differ in zero-ness: FMA contraction of (dr1 x d) rounds
    # differently from the reference's separate multiply and subtract.
    assert np.array_equal(np.all(li == 0, axis=-1), np.all(g("line_ind") == 0, axis=-1))
    assert rel(m.induction_matrix(TOL, pos, cps), g("ind_vec")) <= PARITY
    assert rel(m.induction_matrix3(TOL, pos, cps, nrm), g("ind_nrm")) <= PARITY
    assert rel(m.surface_normal(pos), g("surface_normal")) <= 1e-15
    assert rel(m.surface_average_vec3(pos), g("surface_center")) <= 1e-15
    f = Mesh.line_forces(m, m.compute_dual(), g("circ"), pos, g("velocity"))
    assert rel(f, g("line_forces")) <= 1e-15


def test_overlap_self_entries_are_exact_zeros(torch_cuda):
    """test/pytests/test_mesh.py:105-111 on the GPU."""
    from pyvl_b200.cvl import Mesh

    msh = Mesh(4, [[0, 1, 2, 3]])
    positions = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float64)
    mat = msh.line_induction_matrix(1e-6, positions, positions)
    for i in range(4):
        assert all(mat[i, i, :] == (0, 0, 0))


@pytest.mark.parametrize("name", ["swept_pitching", "flapping"])
def test_full_size_body_matrix_checksums(torch_cuda, name):
    """Full-size (1024 and 4096 ring) body matrices vs the reference's checksums."""
    from pyvl_b200 import workloads
    from pyvl_b200.cvl import Mesh

    gold = np.load(GOLD / "checksums.npz")
    case = workloads.by_name(name)
    t = float(gold[f"{name}/t"])
    m = Mesh(case.n_points, case.elements)
    pos = case.positions_at(t)
    cps = m.surface_average_vec3(pos)
    nrm = m.surface_normal(pos)
    A = m.induction_matrix3(TOL, pos, cps, nrm)
    assert rel(A @ gold[f"{name}/v"], gold[f"{name}/Av"]) <= PARITY
    assert rel(A.T @ gold[f"{name}/w"], gold[f"{name}/ATw"]) <= PARITY
    assert rel(A[gold[f"{name}/ii"], gold[f"{name}/jj"]], gold[f"{name}/Aij"]) <= PARITY
    assert rel(np.diag(A), gold[f"{name}/diag"]) <= PARITY
    assert abs(np.linalg.norm(A) - gold[f"{name}/fro"]) <= PARITY * gold[f"{name}/fro"]


def test_induced_velocity_matches_oracle_contraction(torch_cuda):
    """Fused sum_j K_ij Gamma_j vs the reference's materialised matrix + vecdot (oracle)."""
    from oracle.kernels import OracleMesh
    from pyvl_b200 import workloads
    from pyvl_b200.cvl import Mesh

    case = workloads.swept_pitching(ns=16, nc=8)
    rng = np.random.default_rng(3)
    pos = case.positions_at(0.4)
    pts = rng.normal(size=(777, 3)) * 3
    pts[:10] = pos[:10]  # points on nodes: cut-off
    gam = rng.normal(size=case.n_surfaces)
    om = OracleMesh(case.n_points, case.elements)
    want = np.vecdot(om.induction_matrix(TOL, pos, pts), gam[None, :, None], axis=1)
    m = Mesh(case.n_points, case.elements)
    got = m.induced_velocity(TOL, pos, pts, gam)
    assert rel(got, want) <= PARITY


def _lu_roundtrip(torch, A, b):
    from pyvl_b200 import _lib
    from pyvl_b200.device import Workspace, ptr, stream_ptr

    n = A.shape[0]
    dA = torch.tensor(A, device="cuda")
    ipiv = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws, nb = Workspace.get(_lib.query("pvl_lu_workspace", n))
    _lib.call("pvl_lu_factor", n, ptr(dA), n, ptr(ipiv), ptr(info), ws, nb, stream_ptr())
    db = torch.tensor(b, device="cuda")
    _lib.call("pvl_lu_solve", n, ptr(dA), n, ptr(ipiv), ptr(db), ptr(err), ws, nb, stream_ptr())
    torch.cuda.synchronize()
    return dA.cpu().numpy(), ipiv.cpu().numpy(), int(info.item()), int(err.item()), db.cpu().numpy()


@pytest.mark.parametrize("n,kind", [(64, "dominant"), (200, "dominant"), (1000, "dominant"), (333, "general"),
                                    (130, "general"), (777, "singular_last"), (1000, "mixed"), (1600, "mixed")])
def test_lu_matches_lapack(torch_cuda, n, kind):
    rng = np.random.default_rng(n)
    A = rng.normal(size=(n, n))
    if kind in ("dominant", "mixed"):
        A = A * 1e-3 - 2 * np.pi * np.eye(n)
    if kind == "mixed":
        # the diagonal blocks of panels 5 and 11 (64 columns each) are permuted (antidiagonal, a
        # random permutation): those two panels interchange rows inside their own row block and
        # take the pivoting fallback, every other panel the speculative path -- the fallback runs
        # while the look-ahead's bulk update of the panel before it is in flight
        for p, perm in ((5, np.arange(63, -1, -1)), (11, rng.permutation(64))):
            c0 = 64 * p
            A[c0:c0 + 64, c0:c0 + 64] = rng.normal(size=(64, 64)) * 1e-3
            A[c0 + perm, c0 + np.arange(64)] -= 2 * np.pi
    if kind == "singular_last":
        A[:, -1] = 0.0
    b = rng.normal(size=n)
    LU, ipiv, info, err, x = _lu_roundtrip(torch_cuda, A, b)
    assert err == 0
    lu_ref, piv_ref = la.lu_factor(A)
    if kind == "mixed":
        moved = np.nonzero(piv_ref != np.arange(n))[0] // 64
        assert sorted(set(moved.tolist())) == [5, 11]
    assert np.array_equal(ipiv[:n], piv_ref)
    assert rel(LU, lu_ref) <= 1e-13
    if kind == "singular_last":
        assert info == n
        return
    assert info == 0
    x_ref = la.lu_solve((lu_ref, piv_ref), b)
    assert rel(x, x_ref) <= 1e-12


def test_lu_bordered_sphere(torch_cuda):
    """Closed sphere: the bordered (zero-mean) system vs the numpy/LAPACK oracle."""
    from oracle.solver import bordered_solve

    gold = np.load(GOLD / "sphere.npz")
    A, rhs = gold["A"], gold["rhs"]
    n = A.shape[0]
    K = np.zeros((n + 1, n + 1))
    K[:n, :n] = A
    K[:n, n] = K[n, :n] = 1.0
    LU, ipiv, info, err, x = _lu_roundtrip(torch_cuda, K, np.concatenate([rhs, [0.0]]))
    assert info == 0 and err == 0
    want = bordered_solve(A, rhs, [np.arange(n)])
    assert rel(x[:n], want) <= 1e-12


@pytest.mark.parametrize("factory", ["flapping_small", "sphere"])
def test_tiled_ring_matrix_matches_ring_matrix(factory):
    """pvl_induction_normal_tiled (each line once per control point per ring tile) gives the
    matrix of pvl_induction_normal to rounding, on quads and on triangles."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.device import Workspace, ptr, stream_ptr
    from pyvl_b200.workloads import flapping, icosphere

    case = flapping(ns=48, nc=12, line_rows=2) if factory == "flapping_small" else icosphere(subdiv=3)
    mesh = Mesh(case.n_points, case.elements)
    pos = torch.as_tensor(case.positions_at(0.3), device="cuda")
    cps = torch.as_tensor(mesh.surface_average_vec3(case.positions_at(0.3)), device="cuda")
    nrm = torch.as_tensor(mesh.surface_normal(case.positions_at(0.3)), device="cuda")
    P = mesh.n_surfaces
    d = mesh.device_arrays()
    ws, nb = Workspace.get(_lib.query("pvl_segments_workspace", mesh.n_lines, _lib.PVL_F64))
    a = torch.zeros((P, P), dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    s = stream_ptr()
    _lib.call("pvl_induction_normal", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos), P,
              ptr(d["offsets"]), ptr(d["surface_lines"]), P, ptr(cps), ptr(nrm), case.tol, ptr(a), P, ws, nb, s)
    _lib.call("pvl_induction_normal_tiled", mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos), P,
              ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["tile_offsets"]), ptr(d["tile_lines"]),
              ptr(d["sl_local"]), d["tile_max"], P, ptr(cps), ptr(nrm), case.tol, ptr(b), P, ws, nb, s)
    torch.cuda.synchronize()
    assert (torch.linalg.norm(a - b) / torch.linalg.norm(a)).item() <= 1e-14


def test_far_field_reciprocal_and_series_bounds(torch_cuda):
    """The FP64 pair kernels' far-field arithmetic held to its error bounds: 1/x from the
    hardware seed and one third-order step within an ulp of the rounded quotient; the
    arctangent series (four, eight or sixteen terms by w) within a few ulps of atan(q)/q,
    q = sqrt(w), evaluated in extended precision."""
    torch = torch_cuda
    from pyvl_b200 import _probe
    from pyvl_b200.device import ptr, stream_ptr

    rng = np.random.default_rng(3)
    n = 1 << 20
    x = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-900, 900, n))
    x[:4] = [1.0, 1.5, 2.0 - 2.0**-52, 3.0]
    w = np.concatenate([rng.uniform(0.0, 0.1, n // 2), 10.0 ** rng.uniform(-12, -1, n // 2)])
    w[:6] = [0.0, 1e-4, np.nextafter(1e-4, 1.0), 0.01, np.nextafter(0.01, 1.0), 0.1]
    dx, dw = torch.as_tensor(x, device="cuda"), torch.as_tensor(w, device="cuda")
    rcp, ssum = torch.empty_like(dx), torch.empty_like(dw)
    _probe.call("pvl_probe_far_series", n, ptr(dx), ptr(dw), ptr(rcp), ptr(ssum), stream_ptr())
    torch.cuda.synchronize()
    r, s = rcp.cpu().numpy(), ssum.cpu().numpy()
    want_r = 1.0 / x  # correctly rounded
    assert np.all(np.abs(r - want_r) <= np.spacing(want_r))
    q = np.sqrt(w.astype(np.longdouble))
    want_s = np.where(q > 0, np.arctan(q) / np.where(q > 0, q, 1), 1).astype(np.longdouble)
    err = np.abs(s.astype(np.longdouble) - want_s) / want_s
    assert float(err.max()) <= 4 * 2.0**-53
