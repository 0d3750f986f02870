"""The mixed-precision path on the GPU.

* FP32 LU with tensor-core trailing updates and its explicit inverse: X A ~ I to FP32/TF32
  accuracy, on a vortex-ring system and on a random matrix that needs row interchanges.
* Row-range wake node velocity: FP64 pieces reassemble the full sweep; FP32 far rows stay
  within FP32 rounding.
* MixedSolverEngine: every step judged against the all-FP64 step (FP64 assembly of the same
  state + FP64 LU): circulation within 1e-10 relative, no FP64 fallbacks, few GMRES iterations.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-10


def _lu32_inverse(A64):
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    n = A64.shape[0]
    npad = (n + 63) // 64 * 64
    A32 = torch.zeros((npad, npad), dtype=torch.float32, device="cuda")
    X = torch.zeros_like(A32)
    Y = torch.zeros_like(A32)
    ipiv = torch.zeros(2 * npad, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nb = _lib.query("pvl_lu32_workspace", npad)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    s = stream_ptr()
    _lib.call("pvl_pad_convert_f32", n, ptr(A64), n, ptr(A32), npad, npad, s)
    _lib.call("pvl_lu32_factor", npad, ptr(A32), npad, ptr(ipiv), ptr(info), ptr(err), ptr(ws), nb, s)
    _lib.call("pvl_lu32_inverse", npad, ptr(A32), npad, ipiv.data_ptr() + 4 * npad, ptr(X), npad, ptr(Y), npad,
              ptr(err), ptr(ws), nb, s)
    torch.cuda.synchronize()
    assert int(info.item()) == 0 and int(err.item()) == 0
    perm = ipiv[npad:].long()
    return X, perm, npad


def _apply(X, perm, n, v):
    """z = X v with the permutation already folded into X's columns."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    _lib.call("pvl_gemv_f32mat", n, n, 1.0, ptr(X), X.shape[1], ptr(v), 0.0, ptr(z), stream_ptr())
    torch.cuda.synchronize()
    return z


def test_lu32_inverse_of_ring_system():
    import torch

    from pyvl_b200.cvl import Mesh
    from pyvl_b200.workloads import flapping

    case = flapping(ns=32, nc=8, line_rows=4)
    mesh = Mesh(case.n_points, case.elements)
    pos = case.positions_at(0.37)
    cps = mesh.surface_average_vec3(pos)
    nrm = mesh.surface_normal(pos)
    A = torch.as_tensor(mesh.induction_matrix3(case.tol, pos, cps, nrm), device="cuda")
    X, perm, npad = _lu32_inverse(A)
    n = A.shape[0]
    g = torch.Generator(device="cuda").manual_seed(3)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    x = _apply(X, perm, n, b)
    ref = torch.linalg.solve(A, b)
    rel = (torch.linalg.vector_norm(x - ref) / torch.linalg.vector_norm(ref)).item()
    assert rel < 1e-5, rel  # FP32 factors, small off-diagonal entries through TF32


def test_lu32_inverse_with_pivoting():
    """Rows of a well-conditioned matrix shuffled: partial pivoting must undo the shuffle."""
    import torch

    n = 200  # not a multiple of 64: exercises the identity padding
    g = torch.Generator(device="cuda").manual_seed(11)
    base = 2.0 * torch.eye(n, dtype=torch.float64, device="cuda")
    base += 0.3 * torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    shuffle = torch.randperm(n, generator=torch.Generator().manual_seed(4)).cuda()
    A = base[shuffle].contiguous()
    X, perm, npad = _lu32_inverse(A)
    assert not torch.equal(perm[:n].cpu(), torch.arange(n)), "the shuffled rows need interchanges"
    assert int(perm[:n].max()) < n and torch.equal(perm[n:].cpu(), torch.arange(n, npad))
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    x = _apply(X, perm, n, b)
    ref = torch.linalg.solve(A, b)
    rel = (torch.linalg.vector_norm(x - ref) / torch.linalg.vector_norm(ref)).item()
    assert rel < 1e-3, rel  # TF32 products in the updates: ~2^-11 relative on the off-diagonal part


def test_wake_node_velocity_column_and_row_split():
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.engine import synthetic_full_wake, wake_spec_from_te
    from pyvl_b200.workloads import flapping

    case = flapping(ns=32, nc=8, line_rows=24)
    mesh = Mesh(case.n_points, case.elements)
    t = 0.5
    pos_h = case.positions_at(t)
    spec = wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, t - case.dt)
    wpos, _ = synthetic_full_wake(pos_h, spec, case.freestream, case.dt, seed=2)
    S, R = len(spec.shedding_lines), case.line_rows
    complete = R - 3
    d = mesh.device_arrays()
    pos = torch.as_tensor(pos_h, device="cuda")
    wp = torch.as_tensor(np.ascontiguousarray(wpos), device="cuda")
    g = torch.Generator(device="cuda").manual_seed(5)
    lg = torch.randn(mesh.n_lines, dtype=torch.float64, device="cuda", generator=g)
    u = case.freestream
    nb = max(_lib.query("pvl_line_velocity_workspace", mesh.n_lines, 2 * S * c, p) for c in range(1, complete + 1)
             for p in (_lib.PVL_F64, _lib.PVL_F32))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    s = stream_ptr()

    def run(prec, r0, r1, out, n_cols=2 * S, cols=None):
        _lib.call("pvl_wake_node_velocity_cols", prec, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos),
                  ptr(lg), S, R, complete, r0, r1, n_cols, ptr(cols) if cols is not None else None, ptr(wp),
                  float(u[0]), float(u[1]), float(u[2]), case.tol, ptr(out), ptr(ws), nb, s)

    full = torch.zeros((S, 2, complete, 3), dtype=torch.float64, device="cuda")
    _lib.call("pvl_wake_node_velocity", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos), ptr(lg),
              S, R, complete, ptr(wp), float(u[0]), float(u[1]), float(u[2]), case.tol, ptr(full), ptr(ws), nb, s)
    parts = torch.full_like(full, float("nan"))
    run(_lib.PVL_F64, 0, 5, parts)
    run(_lib.PVL_F64, 5, complete, parts)
    mixed = torch.full_like(full, float("nan"))
    run(_lib.PVL_F64, 0, 5, mixed)
    run(_lib.PVL_F32, 5, complete, mixed)
    torch.cuda.synchronize()
    assert not torch.isnan(parts).any() and not torch.isnan(mixed).any()
    assert torch.allclose(parts, full, rtol=1e-13, atol=1e-13)
    assert torch.equal(mixed[:, :, :5], parts[:, :, :5])
    ind_full = full - torch.as_tensor(u, device="cuda")  # the induced part only
    ind_mixed = mixed - torch.as_tensor(u, device="cuda")
    rel = (torch.linalg.vector_norm(ind_mixed - ind_full) / torch.linalg.vector_norm(ind_full)).item()
    assert rel < 1e-5, rel
    # de-duplicated columns: each representative column gets the full sweep's velocities
    from pyvl_b200.engine import wake_node_columns

    _, cols, slot = wake_node_columns(spec.bordering_nodes)
    assert cols.size < 2 * S
    dcols = torch.as_tensor(cols.astype(np.int32), device="cuda")
    dedup = torch.full((cols.size, complete, 3), float("nan"), dtype=torch.float64, device="cuda")
    run(_lib.PVL_F64, 0, complete, dedup, int(cols.size), dcols)
    torch.cuda.synchronize()
    want = full.reshape(2 * S, complete, 3)[torch.as_tensor(cols.astype(np.int64), device="cuda")]
    assert torch.allclose(dedup, want, rtol=1e-13, atol=1e-13)
    # every other row (pvl_wake_node_velocity_rows, step 2): those rows as in the full sweep,
    # the rows between untouched
    stepped = torch.full_like(full, float("nan"))
    count = (complete - 5 + 1) // 2
    _lib.call("pvl_wake_node_velocity_rows", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos),
              ptr(lg), S, R, complete, 5, count, 2, 2 * S, None, ptr(wp), float(u[0]), float(u[1]), float(u[2]),
              case.tol, ptr(stepped), ptr(ws), nb, s)
    torch.cuda.synchronize()
    assert torch.allclose(stepped[:, :, 5::2], full[:, :, 5::2], rtol=1e-13, atol=1e-13)
    assert torch.isnan(stepped[:, :, 6::2]).all() and torch.isnan(stepped[:, :, :5]).all()
    with pytest.raises(ValueError):  # the last listed row must lie below complete_rows
        _lib.call("pvl_wake_node_velocity_rows", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]),
                  ptr(pos), ptr(lg), S, R, complete, 5, count + 1, 2, 2 * S, None, ptr(wp), float(u[0]),
                  float(u[1]), float(u[2]), case.tol, ptr(stepped), ptr(ws), nb, s)
    # the rows between from their column's neighbours 1 and 3 rows away (pvl_wake_interp_rows)
    interp = full.clone()
    last = complete - 4 if (complete - 4) % 2 == 1 else complete - 5
    _lib.call("pvl_wake_interp_rows", 2 * S, complete, 7, last, ptr(interp), s)
    torch.cuda.synchronize()
    f = full.reshape(2 * S, complete, 3)
    i = torch.arange(7, last + 1, 2, device="cuda")
    want = (9.0 * (f[:, i - 1] + f[:, i + 1]) - (f[:, i - 3] + f[:, i + 3])) / 16.0
    got = interp.reshape(2 * S, complete, 3)
    assert torch.allclose(got[:, i], want, rtol=1e-15, atol=1e-15)
    keep = torch.ones(complete, dtype=torch.bool, device="cuda")
    keep[i] = False
    assert torch.equal(got[:, keep], f[:, keep])
    with pytest.raises(ValueError):  # an interpolated row needs the rows 3 above it
        _lib.call("pvl_wake_interp_rows", 2 * S, complete, 7, complete - 3, ptr(interp), s)
    # at spacing 2 (rows midway between every fourth row): rows 6, 10, 14 from rows +-2, +-6
    spaced = full.clone()
    _lib.call("pvl_wake_interp_rows_spaced", 2 * S, complete, 6, 14, 2, ptr(spaced), s)
    torch.cuda.synchronize()
    i2 = torch.arange(6, 15, 4, device="cuda")
    want = (9.0 * (f[:, i2 - 2] + f[:, i2 + 2]) - (f[:, i2 - 6] + f[:, i2 + 6])) / 16.0
    got = spaced.reshape(2 * S, complete, 3)
    assert torch.allclose(got[:, i2], want, rtol=1e-15, atol=1e-15)
    keep = torch.ones(complete, dtype=torch.bool, device="cuda")
    keep[i2] = False
    assert torch.equal(got[:, keep], f[:, keep])
    with pytest.raises(ValueError):  # rows 6 above the last one needed
        _lib.call("pvl_wake_interp_rows_spaced", 2 * S, complete, 6, complete - 6, 2, ptr(spaced), s)
    # listed rows (pvl_wake_node_velocity_list) of the de-duplicated columns: those rows as in the
    # full sweep, a listed row at or past complete_rows skipped, the other rows untouched
    rows = np.array([2, 3, 9, 10, 11, complete - 1, complete + 4], np.int32)
    d_rows = torch.as_tensor(rows, device="cuda")
    listed = torch.full((cols.size, complete, 3), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("pvl_wake_node_velocity_list", _lib.PVL_F64, mesh.n_points, mesh.n_lines, ptr(d["lines"]), ptr(pos),
              ptr(lg), S, R, complete, rows.size, ptr(d_rows), int(cols.size), ptr(dcols), ptr(wp), float(u[0]),
              float(u[1]), float(u[2]), case.tol, ptr(listed), ptr(ws), nb, s)
    torch.cuda.synchronize()
    r_ok = torch.as_tensor(rows[:-1].astype(np.int64), device="cuda")
    want = full.reshape(2 * S, complete, 3)[torch.as_tensor(cols.astype(np.int64), device="cuda")]
    assert torch.allclose(listed[:, r_ok], want[:, r_ok], rtol=1e-13, atol=1e-13)
    other = torch.ones(complete, dtype=torch.bool, device="cuda")
    other[r_ok] = False
    assert torch.isnan(listed[:, other]).all()


def _mixed_engine(case, **kw):
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, wake_spec_from_te

    mesh = Mesh(case.n_points, case.elements)
    wake = None
    if case.line_rows > 0 and len(case.te_node_pairs):
        wake = wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)
    groups = [(0, case.n_surfaces)] if case.closed else None
    return MixedSolverEngine(mesh, case.freestream, case.tol, wake, groups, **kw)


@pytest.mark.parametrize("factory,kw,steps", [
    ("swept_pitching", dict(line_rows=30), 30),
    ("flapping", dict(ns=64, nc=16, line_rows=40), 40),
])
def test_mixed_steps_judged_against_fp64(factory, kw, steps):
    from pyvl_b200 import workloads

    case = getattr(workloads, factory)(**kw)
    eng = _mixed_engine(case, refresh=10, advect_near_rows=4)
    errs = []
    for it in range(steps):
        t = it * case.dt
        errs.append(eng.step_judged(t, case.positions_at(t), case.velocities_at(t)))
    eng.check_status()
    st = eng.stats
    assert max(errs) <= MIXED_TOL, max(errs)
    assert st["fallbacks"] == 0
    assert max(st["gmres_iters"]) <= 6, st["gmres_iters"]
    assert (steps + 9) // 10 <= st["refreshes"] <= steps // 2  # every 10 steps, earlier after slow solves


def test_mixed_closed_sphere_judged():
    from pyvl_b200.workloads import icosphere

    case = icosphere(subdiv=3)
    eng = _mixed_engine(case, gmres_tol=1e-13)
    for it in range(3):
        t = it * case.dt
        err = eng.step_judged(t, case.positions_at(t), case.velocities_at(t))
        assert err <= MIXED_TOL, err
    assert eng.stats["fallbacks"] == 0


def test_mixed_trajectory_tracks_plain():
    """Whole trajectories, held to the mixed path's 1e-10: the flapping wing (64 x 16) flown
    from t = 0 for 250 steps by the plain FP64 engine and by the mixed engine with its default
    precision bands (FP64 wake term, FP32 advection beyond the first 8 node rows); the wake
    grows to its 100 rows and is then truncated for 150 steps.  Every step's circulation of the
    mixed run is within 1e-10 of the plain run's."""
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flapping

    case = flapping(ns=64, nc=16, line_rows=100)
    mesh = Mesh(case.n_points, case.elements)

    def spec():
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    plain = SolverEngine(mesh, case.freestream, case.tol, spec())
    mixed = MixedSolverEngine(mesh, case.freestream, case.tol, spec())
    worst = 0.0
    for it in range(250):
        t = it * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        plain.step(t, p, v)
        mixed.step(t, p, v)
        a, b = mixed.gamma_host(), plain.gamma_host()
        worst = max(worst, float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    print(f"max trajectory difference over 250 steps: {worst:.3e}")
    assert worst <= MIXED_TOL, worst
    assert mixed.stats["fallbacks"] == 0


def test_mixed_trajectory_with_interpolated_far_rows():
    """As test_mixed_trajectory_tracks_plain, with the advection of every other node row from
    row 48 on interpolated (advect_interp_row=48; 52 of the 100 rows): every step's circulation
    is still within 1e-10 of the plain FP64 run's."""
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flapping

    case = flapping(ns=64, nc=16, line_rows=100)
    mesh = Mesh(case.n_points, case.elements)

    def spec():
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    plain = SolverEngine(mesh, case.freestream, case.tol, spec())
    mixed = MixedSolverEngine(mesh, case.freestream, case.tol, spec(), advect_interp_row=48)
    worst = 0.0
    for it in range(250):
        t = it * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        plain.step(t, p, v)
        mixed.step(t, p, v)
        a, b = mixed.gamma_host(), plain.gamma_host()
        worst = max(worst, float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    print(f"max trajectory difference over 250 steps: {worst:.3e}")
    assert worst <= MIXED_TOL, worst
    assert mixed.stats["fallbacks"] == 0
    with pytest.raises(ValueError):
        MixedSolverEngine(mesh, case.freestream, case.tol, spec(), advect_interp_row=47)


def test_far_stencil_kernels_match_numpy():
    """pvl_gather_points and pvl_stencil_normal_add against numpy on seeded data (bit-exact
    gather; the stencil's sums to rounding), out-of-range indices giving NaN."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr, to_device_u32

    rng = np.random.default_rng(7)
    n_pts, n = 300, 257
    pts = rng.normal(size=(n_pts, 3))
    index = rng.integers(0, n_pts, n).astype(np.uint32)
    index[5] = n_pts  # out of range
    # every device array held by a name until the results are read back: a temporary freed
    # before the launch would hand its block to the next allocation
    d_pts = torch.tensor(pts, device="cuda")
    d_out = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    d_index = to_device_u32(index)
    _lib.call("pvl_gather_points", n, ptr(d_index), n_pts, ptr(d_pts), ptr(d_out), stream_ptr())
    got = d_out.cpu().numpy()
    ok = np.arange(n) != 5
    assert np.array_equal(got[ok], pts[index[ok].astype(np.int64)])
    assert np.isnan(got[5]).all()

    n_cp, n_val = 500, 120
    counts = rng.integers(0, 43, n_cp)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    entries = rng.integers(0, n_val, int(offsets[-1])).astype(np.uint32)
    entries[offsets[3]] = n_val if counts[3] else entries[offsets[3]]
    weights = rng.normal(size=int(offsets[-1]))
    vals, nrm, out0 = rng.normal(size=(n_val, 3)), rng.normal(size=(n_cp, 3)), rng.normal(size=n_cp)
    d_o = torch.tensor(out0, device="cuda")
    d_off, d_ent = to_device_u32(offsets), to_device_u32(entries)
    d_w, d_v, d_n = (torch.tensor(a, device="cuda") for a in (weights, vals, nrm))
    _lib.call("pvl_stencil_normal_add", n_cp, ptr(d_off), entries.size, ptr(d_ent), ptr(d_w), n_val, ptr(d_v),
              ptr(d_n), ptr(d_o), stream_ptr())
    got = d_o.cpu().numpy()
    # offsets past the entries: NaN for the points concerned, nothing read outside the arrays
    bad_off = offsets.copy()
    bad_off[7:] += 5
    d_bad = to_device_u32(bad_off)
    d_o2 = torch.zeros(n_cp, dtype=torch.float64, device="cuda")
    _lib.call("pvl_stencil_normal_add", n_cp, ptr(d_bad), entries.size, ptr(d_ent), ptr(d_w), n_val, ptr(d_v),
              ptr(d_n), ptr(d_o2), stream_ptr())
    got2 = d_o2.cpu().numpy()
    past = bad_off[1:] > entries.size
    assert np.isnan(got2[past]).all() and past.any()
    want = out0.copy()
    for p in range(n_cp):
        k = slice(int(offsets[p]), int(offsets[p + 1]))
        e = entries[k].astype(np.int64)
        if (e >= n_val).any():
            want[p] = np.nan
            continue
        want[p] += nrm[p] @ (weights[k, None] * vals[e]).sum(0)
    bad = np.isnan(want)
    assert bad[3] == bool(counts[3]) and np.isnan(got[bad]).all()
    np.testing.assert_allclose(got[~bad], want[~bad], rtol=1e-12, atol=1e-12)


def test_wake_interp_cols_matches_numpy():
    """pvl_wake_interp_cols against numpy: rows [4, 17) of 9 node columns from the 5 evaluated
    ones by seeded rules; a rule past the entries gives NaN for its column only."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr, to_device_u32

    rng = np.random.default_rng(11)
    n_cols, n_sub, complete = 9, 5, 20
    counts = rng.integers(1, 7, n_cols)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    entries = rng.integers(0, n_sub, int(offsets[-1])).astype(np.uint32)
    weights = rng.normal(size=entries.size)
    sub = rng.normal(size=(n_sub, complete, 3))
    node0 = rng.normal(size=(n_cols, complete, 3))
    d_off, d_ent = to_device_u32(offsets), to_device_u32(entries)
    d_w, d_sub, d_node = (torch.tensor(a, device="cuda") for a in (weights, sub, node0))
    _lib.call("pvl_wake_interp_cols", n_cols, complete, 4, 17, ptr(d_off), entries.size, ptr(d_ent), ptr(d_w),
              n_sub, ptr(d_sub), ptr(d_node), stream_ptr())
    got = d_node.cpu().numpy()
    want = node0.copy()
    for c in range(n_cols):
        k = slice(int(offsets[c]), int(offsets[c + 1]))
        want[c, 4:17] = (weights[k, None, None] * sub[entries[k].astype(np.int64), 4:17]).sum(0)
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)
    bad = offsets.copy()
    bad[-1] += 3
    d_bad = to_device_u32(bad)
    _lib.call("pvl_wake_interp_cols", n_cols, complete, 0, complete, ptr(d_bad), entries.size, ptr(d_ent),
              ptr(d_w), n_sub, ptr(d_sub), ptr(d_node), stream_ptr())
    got = d_node.cpu().numpy()
    assert np.isnan(got[-1]).all() and np.isfinite(got[:-1]).all()
    with pytest.raises(ValueError):
        _lib.call("pvl_wake_interp_cols", n_cols, complete, 3, complete + 1, ptr(d_off), entries.size, ptr(d_ent),
                  ptr(d_w), n_sub, ptr(d_sub), ptr(d_node), stream_ptr())


def test_mixed_trajectory_with_far_wake_stencil():
    """As test_mixed_trajectory_tracks_plain, with the explicit wake term of the far rows
    evaluated at part of the control points and interpolated across each half wing
    (cp_patches; 200 wake rows, chordwise from row 64 = 4 chords, spanwise too from row 160 =
    10 chords, where the coarser 64 x 16 grid's spacing relative to the distance matches the
    128 x 32 wing's from row 192) and the advection of the rows from 64 on evaluated at every
    other node column (wake_col_runs), from row 160 at every fourth row (advect_row4): every
    step's circulation is still within 1e-10 of the plain FP64 run's, and the judged step
    (everything re-assembled in FP64) agrees with the interpolated one to the same bar."""
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flapping

    case = flapping(ns=64, nc=16, line_rows=200)
    mesh = Mesh(case.n_points, case.elements)

    def spec():
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    plain = SolverEngine(mesh, case.freestream, case.tol, spec())
    mixed = MixedSolverEngine(mesh, case.freestream, case.tol, spec(), cp_patches=case.smooth_patches,
                              wake_chord_row=64, wake_span_row=160, wake_col_runs=case.wake_col_runs,
                              advect_col_row=64, advect_row4=160)
    assert mixed._far["n_chord_eval"] < mixed.P and mixed._cols["n_sub"] < mixed.wake["n_cols"]
    worst = 0.0
    for it in range(250):
        t = it * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        plain.step(t, p, v)
        mixed.step(t, p, v)
        a, b = mixed.gamma_host(), plain.gamma_host()
        worst = max(worst, float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    print(f"max trajectory difference over 250 steps: {worst:.3e}")
    assert worst <= MIXED_TOL, worst
    assert mixed.stats["fallbacks"] == 0
    t = 250 * case.dt
    assert mixed.step_judged(t, case.positions_at(t), case.velocities_at(t)) <= MIXED_TOL
    with pytest.raises(ValueError):
        MixedSolverEngine(mesh, case.freestream, case.tol, spec(), cp_patches=case.smooth_patches, near_rows=10)
    with pytest.raises(ValueError):
        MixedSolverEngine(mesh, case.freestream, case.tol, spec(), cp_patches=case.smooth_patches,
                          wake_chord_row=80, wake_span_row=40)


def test_full_wake_graphs_match_direct_launches():
    """Once the wake is full the wake terms and the wake update replay captured graphs (one per
    buffer pair and time step); the circulations and the wake are bit-identical to an engine
    that launches every kernel directly (capture_steps off)."""
    import torch

    from pyvl_b200.workloads import flapping

    case = flapping(ns=32, nc=8, line_rows=32)
    runs = []
    for capture in (True, False):
        eng = _mixed_engine(case, cp_patches=case.smooth_patches, wake_chord_row=8, wake_span_row=16,
                            wake_col_runs=case.wake_col_runs, advect_col_row=8, advect_interp_row=12,
                            advect_row4=16)
        eng.capture_steps = capture
        G = []
        for it in range(50):
            t = it * case.dt
            eng.step(t, case.positions_at(t), case.velocities_at(t))
            G.append(eng.gamma_host())
        runs.append((np.array(G), eng.wake_positions.cpu().numpy(), eng.wake_circulation.cpu().numpy(),
                     len(eng._update_keys), sum(1 for k in eng._step_graphs if k[0] == "wake_terms")))
        torch.cuda.synchronize()
    (g1, p1, c1, nu1, nt1), (g2, p2, c2, nu2, nt2) = runs
    assert nu1 >= 2 and nt1 >= 2 and nu2 == 0 and nt2 == 0
    assert np.array_equal(g1, g2) and np.array_equal(p1, p2) and np.array_equal(c1, c2)


def test_gmres_graph_replay_is_bitwise_identical():
    """The GMRES pieces replayed as captured CUDA graphs give the same circulations, bit for
    bit, as launching them directly."""
    from pyvl_b200.workloads import flapping

    case = flapping(ns=32, nc=8, line_rows=12)
    a = _mixed_engine(case, refresh=5, use_graphs=False, device_solve=False)
    b = _mixed_engine(case, refresh=5, use_graphs=True, device_solve=False)
    for k in range(14):
        t = k * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        a.step(t, p, v)
        b.step(t, p, v)
        assert np.array_equal(a.gamma_host(), b.gamma_host()), k
    assert len(b.graphs) > 2


def test_device_solve_against_host_driven_gmres():
    """The solve driven by the device (one graph launch, conditional WHILE over the Krylov
    columns) and the host-driven GMRES reach the same circulations; both judged against FP64."""
    from pyvl_b200.workloads import flapping

    case = flapping(ns=64, nc=16, line_rows=30)
    dev = _mixed_engine(case, refresh=10)
    host = _mixed_engine(case, refresh=10, device_solve=False)
    assert dev.device_solve and not host.device_solve
    worst = 0.0
    for k in range(30):
        t = k * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        if k % 10 == 9:
            assert dev.step_judged(t, p, v) <= MIXED_TOL
            assert host.step_judged(t, p, v) <= MIXED_TOL
        else:
            dev.step(t, p, v)
            host.step(t, p, v)
        a, b = dev.gamma_host(), host.gamma_host()
        worst = max(worst, float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    sd, sh = dev.stats, host.stats
    print("device iterations", sd["gmres_iters"], "host iterations", sh["gmres_iters"], "worst", worst)
    assert worst <= 1e-9, worst
    assert sd["fallbacks"] == 0 and len(sd["gmres_iters"]) == 30
    assert max(sd["final_rel_residual"]) <= 1e-12
    assert abs(sum(sd["gmres_iters"]) - sum(sh["gmres_iters"])) <= 6


def test_device_solve_fallback_runs_fp64_lu():
    """With a tolerance GMRES cannot meet in one column, every solve takes the FP64 fallback
    inside the graph (conditional IF: LU factorisation + blocked substitution): the
    circulations are the plain FP64 engine's."""
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import flapping

    case = flapping(ns=32, nc=8, line_rows=10)
    mesh = Mesh(case.n_points, case.elements)
    plain = SolverEngine(mesh, case.freestream, case.tol,
                         wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0))
    mixed = _mixed_engine(case, max_iter=1, gmres_tol=1e-300, refresh=5)
    for k in range(8):
        t = k * case.dt
        p, v = case.positions_at(t), case.velocities_at(t)
        plain.step(t, p, v)
        mixed.step(t, p, v)
        a, b = mixed.gamma_host(), plain.gamma_host()
        assert float(np.linalg.norm(a - b) / np.linalg.norm(b)) <= 1e-11, k
    st = mixed.stats
    assert st["fallbacks"] == 8 and st["gmres_iters"] == [1] * 8
    mixed.check_status()
