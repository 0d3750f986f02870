"""Generate the golden vectors in tests/golden/ from the REFERENCE ITSELF.

Run here (where the reference tree is mounted) after oracle/build_ref.sh:

    python tests/golden/make_golden.py [--reference REFERENCE_ROOT]   (default: $PYVL_REFERENCE_ROOT)

It imports the reference's compiled extension (oracle/_ref) and its Python package
and records, for small seeded inputs:

* kernels.npz  -- Mesh topology, induction_matrix / induction_matrix3 /
  line_induction_matrix, surface_normal / surface_average_vec3, dual lines,
  line_forces, dual_normal_criterion / dual_free_edges on several meshes.
* run_flat.npz -- the UNMODIFIED reference ``run_solver`` on the 16 x 4 flat wing,
  10 free-wake steps: circulation history, final wake state, CL per output
  (``postprocess.circulatory_forces``).
* run_<name>.npz -- pitching and flapping wings: a harness that replays
  python/pyvl/solver.py:175-263 step by step with kinematic positions, calling the
  reference's Mesh and WakeModelLineExplicitUnsteady objects.
* sphere.npz  -- a 320-triangle closed sphere: A, b and the reference's LU + mean
  circulation.
* wake_wedge.npz -- the wedge of test/pytests/test_wake_models.py:18-77 after 5 updates.
* checksums.npz -- full-size body matrices (1024 and 4096 rings) reduced to
  A @ v, A^T @ w and sampled entries for seeded v, w.
* checkpoint_flat.json / .npz -- the reference's own JSON solver-state snapshot (run_solver
  with OutputSettings("JSON")) after a 3-step flat-wing run, with its circulation and wake.

``--only NAME`` regenerates one fixture (e.g. ``--only checkpoint``).

The fixtures are small (a few hundred KB in total) and committed.
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import scipy.linalg as la

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402
from pyvl_b200 import workloads  # noqa: E402

TOL = 1e-6


def ref_mesh(pyvl, case):
    return pyvl.Mesh(case.n_points, [np.asarray(e, np.uint32) for e in case.elements])


def oriented_surface_lines(msh):
    """Rebuild the signed ring->line CSR from the reference's public getters."""
    lines = np.array(msh.line_data, np.uint32)
    offsets = [0]
    sl = []
    for i in range(msh.n_surfaces):
        s = msh.get_surface(i)
        for ln in s.lines:
            b, e = int(ln.begin), int(ln.end)
            hit = np.nonzero(((lines[:, 0] == b) & (lines[:, 1] == e)) | ((lines[:, 0] == e) & (lines[:, 1] == b)))[0]
            il = int(hit[0])
            # Surface lines come back reversed for orientation 0 (src/surfaceobject.c:226-233)
            rev = 1 if (lines[il, 0] == b and lines[il, 1] == e) else 0
            sl.append((rev << 31) | il)
        offsets.append(len(sl))
    return lines, np.array(offsets, np.uint32), np.array(sl, np.uint32)


def kernel_cases():
    rng = np.random.default_rng(11)
    out = []
    # the reference's own test mesh (test/pytests/test_mesh.py:18-68)
    pos = np.array([[0, 2, 0.5], [0.4, 2, 0.4], [4, 0.1, 0.2], [3, -0.1, 0.2], [2, 1, 0.2], [2, -1, 3]], np.float64)
    out.append(("mixed", pos, [[0, 1, 2, 3], [2, 3, 4], [0, 1, 4], [2, 4, 5]]))
    # unit square ring whose control points sit on its own nodes (test_mesh.py:105-111)
    out.append(("square", np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float64), [[0, 1, 2, 3]]))
    fw = workloads.flat_wing()
    out.append(("flat", fw.positions, [list(map(int, e)) for e in fw.elements]))
    sp = workloads.swept_pitching(ns=8, nc=4)
    out.append(("swept", sp.positions_at(0.3), [list(map(int, e)) for e in sp.elements]))
    ico = workloads.icosphere(subdiv=1)
    out.append(("ico80", ico.positions, [list(map(int, e)) for e in ico.elements]))
    # a random quad patch with one degenerate (zero-length) line
    p = rng.normal(size=(9, 3))
    p[8] = p[7]
    out.append(("random", p, [[0, 1, 2, 3], [1, 4, 5, 2], [3, 2, 6], [6, 2, 5, 7, 8]]))
    return out, rng


def make_kernels(pyvl):
    cases, rng = kernel_cases()
    data = {}
    for name, pos, elems in cases:
        msh = pyvl.Mesh(pos.shape[0], [np.asarray(e, np.uint32) for e in elems])
        lines, off, sl = oriented_surface_lines(msh)
        n_cp = 7
        cps = np.concatenate([rng.normal(size=(n_cp, 3)) * 2, pos[: min(4, pos.shape[0])]], axis=0)
        # points exactly on segment midpoints exercise the near-singular cutoff
        mids = 0.5 * (pos[lines[:2, 0]] + pos[lines[:2, 1]])
        cps = np.ascontiguousarray(np.concatenate([cps, mids], axis=0))
        nrm = rng.normal(size=cps.shape)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        dual = msh.compute_dual()
        circ = rng.normal(size=msh.n_surfaces)
        vel = rng.normal(size=pos.shape)
        counts, flat = msh.to_element_connectivity()
        d = {
            "positions": pos, "elements_counts": np.array([len(e) for e in elems], np.uint32),
            "elements_flat": np.concatenate([np.asarray(e, np.uint32) for e in elems]),
            "lines": lines, "offsets": off, "surface_lines": sl,
            "cps": cps, "normals": nrm, "circ": circ, "velocity": vel,
            "line_ind": msh.line_induction_matrix(TOL, pos, cps),
            "ind_vec": msh.induction_matrix(TOL, pos, cps),
            "ind_nrm": msh.induction_matrix3(TOL, pos, cps, nrm),
            "surface_normal": msh.surface_normal(pos),
            "surface_center": msh.surface_average_vec3(pos),
            "dual_lines": np.array(dual.line_data, np.uint32),
            "line_forces": pyvl.Mesh.line_forces(msh, dual, circ, pos, vel),
            "to_elem_counts": np.asarray(counts), "to_elem_flat": np.asarray(flat),
            "free_edges": np.asarray(dual.dual_free_edges()),
        }
        if name in ("swept", "mixed", "ico80"):
            d["normal_crit"] = np.asarray(dual.dual_normal_criterion(-0.5, msh.surface_normal(pos)))
        for k, v in d.items():
            data[f"{name}/{k}"] = np.asarray(v)
    np.savez_compressed(HERE / "kernels.npz", **data)


def te_lines_for(msh, te_pairs):
    lines = np.array(msh.line_data, np.uint32)
    idx = []
    for a, b in te_pairs:
        hit = np.nonzero(((lines[:, 0] == a) & (lines[:, 1] == b)) | ((lines[:, 0] == b) & (lines[:, 1] == a)))[0]
        idx.append(int(hit[0]))
    return np.array(sorted(idx), np.uint32)


def make_flat_run(pyvl):
    """Unmodified run_solver + circulatory_forces on the 16 x 4 flat wing."""
    case = workloads.flat_wing()
    geo = pyvl.Geometry("wing", pyvl.ReferenceFrame(), ref_mesh(pyvl, case), case.positions)
    sim = pyvl.SimulationGeometry(geo)
    fc = pyvl.FlowConditionsUniform(*case.freestream)
    settings = pyvl.SolverSettings(fc, pyvl.ModelSettings(TOL), pyvl.TimeSettings(case.nt, case.dt))
    te = te_lines_for(sim.mesh, case.te_node_pairs)
    nds, srf = sim.line_adjecency_information(te)
    wm = pyvl.WakeModelLineExplicitUnsteady(nds, te, srf, TOL, case.t0, case.line_rows)
    import contextlib
    import io

    with contextlib.redirect_stdout(io.StringIO()):
        res = pyvl.run_solver(sim, settings, wm, None)
    forces = pyvl.postprocess.circulatory_forces(res)
    u2 = float(case.freestream @ case.freestream)
    cl = np.array([f.sum(axis=0) @ case.lift_direction() / (0.5 * u2 * case.s_ref) for f in forces])
    last = res.wake_models[-1]
    np.savez_compressed(
        HERE / "run_flat.npz", circulations=res.circulations, cl=cl, forces_last=forces[-1],
        wake_positions=last.wake_positions, wake_circulation=last.circulation,
        shedding_lines=te, harness_circulations=harness_run(pyvl, case)[0],
    )


def harness_run(pyvl, case, with_forces=False):
    """Replay solver.py:175-263 with kinematic positions (reference objects throughout)."""
    msh = ref_mesh(pyvl, case)
    geo = pyvl.Geometry("wing", pyvl.ReferenceFrame(), msh, case.positions)
    sim = pyvl.SimulationGeometry(geo)
    mesh = sim.mesh
    fc = pyvl.FlowConditionsUniform(*case.freestream)
    wm = None
    if case.line_rows > 0:
        te = te_lines_for(mesh, case.te_node_pairs)
        nds, srf = sim.line_adjecency_information(te)
        wm = pyvl.WakeModelLineExplicitUnsteady(nds, te, srf, TOL, case.t0, case.line_rows)
    gammas, cls, snapshots = [], [], []
    for it in range(case.nt):
        t = it * case.dt
        pos = case.positions_at(t)
        vel = case.velocities_at(t)
        cps = mesh.surface_average_vec3(pos)
        cpv = mesh.surface_average_vec3(vel)
        nrm = mesh.surface_normal(pos)
        ev = fc.get_velocity(t, cps)
        ev -= cpv
        rhs = np.empty(case.n_surfaces)
        np.vecdot(nrm, -ev, out=rhs, axis=1)
        A = mesh.induction_matrix3(TOL, pos, cps, nrm)
        if wm is not None and it > 0:
            wm.apply_corrections(cps, nrm, A, rhs)
        g = la.lu_solve(la.lu_factor(A, overwrite_a=True), rhs, overwrite_b=True)
        if case.closed:
            g -= np.mean(g)
        if wm is not None:
            wm.update(t, sim, pos, g, fc)
        gammas.append(np.array(g))
        if with_forces:
            # postprocess/forces.py:10-42 with the kinematic motion velocity
            fs = fc.get_velocity(t, pos)
            induced = np.vecdot(mesh.induction_matrix(TOL, pos, pos), g[None, :, None], axis=1)
            if wm is not None:
                induced += wm.get_velocity(pos)
            f = pyvl.Mesh.line_forces(mesh, sim.dual, g / (2 * np.pi), pos, fs + induced - vel)
            if wm is not None:
                wm.correct_forces(f, sim, pos, g, fc)
            u2 = float(case.freestream @ case.freestream)
            cls.append(f.sum(axis=0) @ case.lift_direction() / (0.5 * u2 * case.s_ref))
    if wm is not None:
        snapshots = (np.array(wm.wake_positions), np.array(wm.circulation))
    return np.array(gammas), np.array(cls), snapshots


def make_kinematic_runs(pyvl):
    runs = {
        "pitch": workloads.swept_pitching(ns=16, nc=4, nt=12, line_rows=8, seed=5),
        "flap": workloads.flapping(ns=16, nc=4, nt=12, line_rows=6),
    }
    for name, case in runs.items():
        g, cl, (wp, wc) = harness_run(pyvl, case, with_forces=True)
        np.savez_compressed(HERE / f"run_{name}.npz", circulations=g, cl=cl, wake_positions=wp,
                            wake_circulation=wc)


def make_sphere(pyvl):
    case = workloads.icosphere(subdiv=2)
    msh = ref_mesh(pyvl, case)
    pos = case.positions
    cps = msh.surface_average_vec3(pos)
    nrm = msh.surface_normal(pos)
    rhs = np.vecdot(nrm, -np.broadcast_to(case.freestream, cps.shape), axis=1)
    A = msh.induction_matrix3(TOL, pos, cps, nrm)
    g, _, _ = harness_run(pyvl, case)
    np.savez_compressed(HERE / "sphere.npz", A=A, rhs=rhs, gamma_ref=g[0])


def make_wedge(pyvl):
    """test/pytests/test_wake_models.py:18-77, recorded after the 5 updates."""
    node_positions = np.array([[0, 1, 0], [3, 1, -0.5], [3, 1, +0.5], [0, -1, 0], [3, -1, -0.5], [3, -1, +0.5]], float)
    geo = pyvl.Geometry("wedge", pyvl.ReferenceFrame(), pyvl.Mesh(6, [[0, 3, 5, 2], [3, 0, 1, 4], [1, 2, 5, 4]]),
                        node_positions)
    sim = pyvl.SimulationGeometry(geo)
    fc = pyvl.FlowConditionsUniform(-1, 0, 0)
    te = sim.te_normal_criterion(-0.5)
    nds, srf = sim.line_adjecency_information(te)
    wm = pyvl.WakeModelLineExplicitUnsteady(nds, te, srf, 1e-6, -1, 5)
    circ_hist = []
    for i in range(5):
        c = 0.01 * np.array((np.sin(i), np.cos(i), 1))
        wm.update(float(i), sim, sim.positions_at_time(0), c, fc)
        circ_hist.append(np.array(wm.circulation))
    np.savez_compressed(HERE / "wake_wedge.npz", te=np.asarray(te), nodes=nds, surfaces=srf,
                        circulation=np.array(circ_hist), wake_positions=wm.wake_positions)


def make_checksums(pyvl):
    data = {}
    rng = np.random.default_rng(17)
    for name, case, t in (("swept_pitching", workloads.swept_pitching(), 0.5),
                          ("flapping", workloads.flapping(), 3.0)):
        msh = ref_mesh(pyvl, case)
        pos = case.positions_at(t)
        cps = msh.surface_average_vec3(pos)
        nrm = msh.surface_normal(pos)
        A = msh.induction_matrix3(TOL, pos, cps, nrm)
        v = rng.normal(size=A.shape[1])
        w = rng.normal(size=A.shape[0])
        ii = rng.integers(0, A.shape[0], 2000)
        jj = rng.integers(0, A.shape[1], 2000)
        data.update({
            f"{name}/t": np.float64(t), f"{name}/v": v, f"{name}/w": w,
            f"{name}/Av": A @ v, f"{name}/ATw": A.T @ w, f"{name}/ii": ii, f"{name}/jj": jj,
            f"{name}/Aij": A[ii, jj], f"{name}/diag": np.diag(A).copy(),
            f"{name}/fro": np.float64(np.linalg.norm(A)),
        })
    np.savez_compressed(HERE / "checksums.npz", **data)


def make_frames(pyvl):
    """ReferenceFrame transforms (src/referenceframeobject.c) and the Python frame subclasses."""
    rng = np.random.default_rng(23)
    RF = pyvl.ReferenceFrame
    f0 = RF(rng.normal(size=3), rng.normal(size=3) * 2)
    f1 = RF(rng.normal(size=3), rng.normal(size=3) * 2, f0)
    f2 = RF(rng.normal(size=3), (-7.0, 0.3, 11.0), f1)
    x = rng.normal(size=(5, 4, 3))
    data = {"x": x}
    for name, f in (("f0", f0), ("f1", f1), ("f2", f2)):
        data[f"{name}/angles"] = f.angles
        data[f"{name}/offset"] = f.offset
        data[f"{name}/rot"] = f.rotation_matrix
        data[f"{name}/rot_inv"] = f.rotation_matrix_inverse
        for fn in ("from_parent_with_offset", "from_parent_without_offset", "to_parent_with_offset",
                   "to_parent_without_offset", "from_global_with_offset", "from_global_without_offset",
                   "to_global_with_offset", "to_global_without_offset"):
            data[f"{name}/{fn}"] = getattr(f, fn)(x)
        data[f"{name}/rot_x"] = f.rotate_x(2.1).angles
        data[f"{name}/rot_y"] = f.rotate_y(-1.1).angles
        data[f"{name}/rot_z"] = f.rotate_z(7.5).angles
    data["angles_from_rotation"] = RF.angles_from_rotation(f2.rotation_matrix)
    tr = pyvl.TranslatingReferenceFrame((1, 2, 3), (0.1, 0.2, 0.3), (0.5, -1, 2), f0, 0.5)
    trt = tr.at_time(2.25)
    data["translating/offset"] = trt.offset
    data["translating/angles"] = trt.angles
    v = np.zeros((7, 3))
    p = rng.normal(size=(7, 3))
    trt.add_velocity(p, v)
    data["translating/p"] = p
    data["translating/velocity"] = v
    rr = pyvl.RotorReferenceFrame((0, 1, 0), (0.3, 0.0, 0.2), None, (0.1, 0.2, 2.0), 0.0)
    rrt = rr.at_time(1.7)
    data["rotor/offset"] = rrt.offset
    data["rotor/angles"] = rrt.angles
    v = np.zeros((7, 3))
    rrt.add_velocity(p, v)
    data["rotor/velocity"] = v
    np.savez_compressed(HERE / "frames.npz", **data)


def make_checkpoint(pyvl):
    """A solver-state snapshot written by the reference's own JSON output (run_solver with
    OutputSettings("JSON"), solver.py:251-262) after the last step of a 3-step flat-wing run."""
    import contextlib
    import io
    import shutil
    import tempfile

    case = workloads.flat_wing(nt=3, line_rows=3)
    geo = pyvl.Geometry("wing", pyvl.ReferenceFrame(), ref_mesh(pyvl, case), case.positions)
    sim = pyvl.SimulationGeometry(geo)
    fc = pyvl.FlowConditionsUniform(*case.freestream)
    settings = pyvl.SolverSettings(fc, pyvl.ModelSettings(TOL), pyvl.TimeSettings(case.nt, case.dt))
    te = te_lines_for(sim.mesh, case.te_node_pairs)
    nds, srf = sim.line_adjecency_information(te)
    wm = pyvl.WakeModelLineExplicitUnsteady(nds, te, srf, TOL, case.t0, case.line_rows)
    with tempfile.TemporaryDirectory() as tmp:
        out = pyvl.OutputSettings("JSON", lambda i, t: f"{tmp}/state_{i}.json")
        with contextlib.redirect_stdout(io.StringIO()):
            res = pyvl.run_solver(sim, settings, wm, out)
        shutil.copy(f"{tmp}/state_{case.nt - 1}.json", HERE / "checkpoint_flat.json")
    np.savez_compressed(HERE / "checkpoint_flat.npz", circulation=res.circulations[-1],
                        wake_positions=res.wake_models[-1].wake_positions,
                        wake_circulation=res.wake_models[-1].circulation)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (default: $PYVL_REFERENCE_ROOT)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    pyvl = ref.load_pyvl(args.reference)
    if args.only:
        globals()[f"make_{args.only}"](pyvl)
        return
    make_kernels(pyvl)
    make_flat_run(pyvl)
    make_kinematic_runs(pyvl)
    make_sphere(pyvl)
    make_wedge(pyvl)
    make_checksums(pyvl)
    make_frames(pyvl)
    make_checkpoint(pyvl)
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
