"""Numpy restatement of the reference solver loop and free-wake model -- ORACLE ONLY.

Follows python/pyvl/solver.py:175-263 (one ``run_solver`` iteration),
python/pyvl/wake_models.py:17-330 (``WakeModelLineExplicitUnsteady``) and
python/pyvl/postprocess/forces.py:10-42 (``circulatory_forces``), with the pair
kernels from oracle.c and the dense solve from scipy LAPACK (``lu_factor`` /
``lu_solve``, the reference's own call, solver.py:223-227).

Positions and velocities come from a workload's kinematics instead of a chain of
ReferenceFrame objects; for a rigid static frame the two are identical, which
tests/test_oracle_pins.py checks against the reference's own ``run_solver``.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as la

from .kernels import INVALID_ID, OracleMesh, line_forces


def wake_ring_connectivity(line_rows: int, n_lines: int) -> np.ndarray:
    """Wake rings (n_lines * line_rows, 4): restates _create_wake_mesh, wake_models.py:35-52."""
    npr = line_rows + 1
    rc = np.empty((n_lines, line_rows, 4), np.uint32)
    r = np.arange(line_rows, dtype=np.uint32)
    rc[:, :, 0] = r
    rc[:, :, 1] = r + npr
    rc[:, :, 2] = r + npr + 1
    rc[:, :, 3] = r + 1
    rc[...] += (2 * npr * np.arange(n_lines, dtype=np.uint32))[:, None, None]
    return rc.reshape((-1, 4))


class OracleWake:
    """State and operations of WakeModelLineExplicitUnsteady (wake_models.py:17-330)."""

    def __init__(self, bordering_nodes, shedding_lines, adjacent_surfaces, vortex_tol, time, line_rows,
                 mesh_cls=OracleMesh):
        # wake_models.py:54-81
        self.shedding_lines = np.array(shedding_lines, np.uint64)
        S = self.shedding_lines.size
        self.wake_positions = np.zeros((S, 2, line_rows + 1, 3), np.float64)
        self.line_rows = int(line_rows)
        self.bordering_nodes = np.array(bordering_nodes, np.uint64)
        self.adjacent_surfaces = np.array(adjacent_surfaces, np.uint64)
        self.vortex_tol = float(vortex_tol)
        self.circulation = np.zeros((S, line_rows), np.float64)
        self.wake_mesh = mesh_cls(2 * (line_rows + 1) * S, wake_ring_connectivity(line_rows, S))
        self.current_time = float(time)
        self.step_count = 0

    def update(self, time, mesh: OracleMesh, positions, circulation, freestream, self_induction: bool = False):
        """Advect, re-pin, collapse, shift and shed: wake_models.py:83-157.  With self_induction
        (an option the reference does not have) every node also moves with the velocity the
        wake itself induces, evaluated on the wake as it was when the update began."""
        dt = time - self.current_time
        self.current_time = time
        bn = self.bordering_nodes.astype(np.int64)
        if self.step_count == 0:
            self.wake_positions[:, 0, 0, :] = positions[bn[:, 0], :]
            self.wake_positions[:, 1, 0, :] = positions[bn[:, 1], :]
            self.step_count = 1
        complete_rows = min(self.step_count, self.line_rows)
        wake_vel = None
        if self_induction:
            wake_vel = self.get_velocity(self.wake_positions.reshape((-1, 3))).reshape(self.wake_positions.shape)
        for i in reversed(range(complete_rows)):
            old_pos = self.wake_positions[:, :, i, :]
            flat = np.array(old_pos.reshape((-1, 3)), np.float64)
            vel = np.broadcast_to(freestream, flat.shape).copy()
            ind = mesh.induction_matrix(self.vortex_tol, positions, flat)
            vel += np.vecdot(ind, circulation[None, :, None], axis=1)
            if wake_vel is not None:
                vel += wake_vel[:, :, i, :].reshape((-1, 3))
            self.wake_positions[:, :, i + 1, :] = old_pos + vel.reshape(old_pos.shape) * dt
        self.wake_positions[:, 0, 0, :] = positions[bn[:, 0], :]
        self.wake_positions[:, 1, 0, :] = positions[bn[:, 1], :]
        if complete_rows != self.line_rows:
            self.wake_positions[:, :, complete_rows + 1:, :] = self.wake_positions[:, :, complete_rows, :][:, :, None, :]
        self.circulation[:, 1:] = self.circulation[:, :-1]
        self.circulation[:, 0] = 0
        adj = self.adjacent_surfaces
        mask = adj != INVALID_ID
        self.circulation[mask[:, 1], 0] += circulation[adj[mask[:, 1], 1].astype(np.int64)]
        self.circulation[mask[:, 0], 0] -= circulation[adj[mask[:, 0], 0].astype(np.int64)]
        self.step_count += 1

    def get_velocity(self, positions):
        """Wake-induced velocity at points: wake_models.py:159-175."""
        ind = self.wake_mesh.induction_matrix(self.vortex_tol, self.wake_positions.reshape((-1, 3)), positions)
        return np.vecdot(ind, self.circulation.reshape((1, -1, 1)), axis=1)

    def apply_corrections(self, control_pts, normals, mat_in, rhs_in):
        """Implicit (row 0) and explicit (rows >= 1) corrections: wake_models.py:177-223."""
        S = self.shedding_lines.size
        ind = self.wake_mesh.induction_matrix3(
            self.vortex_tol, self.wake_positions.reshape((-1, 3)), control_pts, normals
        ).reshape((control_pts.shape[0], S, self.line_rows))
        implicit = ind[:, :, 0]
        explicit = ind[:, :, 1:].reshape((control_pts.shape[0], -1))
        for i_line in range(S):
            correction = implicit[:, i_line]
            s1 = self.adjacent_surfaces[i_line, 1]
            if s1 != INVALID_ID:
                mat_in[:, int(s1)] -= correction
            s2 = self.adjacent_surfaces[i_line, 0]
            if s2 != INVALID_ID:
                mat_in[:, int(s2)] += correction
        circ = self.circulation.reshape((S, self.line_rows))[:, 1:].reshape((-1,))
        rhs_in[:] += np.vecdot(explicit, circ[None, :], axis=1)

    def correct_forces(self, line_forces_arr, mesh: OracleMesh, positions, circulation, freestream):
        """Subtract the first-wake-row TE force: wake_models.py:293-330."""
        S = self.shedding_lines.size
        tmp = OracleMesh(4 * S, wake_ring_connectivity(1, S))
        dual = tmp.dual_lines()
        cpts = np.ascontiguousarray(self.wake_positions[:, :, 0:2, :].reshape(-1, 3))
        circ = np.ascontiguousarray(self.circulation[:, 0] / (2 * np.pi))
        fs = np.broadcast_to(freestream, cpts.shape)
        ind_v = np.vecdot(mesh.induction_matrix(self.vortex_tol, positions, cpts), circulation[None, :, None], axis=1)
        self_v = self.get_velocity(cpts)
        forces = line_forces(tmp, dual, circ, cpts, fs + ind_v + self_v)
        for i, i_line in enumerate(self.shedding_lines):
            line_forces_arr[int(i_line), :] -= forces[4 * i + 1, :]


def shedding_setup(mesh: OracleMesh, te_node_pairs):
    """Shedding lines, bordering nodes and adjacent rings for given TE node pairs.

    Lines are found by their node pair; bordering nodes and adjacent rings follow
    SimulationGeometry.line_adjecency_information, geometry.py:654-681.
    """
    lookup = {}
    for il, (a, b) in enumerate(mesh.lines):
        lookup[(int(a), int(b))] = il
        lookup[(int(b), int(a))] = il
    shed = np.array(sorted(lookup[(int(a), int(b))] for a, b in te_node_pairs), np.uint64)
    dual = mesh.dual_lines()
    nodes = mesh.lines[shed.astype(np.int64)].astype(np.uint64)
    adj = dual[shed.astype(np.int64)].astype(np.uint64)
    return shed, nodes, adj


def bordered_solve(A, b, groups):
    """Solve A x + E lam = b, E^T x = 0 (one zero-mean constraint per closed group)."""
    n = A.shape[0]
    m = len(groups)
    K = np.zeros((n + m, n + m))
    K[:n, :n] = A
    for j, g in enumerate(groups):
        K[g, n + j] = 1.0
        K[n + j, g] = 1.0
    rhs = np.concatenate([b, np.zeros(m)])
    return la.lu_solve(la.lu_factor(K), rhs)[:n]


class OracleRun:
    """One run of the reference solver loop (solver.py:175-263) on a workload Case.

    ``mesh_cls`` supplies the pair kernels: OracleMesh (the C restatement, oracle.c) by default;
    oracle/refbench.py passes an adapter over the reference's own compiled extension."""

    def __init__(self, case, closed_mode: str = "reference", wake_self_induction: bool = False, mesh_cls=OracleMesh):
        self.case = case
        self.wake_self_induction = wake_self_induction
        self.mesh = mesh_cls(case.n_points, case.elements)
        self.closed_mode = closed_mode
        self.wake = None
        if case.line_rows > 0 and len(case.te_node_pairs):
            shed, nodes, adj = shedding_setup(self.mesh, case.te_node_pairs)
            self.wake = OracleWake(nodes, shed, adj, case.tol, case.t0, case.line_rows, mesh_cls)
        self.iteration = 0
        self.history = []

    def assemble(self, time):
        """Positions, control points, normals, RHS and the corrected system (solver.py:178-220)."""
        c = self.case
        pos = c.positions_at(time)
        vel = c.velocities_at(time)
        cps = self.mesh.surface_average_vec3(pos)
        cpv = self.mesh.surface_average_vec3(vel)
        nrm = self.mesh.surface_normal(pos)
        ev = np.broadcast_to(c.freestream, cps.shape) - cpv
        rhs = np.vecdot(nrm, -ev, axis=1)
        A = self.mesh.induction_matrix3(c.tol, pos, cps, nrm)
        if self.wake is not None and self.iteration > 0:
            self.wake.apply_corrections(cps, nrm, A, rhs)
        return pos, cps, nrm, A, rhs

    def solve(self, A, rhs):
        """LU solve + closed-body mean removal (solver.py:223-233), or the bordered system."""
        if self.case.closed and self.closed_mode == "bordered":
            return bordered_solve(A, rhs, [np.arange(A.shape[0])])
        g = la.lu_solve(la.lu_factor(A), rhs)
        if self.case.closed:
            g = g - np.mean(g)
        return g

    def step(self):
        time = self.iteration * self.case.dt
        pos, cps, nrm, A, rhs = self.assemble(time)
        gamma = self.solve(A, rhs)
        if self.wake is not None:
            self.wake.update(time, self.mesh, pos, gamma, self.case.freestream, self.wake_self_induction)
        self.history.append(gamma)
        self.iteration += 1
        return gamma

    def forces(self, time, gamma):
        """Line forces at output time t: restates postprocess/forces.py:10-42."""
        c = self.case
        pos = c.positions_at(time)
        fs = np.broadcast_to(c.freestream, pos.shape)
        induced = np.vecdot(self.mesh.induction_matrix(c.tol, pos, pos), gamma[None, :, None], axis=1)
        motion = c.velocities_at(time)
        if self.wake is not None:
            induced = induced + self.wake.get_velocity(pos)
        f = line_forces(self.mesh, self.mesh.dual_lines(), gamma / (2 * np.pi), pos, fs + induced - motion)
        if self.wake is not None:
            self.wake.correct_forces(f, self.mesh, pos, gamma, c.freestream)
        return f

    def cl(self, time, gamma):
        """CL = (sum F) . l / (0.5 |U|^2 S_ref) with rho = 1."""
        f = self.forces(time, gamma)
        u2 = float(np.dot(self.case.freestream, self.case.freestream))
        return float(f.sum(axis=0) @ self.case.lift_direction() / (0.5 * u2 * self.case.s_ref))
