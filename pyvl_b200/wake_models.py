"""Free-wake model with explicit Euler advection of shed vortex lines.

Mirrors WakeModelLineExplicitUnsteady (python/pyvl/wake_models.py:17-330): same
constructor, state arrays and methods.  Its numpy-facing methods run on the GPU kernels
(fused contractions, no materialised induction matrices); ``run_solver`` keeps the same
state resident on the device instead (pyvl_b200.engine).
"""

from __future__ import annotations

import numpy as np
from numpy import typing as npt

from .cvl import INVALID_ID, Mesh
from .engine import wake_ring_connectivity
from .fio.io_common import HirearchicalMap
from .wake import WakeModel


class WakeModelLineExplicitUnsteady(WakeModel):
    """Wake rings behind shedding lines, advected by the free stream and the body."""

    @staticmethod
    def _create_wake_mesh(line_rows: int, n_lines: int) -> Mesh:
        """Wake strips, ring (s, r) = s * line_rows + r (wake_models.py:35-52)."""
        return Mesh(2 * (line_rows + 1) * n_lines, wake_ring_connectivity(line_rows, n_lines))

    def __init__(self, bordering_nodes, shedding_lines, adjacent_surfaces, vortex_tol: float, time: float,
                 line_rows: int) -> None:
        if len(shedding_lines) == 0:
            raise RuntimeError("The geometry has no edges which would shed any wake.")
        self.shedding_lines = np.array(shedding_lines, np.uint)
        self.wake_positions = np.empty((self.shedding_lines.size, 2, line_rows + 1, 3), np.float64)
        self.line_rows = int(line_rows)
        self.bordering_nodes = np.array(bordering_nodes, np.uint)
        self.adjacent_surfaces = np.array(adjacent_surfaces)
        self.vortex_tol = float(vortex_tol)
        self.circulation = np.zeros((self.shedding_lines.size, line_rows), np.float64)
        self.wake_mesh = WakeModelLineExplicitUnsteady._create_wake_mesh(line_rows, self.shedding_lines.size)
        self.current_time = time
        self.step_count = 0

    # ------------------------------------------------------------------ time stepping
    def update(self, time, geometry, positions, circulation, flow) -> None:
        """Advance to `time` (wake_models.py:83-157): advect every complete row with the
        free stream plus the body's induced velocity, re-pin row 0 to the trailing edge,
        collapse the rows not yet reached, shift the circulations and shed the new row."""
        positions = np.ascontiguousarray(positions, np.float64)
        circulation = np.ascontiguousarray(circulation, np.float64)
        dt = time - self.current_time
        self.current_time = time
        bn = self.bordering_nodes.astype(np.int64)
        if self.step_count == 0:
            self.wake_positions[:, 0, 0, :] = positions[bn[:, 0], :]
            self.wake_positions[:, 1, 0, :] = positions[bn[:, 1], :]
            self.step_count = 1
        complete = min(self.step_count, self.line_rows)
        old = np.ascontiguousarray(self.wake_positions[:, :, :complete, :])
        pts = old.reshape(-1, 3)
        vel = np.asarray(flow.get_velocity(time, pts), np.float64)
        vel = vel + geometry.mesh.induced_velocity(self.vortex_tol, positions, pts, circulation)
        self.wake_positions[:, :, 1: complete + 1, :] = old + vel.reshape(old.shape) * dt
        self.wake_positions[:, 0, 0, :] = positions[bn[:, 0], :]
        self.wake_positions[:, 1, 0, :] = positions[bn[:, 1], :]
        if complete != self.line_rows:
            self.wake_positions[:, :, complete + 1:, :] = self.wake_positions[:, :, complete, :][:, :, None, :]
        self.circulation[:, 1:] = self.circulation[:, :-1]
        self.circulation[:, 0] = 0
        mask = self.adjacent_surfaces != INVALID_ID
        self.circulation[mask[:, 1], 0] += circulation[self.adjacent_surfaces[mask[:, 1], 1].astype(np.int64)]
        self.circulation[mask[:, 0], 0] -= circulation[self.adjacent_surfaces[mask[:, 0], 0].astype(np.int64)]
        self.step_count += 1

    def get_velocity(self, positions) -> npt.NDArray[np.float64]:
        """Velocity the wake induces at `positions` (wake_models.py:159-175), fused."""
        pts = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        return self.wake_mesh.induced_velocity(self.vortex_tol, self.wake_positions.reshape(-1, 3), pts,
                                               self.circulation.reshape(-1))

    def apply_corrections(self, control_pts, normals, mat_in, rhs_in) -> None:
        """Implicit first row into mat_in, explicit rows into rhs_in (wake_models.py:177-223).

        The first-row ring inductions come from the fused normal-induction kernel on those
        rings only; the explicit rows are one fused contraction with their circulations."""
        from .engine import wake_row0_mesh

        cps = np.ascontiguousarray(control_pts, np.float64)
        nrm = np.ascontiguousarray(normals, np.float64)
        wpos = np.ascontiguousarray(self.wake_positions.reshape(-1, 3))
        S, R = self.shedding_lines.size, self.line_rows
        implicit = wake_row0_mesh(self.wake_mesh, S, R).induction_matrix3(self.vortex_tol, wpos, cps, nrm)
        for i_line in range(S):
            correction = implicit[:, i_line]
            s1 = self.adjacent_surfaces[i_line, 1]
            if s1 != INVALID_ID:
                mat_in[:, s1] -= correction
            s2 = self.adjacent_surfaces[i_line, 0]
            if s2 != INVALID_ID:
                mat_in[:, s2] += correction
        if R > 1:
            circ = self.circulation.copy()
            circ[:, 0] = 0.0
            v = self.wake_mesh.induced_velocity(self.vortex_tol, wpos, cps, circ.reshape(-1))
            rhs_in[:] += np.einsum("ij,ij->i", v, nrm)

    def correct_forces(self, line_forces, geometry, positions, circulation, flow) -> None:
        """Remove the force on the first wake row's leading line (wake_models.py:293-330)."""
        tmp_mesh = WakeModelLineExplicitUnsteady._create_wake_mesh(1, self.shedding_lines.size)
        dual = tmp_mesh.compute_dual()
        cpts = np.ascontiguousarray(self.wake_positions[:, :, 0:2, :].reshape(-1, 3))
        circ = np.ascontiguousarray(self.circulation[:, 0] / (2 * np.pi))
        freestream = flow.get_velocity(self.current_time, cpts)
        ind_v = geometry.mesh.induced_velocity(self.vortex_tol, np.ascontiguousarray(positions, np.float64), cpts,
                                               np.ascontiguousarray(circulation, np.float64))
        self_v = self.get_velocity(cpts)
        forces = Mesh.line_forces(tmp_mesh, dual, circ, cpts, freestream + ind_v + self_v)
        for i, i_line in enumerate(self.shedding_lines):
            line_forces[int(i_line), :] -= forces[4 * i + 1, :]

    # ------------------------------------------------------------------ state
    def save(self) -> HirearchicalMap:
        out = HirearchicalMap()
        out.insert_array("bordering_nodes", self.bordering_nodes)
        out.insert_array("adjacent_surfaces", self.adjacent_surfaces)
        out.insert_array("shedding_lines", self.shedding_lines)
        out.insert_scalar("current_time", float(self.current_time))
        out.insert_int("step_count", int(self.step_count))
        out.insert_int("line_rows", int(self.line_rows))
        out.insert_array("wake_positions", self.wake_positions)
        out.insert_scalar("vortex_tol", float(self.vortex_tol))
        out.insert_array("circulation", self.circulation)
        return out

    @classmethod
    def load(cls, group: HirearchicalMap):
        out = cls(group.get_array("bordering_nodes"), group.get_array("shedding_lines"),
                  group.get_array("adjacent_surfaces"), group.get_scalar("vortex_tol"),
                  group.get_scalar("current_time"), group.get_int("line_rows"))
        out.circulation[...] = group.get_array("circulation")
        out.wake_positions[...] = group.get_array("wake_positions")
        out.step_count = group.get_int("step_count")
        return out

    def copy_state(self):
        """A snapshot with copied arrays and a shared wake mesh (no topology rebuild)."""
        new = object.__new__(type(self))
        new.__dict__.update(self.__dict__)
        new.wake_positions = self.wake_positions.copy()
        new.circulation = self.circulation.copy()
        return new
