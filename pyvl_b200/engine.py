"""Device-resident UVLM time stepping: the hot path of ``run_solver`` on one GPU.

One :meth:`SolverEngine.step` is one iteration of the reference's solver loop
(python/pyvl/solver.py:175-239) with the free wake of
``WakeModelLineExplicitUnsteady`` (python/pyvl/wake_models.py:83-223):

1. control points, control-point velocities, normals and the no-penetration RHS
   (solver.py:194-206)                                     -> pvl_surface_*, pvl_rhs
2. body influence matrix (solver.py:209)                   -> pvl_induction_normal
3. wake corrections for iteration > 0 (solver.py:217-220):
   implicit first wake row folded into the TE-adjacent columns, explicit rows contracted
   with the wake circulations into the RHS (wake_models.py:199-223)
                                                            -> pvl_induction_normal on the
   first-row rings, pvl_wake_fold_implicit, pvl_line_circulation + pvl_line_velocity
4. dense solve (solver.py:223-227)                         -> pvl_lu_factor / pvl_lu_solve
   closed bodies: the bordered zero-mean system, then the mean removal of solver.py:229-233
5. wake update (solver.py:236-239, wake_models.py:111-157): node velocities from the body
   (pvl_wake_node_velocity), Euler advection + re-pin + collapse (pvl_wake_advect),
   circulation shift + shed (pvl_wake_shed).

Every buffer is allocated once; positions and velocities of the body for the step are the
only inputs, the ring circulations the output.  Wake positions and circulations stay on
the device (double-buffered) and are copied out only on request.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .cvl import INVALID_ID, Mesh
from .device import ptr, require_cuda, stream_ptr, to_device, to_device_u32


def wake_ring_connectivity(line_rows: int, n_shed: int) -> np.ndarray:
    """Rings of the wake strips: strip s, row r -> nodes (s,0,r), (s,1,r), (s,1,r+1), (s,0,r+1).

    Same node numbering and ring order as the reference's wake mesh
    (python/pyvl/wake_models.py:35-52), so wake ring s*line_rows + r holds circulation[s, r].
    """
    npr = line_rows + 1
    r = np.arange(line_rows, dtype=np.uint64)
    base = (2 * npr * np.arange(n_shed, dtype=np.uint64))[:, None]
    rc = np.empty((n_shed, line_rows, 4), np.uint64)
    rc[:, :, 0] = r + base
    rc[:, :, 1] = r + npr + base
    rc[:, :, 2] = r + npr + 1 + base
    rc[:, :, 3] = r + 1 + base
    return rc.reshape(-1, 4).astype(np.uint32)


def wake_row0_mesh(wake_mesh: Mesh, n_shed: int, line_rows: int) -> Mesh:
    """The first-row rings (ring s * line_rows of each strip) over the wake mesh's lines and
    points: their induction is the implicit part of the wake correction."""
    off = wake_mesh.surface_offsets
    sl = wake_mesh.surface_lines
    rows0 = np.arange(n_shed) * line_rows
    cnt = (off[rows0 + 1] - off[rows0]).astype(np.uint32)
    off0 = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
    sl0 = np.concatenate([sl[off[r]: off[r + 1]] for r in rows0]).astype(np.uint32)
    return Mesh._from_arrays(wake_mesh.n_points, wake_mesh.line_data.copy(), off0, sl0)


@dataclass
class WakeSpec:
    """What the wake model needs from the geometry (wake_models.py:54-81)."""

    shedding_lines: np.ndarray     # (S,) body line ids
    bordering_nodes: np.ndarray    # (S, 2) body node ids (line begin, end)
    adjacent_surfaces: np.ndarray  # (S, 2) ring ids on either side (INVALID_ID where none)
    line_rows: int
    time: float                    # wake model start time (first update's dt = t0 - time)


def wake_spec_from_te(mesh: Mesh, te_node_pairs, line_rows: int, time: float) -> WakeSpec:
    """Shedding lines from trailing-edge node pairs, with their bordering nodes and the rings
    on either side (SimulationGeometry.line_adjecency_information, python/pyvl/geometry.py:654-681).
    Lines are taken in ascending id order like the reference's edge criteria return them."""
    lines = mesh.line_data
    lookup = {}
    for il, (a, b) in enumerate(lines):
        lookup[(int(a), int(b))] = il
        lookup[(int(b), int(a))] = il
    shed = np.array(sorted(lookup[(int(a), int(b))] for a, b in te_node_pairs), np.int64)
    dual = mesh.compute_dual().line_data
    return WakeSpec(shed.astype(np.uint32), lines[shed].astype(np.uint32), dual[shed].astype(np.uint32),
                    int(line_rows), float(time))


def synthetic_full_wake(body_positions: np.ndarray, spec: WakeSpec, freestream, dt: float, seed: int = 0):
    """Seeded full-wake state behind the shedding lines of `spec` (workloads.synthetic_full_wake)."""
    from .workloads import synthetic_full_wake as _swf

    te = np.asarray(body_positions, np.float64)[np.asarray(spec.bordering_nodes, np.int64)]
    return _swf(te, spec.line_rows, freestream, dt, seed)


class SolverEngine:
    """Plain FP64 UVLM stepping with the wake resident on the device."""

    def __init__(self, mesh: Mesh, freestream, tol: float, wake: WakeSpec | None = None,
                 closed_groups: list[tuple[int, int]] | None = None):
        self.dev = require_cuda()
        self.mesh = mesh
        self.tol = float(tol)
        self.u_inf = np.asarray(freestream, np.float64).reshape(3)
        self.P = mesh.n_surfaces
        self.groups = [(int(a), int(b)) for a, b in (closed_groups or []) if b > a]
        self.m = len(self.groups)
        self.N = self.P + self.m
        self.iteration = 0
        f64 = dict(dtype=torch.float64, device=self.dev)
        d = mesh.device_arrays()
        self.d_body = d
        self.pos = torch.zeros((mesh.n_points, 3), **f64)
        self.vel = torch.zeros((mesh.n_points, 3), **f64)
        self.cps = torch.zeros((self.P, 3), **f64)
        self.cpv = torch.zeros((self.P, 3), **f64)
        self.nrm = torch.zeros((self.P, 3), **f64)
        self.rhs = torch.zeros(self.N, **f64)
        self.A = torch.zeros((self.N, self.N), **f64)
        self.gamma = torch.zeros(self.P, **f64)
        self.body_line_gamma = torch.zeros(max(mesh.n_lines, 1), **f64)
        self.ipiv = torch.zeros(2 * self.N, dtype=torch.int32, device=self.dev)
        self.info = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        if self.m:
            goff = np.array([a for a, _ in self.groups] + [self.groups[-1][1]], np.uint32)
            contiguous = all(self.groups[i][1] == self.groups[i + 1][0] for i in range(self.m - 1))
            if not contiguous:
                raise ValueError("closed groups must be contiguous ranges of rings")
            self.goff = to_device_u32(goff, self.dev)
        self.wake = None
        if wake is not None:
            self._init_wake(wake)
        self._ws_bytes = self._workspace_bytes()
        self.ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=self.dev)
        self.h_pos = torch.empty((mesh.n_points, 3), dtype=torch.float64, pin_memory=True)
        self.h_vel = torch.empty((mesh.n_points, 3), dtype=torch.float64, pin_memory=True)
        self.h_gamma = torch.empty(self.P, dtype=torch.float64, pin_memory=True)

    # ------------------------------------------------------------------ setup
    def _init_wake(self, w: WakeSpec) -> None:
        S = int(np.asarray(w.shedding_lines).size)
        R = int(w.line_rows)
        if S == 0:
            raise RuntimeError("The geometry has no edges which would shed any wake.")
        adj = np.asarray(w.adjacent_surfaces, np.int64).reshape(S, 2)
        bn = np.asarray(w.bordering_nodes, np.int64).reshape(S, 2)
        ok = (adj == INVALID_ID) | ((adj >= 0) & (adj < self.P))
        if not ok.all():
            raise ValueError("adjacent surfaces out of range")
        if bn.min() < 0 or bn.max() >= self.mesh.n_points:
            raise ValueError("bordering nodes out of range")
        wmesh = Mesh(2 * (R + 1) * S, wake_ring_connectivity(R, S))
        # first-row rings (r = 0) as their own CSR over the wake's lines
        row0 = wake_row0_mesh(wmesh, S, R)
        off0, sl0 = row0.surface_offsets, row0.surface_lines
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.wake = {
            "S": S, "R": R, "mesh": wmesh, "d": wmesh.device_arrays(),
            "off0": to_device_u32(off0, self.dev), "sl0": to_device_u32(sl0, self.dev),
            "adj": to_device_u32(adj.astype(np.uint32), self.dev),
            "bn": to_device_u32(bn.astype(np.uint32), self.dev),
            "pos": [torch.zeros((S, 2, R + 1, 3), **f64), torch.zeros((S, 2, R + 1, 3), **f64)],
            "circ": [torch.zeros((S, R), **f64), torch.zeros((S, R), **f64)],
            "cur": 0,    # current buffer of "pos"
            "ccur": 0,   # current buffer of "circ"
            "implicit": torch.zeros((self.P, S), **f64),
            "node_vel": torch.zeros((S, 2, R, 3), **f64),
            "line_gamma": torch.zeros(max(wmesh.n_lines, 1), **f64),
            "time": float(w.time),
            "step_count": 0,
        }

    def _workspace_bytes(self) -> int:
        L = self.mesh.n_lines
        need = [
            _lib.query("pvl_segments_workspace", L, _lib.PVL_F64),
            _lib.query("pvl_lu_workspace", self.N),
            _lib.query("pvl_lu_solve_workspace", self.N),
        ]
        if self.wake is not None:
            w = self.wake
            Lw = w["mesh"].n_lines
            need += [
                _lib.query("pvl_segments_workspace", Lw, _lib.PVL_F64),
                _lib.query("pvl_line_velocity_workspace", Lw, self.P, _lib.PVL_F64),
                _lib.query("pvl_wake_node_velocity_workspace", L, w["S"], w["R"], _lib.PVL_F64),
            ]
        return max(need) + 256

    # ------------------------------------------------------------------ state access
    @property
    def wake_positions(self) -> torch.Tensor:
        return self.wake["pos"][self.wake["cur"]]

    @property
    def wake_circulation(self) -> torch.Tensor:
        return self.wake["circ"][self.wake["ccur"]]

    def set_wake_state(self, positions, circulation, step_count: int, time: float) -> None:
        """Load a wake state (e.g. from WakeModelLineExplicitUnsteady.save/load)."""
        w = self.wake
        w["pos"][w["cur"]].copy_(to_device(positions).reshape(w["pos"][0].shape))
        w["circ"][w["ccur"]].copy_(to_device(circulation).reshape(w["circ"][0].shape))
        w["step_count"] = int(step_count)
        w["time"] = float(time)

    # ------------------------------------------------------------------ the step
    def load_inputs(self, positions, velocities) -> None:
        """Copy this step's body positions/velocities to the device (pinned, async)."""
        for host, dev, src in ((self.h_pos, self.pos, positions), (self.h_vel, self.vel, velocities)):
            if isinstance(src, torch.Tensor) and src.is_cuda:
                dev.copy_(src.reshape(dev.shape))
            else:
                host.numpy()[...] = np.asarray(src, np.float64).reshape(host.shape)
                dev.copy_(host, non_blocking=True)

    def assemble_body_only(self) -> None:
        """Control points, normals, RHS for a uniform stream and the body matrix."""
        s = stream_ptr()
        d, P = self.d_body, self.P
        msh = self.mesh
        _lib.call("pvl_surface_average", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.pos), ptr(self.cps), s)
        _lib.call("pvl_surface_average", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.vel), ptr(self.cpv), s)
        _lib.call("pvl_surface_normal", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.pos), ptr(self.nrm), s)
        u = self.u_inf
        _lib.call("pvl_rhs", P, ptr(self.nrm), None, float(u[0]), float(u[1]), float(u[2]), ptr(self.cpv),
                  ptr(self.rhs), s)
        ws, nb = ptr(self.ws), self._ws_bytes
        _lib.call("pvl_induction_normal", _lib.PVL_F64, msh.n_points, msh.n_lines, ptr(d["lines"]), ptr(self.pos), P,
                  ptr(d["offsets"]), ptr(d["surface_lines"]), P, ptr(self.cps), ptr(self.nrm), self.tol, ptr(self.A),
                  self.N, ws, nb, s)

    def border(self) -> None:
        """Zero-mean rows/columns of the closed bodies (bordered system)."""
        if self.m:
            _lib.call("pvl_border_groups", self.P, self.m, ptr(self.goff), ptr(self.A), self.N, ptr(self.rhs),
                      stream_ptr())

    def assemble(self) -> None:
        """The corrected system of this iteration (solver.py:194-220)."""
        self.assemble_body_only()
        if self.wake is not None and self.iteration > 0:
            self._wake_corrections()
        self.border()

    def _wake_corrections(self) -> None:
        """Implicit first row into A, explicit rows into the RHS (wake_models.py:199-223)."""
        s = stream_ptr()
        w = self.wake
        S, R = w["S"], w["R"]
        wm, wd = w["mesh"], w["d"]
        wpos = self.wake_positions.reshape(-1, 3)
        ws, nb = ptr(self.ws), self._ws_bytes
        _lib.call("pvl_induction_normal", _lib.PVL_F64, wm.n_points, wm.n_lines, ptr(wd["lines"]), ptr(wpos), S,
                  ptr(w["off0"]), ptr(w["sl0"]), self.P, ptr(self.cps), ptr(self.nrm), self.tol, ptr(w["implicit"]),
                  S, ws, nb, s)
        _lib.call("pvl_wake_fold_implicit", self.P, S, ptr(w["implicit"]), ptr(w["adj"]), ptr(self.A), self.N, s)
        if R > 1:
            _lib.call("pvl_line_circulation", wm.n_lines, ptr(wd["map_offsets"]), ptr(wd["map_entries"]),
                      ptr(self.wake_circulation), R, ptr(w["line_gamma"]), s)
            _lib.call("pvl_line_velocity", _lib.PVL_F64, wm.n_points, wm.n_lines, ptr(wd["lines"]), ptr(wpos),
                      ptr(w["line_gamma"]), self.P, ptr(self.cps), ptr(self.nrm), self.tol, 1.0, 1.0, ptr(self.rhs),
                      ws, nb, s)

    def solve(self) -> None:
        s = stream_ptr()
        ws, nb = ptr(self.ws), self._ws_bytes
        _lib.call("pvl_lu_factor", self.N, ptr(self.A), self.N, ptr(self.ipiv), ptr(self.info), ws, nb, s)
        _lib.call("pvl_lu_solve", self.N, ptr(self.A), self.N, ptr(self.ipiv), ptr(self.rhs), ptr(self.err), ws, nb, s)
        self.gamma.copy_(self.rhs[: self.P])
        if self.m:
            _lib.call("pvl_group_mean_remove", self.m, ptr(self.goff), ptr(self.gamma), s)

    def wake_update(self, time: float) -> None:
        """Advance the wake to `time` (wake_models.py:111-157)."""
        s = stream_ptr()
        w = self.wake
        S, R = w["S"], w["R"]
        dt = float(time) - w["time"]
        w["time"] = float(time)
        if w["step_count"] == 0:
            # first update: pin row 0 to the trailing edge before it is advected
            self._advect(0, 0.0)
            w["step_count"] = 1
        complete = min(w["step_count"], R)
        msh, d = self.mesh, self.d_body
        _lib.call("pvl_line_circulation", msh.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(self.gamma), 0,
                  ptr(self.body_line_gamma), s)
        u = self.u_inf
        _lib.call("pvl_wake_node_velocity", _lib.PVL_F64, msh.n_points, msh.n_lines, ptr(d["lines"]), ptr(self.pos),
                  ptr(self.body_line_gamma), S, R, complete, ptr(self.wake_positions), float(u[0]), float(u[1]),
                  float(u[2]), self.tol, ptr(w["node_vel"]), ptr(self.ws), self._ws_bytes, s)
        self._advect(complete, dt)
        c = w["ccur"]
        _lib.call("pvl_wake_shed", S, R, ptr(w["circ"][c]), ptr(w["adj"]), ptr(self.gamma), ptr(w["circ"][1 - c]), s)
        w["ccur"] = 1 - c
        w["step_count"] += 1

    def _advect(self, complete: int, dt: float) -> None:
        s = stream_ptr()
        w = self.wake
        cur = w["cur"]
        _lib.call("pvl_wake_advect", w["S"], w["R"], complete, ptr(w["pos"][cur]), ptr(w["node_vel"]), dt,
                  ptr(self.pos), ptr(w["bn"]), ptr(w["pos"][1 - cur]), s)
        w["cur"] = 1 - cur

    def step(self, time: float, positions, velocities) -> torch.Tensor:
        """One solver iteration at `time`; returns the ring circulations (device tensor)."""
        self.load_inputs(positions, velocities)
        self.assemble()
        self.solve()
        if self.wake is not None:
            self.wake_update(time)
        self.iteration += 1
        return self.gamma

    def gamma_host(self) -> np.ndarray:
        self.h_gamma.copy_(self.gamma, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_gamma.numpy().copy()

    def check_status(self) -> None:
        """Raise if the last solve reported a zero pivot or a timed-out wait."""
        info, err = int(self.info.item()), int(self.err.item())
        if err:
            raise _lib.PvlError(_lib.PVL_ERR_TIMEOUT, "a wavefront wait in the triangular solve timed out")
        if info:
            raise _lib.PvlError(_lib.PVL_ERR_SINGULAR, f"exactly singular system: U[{info - 1},{info - 1}] == 0")
