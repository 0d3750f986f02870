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
                                                            -> pvl_induction_normal_tiled on
   the first-row rings, pvl_wake_fold_implicit, pvl_line_circulation + pvl_line_velocity over the
   lines of the rows shed so far
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

import ctypes
from collections import deque
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .cvl import INVALID_ID, Mesh
from .device import ptr, require_cuda, stream_ptr, to_device, to_device_u32

# pvl_gmres_status (include/pvl_b200.h) and the number of solves whose status may be in flight
_GMRES_STATUS = np.dtype([("iterations", "<u4"), ("converged", "<u4"), ("initial_rel_residual", "<f8"),
                          ("final_rel_residual", "<f8")])
_STATUS_RING = 4  # at most one record is pending when a solve is launched
_HOST_RING = 4    # pinned result buffers of gamma_host_async


class HostResult:
    """A device-to-host copy in flight (SolverEngine.gamma_host_async)."""

    def __init__(self, buf: torch.Tensor, event: torch.cuda.Event):
        self._buf, self._event = buf, event

    def result(self) -> np.ndarray:
        self._event.synchronize()
        return self._buf.numpy().copy()


def wake_ring_connectivity(line_rows: int, n_shed: int, bordering_nodes=None) -> np.ndarray:
    """Rings of the wake strips: strip s, row r -> nodes (s,0,r), (s,1,r), (s,1,r+1), (s,0,r+1).

    Same node numbering and ring order as the reference's wake mesh
    (python/pyvl/wake_models.py:35-52), so wake ring s*line_rows + r holds circulation[s, r].
    With ``bordering_nodes`` ((n_shed, 2) body node ids), node columns that start at the same
    body node -- the shared trailing-edge node of adjacent strips -- are referenced through
    one representative column (``wake_node_columns``).  Those columns hold bitwise identical
    positions at every step (same start, same advection), so the two coincident streamwise
    segments of neighbouring strips become one line carrying the difference of the two
    strips' circulations: the same induced velocity in exact arithmetic with a third fewer
    wake lines.
    """
    npr = line_rows + 1
    r = np.arange(line_rows, dtype=np.uint64)
    base = (2 * npr * np.arange(n_shed, dtype=np.uint64))[:, None]
    rc = np.empty((n_shed, line_rows, 4), np.uint64)
    rc[:, :, 0] = r + base
    rc[:, :, 1] = r + npr + base
    rc[:, :, 2] = r + npr + 1 + base
    rc[:, :, 3] = r + 1 + base
    rc = rc.reshape(-1, 4)
    if bordering_nodes is not None:
        rep, _, _ = wake_node_columns(bordering_nodes)
        col, row = rc // npr, rc % npr
        rc = rep.astype(np.uint64)[col] * npr + row
    return rc.astype(np.uint32)


def wake_node_columns(bordering_nodes):
    """Node columns (strip side s*2 + side) of the wake that start at the same body node.

    Returns (rep, cols, slot): rep[c] the first column with column c's body node, cols the
    distinct representatives in ascending order and slot[c] the position of rep[c] in cols.
    """
    bn = np.asarray(bordering_nodes, np.int64).reshape(-1)
    first = {}
    rep = np.empty(bn.size, np.int64)
    for c, node in enumerate(bn):
        rep[c] = first.setdefault(int(node), c)
    cols = np.unique(rep)
    slot = np.searchsorted(cols, rep)
    return rep, cols.astype(np.uint32), slot.astype(np.uint32)


# midpoint value of the quintic through six equally spaced samples at -5, -3, -1, +1, +3, +5
_MID6 = ((-5, 3.0 / 256), (-3, -25.0 / 256), (-1, 150.0 / 256), (1, 150.0 / 256), (3, -25.0 / 256), (5, 3.0 / 256))


def _midpoint_rules(n: int) -> list:
    """Per sample of a smooth run of n: [(sample, weight), ...].  Odd samples with five samples
    on either side take the quintic midpoint rule of their even neighbours, the rest are
    evaluated ([(itself, 1.0)])."""
    return [[(j + o, w) for o, w in _MID6] if j % 2 and 5 <= j <= n - 6 else [(j, 1.0)] for j in range(n)]


def far_wake_stencil(n_rings: int, patches) -> dict:
    """Where the far wake term is evaluated and how the other control points get it.

    ``patches``: (ring0, n_span, n_chord) blocks of rings ring0 + i * n_chord + j whose control
    points (and normals) are smooth functions of (i, j) — a kink, e.g. a twist linear in |y|,
    splits a wing into two patches.  Rings outside every patch are always evaluated.  Two
    bands: in the chord band a point takes its chordwise rule (``_midpoint_rules`` along j), in
    the span band the product of its spanwise and chordwise rules.  Returns ``index`` (rings to
    gather: the span band's evaluated rings first, n_span_eval of them, then the rest of the
    chord band's, n_chord_eval in all) and the CSR stencil (offsets, entries, weights) over the
    values [chord band at the n_chord_eval points; span band at the first n_span_eval]: ring p
    receives sum_k weights[k] values[entries[k]] in both bands together.
    """
    chord_rule = [[(p, 1.0)] for p in range(n_rings)]
    span_rule = [[(p, 1.0)] for p in range(n_rings)]
    owner = np.full(n_rings, -1, np.int64)
    for k, (r0, ns, nc) in enumerate(patches):
        r0, ns, nc = int(r0), int(ns), int(nc)
        if r0 < 0 or ns <= 0 or nc <= 0 or r0 + ns * nc > n_rings:
            raise ValueError(f"patch {k} ({r0}, {ns}, {nc}) outside the {n_rings} rings")
        blk = owner[r0:r0 + ns * nc]
        if (blk >= 0).any():
            raise ValueError(f"patch {k} overlaps another patch")
        blk[:] = k
        cr, sr = _midpoint_rules(nc), _midpoint_rules(ns)
        for i in range(ns):
            for j in range(nc):
                p = r0 + i * nc + j
                chord_rule[p] = [(r0 + i * nc + jj, w) for jj, w in cr[j]]
                span_rule[p] = [(r0 + ii * nc + j, w) for ii, w in sr[i]]
    chord_eval = np.array([len(r) == 1 for r in chord_rule])
    both_eval = chord_eval & np.array([len(r) == 1 for r in span_rule])
    index = np.concatenate([np.nonzero(both_eval)[0], np.nonzero(chord_eval & ~both_eval)[0]])
    pos = np.full(n_rings, -1, np.int64)
    pos[index] = np.arange(index.size)
    n_chord, n_span = int(index.size), int(both_eval.sum())
    offsets = np.zeros(n_rings + 1, np.int64)
    entries, weights = [], []
    for p in range(n_rings):
        terms = [(int(pos[q]), w) for q, w in chord_rule[p]]
        for q, ws in span_rule[p]:
            terms += [(n_chord + int(pos[qq]), ws * wc) for qq, wc in chord_rule[q]]
        entries += [e for e, _ in terms]
        weights += [w for _, w in terms]
        offsets[p + 1] = len(entries)
    return {"index": index.astype(np.uint32), "n_chord_eval": n_chord, "n_span_eval": n_span,
            "offsets": offsets.astype(np.uint32), "entries": np.asarray(entries, np.uint32),
            "weights": np.asarray(weights, np.float64)}


def column_stencil(n_cols: int, runs) -> dict:
    """Which wake node columns the far-row advection evaluates and how the others get theirs.

    ``runs``: (col0, n) runs of consecutive node columns (in the de-duplicated column order)
    whose wake nodes are smooth functions of the column index; runs may share their end
    columns only (the trailing-edge node at a kink).  Odd columns of a run with five columns
    on either side take the quintic midpoint rule of their even neighbours (_midpoint_rules);
    the rest are evaluated.  Returns ``sub`` (the evaluated columns, ascending) and the CSR
    rule of every column over positions in ``sub`` (offsets, entries, weights)."""
    count = np.zeros(n_cols, np.int64)
    runs = [(int(c0), int(n)) for c0, n in runs]
    for c0, n in runs:
        if c0 < 0 or n <= 0 or c0 + n > n_cols:
            raise ValueError(f"column run ({c0}, {n}) outside the {n_cols} node columns")
        count[c0:c0 + n] += 1
    rules = [[(c, 1.0)] for c in range(n_cols)]
    for c0, n in runs:
        for j, r in enumerate(_midpoint_rules(n)):
            if len(r) > 1:
                if count[c0 + j] > 1:
                    raise ValueError(f"column runs overlap at column {c0 + j}, inside a run")
                rules[c0 + j] = [(c0 + jj, w) for jj, w in r]
    sub = np.array([c for c in range(n_cols) if len(rules[c]) == 1], np.int64)
    pos = np.full(n_cols, -1, np.int64)
    pos[sub] = np.arange(sub.size)
    offsets = np.zeros(n_cols + 1, np.int64)
    entries, weights = [], []
    for c in range(n_cols):
        entries += [int(pos[q]) for q, _ in rules[c]]
        weights += [w for _, w in rules[c]]
        offsets[c + 1] = len(entries)
    return {"sub": sub, "offsets": offsets.astype(np.uint32), "entries": np.asarray(entries, np.uint32),
            "weights": np.asarray(weights, np.float64)}


def _node_velocity_workspace(n_lines: int, n_cols: int, rows: int, precision: int) -> int:
    """Largest sweep workspace over every row count 1..rows the growing wake passes through."""
    return max(_lib.query("pvl_line_velocity_workspace", n_lines, n_cols * c, precision) for c in range(1, rows + 1))


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
                 closed_groups: list[tuple[int, int]] | None = None, wake_self_induction: bool = False):
        self.dev = require_cuda()
        # off by default (the reference's wake moves with the freestream and the body only)
        self.wake_self_induction = bool(wake_self_induction)
        self.mesh = mesh
        self.tol = float(tol)
        self.u_inf = np.asarray(freestream, np.float64).reshape(3)
        self.P = mesh.n_surfaces
        self.groups = [(int(a), int(b)) for a, b in (closed_groups or []) if b > a]
        self.m = len(self.groups)
        self.N = self.P + self.m
        self.iteration = 0
        # pieces of a step that touch only fixed buffers run as CUDA graphs captured on first use
        # (one replay instead of a launch per kernel from Python)
        self.capture_steps = True
        self._step_graphs: dict = {}
        self.replayed_kernels = 0  # this library's kernels run by those replays
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
        # set by the RHS kernel when a NaN or infinity reaches the system; held until check_status
        self.nonfinite = torch.zeros(1, dtype=torch.int32, device=self.dev)
        if self.m:
            goff = np.array([a for a, _ in self.groups] + [self.groups[-1][1]], np.uint32)
            contiguous = all(self.groups[i][1] == self.groups[i + 1][0] for i in range(self.m - 1))
            if not contiguous:
                raise ValueError("closed groups must be contiguous ranges of rings")
            self.goff = to_device_u32(goff, self.dev)
        self.wake = None
        self._far = None  # far-wake stencil of the explicit wake term (MixedSolverEngine cp_patches)
        if wake is not None:
            self._init_wake(wake)
        self._ws_bytes = self._workspace_bytes()
        self.ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=self.dev)
        self.h_pos = torch.empty((mesh.n_points, 3), dtype=torch.float64, pin_memory=True)
        self.h_vel = torch.empty((mesh.n_points, 3), dtype=torch.float64, pin_memory=True)
        self.h_gamma = torch.empty(self.P, dtype=torch.float64, pin_memory=True)
        self._h2d_done = None  # event after the last copy out of h_pos / h_vel

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
        wmesh = Mesh(2 * (R + 1) * S, wake_ring_connectivity(R, S, bn))
        _, cols, slot = wake_node_columns(bn)
        valid = adj[adj != INVALID_ID]
        # each ring adjacent to at most one shedding line side: the fold may run in parallel
        self._fold_fn = ("pvl_wake_fold_implicit_distinct" if np.unique(valid).size == valid.size
                         else "pvl_wake_fold_implicit")
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.wake = {
            "S": S, "R": R, "mesh": wmesh, "d": wmesh.device_arrays(),
            "adj": to_device_u32(adj.astype(np.uint32), self.dev),
            "bn": to_device_u32(bn.astype(np.uint32), self.dev),
            "pos": [torch.zeros((S, 2, R + 1, 3), **f64), torch.zeros((S, 2, R + 1, 3), **f64)],
            "circ": [torch.zeros((S, R), **f64), torch.zeros((S, R), **f64)],
            "cur": 0,    # current buffer of "pos"
            "ccur": 0,   # current buffer of "circ"
            "implicit": torch.zeros((self.P, S), **f64),
            "cols": to_device_u32(cols, self.dev),
            "slot": to_device_u32(slot, self.dev),
            "n_cols": int(cols.size),
            "node_vel": torch.zeros((int(cols.size), R, 3), **f64),
            "self_line_gamma": torch.zeros(max(wmesh.n_lines, 1), **f64),
            "node_vel_self": torch.zeros((int(cols.size), R, 3), **f64),
            "time": float(w.time),
            "step_count": 0,
        }
        # The explicit wake term runs over the same wake in row-major ring order (ring r*S + s):
        # lines are then numbered row band by row band, so the lines of rows < k are the first
        # lines_upto[k], and a wake that has shed k rows is swept over that prefix only (rows
        # not yet shed carry no circulation).  Its first S rings are row 0, the implicit block.
        rc = wake_ring_connectivity(R, S, bn).reshape(S, R, 4).transpose(1, 0, 2).reshape(-1, 4)
        rm = Mesh(2 * (R + 1) * S, rc)
        off_rm, ids = rm.surface_offsets, (rm.surface_lines & 0x7FFFFFFF).astype(np.int64)
        run = np.maximum.accumulate(ids) + 1
        self.wake.update({
            "rm": rm, "rm_d": rm.device_arrays(),
            "lines_upto": [0] + [int(run[int(off_rm[k * S]) - 1]) for k in range(1, R + 1)],
            "circ_rs": torch.zeros((R, S), **f64),
            "rm_line_gamma": torch.zeros(max(rm.n_lines, 1), **f64),
        })
        self.n_near_lines = rm.n_lines  # lines of the explicit term evaluated in FP64 (all)

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
                _node_velocity_workspace(L, w["n_cols"], w["R"], _lib.PVL_F64),
            ]
            if self.wake_self_induction:
                need.append(_node_velocity_workspace(Lw, w["n_cols"], w["R"], _lib.PVL_F64))
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
        """Copy this step's body positions/velocities to the device (pinned, async).

        The pinned staging buffers are reused every step: before one is overwritten, the host
        waits until the device has consumed the previous copy out of it (otherwise a host that
        runs steps ahead of the device would hand a pending copy the next step's data)."""
        if self._h2d_done is not None:
            self._h2d_done.synchronize()
            self._h2d_done = None
        staged = False
        for host, dev, src in ((self.h_pos, self.pos, positions), (self.h_vel, self.vel, velocities)):
            if isinstance(src, torch.Tensor) and src.is_cuda:
                dev.copy_(src.reshape(dev.shape))
            else:
                host.numpy()[...] = np.asarray(src, np.float64).reshape(host.shape)
                dev.copy_(host, non_blocking=True)
                staged = True
        if staged:
            self._h2d_done = torch.cuda.Event()
            self._h2d_done.record()

    def captured(self, key, fn, store: dict | None = None) -> None:
        """Run ``fn`` (launches on fixed buffers only, no host reads) as the CUDA graph captured
        under ``key`` on its first use (kept in ``store``, by default the engine's own table);
        directly when ``capture_steps`` is off."""
        if not self.capture_steps:
            fn()
            return
        graphs = self._step_graphs if store is None else store
        entry = graphs.get(key)
        if entry is None:
            n0 = _lib.lib().pvl_launch_count()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn()
            entry = (g, int(_lib.lib().pvl_launch_count() - n0))
            graphs[key] = entry
        entry[0].replay()
        self.replayed_kernels += entry[1]

    def assemble_body_only(self, buf: dict | None = None) -> None:
        """Control points, normals, RHS for a uniform stream and the body matrix (into ``buf``,
        a set of pos/vel/cps/cpv/nrm/rhs/A/ws buffers, or the engine's own: then as one
        captured graph)."""
        if buf is None:
            self.captured("body", lambda: self._assemble_body(None))
        else:
            self._assemble_body(buf)

    def _assemble_body(self, buf: dict | None) -> None:
        s = stream_ptr()
        d, P = self.d_body, self.P
        msh = self.mesh
        b = buf or {"pos": self.pos, "vel": self.vel, "cps": self.cps, "cpv": self.cpv, "nrm": self.nrm,
                    "rhs": self.rhs, "A": self.A, "ws": self.ws}
        _lib.call("pvl_surface_average", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(b["pos"]), ptr(b["cps"]), s)
        _lib.call("pvl_surface_average", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(b["vel"]), ptr(b["cpv"]), s)
        _lib.call("pvl_surface_normal", P, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(b["pos"]), ptr(b["nrm"]), s)
        u = self.u_inf
        _lib.call("pvl_rhs", P, ptr(b["nrm"]), None, float(u[0]), float(u[1]), float(u[2]), ptr(b["cpv"]),
                  ptr(b["rhs"]), ptr(self.nonfinite), s)
        ws = b["ws"]
        _lib.call("pvl_induction_normal_tiled", msh.n_points, msh.n_lines, ptr(d["lines"]), ptr(b["pos"]), P,
                  ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["tile_offsets"]), ptr(d["tile_lines"]),
                  ptr(d["sl_local"]), d["tile_max"], P, ptr(b["cps"]), ptr(b["nrm"]), self.tol, ptr(b["A"]), self.N,
                  ptr(ws), ws.numel(), s)

    def border(self) -> None:
        """Zero-mean rows/columns of the closed bodies (bordered system)."""
        if self.m:
            _lib.call("pvl_border_groups", self.P, self.m, ptr(self.goff), ptr(self.A), self.N, ptr(self.rhs),
                      stream_ptr())

    def assemble(self) -> None:
        """The corrected system of this iteration (solver.py:194-220)."""
        self.assemble_body_only()
        if self.wake is not None and self.iteration > 0:
            self._wake_terms()
        self.border()

    def _wake_full(self) -> bool:
        """The wake has all its rows: every launch of a wake phase then depends only on which
        of the double-buffered positions and circulations are current."""
        return self.capture_steps and self.wake["step_count"] >= self.wake["R"]

    def _wake_terms(self) -> None:
        """_wake_corrections, as a captured graph per (positions, circulations) buffer pair once
        the wake is full (while it grows every step has other sizes)."""
        w = self.wake
        if self._wake_full():
            self.captured(("wake_terms", w["cur"], w["ccur"]), self._wake_corrections)
        else:
            self._wake_corrections()

    def _wake_corrections(self, fp64_only: bool = False) -> None:
        """Implicit first row into A, explicit rows into the RHS (wake_models.py:199-223).

        Both over the row-major wake: the implicit block is its first S rings (row 0 of every
        strip, in strip order) at the control points, folded into the columns of the rings
        that shed them; the explicit term sweeps the lines of the rows shed so far with the
        line circulations of rows >= 1, in FP64 for the first ``n_near_lines`` lines and in
        FP32 beyond (all FP64 unless a subclass says otherwise, or with ``fp64_only``).  With a
        far-wake stencil (``_far``, the mixed engine's ``cp_patches``) and not ``fp64_only``, the
        rows from its chord row on are evaluated at part of the control points only."""
        s = stream_ptr()
        w = self.wake
        S, R = w["S"], w["R"]
        rm, d = w["rm"], w["rm_d"]
        wpos = self.wake_positions.reshape(-1, 3)
        ws, nb = ptr(self.ws), self._ws_bytes
        # the implicit block needs the segments of row 0's lines only (the first lines_upto[1])
        _lib.call("pvl_induction_normal_tiled", rm.n_points, w["lines_upto"][1], ptr(d["lines"]), ptr(wpos), S,
                  ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["tile_offsets"]), ptr(d["tile_lines"]),
                  ptr(d["sl_local"]), d["tile_max"], self.P, ptr(self.cps), ptr(self.nrm), self.tol,
                  ptr(w["implicit"]), S, ws, nb, s)
        _lib.call(self._fold_fn, self.P, S, ptr(w["implicit"]), ptr(w["adj"]), ptr(self.A), self.N, s)
        active = w["lines_upto"][min(w["step_count"], R)]
        if R <= 1 or active == 0:
            return
        crs = w["circ_rs"]
        crs.copy_(self.wake_circulation.t())
        crs[0].zero_()  # row 0 is implicit
        lg = w["rm_line_gamma"]
        _lib.call("pvl_line_circulation", rm.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(crs), 0,
                  ptr(lg), s)
        far = None if fp64_only else self._far
        if far is not None and min(w["step_count"], R) > far["chord_row"]:
            self._far_wake_term(active, lg, wpos, s)
            return
        near = active if fp64_only else min(self.n_near_lines, active)
        lines = d["lines"]
        _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, near, ptr(lines), ptr(wpos), ptr(lg), self.P,
                  ptr(self.cps), ptr(self.nrm), self.tol, 1.0, 1.0, ptr(self.rhs), ws, nb, s)
        if active > near:
            _lib.call("pvl_line_velocity", _lib.PVL_F32, rm.n_points, active - near, lines.data_ptr() + 8 * near,
                      ptr(wpos), lg.data_ptr() + 8 * near, self.P, ptr(self.cps), ptr(self.nrm), self.tol, 1.0, 1.0,
                      ptr(self.rhs), ws, nb, s)

    def _far_wake_term(self, active: int, lg: torch.Tensor, wpos: torch.Tensor, s) -> None:
        """The explicit wake term with the far rows interpolated across the control points.

        Rows below the chord row: every control point, into the RHS.  Rows from the chord row to
        the span row: velocities at the chord band's evaluated points; rows beyond: at the span
        band's (a prefix of the same gathered points); then every RHS entry takes its stencil of
        the two (pvl_stencil_normal_add)."""
        f, w = self._far, self.wake
        rm, d = w["rm"], w["rm_d"]
        lines, up = d["lines"], w["lines_upto"]
        a = up[f["chord_row"]]
        b = active if f["span_row"] is None else max(a, min(up[f["span_row"]], active))
        ws, nb = ptr(self.ws), self._ws_bytes
        n_c, n_s = f["n_chord_eval"], f["n_span_eval"]
        pts, vals = f["pts"], f["vals"]
        _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, a, ptr(lines), ptr(wpos), ptr(lg), self.P,
                  ptr(self.cps), ptr(self.nrm), self.tol, 1.0, 1.0, ptr(self.rhs), ws, nb, s)
        _lib.call("pvl_gather_points", n_c, ptr(f["index"]), self.P, ptr(self.cps), ptr(pts), s)
        _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, b - a, lines.data_ptr() + 8 * a, ptr(wpos),
                  lg.data_ptr() + 8 * a, n_c, ptr(pts), None, self.tol, 1.0, 0.0, ptr(vals), ws, nb, s)
        _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, active - b, lines.data_ptr() + 8 * b, ptr(wpos),
                  lg.data_ptr() + 8 * b, n_s, ptr(pts), None, self.tol, 1.0, 0.0, vals.data_ptr() + 24 * n_c,
                  ws, nb, s)
        _lib.call("pvl_stencil_normal_add", self.P, ptr(f["offsets"]), f["entries"].numel(), ptr(f["entries"]),
                  ptr(f["weights"]), n_c + n_s, ptr(vals), ptr(self.nrm), ptr(self.rhs), s)

    def solve(self) -> None:
        ws, nb = ptr(self.ws), self._ws_bytes
        # the factorisation's ~5 launches per 64-column panel run as one captured graph (fixed buffers)
        self.captured(("lu", ws, nb), lambda: _lib.call("pvl_lu_factor", self.N, ptr(self.A), self.N, ptr(self.ipiv),
                                                        ptr(self.info), ws, nb, stream_ptr()))
        _lib.call("pvl_lu_solve", self.N, ptr(self.A), self.N, ptr(self.ipiv), ptr(self.rhs), ptr(self.err), ws, nb,
                  stream_ptr())
        self.gamma.copy_(self.rhs[: self.P])
        if self.m:
            _lib.call("pvl_group_mean_remove", self.m, ptr(self.goff), ptr(self.gamma), stream_ptr())

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
        _lib.call("pvl_wake_node_velocity_cols", _lib.PVL_F64, msh.n_points, msh.n_lines, ptr(d["lines"]),
                  ptr(self.pos), ptr(self.body_line_gamma), S, R, complete, 0, complete, w["n_cols"], ptr(w["cols"]),
                  ptr(self.wake_positions), float(u[0]), float(u[1]), float(u[2]), self.tol, ptr(w["node_vel"]),
                  ptr(self.ws), self._ws_bytes, s)
        if self.wake_self_induction:
            self._add_wake_self_velocity(complete)
        self._advect(complete, dt)
        c = w["ccur"]
        _lib.call("pvl_wake_shed", S, R, ptr(w["circ"][c]), ptr(w["adj"]), ptr(self.gamma), ptr(w["circ"][1 - c]), s)
        w["ccur"] = 1 - c
        w["step_count"] += 1

    def _add_wake_self_velocity(self, complete: int) -> None:
        """node_vel += the velocity the whole wake (every row, row 0 included) induces at the
        advecting nodes, from the wake as it is before this update (FP64).  An option: the
        reference's wake_models.py:113-137 moves the wake with the freestream and the body only."""
        s = stream_ptr()
        w = self.wake
        S, R = w["S"], w["R"]
        wm, wd = w["mesh"], w["d"]
        _lib.call("pvl_line_circulation", wm.n_lines, ptr(wd["map_offsets"]), ptr(wd["map_entries"]),
                  ptr(self.wake_circulation), 0, ptr(w["self_line_gamma"]), s)
        _lib.call("pvl_wake_node_velocity_cols", _lib.PVL_F64, wm.n_points, wm.n_lines, ptr(wd["lines"]),
                  ptr(self.wake_positions.reshape(-1, 3)), ptr(w["self_line_gamma"]), S, R, complete, 0, complete,
                  w["n_cols"], ptr(w["cols"]), ptr(self.wake_positions), 0.0, 0.0, 0.0, self.tol,
                  ptr(w["node_vel_self"]), ptr(self.ws), self._ws_bytes, s)
        _lib.call("pvl_axpy_f64", w["n_cols"] * complete * 3, 1.0, ptr(w["node_vel_self"]), ptr(w["node_vel"]), s)

    def _advect(self, complete: int, dt: float) -> None:
        s = stream_ptr()
        w = self.wake
        cur = w["cur"]
        _lib.call("pvl_wake_advect_cols", w["S"], w["R"], complete, ptr(w["pos"][cur]), ptr(w["node_vel"]),
                  ptr(w["slot"]), w["n_cols"], dt, ptr(self.pos), ptr(w["bn"]), ptr(w["pos"][1 - cur]), s)
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

    def gamma_host_async(self) -> "HostResult":
        """Start copying this step's circulations to the host and return at once; the returned
        object's ``result()`` waits for that copy only.  A caller can enqueue the next step
        before reading this one, so the GPU does not idle while the host reads the result.
        Results come from a small ring of pinned buffers: read each one before starting more
        than ``_HOST_RING - 1`` further copies."""
        if not hasattr(self, "_h_ring"):
            self._h_ring = [torch.empty(self.P, dtype=torch.float64, pin_memory=True) for _ in range(_HOST_RING)]
            self._h_next = 0
        buf = self._h_ring[self._h_next]
        self._h_next = (self._h_next + 1) % _HOST_RING
        buf.copy_(self.gamma, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        return HostResult(buf, ev)

    def check_status(self) -> None:
        """Raise if a step since the last check met a NaN or infinity in its inputs, or if the
        last solve reported a zero pivot or a timed-out wait (one host synchronisation)."""
        info, err, bad = (int(v) for v in torch.cat([self.info, self.err, self.nonfinite]).tolist())
        if bad:
            self.nonfinite.zero_()
            raise _lib.PvlError(_lib.PVL_ERR_NONFINITE,
                                "a NaN or infinity reached the right-hand side (positions, velocities or stream)")
        if err:
            raise _lib.PvlError(_lib.PVL_ERR_TIMEOUT, "a wavefront wait in the triangular solve timed out")
        if info:
            raise _lib.PvlError(_lib.PVL_ERR_SINGULAR, f"exactly singular system: U[{info - 1},{info - 1}] == 0")


class RefreshPolicy:
    """When the mixed solve rebuilds its FP32 preconditioner, from the Krylov iteration counts
    of the solves since the last rebuild (host logic only).

    A rebuild is due every ``period`` steps when that is set; otherwise, with no rebuild in
    flight and at least two steps since the last one, when the latest solve needed
    ``on_iters`` iterations and at least 3 more than the fewest since the last rebuild (a
    stale preconditioner), or when the iterations above that fewest count add up to
    ``excess`` (a preconditioner that costs one extra column per step is kept for a while: a
    rebuild costs as much as a few hundred columns)."""

    def __init__(self, on_iters: int, excess: int, period: int | None = None):
        self.on_iters = int(on_iters)
        self.excess_limit = int(excess)
        self.period = None if period is None else int(period)
        self.best: int | None = None  # fewest iterations of a solve since the last rebuild
        self.excess = 0               # iterations above that since the last rebuild
        self.last: int | None = None  # the latest solve's count

    def observe(self, counts) -> None:
        """Take the iteration counts of further solves, in order."""
        for k in counts:
            k = int(k)
            self.best = k if self.best is None else min(self.best, k)
            self.excess += k - self.best
            self.last = k

    def rebuilt(self) -> None:
        self.best = None
        self.excess = 0

    def due(self, steps_since_rebuild: int, idle: bool) -> bool:
        if self.period is not None and steps_since_rebuild >= self.period:
            return True
        slow = self.last is not None and self.last >= self.on_iters and (
            self.best is None or self.last >= self.best + 3)
        return idle and steps_since_rebuild >= 2 and (slow or self.excess >= self.excess_limit)


class MixedSolverEngine(SolverEngine):
    """The mixed-precision step: the FP64 system solved to FP64 accuracy with cheaper arithmetic.

    * Body matrix, implicit wake row and every residual stay FP64.
    * The solve is right-preconditioned GMRES with FP64 vectors and FP64 residuals against the
      FP64 matrix.  The preconditioner is the explicit inverse of an FP32 LU factorisation of
      the system (trailing updates and the triangular inversion's rank-64 updates on the
      tensor cores in TF32, pvl_lu32_factor / pvl_lu32_inverse), applied as one FP32
      matrix-vector product per iteration.  It is rebuilt (on a side stream while the steps go
      on) when it has gone stale: at once when a solve needed ``refresh_on_iters`` iterations
      and at least 3 more than the best count since the last rebuild, or when the iterations
      above that best count add up to ``refresh_excess`` (a rebuild costs as much as a few
      hundred Krylov columns, so a preconditioner that costs one extra column per step is kept
      for a while), and in any case every ``refresh`` steps when that is set.  If GMRES has not reached ``gmres_tol``
      (relative residual) after ``max_iter`` iterations the step falls back to the plain FP64
      factorisation.
    * The explicit wake term runs in FP64 for the wake rows below ``near_rows`` and in FP32
      beyond.  The default keeps every row FP64: the far wake still carries a large share of
      the normal wash (co-located segments of neighbouring strips and the long trailing
      lines), and FP32 rounding of those terms alone moves the circulation by ~1e-8.
    * The advection sweep runs in FP64 for wake node rows below ``advect_near_rows`` and in
      FP32 beyond; it moves the wake and does not enter this step's solve.  From row
      ``advect_interp_row`` on (even; None: never) only every other row is evaluated and the
      rows between take the midpoint value of the cubic through their column's neighbours 1
      and 3 rows away (pvl_wake_interp_rows): far from the body its induced velocity varies
      slowly along a node column.  On the 128x32 flapping wing, 2000 steps, interpolating from
      row 128 keeps every step's circulation within 1.4e-11 of the plain FP64 run (from row 64:
      5.6e-11; row 32: 1.4e-10, over the 1e-10 bar).
    * With ``wake_col_runs`` (runs of smooth wake node columns, ``column_stencil``) the
      advection of the rows from ``advect_col_row`` on is evaluated at every other node column
      (plus those within five of a run end) and interpolated between them by the quintic
      midpoint rule, and from ``advect_row4`` on (even, at least ``advect_interp_row`` + 4;
      None: never) at every fourth row only, the rows between by the cubic midpoint rule at
      spacing 2, then 1.  On the flapping wing, columns from row 64: 4.5e-11; every fourth row
      from 136 or 192: no measurable change (4.4e-11 overall).  Default off (no runs given).
    * With ``cp_patches`` (smooth (ring0, n_span, n_chord) blocks of the body's ring grid,
      ``far_wake_stencil``) the explicit wake term of the rows from ``wake_chord_row`` on is
      evaluated at every other chordwise control point (plus those within five of a patch
      edge) and interpolated between them by the quintic midpoint rule, and from
      ``wake_span_row`` on (None: never) at every other spanwise one too: seen from the body,
      wake rows four or more chords away vary slowly across a patch.  On the 128x32 flapping
      wing (two patches, split at the root where the twist has its kink), 2000 steps, every
      step's circulation stays within 1.4e-11 of the plain FP64 run with the chordwise rule
      from row 64 and within 1.0e-11 with both from row 192; the cubic rule, the product
      rule from row 64, or a patch across the kink go over the 1e-10 bar.  Default off.
    ``judge()`` re-assembles the step's system entirely in FP64 and solves it with the FP64
    factorisation, which is how the mixed answer's error is measured.
    """

    def __init__(self, mesh: Mesh, freestream, tol: float, wake: WakeSpec | None = None, closed_groups=None,
                 refresh: int | None = None, near_rows: int | None = None, advect_near_rows: int = 8,
                 gmres_tol: float = 1e-12, max_iter: int = 20, async_refresh: bool = True,
                 refresh_on_iters: int = 5, use_graphs: bool = True, wake_self_induction: bool = False,
                 device_solve: bool = True, refresh_excess: int = 128, advect_interp_row: int | None = 128,
                 cp_patches=None, wake_chord_row: int = 64, wake_span_row: int | None = 192,
                 wake_col_runs=None, advect_col_row: int = 64, advect_row4: int | None = 136):
        super().__init__(mesh, freestream, tol, wake, closed_groups, wake_self_induction)
        if advect_interp_row is not None and (int(advect_interp_row) < 4 or int(advect_interp_row) % 2):
            raise ValueError("advect_interp_row must be even and at least 4 (or None)")
        self.advect_interp_row = None if advect_interp_row is None else int(advect_interp_row)
        self.advect_row4 = None if advect_row4 is None else int(advect_row4)
        if self.advect_row4 is not None and (self.advect_row4 % 2 or self.advect_interp_row is None
                                             or self.advect_row4 < self.advect_interp_row + 4):
            raise ValueError("advect_row4 must be even and at least advect_interp_row + 4 (or None)")
        self._update_keys: set = set()  # captured wake_update graphs (full wake)
        self.refresh = None if refresh is None else int(refresh)
        self.refresh_excess = int(refresh_excess)
        self._iters_seen = 0      # solves the refresh policy has looked at
        self.gmres_tol = float(gmres_tol)
        self.max_iter = int(max_iter)
        n = self.N
        self.npad = ((n + 63) // 64) * 64
        f32 = dict(dtype=torch.float32, device=self.dev)
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.A32 = torch.zeros((self.npad, self.npad), **f32)
        self.Xinv = torch.zeros((self.npad, self.npad), **f32)
        self.Xnew = torch.zeros((self.npad, self.npad), **f32)
        self.Yscr = torch.zeros((self.npad, self.npad), **f32)
        self.rws = torch.empty(int(_lib.query("pvl_lu32_workspace", self.npad)) + 256, dtype=torch.uint8,
                               device=self.dev)
        self.async_refresh = bool(async_refresh)
        self.refresh_on_iters = int(refresh_on_iters)  # a solve that needed this many iterations refreshes early
        self.policy = RefreshPolicy(self.refresh_on_iters, self.refresh_excess, self.refresh)
        self.side = torch.cuda.Stream(device=self.dev)
        self.refresh_done = None
        self.ipiv32 = torch.zeros(2 * self.npad, dtype=torch.int32, device=self.dev)
        # status words of a rebuild (zero pivot of the FP32 factorisation, a tensor-core GEMM wait
        # that ran out), side by side so that one copy brings both to the host
        self.rstat = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.info32, self.err32 = self.rstat[0:1], self.rstat[1:2]
        self._h_rstat = torch.zeros(2, dtype=torch.int32, pin_memory=True)
        self._precond_backoff = 0  # steps to wait after a rebuild that failed before trying again
        m = self.max_iter
        self.V = torch.zeros((m + 1, n), **f64)
        self.Z = torch.zeros((m, n), **f64)
        self.W = torch.zeros((m, n), **f64)  # A z_j of the device-driven solve
        self.r0 = torch.zeros(n, **f64)
        self.wv = torch.zeros(n, **f64)
        self.Hd = torch.zeros((m, 2 * (m + 2)), **f64)  # column j: h[0..j+1] and basis_project scratch
        self.h_H = torch.zeros((m, 2 * (m + 2)), dtype=torch.float64, pin_memory=True)
        self.scal = torch.zeros(2, **f64)
        self.h_sc = torch.zeros(2, dtype=torch.float64, pin_memory=True)
        self.h_y = torch.zeros(m, dtype=torch.float64, pin_memory=True)
        self.spec_iters = 2
        self.use_graphs = bool(use_graphs)
        self.graphs: dict = {}
        self.y = torch.zeros(m, **f64)
        self.x = torch.zeros(n, **f64)
        self.b_saved = torch.zeros(n, **f64)
        self.have_precond = False
        self.steps_since_refresh = 0
        self._stats = {"gmres_iters": [], "fallbacks": 0, "refreshes": 0, "refresh_failures": 0,
                       "initial_rel_residual": [], "final_rel_residual": [], "judge": []}
        # device-driven solve (pvl_gmres_graph_*): buffers captured by the graph, status ring
        self.device_solve = bool(device_solve)
        if self.device_solve and self.max_iter > int(_lib.query("pvl_gmres_max_iter")):
            raise ValueError(f"max_iter {self.max_iter} > {int(_lib.query('pvl_gmres_max_iter'))} of the device solve")
        self.v32 = torch.zeros(n, dtype=torch.float32, device=self.dev)
        self.ctl = torch.zeros(int(_lib.query("pvl_gmres_ctl_bytes")), dtype=torch.uint8, device=self.dev)
        self.status_dev = torch.zeros(_GMRES_STATUS.itemsize, dtype=torch.uint8, device=self.dev)
        self._status_ring = torch.zeros((_STATUS_RING, _GMRES_STATUS.itemsize), dtype=torch.uint8, pin_memory=True)
        self._pending: deque = deque()
        self._next_slot = 0
        self._graph = 0
        self._graph_key = None
        need = 0
        if self.wake is not None:
            need = max(need, self._init_row_major_wake(near_rows, advect_near_rows))
            if cp_patches is not None:
                need = max(need, self._init_far_stencil(cp_patches, wake_chord_row, wake_span_row))
            self._cols = None  # node-column stencil of the far-row advection (wake_col_runs)
            if wake_col_runs is not None:
                need = max(need, self._init_col_stencil(wake_col_runs, advect_col_row))
        if need + 256 > self._ws_bytes:
            self._ws_bytes = need + 256
            self.ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=self.dev)

    # ------------------------------------------------------------------ wake in row-major ring order
    def _init_row_major_wake(self, near_rows: int | None, advect_near_rows: int) -> int:
        """Precision bands of the wake terms and their workspace."""
        w = self.wake
        S, R = w["S"], w["R"]
        rm = w["rm"]
        self.near_rows = R if near_rows is None else max(1, min(int(near_rows), R))
        self.advect_near_rows = max(0, min(int(advect_near_rows), R))
        self.n_near_lines = w["lines_upto"][self.near_rows]  # lines of rows < near_rows come first
        L, P = self.mesh.n_lines, self.P
        need = [_lib.query("pvl_segments_workspace", rm.n_lines, _lib.PVL_F64),
                _lib.query("pvl_line_velocity_workspace", self.n_near_lines, P, _lib.PVL_F64),
                _lib.query("pvl_line_velocity_workspace", max(rm.n_lines - self.n_near_lines, 1), P, _lib.PVL_F32)]
        nc = w["n_cols"]
        for c in range(1, R + 1):  # every row split the advection can see as the wake grows
            nr = min(self.advect_near_rows, c)
            if nr:
                need.append(_lib.query("pvl_line_velocity_workspace", L, nc * nr, _lib.PVL_F64))
            if c > nr:
                need.append(_lib.query("pvl_line_velocity_workspace", L, nc * (c - nr), _lib.PVL_F32))
        return max(need)

    def _init_far_stencil(self, patches, chord_row: int, span_row: int | None) -> int:
        """Device copy of far_wake_stencil(patches) and the workspace of its two sweeps."""
        w = self.wake
        R = w["R"]
        if self.near_rows < R:
            raise ValueError("cp_patches needs the explicit wake term in FP64 (near_rows None)")
        chord_row = int(chord_row)
        if chord_row < 1 or (span_row is not None and int(span_row) < chord_row):
            raise ValueError("need 1 <= wake_chord_row <= wake_span_row")
        span_row = None if span_row is None else min(int(span_row), R)
        chord_row = min(chord_row, R)
        plan = far_wake_stencil(self.P, patches)
        n_c, n_s = plan["n_chord_eval"], plan["n_span_eval"]
        f64 = dict(dtype=torch.float64, device=self.dev)
        self._far = {
            "chord_row": chord_row, "span_row": span_row, "n_chord_eval": n_c, "n_span_eval": n_s,
            "index": to_device_u32(plan["index"], self.dev), "offsets": to_device_u32(plan["offsets"], self.dev),
            "entries": to_device_u32(plan["entries"], self.dev),
            "weights": torch.as_tensor(plan["weights"]).to(self.dev),
            "pts": torch.zeros((max(n_c, 1), 3), **f64), "vals": torch.zeros((max(n_c + n_s, 1), 3), **f64),
        }
        up, n_all = w["lines_upto"], w["rm"].n_lines
        b = n_all if span_row is None else up[span_row]
        return max(_lib.query("pvl_line_velocity_workspace", max(b - up[chord_row], 1), max(n_c, 1), _lib.PVL_F64),
                   _lib.query("pvl_line_velocity_workspace", max(n_all - b, 1), max(n_s, 1), _lib.PVL_F64))

    def _init_col_stencil(self, runs, col_row: int) -> int:
        """Device copy of column_stencil(runs), the row lists and the velocity buffer of the
        evaluated columns; returns the workspace of their sweeps."""
        w = self.wake
        col_row = max(int(col_row), self.advect_near_rows)
        ri = self.advect_interp_row
        if ri is not None and col_row > ri:
            raise ValueError("advect_col_row must not exceed advect_interp_row")
        plan = column_stencil(w["n_cols"], runs)
        sub = plan["sub"]
        cols = w["cols"].cpu().numpy().view(np.uint32)
        R = w["R"]
        self._cols = {"row": col_row}
        # the evaluated rows from col_row on for every row count 1..R: row k of ``lists``
        lists = np.zeros((R + 1, R), np.uint32)
        lens = [0] * (R + 1)
        for c in range(1, R + 1):
            rows = self._advect_schedule(c)[5]
            lists[c, :len(rows)] = rows
            lens[c] = len(rows)
        self._cols.update({
            "lists": to_device_u32(lists, self.dev), "list_len": lens,
            "n_sub": int(sub.size), "ids": to_device_u32(cols[sub], self.dev),
            "offsets": to_device_u32(plan["offsets"], self.dev), "entries": to_device_u32(plan["entries"], self.dev),
            "weights": torch.as_tensor(plan["weights"]).to(self.dev),
            "vel": torch.zeros((max(int(sub.size), 1), R, 3), dtype=torch.float64, device=self.dev),
        })
        L = self.mesh.n_lines
        return max(_lib.query("pvl_line_velocity_workspace", L, max(int(sub.size) * n, 1), _lib.PVL_F32)
                   for n in set(lens))

    # ------------------------------------------------------------------ preconditioner
    def refresh_preconditioner(self, wait: bool = True) -> None:
        """FP32 LU of the current system (tensor-core trailing updates) and its explicit inverse.

        With ``wait`` (the first refresh, or ``async_refresh=False``) the new inverse is built on
        the current stream and used at once.  Otherwise the system is converted to FP32 on the
        current stream and factorised and inverted on a side stream into a second buffer, with
        its own workspace; the solves keep the previous inverse until the new one is complete
        (``_adopt_refresh``), so the refresh overlaps the following steps' work."""
        s = stream_ptr()
        n, npad = self.N, self.npad
        self._finish_refresh()  # never two refreshes in flight
        self._stats["refreshes"] += 1  # rebuilds started (those that failed are refresh_failures)
        _lib.call("pvl_pad_convert_f32", n, ptr(self.A), self.N, ptr(self.A32), npad, npad, s)
        target = self.Xinv if wait else self.Xnew

        def build(stream):
            ws, nb = ptr(self.rws), self.rws.numel()
            _lib.call("pvl_lu32_factor", npad, ptr(self.A32), npad, ptr(self.ipiv32), ptr(self.info32),
                      ptr(self.err32), ws, nb, stream)
            perm = self.ipiv32.data_ptr() + 4 * npad
            _lib.call("pvl_lu32_inverse", npad, ptr(self.A32), npad, perm, ptr(target), npad, ptr(self.Yscr), npad,
                      ptr(self.err32), ws, nb, stream)
            # the status words travel with the rebuild; the host reads them when it adopts it
            self._h_rstat.copy_(self.rstat, non_blocking=True)

        if wait:
            build(s)
            torch.cuda.current_stream().synchronize()
            if not self._rebuild_ok():
                self.have_precond = False
                self._precond_backoff = 25
                return
        else:
            converted = torch.cuda.Event()
            converted.record()
            with torch.cuda.stream(self.side):
                self.side.wait_event(converted)
                build(stream_ptr())
                self.refresh_done = torch.cuda.Event()
                self.refresh_done.record()
        self.have_precond = True
        self.steps_since_refresh = 0
        self.policy.rebuilt()

    def _adopt_refresh(self) -> None:
        """Switch to the side stream's new inverse once it is complete (no host wait).  It is
        copied into the inverse's fixed buffer, which the captured solve graphs read."""
        if self.refresh_done is not None and self.refresh_done.query():
            self._finish_refresh()

    def wait_refresh(self) -> None:
        """Make the current stream wait for a preconditioner rebuild still running on the side
        stream and adopt it (e.g. at the end of a warm-up, so that a rebuild started there is
        not timed as part of the steps that follow)."""
        self._finish_refresh()

    def join_side_stream(self) -> None:
        """Make the current stream wait for everything enqueued on the side stream so far (a
        rebuild in flight stays in flight for the host): an event recorded after this covers
        the side stream's work too."""
        ev = torch.cuda.Event()
        ev.record(self.side)
        torch.cuda.current_stream().wait_event(ev)

    def _rebuild_ok(self) -> bool:
        """Whether the rebuild whose status words reached the host is usable: no exactly zero
        FP32 pivot and no tensor-core wait that ran out.  A failed one is counted and dropped."""
        info, err = (int(v) for v in self._h_rstat.tolist())
        if info or err:
            self._stats["refresh_failures"] += 1
            return False
        return True

    def _finish_refresh(self) -> None:
        """Adopt a refresh still in flight: the host waits for its status words (long done when
        the policy adopts it) and, if it succeeded, the current stream waits for it and copies
        the new inverse into place; a failed rebuild leaves the previous inverse in use."""
        if self.refresh_done is not None:
            self.refresh_done.synchronize()
            if self._rebuild_ok():
                torch.cuda.current_stream().wait_event(self.refresh_done)
                self.Xinv.copy_(self.Xnew)
            self.refresh_done = None

    # ------------------------------------------------------------------ GMRES
    def _arnoldi(self, j: int) -> None:
        """Column j of the right-preconditioned Arnoldi process, entirely on the device:
        Z_j = M V_j, w = A Z_j, two classical Gram-Schmidt passes into Hd[j][0..j],
        Hd[j][j+1] = ||w||, V_{j+1} = w / ||w||."""
        s = stream_ptr()
        n = self.N
        hj = self.Hd[j]
        _lib.call("pvl_gemv_f32mat", n, n, 1.0, ptr(self.Xinv), self.npad, ptr(self.V[j]), 0.0, ptr(self.Z[j]), s)
        _lib.call("pvl_gemv_f64", n, n, 1.0, ptr(self.A), self.N, ptr(self.Z[j]), 0.0, ptr(self.wv), s)
        for _ in range(2):
            _lib.call("pvl_basis_project", n, j + 1, ptr(self.V), n, ptr(self.wv), ptr(hj), s)
        _lib.call("pvl_normalize", n, ptr(self.wv), ptr(self.V[j + 1]), hj.data_ptr() + 8 * (j + 1), s)

    def _replay(self, key, fn) -> None:
        """Run ``fn`` as a CUDA graph captured on first use under ``key`` (every buffer the
        solve touches has a fixed address), or directly when graphs are off."""
        if not self.use_graphs:
            fn()
            return
        g = self.graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn()
            self.graphs[key] = g
        g.replay()

    def _gmres_start(self) -> None:
        s = stream_ptr()
        n = self.N
        self.wv.copy_(self.rhs)
        _lib.call("pvl_gemv_f64", n, n, -1.0, ptr(self.A), self.N, ptr(self.x), 1.0, ptr(self.wv), s)
        _lib.call("pvl_normalize", n, ptr(self.rhs), None, self.scal.data_ptr(), s)
        _lib.call("pvl_normalize", n, ptr(self.wv), ptr(self.V[0]), self.scal.data_ptr() + 8, s)
        self.Hd.zero_()

    def _gmres_finish(self, k: int) -> None:
        s = stream_ptr()
        n = self.N
        if k:
            _lib.call("pvl_combine", n, k, ptr(self.Z), n, ptr(self.y), ptr(self.x), s)
        self.wv.copy_(self.rhs)
        _lib.call("pvl_gemv_f64", n, n, -1.0, ptr(self.A), self.N, ptr(self.x), 1.0, ptr(self.wv), s)
        _lib.call("pvl_normalize", n, ptr(self.wv), None, self.scal.data_ptr(), s)

    def solve_mixed(self, x0: torch.Tensor | None = None) -> bool:
        """Right-preconditioned GMRES on A x = b in FP64; True if the relative residual met gmres_tol.

        The Arnoldi columns run on the device without host round trips (each a replayed CUDA
        graph); the host reads the small Hessenberg matrix after as many columns as the
        previous solve needed and then column by column, applies the Givens rotations and forms
        the update.  The true FP64 residual b - A x decides convergence."""
        n = self.N
        self._maybe_refresh()
        if not self.have_precond:
            return False  # the caller falls back to the FP64 LU
        x = self.x
        if x0 is not None:
            x.copy_(x0.reshape(-1)[:n])
        else:
            x[: self.P].copy_(self.gamma)  # the previous step's circulation
        sc = self.scal
        self._replay("start", self._gmres_start)
        m = self.max_iter
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        k, done, first = 0, False, True
        bnorm = beta = target = 0.0
        while k < m and not done:
            nxt = min(m, k + (self.spec_iters if first else 1))
            for j in range(k, nxt):
                self._replay(("col", j), lambda j=j: self._arnoldi(j))
            self.h_H[: nxt].copy_(self.Hd[: nxt], non_blocking=True)
            if first:
                self.h_sc.copy_(sc, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            if first:
                bnorm, beta = float(self.h_sc[0]), float(self.h_sc[1])
                self._stats["initial_rel_residual"].append(beta / max(bnorm, 1e-300))
                target = self.gmres_tol * bnorm
                g[0] = beta
                first = False
                if beta <= target:
                    k, done = 0, True
                    break
            hh = self.h_H.numpy()
            for j in range(k, nxt):
                H[: j + 2, j] = hh[j, : j + 2]
                hnext = H[j + 1, j]
                for i in range(j):  # previous Givens rotations
                    t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                    H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                    H[i, j] = t
                den = float(np.hypot(H[j, j], H[j + 1, j]))
                cs[j], sn[j] = (1.0, 0.0) if den == 0.0 else (H[j, j] / den, H[j + 1, j] / den)
                H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
                H[j + 1, j] = 0.0
                g[j + 1] = -sn[j] * g[j]
                g[j] = cs[j] * g[j]
                k = j + 1
                if abs(g[j + 1]) <= target or hnext == 0.0:  # converged, or the Krylov space is exhausted
                    done = True
                    break
        if k:
            yk = np.zeros(k)
            for i in range(k - 1, -1, -1):  # back substitution with the rotated Hessenberg
                yk[i] = (g[i] - H[i, i + 1:k] @ yk[i + 1:]) / H[i, i] if H[i, i] != 0.0 else 0.0
            self.h_y[:k] = torch.from_numpy(yk)
            self.y[:k].copy_(self.h_y[:k], non_blocking=True)
            self.spec_iters = max(1, k)
        # the true FP64 residual decides
        self._replay(("finish", k), lambda: self._gmres_finish(k))
        rel = float(sc[0].item()) / max(bnorm, 1e-300)
        self._stats["gmres_iters"].append(k)
        self._stats["final_rel_residual"].append(rel)
        return rel <= self.gmres_tol

    def _maybe_refresh(self) -> None:
        """Adopt a finished refresh; start a new one when the preconditioner has gone stale
        (the policy of the class docstring)."""
        self._adopt_refresh()
        its = self._stats["gmres_iters"]
        self.policy.observe(its[self._iters_seen:])
        self._iters_seen = len(its)
        if self._precond_backoff > 0:
            self._precond_backoff -= 1
        elif not self.have_precond:
            self.refresh_preconditioner(wait=True)
        elif self.policy.due(self.steps_since_refresh, idle=self.refresh_done is None):
            self.refresh_preconditioner(wait=not self.async_refresh)
        self.steps_since_refresh += 1

    # ------------------------------------------------------------------ device-driven solve
    def _ensure_graph(self) -> None:
        key = (int(self.ws.data_ptr()), self._ws_bytes)
        if self._graph and self._graph_key == key:
            return
        self._destroy_graph()
        n = self.N
        h = ctypes.c_uint64(0)
        _lib.call("pvl_gmres_graph_create", n, ptr(self.A), n, ptr(self.Xinv), self.npad, ptr(self.rhs), ptr(self.x),
                  ptr(self.V), ptr(self.Z), ptr(self.W), ptr(self.r0), ptr(self.wv), ptr(self.v32), ptr(self.ctl),
                  self.max_iter, self.gmres_tol, ptr(self.ipiv), ptr(self.info), ptr(self.ws), self._ws_bytes, ptr(self.gamma),
                  self.P, self.m, ptr(self.goff) if self.m else None, ptr(self.status_dev), ctypes.byref(h))
        self._graph = int(h.value)
        self._graph_key = key

    def _destroy_graph(self) -> None:
        if self._graph:
            self._collect_status(block=True)
            _lib.call("pvl_gmres_graph_destroy", self._graph)
            self._graph = 0

    def __del__(self):
        try:
            self._destroy_graph()
        except Exception:
            pass

    def _collect_status(self, block: bool) -> None:
        """Move the status records of finished device solves into the statistics."""
        while self._pending:
            slot, ev = self._pending[0]
            if block:
                ev.synchronize()
            elif not ev.query():
                break
            self._pending.popleft()
            rec = np.frombuffer(self._status_ring[slot].numpy().tobytes(), dtype=_GMRES_STATUS)[0]
            it, ok = int(rec["iterations"]), bool(rec["converged"])
            st = self._stats
            st["gmres_iters"].append(it)
            st["initial_rel_residual"].append(float(rec["initial_rel_residual"]))
            st["final_rel_residual"].append(float(rec["final_rel_residual"]))
            if not ok:
                st["fallbacks"] += 1
            _lib.call("pvl_gmres_graph_account", self._graph, it, 0 if ok else 1)

    @property
    def stats(self) -> dict:
        """Solve statistics (waits for the device solves still in flight)."""
        self._collect_status(block=True)
        return self._stats

    def _solve_device(self, x0: torch.Tensor | None) -> None:
        """The whole solve as one graph launch (pvl_gmres_graph_create): GMRES driven by the
        device to convergence, the FP64 fallback inside the graph; no host synchronisation.
        The status of each solve is read back later (``stats``); the host waits here for the
        previous solve's record (finished by the time the GPU works through the wake update and
        this step's assembly, which are queued behind it), so that the refresh policy sees every
        iteration count in time."""
        self._collect_status(block=True)
        self._maybe_refresh()
        if not self.have_precond:  # no usable preconditioner (its rebuild failed): the FP64 LU
            self._stats["fallbacks"] += 1
            SolverEngine.solve(self)
            return
        if x0 is not None:
            self.x.copy_(x0.reshape(-1)[: self.N])
        else:
            self.x[: self.P].copy_(self.gamma)  # the previous step's circulation
        self._ensure_graph()
        _lib.call("pvl_gmres_graph_launch", self._graph, stream_ptr())
        slot = self._next_slot
        self._next_slot = (slot + 1) % _STATUS_RING
        self._status_ring[slot].copy_(self.status_dev, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._pending.append((slot, ev))

    def solve(self, x0: torch.Tensor | None = None) -> None:
        if self.device_solve:
            self._solve_device(x0)
            return
        self.b_saved.copy_(self.rhs)
        if self.solve_mixed(x0):
            self.gamma.copy_(self.x[: self.P])
            if self.m:
                _lib.call("pvl_group_mean_remove", self.m, ptr(self.goff), ptr(self.gamma), stream_ptr())
            return
        self._stats["fallbacks"] += 1
        self.rhs.copy_(self.b_saved)
        super().solve()

    def assemble_rest(self) -> None:
        """The wake corrections and the closed-body border, the body part already in place."""
        if self.wake is not None and self.iteration > 0:
            self._wake_terms()
        self.border()

    def begin_step(self, positions, velocities) -> None:
        """Inputs and body assembly of this step."""
        self.load_inputs(positions, velocities)
        self.assemble_body_only()

    def step(self, time: float, positions, velocities, x0: torch.Tensor | None = None) -> torch.Tensor:
        self.begin_step(positions, velocities)
        self.assemble_rest()
        self.solve(x0)
        if self.wake is not None:
            self.wake_update(time)
        self.iteration += 1
        return self.gamma

    # ------------------------------------------------------------------ error against FP64
    def judge(self) -> float:
        """Relative error of the current circulation against the all-FP64 step.

        Call after assemble/solve and before the wake update of a step (``step_judged`` does
        this): the system is re-assembled in FP64 (body, implicit and explicit wake terms) and
        solved with the FP64 factorisation; the mixed circulation is kept."""
        mixed = self.gamma.clone()
        self.assemble_body_only()
        if self.wake is not None and self.iteration > 0:
            self._wake_corrections(fp64_only=True)
        self.border()
        SolverEngine.solve(self)
        ref = self.gamma.clone()
        self.last_judge_ref = ref  # the all-FP64 circulation of the judged state
        self.gamma.copy_(mixed)
        err = float((torch.linalg.vector_norm(mixed - ref) / torch.linalg.vector_norm(ref)).item())
        self._stats["judge"].append(err)
        return err

    def step_judged(self, time: float, positions, velocities, x0: torch.Tensor | None = None) -> float:
        self.load_inputs(positions, velocities)
        self.assemble()
        self.solve(x0)
        err = self.judge()
        if self.wake is not None:
            self.wake_update(time)
        self.iteration += 1
        return err

    def wake_update(self, time: float) -> None:
        """As the plain update, with the advection sweep split into FP64 near rows and FP32 far rows."""
        w = self.wake
        R = w["R"]
        dt = float(time) - w["time"]
        w["time"] = float(time)
        if w["step_count"] == 0:
            self._advect(0, 0.0)
            w["step_count"] = 1
        complete = min(w["step_count"], R)
        cur, c = w["cur"], w["ccur"]
        key = ("wake_update", cur, c, dt)
        if self._wake_full() and (key in self._update_keys or len(self._update_keys) < 8):
            # one graph per buffer pair and time step (a few distinct dt at most)
            self._update_keys.add(key)
            self.captured(key, lambda: self._update_launches(complete, dt, cur, c))
        else:
            self._update_launches(complete, dt, cur, c)
        w["cur"], w["ccur"] = 1 - cur, 1 - c
        w["step_count"] += 1

    def _advect_schedule(self, complete: int):
        """How the advection of a wake with ``complete`` rows is evaluated: rows below nr in
        FP64, the rest in FP32; from ri (advect_interp_row, when interp) even rows only up to
        the tail (the odd rows between from their neighbours), every row from tail on; from ac
        (< complete when the column stencil applies) at the evaluated node columns only, whose
        rows are then listed in ``rows`` (ascending).  With the column stencil and r4
        (advect_row4, when four) every fourth row from r4 up to T, every row from T on (T a
        multiple of 4, 5 to 8 rows below complete): the rows midway between from the rows 2 and
        6 away, then the odd rows up to T - 1.  Returns (nr, interp, mid, tail, ac, rows, four,
        T); the interpolated rows are ``_row_passes``."""
        nr = min(self.advect_near_rows, complete)
        ri = self.advect_interp_row
        interp = ri is not None and ri >= nr and complete >= ri + 8
        mid = ri if interp else complete
        tail = (complete - 4) | 1 if interp else complete  # first odd row without 3 rows above it
        cs = self._cols
        ac = cs["row"] if cs is not None and complete > cs["row"] else complete  # ac <= mid
        r4 = self.advect_row4
        T = ((complete - 5) // 4) * 4
        four = interp and ac < complete and r4 is not None and T >= r4 + 8
        rows = []
        if ac < complete:
            if four:
                rows = list(range(ac, mid)) + list(range(ri, r4, 2)) + list(range(r4, T, 4)) + list(range(T, complete))
            elif interp:
                rows = list(range(ac, mid)) + list(range(ri, tail, 2)) + list(range(tail, complete))
            else:
                rows = list(range(ac, complete))
        return nr, interp, mid, tail, ac, rows, four, T

    def _row_passes(self, complete: int) -> list:
        """(first row, last row, half spacing) of the row interpolations, in order."""
        _, interp, _, tail, _, _, four, T = self._advect_schedule(complete)
        ri = self.advect_interp_row
        if four:
            return [(self.advect_row4 + 2, T - 2, 2), (ri + 1, T - 1, 1)]
        return [(ri + 1, tail - 2, 1)] if interp else []

    def _update_launches(self, complete: int, dt: float, cur: int, c: int) -> None:
        """The launches of wake_update from positions pos[cur] and circulations circ[c] into the
        other buffers (no host state changes: they may be captured once and replayed)."""
        s = stream_ptr()
        w = self.wake
        S, R = w["S"], w["R"]
        wpos = w["pos"][cur]
        msh, d = self.mesh, self.d_body
        _lib.call("pvl_line_circulation", msh.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(self.gamma), 0,
                  ptr(self.body_line_gamma), s)
        u = self.u_inf
        nr, interp, mid, tail, ac, _, _, _ = self._advect_schedule(complete)
        ri = self.advect_interp_row
        cs = self._cols
        # (precision, row, count, step, columns, column list, output) of the banded sweeps
        all_cols = (w["n_cols"], w["cols"], w["node_vel"])
        bands = [(_lib.PVL_F64, 0, nr, 1) + all_cols, (_lib.PVL_F32, nr, min(ac, mid) - nr, 1) + all_cols]
        if ac == complete and interp:
            bands += [(_lib.PVL_F32, ri, (tail - ri + 1) // 2, 2) + all_cols,
                      (_lib.PVL_F32, tail, complete - tail, 1) + all_cols]
        for prec, r0, count, step, n_c, col_list, out in bands:
            if count > 0:
                _lib.call("pvl_wake_node_velocity_rows", prec, msh.n_points, msh.n_lines, ptr(d["lines"]),
                          ptr(self.pos), ptr(self.body_line_gamma), S, R, complete, r0, count, step, n_c,
                          ptr(col_list), ptr(wpos), float(u[0]), float(u[1]), float(u[2]), self.tol,
                          ptr(out), ptr(self.ws), self._ws_bytes, s)
        if ac < complete:
            # every evaluated row from ac on, at the evaluated node columns, in one sweep (the row
            # list of this row count, precomputed), then the other columns from their rule
            n_list = cs["list_len"][complete]
            _lib.call("pvl_wake_node_velocity_list", _lib.PVL_F32, msh.n_points, msh.n_lines, ptr(d["lines"]),
                      ptr(self.pos), ptr(self.body_line_gamma), S, R, complete, n_list,
                      cs["lists"].data_ptr() + 4 * R * complete, cs["n_sub"], ptr(cs["ids"]), ptr(wpos),
                      float(u[0]), float(u[1]), float(u[2]), self.tol, ptr(cs["vel"]), ptr(self.ws), self._ws_bytes, s)
            _lib.call("pvl_wake_interp_cols", w["n_cols"], complete, ac, complete, ptr(cs["offsets"]),
                      cs["entries"].numel(), ptr(cs["entries"]), ptr(cs["weights"]), cs["n_sub"], ptr(cs["vel"]),
                      ptr(w["node_vel"]), s)
        for first, last, half in self._row_passes(complete):
            _lib.call("pvl_wake_interp_rows_spaced", w["n_cols"], complete, first, last, half, ptr(w["node_vel"]), s)
        if self.wake_self_induction:
            self._add_wake_self_velocity(complete)
        _lib.call("pvl_wake_advect_cols", S, R, complete, ptr(wpos), ptr(w["node_vel"]), ptr(w["slot"]), w["n_cols"],
                  dt, ptr(self.pos), ptr(w["bn"]), ptr(w["pos"][1 - cur]), s)
        _lib.call("pvl_wake_shed", S, R, ptr(w["circ"][c]), ptr(w["adj"]), ptr(self.gamma), ptr(w["circ"][1 - c]), s)
