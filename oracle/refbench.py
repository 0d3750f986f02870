"""CPU baseline of one full-wake UVLM step with the reference's own code -- ORACLE ONLY.

Used by bench.py (its ``cpu_baseline`` object and ``--impl reference``).  The pair work
runs in the reference's compiled extension (oracle/_ref, built from the reference's
sources: Mesh.induction_matrix3 / induction_matrix, OpenMP over all host cores); the
dense solve is scipy's LAPACK lu_factor / lu_solve (the reference's call,
python/pyvl/solver.py:223-227); the glue between them restates solver.py:178-239 and
wake_models.py:111-223 with numpy.

A full step at 4096 rings and a 400-row wake takes tens of seconds on a few cores, so one
timed "step" is a bounded sample: body geometry, body matrix and the LU at full size, the
wake correction and the wake advection on 1/F of their points, scaled by F.  The pair
cost is linear in the number of points, so the scaled sample estimates the full step;
``step(t, whole=True)`` runs every control point and wake node, which checks the estimate.
"""

from __future__ import annotations

import os
import time

import numpy as np


def _threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


class ReferenceStep:
    """State for timing the reference's step on a workload with a full synthetic wake."""

    def __init__(self, case, wake_pos, wake_circ, bordering_nodes, adjacent, fraction: int = 16):
        os.environ.setdefault("OMP_NUM_THREADS", str(_threads()))
        from . import ref
        from .solver import wake_ring_connectivity

        cvl = ref.load_cvl()
        self.case = case
        self.F = int(fraction)
        self.mesh = cvl.Mesh(case.n_points, [np.asarray(e, np.uint32) for e in case.elements])
        S, R = wake_circ.shape
        t0 = time.perf_counter()
        self.wake_mesh = cvl.Mesh(2 * (R + 1) * S, wake_ring_connectivity(R, S))
        self.wake_mesh_seconds = time.perf_counter() - t0
        self.wake_pos = np.ascontiguousarray(wake_pos, np.float64)
        self.wake_circ = np.ascontiguousarray(wake_circ, np.float64)
        self.bn = np.asarray(bordering_nodes, np.int64)
        self.adj = np.asarray(adjacent, np.int64)
        self.S, self.R = S, R
        self.threads = int(os.environ.get("OMP_NUM_THREADS", _threads()))

    def step(self, t: float, fraction: int | None = None, whole: bool = False) -> dict:
        """One step with the wake phases on every ``fraction``-th control point and wake node,
        scaled by ``fraction`` (the sampled estimate); with ``whole``, the wake phases run on
        all ``fraction`` interleaved subsets in turn, i.e. on every control point and wake node
        (a measured whole step whose largest reference buffers are 1/fraction of a single call's:
        the line buffer of one call over all 102,400 wake nodes alone would be ~20 GB).
        Returns the phase times and the (estimated or measured) step time."""
        import scipy.linalg as la
        from threadpoolctl import threadpool_limits

        c, tol = self.case, self.case.tol
        F = self.F if fraction is None else int(fraction)
        ph = {"corrections": 0.0, "advection": 0.0}
        with threadpool_limits(limits=self.threads):
            t0 = time.perf_counter()
            pos = c.positions_at(t)
            vel = c.velocities_at(t)
            cps = self.mesh.surface_average_vec3(pos)
            cpv = self.mesh.surface_average_vec3(vel)
            nrm = self.mesh.surface_normal(pos)
            rhs = np.vecdot(nrm, -(np.broadcast_to(c.freestream, cps.shape) - cpv), axis=1)
            A = self.mesh.induction_matrix3(tol, pos, cps, nrm)
            ph["body"] = time.perf_counter() - t0
            # wake corrections on every F-th control point (wake_models.py:199-223)
            for off in range(F if whole else 1):
                t0 = time.perf_counter()
                sel = np.arange(off, cps.shape[0], F)
                ind = self.wake_mesh.induction_matrix3(tol, self.wake_pos.reshape(-1, 3),
                                                       np.ascontiguousarray(cps[sel]),
                                                       np.ascontiguousarray(nrm[sel])).reshape(sel.size, self.S,
                                                                                               self.R)
                implicit = ind[:, :, 0]
                for i in range(self.S):
                    if self.adj[i, 1] != 0x7FFFFFFF:
                        A[sel, self.adj[i, 1]] -= implicit[:, i]
                    if self.adj[i, 0] != 0x7FFFFFFF:
                        A[sel, self.adj[i, 0]] += implicit[:, i]
                rhs[sel] += np.vecdot(ind[:, :, 1:].reshape(sel.size, -1),
                                      self.wake_circ[:, 1:].reshape(-1)[None, :], axis=1)
                del ind, implicit
                ph["corrections"] += time.perf_counter() - t0
            t0 = time.perf_counter()
            g = la.lu_solve(la.lu_factor(A, overwrite_a=True), rhs, overwrite_b=True)
            ph["solve"] = time.perf_counter() - t0
            # advection of every F-th wake node (wake_models.py:120-128)
            all_nodes = self.wake_pos[:, :, : self.R, :].reshape(-1, 3)
            for off in range(F if whole else 1):
                t0 = time.perf_counter()
                nodes = np.ascontiguousarray(all_nodes[off::F])
                v = np.broadcast_to(c.freestream, nodes.shape) + np.vecdot(
                    self.mesh.induction_matrix(tol, pos, nodes), g[None, :, None], axis=1)
                _ = nodes + v * c.dt
                ph["advection"] += time.perf_counter() - t0
        scale = 1 if whole else F
        ph["step_estimate"] = ph["body"] + ph["solve"] + scale * (ph["corrections"] + ph["advection"])
        return ph


class ReferenceMesh:
    """The reference's compiled ``Mesh`` (oracle/_ref) behind the interface OracleRun uses
    (lines, dual_lines, surface averages and normals, induction_matrix / induction_matrix3), so
    that the solver-loop restatement of oracle/solver.py runs on the reference's own kernels."""

    def __init__(self, n_points: int, elements):
        from . import ref

        self._m = ref.load_cvl().Mesh(int(n_points), [np.asarray(e, np.uint32) for e in elements])
        self.n_points = int(n_points)
        self.lines = np.asarray(self._m.line_data, np.uint32).reshape(-1, 2)
        self._dual = None

    @property
    def n_lines(self) -> int:
        return int(self.lines.shape[0])

    def dual_lines(self):
        if self._dual is None:
            self._dual = np.asarray(self._m.compute_dual().line_data, np.uint32).reshape(-1, 2)
        return self._dual

    def surface_average_vec3(self, v):
        return self._m.surface_average_vec3(np.ascontiguousarray(v, np.float64))

    def surface_normal(self, p):
        return self._m.surface_normal(np.ascontiguousarray(p, np.float64))

    def induction_matrix(self, tol, positions, cpts):
        return self._m.induction_matrix(float(tol), np.ascontiguousarray(positions, np.float64),
                                        np.ascontiguousarray(cpts, np.float64))

    def induction_matrix3(self, tol, positions, cpts, normals):
        return self._m.induction_matrix3(float(tol), np.ascontiguousarray(positions, np.float64),
                                         np.ascontiguousarray(cpts, np.float64), np.ascontiguousarray(normals, np.float64))


def reference_case_steps(cases, steps: int) -> tuple[float, int]:
    """Run each case for `steps` solver iterations with the reference's kernels (OracleRun over
    ReferenceMesh, LAPACK solve), all host cores; returns (seconds, case-steps)."""
    from threadpoolctl import threadpool_limits

    from .solver import OracleRun

    os.environ.setdefault("OMP_NUM_THREADS", str(_threads()))
    total = 0.0
    with threadpool_limits(limits=int(os.environ["OMP_NUM_THREADS"])):
        for c in cases:
            run = OracleRun(c, mesh_cls=ReferenceMesh)
            t0 = time.perf_counter()
            for _ in range(steps):
                run.step()
            total += time.perf_counter() - t0
    return total, len(cases) * steps
