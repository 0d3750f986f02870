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
cost is linear in the number of points, so the scaled sample estimates the full step.
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

    def step(self, t: float) -> dict:
        """One sampled step; returns the phase times and the extrapolated full-step time."""
        import scipy.linalg as la
        from threadpoolctl import threadpool_limits

        c, tol, F = self.case, self.case.tol, self.F
        ph = {}
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
            t0 = time.perf_counter()
            sel = np.arange(0, cps.shape[0], F)
            ind = self.wake_mesh.induction_matrix3(tol, self.wake_pos.reshape(-1, 3), np.ascontiguousarray(cps[sel]),
                                                   np.ascontiguousarray(nrm[sel])).reshape(sel.size, self.S, self.R)
            implicit = ind[:, :, 0]
            for i in range(self.S):
                if self.adj[i, 1] != 0x7FFFFFFF:
                    A[sel, self.adj[i, 1]] -= implicit[:, i]
                if self.adj[i, 0] != 0x7FFFFFFF:
                    A[sel, self.adj[i, 0]] += implicit[:, i]
            rhs[sel] += np.vecdot(ind[:, :, 1:].reshape(sel.size, -1), self.wake_circ[:, 1:].reshape(-1)[None, :],
                                  axis=1)
            ph["corrections_sample"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            g = la.lu_solve(la.lu_factor(A, overwrite_a=True), rhs, overwrite_b=True)
            ph["solve"] = time.perf_counter() - t0
            # advection of every F-th wake node (wake_models.py:120-128)
            t0 = time.perf_counter()
            nodes = np.ascontiguousarray(self.wake_pos[:, :, : self.R, :].reshape(-1, 3)[::F])
            v = np.broadcast_to(c.freestream, nodes.shape) + np.vecdot(
                self.mesh.induction_matrix(tol, pos, nodes), g[None, :, None], axis=1)
            _ = nodes + v * c.dt
            ph["advection_sample"] = time.perf_counter() - t0
        ph["step_estimate"] = ph["body"] + ph["solve"] + F * (ph["corrections_sample"] + ph["advection_sample"])
        return ph
