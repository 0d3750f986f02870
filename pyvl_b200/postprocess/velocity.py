"""Velocity fields (python/pyvl/postprocess/velocity.py:11-89), fused on the GPU."""

from __future__ import annotations

import numpy as np
import numpy.typing as npt


def _velocity(results, i: int, t: float, cpts) -> npt.NDArray[np.float64]:
    tol = results.settings.model_settings.vortex_limit
    pos = results.geometry.positions_at_time(t)
    v = results.geometry.mesh.induced_velocity(tol, pos, cpts, results.circulations[i, :])
    v = v + results.settings.flow_conditions.get_velocity(t, cpts)
    wm = results.wake_models[i]
    if wm is not None:
        v = v + wm.get_velocity(cpts)
    return v


def compute_velocities(results, positions: npt.NDArray) -> npt.NDArray[np.float64]:
    """(n_outputs, N, 3) velocities at the same points for every output step."""
    cpts = np.ascontiguousarray(positions, dtype=np.float64)
    if cpts.ndim != 2 or cpts.shape[1] != 3:
        raise ValueError("Positions must be an array of 3 component position vectors.")
    times = results.settings.time_settings.output_times
    out = np.empty((times.size, cpts.shape[0], 3), np.float64)
    for i, t in enumerate(times):
        out[i] = _velocity(results, i, t, cpts)
    return out


def compute_velocities_variable(results, positions) -> list[npt.NDArray[np.float64]]:
    """Velocities at a different point set for every output step."""
    out = []
    for i, (t, pts) in enumerate(zip(results.settings.time_settings.output_times, positions, strict=True)):
        cpts = np.ascontiguousarray(pts, dtype=np.float64)
        if cpts.ndim != 2 or cpts.shape[1] != 3:
            raise ValueError("Positions must be an array of 3 component position vectors.")
        out.append(_velocity(results, i, t, cpts))
    return out
