"""Dynamic pressure (python/pyvl/postprocess/pressure.py:11-107), fused on the GPU."""

from __future__ import annotations

import numpy as np
import numpy.typing as npt


def compute_surface_dynamic_pressure(results) -> list[npt.NDArray[np.float64]]:
    """Dynamic pressure at the ring centres for every output step."""
    tol = results.settings.model_settings.vortex_limit
    flow = results.settings.flow_conditions
    out = []
    for i, t in enumerate(results.settings.time_settings.output_times):
        geo = results.geometry
        pos = geo.positions_at_time(t)
        cpts = geo.mesh.surface_average_vec3(pos)
        induced = geo.mesh.induced_velocity(tol, pos, cpts, results.circulations[i, :])
        induced = induced - geo.mesh.surface_average_vec3(geo.velocity_at_time(t))
        fs = flow.get_velocity(t, cpts)
        wm = results.wake_models[i]
        if wm is not None:
            induced = induced + wm.get_velocity(cpts)
        p = np.einsum("ij,ij->i", induced, 0.5 * induced + fs)
        out.append(-flow.get_density(t, cpts) * p)
    return out


def compute_dynamic_pressure_variable(results, positions) -> list[npt.NDArray[np.float64]]:
    """Dynamic pressure at a different point set for every output step."""
    tol = results.settings.model_settings.vortex_limit
    flow = results.settings.flow_conditions
    out = []
    for i, (t, pts) in enumerate(zip(results.settings.time_settings.output_times, positions, strict=True)):
        cpts = np.ascontiguousarray(pts, dtype=np.float64)
        if cpts.ndim != 2 or cpts.shape[1] != 3:
            raise ValueError("Positions must be an array of 3 component position vectors.")
        pos = results.geometry.positions_at_time(t)
        induced = results.geometry.mesh.induced_velocity(tol, pos, cpts, results.circulations[i, :])
        fs = flow.get_velocity(t, cpts)
        wm = results.wake_models[i]
        if wm is not None:
            induced = induced + wm.get_velocity(cpts)
        p = np.einsum("ij,ij->i", induced, 0.5 * induced + fs)
        out.append(-flow.get_density(t, cpts) * p)
    return out
