"""Circulatory line forces (python/pyvl/postprocess/forces.py:10-42) and the lift coefficient."""

from __future__ import annotations

import numpy as np
import numpy.typing as npt

from ..cvl import Mesh


def circulatory_forces(results) -> list[npt.NDArray[np.float64]]:
    """Kutta-Joukowski force on every body line at each output time.

    The body's induced velocity at the nodes is one fused contraction (no
    (n_points, n_surfaces, 3) matrix); the wake's comes from its get_velocity."""
    out = []
    tol = results.settings.model_settings.vortex_limit
    flow = results.settings.flow_conditions
    for i, t in enumerate(results.settings.time_settings.output_times):
        gamma = results.circulations[i, :]
        positions = results.geometry.positions_at_time(t)
        freestream = flow.get_velocity(t, positions)
        induced = results.geometry.mesh.induced_velocity(tol, positions, positions, gamma)
        motion = results.geometry.velocity_at_time(t)
        wm = results.wake_models[i]
        if wm is not None:
            induced = induced + wm.get_velocity(positions)
        forces = Mesh.line_forces(results.geometry.mesh, results.geometry.dual, gamma / (2 * np.pi), positions,
                                  freestream + induced - motion)
        if wm is not None:
            wm.correct_forces(forces, results.geometry, positions, gamma, flow)
        out.append(forces)
    return out


def lift_coefficient(forces: npt.NDArray[np.float64], freestream, s_ref: float) -> float:
    """CL = (sum of line forces) . l / (0.5 |U|^2 S_ref), l the unit normal to U in the x-z plane
    (rho = 1: the line forces carry no density, src/meshobject.c:1389-1392)."""
    u = np.asarray(freestream, np.float64)
    lift = np.array([-u[2], 0.0, u[0]])
    lift /= np.linalg.norm(lift)
    return float(np.asarray(forces).sum(axis=0) @ lift / (0.5 * float(u @ u) * s_ref))
