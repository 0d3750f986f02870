"""The solver loop (python/pyvl/solver.py:21-279).

``run_solver(geometry, settings, wake_model, output_settings)`` keeps the reference's
signature and results.  Each iteration computes node positions and velocities from the
bodies' reference frames on the host (as the reference does, solver.py:178-197) and hands
them to a :class:`~pyvl_b200.engine.SolverEngine`, which assembles, corrects and solves the
system and advances the wake on the GPU.  With a ``WakeModelLineExplicitUnsteady`` the wake
state stays on the device between iterations and is copied into the model object at every
output step; any other WakeModel is driven through its own methods (its corrections are
applied to the system on the host, then the system is solved on the GPU).

Closed bodies: the reference solves the singular system by LU and then removes each closed
body's mean circulation (solver.py:229-233).  Here the zero-mean condition is imposed as a
bordered system (one Lagrange multiplier per closed body), the well-posed form of the same
constraint; the mean removal is then applied as well.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path
from time import perf_counter
from typing import Callable, Literal

import numpy as np
import numpy.typing as npt
import torch

from .cvl import ReferenceFrame
from .engine import SolverEngine, WakeSpec
from .fio.io_common import HirearchicalMap
from .fio.io_json import serialize_json
from .flow_conditions import FlowConditionsUniform
from .geometry import SimulationGeometry
from .settings import SolverSettings
from .wake import WakeModel
from .wake_models import WakeModelLineExplicitUnsteady


class SolverResults:
    """Circulations and wake snapshots at the output times (solver.py:21-39)."""

    def __init__(self, geo: SimulationGeometry, settings: SolverSettings):
        self.geometry = geo
        self.settings = SolverSettings(flow_conditions=settings.flow_conditions,
                                       model_settings=settings.model_settings,
                                       time_settings=settings.time_settings)
        self.wake_models: list[WakeModel | None] = []
        self.circulations = np.empty((settings.time_settings.output_times.size, geo.n_surfaces), np.float64)


class SolverState:
    """State of the solver at one iteration (solver.py:42-108)."""

    def __init__(self, geometry: SimulationGeometry, settings: SolverSettings, wake_model: WakeModel | None) -> None:
        self.geometry = geometry
        self.positions = np.empty((geometry.n_points, 3), np.float64)
        self.normals = np.empty((geometry.n_surfaces, 3), np.float64)
        self.control_points = np.empty((geometry.n_surfaces, 3), np.float64)
        self.cp_velocity = np.empty((geometry.n_surfaces, 3), np.float64)
        self.circulation = np.empty((geometry.n_surfaces,), np.float64)
        self.settings = settings
        self.wake_model = wake_model
        self.iteration = 0

    def save(self) -> HirearchicalMap:
        out = HirearchicalMap()
        out.insert_array("positions", self.positions)
        out.insert_array("normals", self.normals)
        out.insert_array("control_points", self.control_points)
        out.insert_array("cp_velocity", self.cp_velocity)
        out.insert_array("circulation", self.circulation)
        out.insert_int("iteration", self.iteration)
        out.insert_hirearchycal_map("solver_settings", self.settings.save())
        out.insert_hirearchycal_map("simulation_geometry", self.geometry.save())
        if self.wake_model is not None:
            wm = HirearchicalMap()
            wm.insert_type("type", type(self.wake_model))
            wm.insert_hirearchycal_map("data", self.wake_model.save())
            out.insert_hirearchycal_map("wake_model", wm)
        return out

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        geometry = SimulationGeometry.load(hmap.get_hirearchical_map("simulation_geometry"))
        settings = SolverSettings.load(hmap.get_hirearchical_map("solver_settings"))
        wake_model = None
        if "wake_model" in hmap:
            wm = hmap.get_hirearchical_map("wake_model")
            wake_model = wm.get_type("type").load(wm.get_hirearchical_map("data"))
        self = cls(geometry=geometry, settings=settings, wake_model=wake_model)
        self.iteration = hmap.get_int("iteration")
        self.positions[:] = hmap.get_array("positions")
        self.normals[:] = hmap.get_array("normals")
        self.control_points[:] = hmap.get_array("control_points")
        self.circulation[:] = hmap.get_array("circulation")
        self.cp_velocity[:] = hmap.get_array("cp_velocity")
        return self


OutputFileType = Literal["HDF5", "JSON"]


@dataclass(init=False, eq=False, frozen=True)
class OutputSettings:
    """File format and naming callback of solver output (solver.py:114-142)."""

    naming_callback: Callable[[int, float], str | Path]
    serialization_fn: Callable

    def __init__(self, ftype: OutputFileType, naming_callback: Callable[[int, float], str | Path]) -> None:
        if ftype == "JSON":
            fn = serialize_json
        elif ftype == "HDF5":
            from .fio.io_hdf5 import serialize_hdf5 as fn  # needs h5py
        else:
            raise ValueError(f"The file type {ftype=} is not valid.")
        object.__setattr__(self, "serialization_fn", fn)
        object.__setattr__(self, "naming_callback", naming_callback)


def _frame_kinematics(geometry: SimulationGeometry, time: float, state: SolverState) -> np.ndarray:
    """Positions, control points, velocities and normals from the frames (solver.py:178-197)."""
    vel_all = np.zeros((geometry.n_points, 3), np.float64)
    for name in geometry:
        info = geometry[name]
        rf: ReferenceFrame | None = info.rf.at_time(time)
        positions = np.array(info.pos)
        velocities = np.zeros_like(positions)
        while rf is not None:
            positions = rf.to_parent_with_offset(positions, positions)
            rf.add_velocity(positions, velocities)
            velocities = rf.to_parent_without_offset(velocities, velocities)
            rf = rf.parent
        state.positions[info.points] = positions
        vel_all[info.points] = velocities
    return vel_all


def _closed_groups(geometry: SimulationGeometry) -> list[tuple[int, int]]:
    return [(geometry[n].surfaces.start, geometry[n].surfaces.stop) for n in geometry if geometry[n].closed]


def run_solver(geometry: SimulationGeometry, settings: SolverSettings, wake_model: WakeModel | None,
               output_settings: OutputSettings | None, verbose: bool = True) -> SolverResults:
    """Run the flow solver over the time settings (solver.py:145-265)."""
    results = SolverResults(geometry, settings)
    ts = settings.time_settings
    times = np.array((0,), np.float64) if ts is None else np.arange(ts.nt) * ts.dt
    tol = settings.model_settings.vortex_limit
    flow = settings.flow_conditions
    uniform = isinstance(flow, FlowConditionsUniform)
    resident = isinstance(wake_model, WakeModelLineExplicitUnsteady) and uniform
    spec = None
    if resident:
        spec = WakeSpec(wake_model.shedding_lines.astype(np.uint32), wake_model.bordering_nodes.astype(np.uint32),
                        wake_model.adjacent_surfaces.astype(np.uint32), wake_model.line_rows,
                        float(wake_model.current_time))
    engine = SolverEngine(geometry.mesh, flow.velocity if uniform else np.zeros(3), tol, spec,
                          _closed_groups(geometry))
    if resident and wake_model.step_count > 0:
        engine.set_wake_state(wake_model.wake_positions, wake_model.circulation, wake_model.step_count,
                              wake_model.current_time)
    state = SolverState(geometry, settings, wake_model)
    i_out = 0
    for iteration, time in enumerate(times):
        state.iteration = iteration
        t_begin = perf_counter()
        velocities = _frame_kinematics(geometry, float(time), state)
        engine.iteration = iteration
        engine.load_inputs(state.positions, velocities)
        if uniform and (resident or wake_model is None):
            engine.assemble()
        else:
            # general flow field or wake model: RHS and corrections on the host, solve on the GPU
            engine.assemble_body_only()
            cps = engine.cps.cpu().numpy()
            nrm = engine.nrm.cpu().numpy()
            cpv = engine.cpv.cpu().numpy()
            ev = flow.get_velocity(time, cps) - cpv
            rhs = np.vecdot(nrm, -ev, axis=1)
            A = engine.A[: engine.P, : engine.P].cpu().numpy()
            if wake_model is not None and iteration > 0:
                wake_model.apply_corrections(cps, nrm, A, rhs)
            engine.A[: engine.P, : engine.P].copy_(torch.from_numpy(A))
            engine.rhs[: engine.P].copy_(torch.from_numpy(rhs))
            engine.border()
        engine.solve()
        circulation = engine.gamma_host()
        engine.check_status()
        state.control_points[:] = engine.cps.cpu().numpy()
        state.normals[:] = engine.nrm.cpu().numpy()
        state.cp_velocity[:] = engine.cpv.cpu().numpy()
        state.circulation[:] = circulation
        if wake_model is not None:
            if resident:
                engine.wake_update(float(time))
            else:
                wake_model.update(time, geometry, state.positions, circulation, flow)
        t_end = perf_counter()
        if ts is None or ts.output_interval is None or iteration % ts.output_interval == 0:
            results.circulations[i_out, :] = circulation
            if wake_model is not None:
                if resident:
                    _sync_wake(engine, wake_model)
                results.wake_models.append(wake_model.copy_state() if hasattr(wake_model, "copy_state")
                                           else type(wake_model).load(wake_model.save()))
            else:
                results.wake_models.append(None)
            if output_settings is not None:
                output_settings.serialization_fn(state.save(), output_settings.naming_callback(iteration, time))
            i_out += 1
        if verbose:
            print(f"Finished iteration {iteration} out of {len(times)} in {t_end - t_begin:g} seconds.")
    if resident:
        _sync_wake(engine, wake_model)
    return results


def _sync_wake(engine: SolverEngine, wm: WakeModelLineExplicitUnsteady) -> None:
    wm.wake_positions[...] = engine.wake_positions.cpu().numpy()
    wm.circulation[...] = engine.wake_circulation.cpu().numpy()
    wm.step_count = int(engine.wake["step_count"])
    wm.current_time = engine.wake["time"]


def compute_induced_velocities(state: SolverState, positions: npt.ArrayLike) -> npt.NDArray:
    """Velocity induced by the body's circulation at arbitrary points (solver.py:268-279), fused."""
    points = np.asarray(positions, np.float64).reshape((-1, 3))
    return state.geometry.mesh.induced_velocity(state.settings.model_settings.vortex_limit, state.positions, points,
                                                state.circulation)
