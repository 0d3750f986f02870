"""pyvl_b200: the UVLM hot path of PyVL (python/pyvl/__init__.py) on one B200.

The names the reference package exports are re-exported here: Mesh, Line, Surface,
GeoID, ReferenceFrame, INVALID_ID, Geometry, SimulationGeometry, the flow conditions,
settings, reference frames, run_solver, the wake models, HirearchicalMap and postprocess.
Their compute runs in libpvl_b200.so (hand-written sm_100a kernels behind a C ABI, see
include/pvl_b200.h); PyTorch only provides device memory and streams.

Attributes load lazily, so ``pyvl_b200.workloads`` (seeded test and benchmark geometries)
imports without touching CUDA.
"""

from __future__ import annotations

import importlib

_EXPORTS = {
    "GeoID": "cvl", "Line": "cvl", "Surface": "cvl", "Mesh": "cvl", "ReferenceFrame": "cvl", "INVALID_ID": "cvl",
    "HirearchicalMap": "fio.io_common",
    "FlowConditions": "flow_conditions", "FlowConditionsUniform": "flow_conditions",
    "FlowConditionsRotating": "flow_conditions",
    "Geometry": "geometry", "SimulationGeometry": "geometry",
    "RotorReferenceFrame": "reference_frames", "TranslatingReferenceFrame": "reference_frames",
    "ModelSettings": "settings", "SolverSettings": "settings", "TimeSettings": "settings",
    "OutputSettings": "solver", "run_solver": "solver", "compute_induced_velocities": "solver",
    "SolverResults": "solver", "SolverState": "solver",
    "WakeModel": "wake", "WakeModelLineExplicitUnsteady": "wake_models",
    "SolverEngine": "engine", "WakeSpec": "engine",
}

__all__ = sorted(_EXPORTS) + ["postprocess", "workloads"]


def __getattr__(name: str):
    if name in _EXPORTS:
        mod = importlib.import_module(f"{__name__}.{_EXPORTS[name]}")
        value = getattr(mod, name)
        globals()[name] = value
        return value
    if name in ("postprocess", "workloads", "engine", "cvl", "fio"):
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
