"""Solver settings dataclasses (python/pyvl/settings.py:13-231)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

from .fio.io_common import HirearchicalMap
from .flow_conditions import FlowConditions


@dataclass(frozen=True)
class TimeSettings:
    """nt steps of dt; output every ``output_interval`` steps (all when None)."""

    nt: int
    dt: float
    output_interval: int | None = None

    @property
    def simulation_times(self) -> npt.NDArray[np.float64]:
        return np.arange(self.nt, dtype=np.float64) * np.float64(self.dt)

    @property
    def output_times(self) -> npt.NDArray[np.float64]:
        if self.output_interval is None or self.output_interval == 0:
            return self.simulation_times
        return np.float64(self.dt) * np.arange(self.nt, step=self.output_interval, dtype=np.float64)

    def save(self) -> HirearchicalMap:
        hm = HirearchicalMap()
        hm.insert_int("nt", self.nt)
        hm.insert_scalar("dt", self.dt)
        if self.output_interval is not None:
            hm.insert_int("output_interval", self.output_interval)
        return hm

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        oi = hmap.get_int("output_interval") if "output_interval" in hmap else None
        return cls(nt=hmap.get_int("nt"), dt=hmap.get_scalar("dt"), output_interval=oi)


@dataclass
class ModelSettings:
    """``vortex_limit``: the cut-off distance below which a segment induces nothing."""

    vortex_limit: float

    def save(self) -> HirearchicalMap:
        hm = HirearchicalMap()
        hm.insert_scalar("vortex_limit", self.vortex_limit)
        return hm

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        return cls(vortex_limit=hmap.get_scalar("vortex_limit"))


@dataclass(frozen=True)
class SolverSettings:
    """Flow conditions, model settings and time settings of a run."""

    flow_conditions: FlowConditions
    model_settings: ModelSettings
    time_settings: TimeSettings = TimeSettings(1, 1, None)

    def save(self) -> HirearchicalMap:
        hm = HirearchicalMap()
        fc = HirearchicalMap()
        fc.insert_type("type", type(self.flow_conditions))
        fc.insert_hirearchycal_map("data", self.flow_conditions.save())
        hm.insert_hirearchycal_map("flow_conditions", fc)
        hm.insert_hirearchycal_map("model_settings", self.model_settings.save())
        hm.insert_hirearchycal_map("time_settings", self.time_settings.save())
        return hm

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        fc = hmap.get_hirearchical_map("flow_conditions")
        flow = fc.get_type("type").load(fc.get_hirearchical_map("data"))
        return cls(flow_conditions=flow,
                   model_settings=ModelSettings.load(hmap.get_hirearchical_map("model_settings")),
                   time_settings=TimeSettings.load(hmap.get_hirearchical_map("time_settings")))
