"""Free-stream definitions (python/pyvl/flow_conditions.py:15-541).

``FlowConditionsUniform`` is evaluated on the device by the solver kernels (its velocity
enters pvl_rhs and pvl_wake_node_velocity as three numbers); any other FlowConditions is
evaluated with numpy at the points the solver hands it.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

from .fio.io_common import HirearchicalMap


class FlowConditions(ABC):
    """Velocity, density and pressure fields of the flow (flow_conditions.py:15-140)."""

    @abstractmethod
    def get_velocity(self, time: float, positions: npt.NDArray[np.float64],
                     out_array: npt.NDArray[np.float64] | None = None) -> npt.NDArray[np.float64]: ...

    @abstractmethod
    def get_density(self, time: float, positions: npt.NDArray[np.float64],
                    out_array: npt.NDArray[np.float64] | None = None) -> npt.NDArray[np.float64]: ...

    @abstractmethod
    def get_pressure(self, time: float, positions: npt.NDArray[np.float64],
                     out_array: npt.NDArray[np.float64] | None = None) -> npt.NDArray[np.float64]: ...

    @abstractmethod
    def save(self) -> HirearchicalMap: ...

    @classmethod
    @abstractmethod
    def load(cls, hmap: HirearchicalMap): ...


def _fill(value, positions, out_array):
    if out_array is not None:
        out_array[...] = value
        return out_array
    return np.full(np.shape(positions)[0], value, np.float64)


@dataclass(frozen=True)
class FlowConditionsUniform(FlowConditions):
    """Uniform velocity (vx, vy, vz), constant density and static pressure (:142-328)."""

    vx: float
    vy: float
    vz: float
    rho: float = 1.225
    p_stat: float = 101325

    @property
    def velocity(self) -> npt.NDArray[np.float64]:
        return np.array((self.vx, self.vy, self.vz), np.float64)

    def get_velocity(self, time, positions, out_array=None):
        v = self.velocity
        if out_array is not None:
            out_array[:, :] = v[None, :]
            return out_array
        return np.full_like(np.asarray(positions, np.float64), v)

    def get_density(self, time, positions, out_array=None):
        return _fill(self.rho, positions, out_array)

    def get_pressure(self, time, positions, out_array=None):
        return _fill(self.p_stat, positions, out_array)

    def save(self) -> HirearchicalMap:
        hm = HirearchicalMap()
        hm.insert_array("velocity", (self.vx, self.vy, self.vz))
        return hm

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        return cls(*hmap.get_array("velocity"))


@dataclass(frozen=True)
class FlowConditionsRotating(FlowConditions):
    """Rotation about a centre: v(r) = (r - r0) x omega (:331-541)."""

    center_x: float
    center_y: float
    center_z: float
    omega_x: float
    omega_y: float
    omega_z: float
    rho: float = 1.225
    p_stat: float = 101325.0

    def get_velocity(self, time, positions, out_array=None):
        pos = np.asarray(positions, np.float64) - np.array(((self.center_x, self.center_y, self.center_z),))
        return np.cross(pos, np.array((self.omega_x, self.omega_y, self.omega_z), np.float64))

    def get_density(self, time, positions, out_array=None):
        return _fill(self.rho, positions, out_array)

    def get_pressure(self, time, positions, out_array=None):
        return _fill(self.p_stat, positions, out_array)

    def save(self) -> HirearchicalMap:
        hm = HirearchicalMap()
        hm.insert_array("center", (self.center_x, self.center_y, self.center_z))
        hm.insert_array("omega", (self.omega_x, self.omega_y, self.omega_z))
        return hm

    @classmethod
    def load(cls, hmap: HirearchicalMap):
        return cls(*(*hmap.get_array("center"), *hmap.get_array("omega")))
