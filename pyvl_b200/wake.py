"""The wake-model interface (python/pyvl/wake.py:16-157)."""

from __future__ import annotations

from abc import ABC, abstractmethod

import numpy as np
from numpy import typing as npt

from .fio.io_common import HirearchicalMap


class WakeModel(ABC):
    """A wake model: updated every iteration, corrects the system (implicit and explicit
    parts), gives its induced velocity, corrects forces, saves and loads its state."""

    @abstractmethod
    def update(self, time: float, geometry, positions: npt.NDArray[np.float64],
               circulation: npt.NDArray[np.float64], flow) -> None: ...

    @abstractmethod
    def apply_corrections(self, control_pts: npt.NDArray[np.float64], normals: npt.NDArray[np.float64],
                          mat_in: npt.NDArray[np.float64], rhs_in: npt.NDArray[np.float64]) -> None: ...

    @abstractmethod
    def get_velocity(self, positions: npt.NDArray[np.float64]) -> npt.NDArray[np.float64]: ...

    @abstractmethod
    def correct_forces(self, line_forces: npt.NDArray[np.float64], geometry, positions: npt.NDArray[np.float64],
                       circulation: npt.NDArray[np.float64], flow) -> None: ...

    @abstractmethod
    def save(self) -> HirearchicalMap: ...

    @classmethod
    @abstractmethod
    def load(cls, group: HirearchicalMap): ...
