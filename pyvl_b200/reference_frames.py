"""Moving reference frames (python/pyvl/reference_frames.py:15-322)."""

from __future__ import annotations

import numpy as np

from .cvl import ReferenceFrame
from .fio.io_common import HirearchicalMap


class TranslatingReferenceFrame(ReferenceFrame):
    """Frame moving with constant velocity: r'(t) = R r + d + v (t - t0)."""

    def __new__(cls, offset=(0, 0, 0), theta=(0, 0, 0), velocity=(0, 0, 0), parent=None, time: float = 0.0):
        self = super().__new__(cls, offset=offset, theta=theta, parent=parent)
        self.vel = np.array(velocity, np.float64).reshape((3,))
        self.time = float(time)
        return self

    def at_time(self, t: float) -> TranslatingReferenceFrame:
        dt = t - self.time
        return TranslatingReferenceFrame(offset=self.offset + dt * self.vel, velocity=self.vel, time=t,
                                         parent=self.parent.at_time(t) if self.parent is not None else None,
                                         theta=self.angles)

    def save(self, group: HirearchicalMap) -> None:
        group.insert_array("velocity", self.vel)
        group.insert_scalar("time", self.time)
        group.insert_array("offset", self.offset)
        group.insert_array("angles", self.angles)

    @classmethod
    def load(cls, group: HirearchicalMap, parent=None):
        return cls(group.get_array("offset"), group.get_array("angles"), group.get_array("velocity"), parent,
                   group.get_scalar("time"))

    def add_velocity(self, positions, velocity, /) -> None:
        super().add_velocity(positions, velocity)
        velocity[:, :] += self.vel[None, :]


class RotorReferenceFrame(ReferenceFrame):
    """Frame rotating with constant angular velocity omega about its origin."""

    def __new__(cls, offset=(0, 0, 0), theta=(0, 0, 0), parent=None, omega=(0, 0, 0), time: float = 0.0):
        self = super().__new__(cls, offset=offset, theta=theta, parent=parent)
        self.omega = np.array(omega, np.float64).reshape((3,))
        self.time = time
        return self

    @staticmethod
    def _rotate(omega, r, dt: float):
        """Rotate r about the axis omega by |omega| dt (reference_frames.py:205-235)."""
        w = np.linalg.norm(omega)
        if w == 0:
            return np.array(r)
        d = omega / w
        rp = np.dot(r, d) * d
        v1 = r - rp
        v2 = np.cross(r, d)
        phi = np.arctan2(v2, v1)
        rad = np.hypot(v1, v2)
        return rp + rad * np.cos(phi + w * dt)

    def at_time(self, t: float) -> RotorReferenceFrame:
        m = self.rotation_matrix
        for i in range(3):
            m[i, :] = RotorReferenceFrame._rotate(self.omega, m[i, :], t - self.time)
        return RotorReferenceFrame(self.offset, ReferenceFrame.angles_from_rotation(m),
                                   self.parent.at_time(t) if self.parent else None, self.omega, t)

    def __repr__(self) -> str:
        o, a = self.offset, self.angles
        return (f"{type(self).__name__}({o[0]:g}, {o[1]:g}, {o[2]:g}, {a[0]:g}, {a[1]:g}, {a[2]:g}, "
                f"{self.parent}, time={self.time:g}, omega={self.omega})")

    def save(self, group: HirearchicalMap) -> None:
        group.insert_array("offset", self.offset)
        group.insert_array("angles", self.angles)
        group.insert_array("omega", self.omega)
        group.insert_scalar("time", self.time)

    @classmethod
    def load(cls, group: HirearchicalMap, parent=None):
        return cls(offset=group.get_array("offset"), theta=group.get_array("angles"), parent=parent,
                   omega=group.get_array("omega"), time=group.get_scalar("time"))

    def add_velocity(self, positions, velocity, /) -> None:
        super().add_velocity(positions, velocity)
        velocity[:, :] += np.cross(positions, self.omega[None, :])
