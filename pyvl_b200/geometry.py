"""Geometry containers (python/pyvl/geometry.py:91-731).

``Geometry`` is one body: a Mesh, its node positions in the body frame and a
ReferenceFrame.  ``SimulationGeometry`` merges bodies into one mesh, detects closed
bodies (every dual line has both rings) and finds shedding edges.  Plotting helpers of the
reference (pyvista) have no counterpart here.
"""

from __future__ import annotations

from collections.abc import Iterator, Mapping, Sequence
from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

from .cvl import INVALID_ID, Mesh, ReferenceFrame
from .fio.io_common import HirearchicalMap


def mesh_to_serial(m: Mesh) -> HirearchicalMap:
    out = HirearchicalMap()
    out.insert_int("n_points", m.n_points)
    counts, flat = m.to_element_connectivity()
    out.insert_array("n_per_element", counts)
    out.insert_array("flattened_elements", flat)
    return out


def mesh_from_serial(group: HirearchicalMap) -> Mesh:
    counts = group.get_array("n_per_element")
    flat = np.asarray(group.get_array("flattened_elements"), np.uint32)
    offsets = np.pad(np.cumsum(counts), (1, 0))
    return Mesh(group.get_int("n_points"), [flat[offsets[i]: offsets[i + 1]] for i in range(counts.size)])


def rf_to_serial(rf: ReferenceFrame) -> HirearchicalMap:
    out = HirearchicalMap()
    out.insert_type("type", type(rf))
    data = HirearchicalMap()
    rf.save(data)
    out.insert_hirearchycal_map("data", data)
    if rf.parent is not None:
        out.insert_hirearchycal_map("parent", rf_to_serial(rf.parent))
    return out


def rf_from_serial(group: HirearchicalMap) -> ReferenceFrame:
    cls = group.get_type("type")
    parent = rf_from_serial(group.get_hirearchical_map("parent")) if "parent" in group else None
    return cls.load(group=group.get_hirearchical_map("data"), parent=parent)


@dataclass(init=False, frozen=True, eq=False)
class Geometry:
    """One body: label, reference frame, mesh and body-frame node positions (:91-358)."""

    label: str
    reference_frame: ReferenceFrame
    positions: npt.NDArray[np.float64]
    msh: Mesh

    def __init__(self, label: str, reference_frame: ReferenceFrame, mesh: Mesh, positions) -> None:
        if not isinstance(label, str):
            raise TypeError(f"label must be a string, instead it was {type(label).__name__}.")
        if not isinstance(reference_frame, ReferenceFrame):
            raise TypeError(f"reference_frame must be a ReferenceFrame, instead it was {type(reference_frame).__name__}.")
        if not isinstance(mesh, Mesh):
            raise TypeError(f"mesh must be a either Mesh object, instead it was {type(mesh)}.")
        try:
            pos = np.array(positions, np.float64).reshape((-1, 3))
        except Exception as e:
            raise ValueError("Positions must be a (N, 3) array.") from e
        object.__setattr__(self, "label", label)
        object.__setattr__(self, "reference_frame", reference_frame)
        object.__setattr__(self, "positions", pos)
        object.__setattr__(self, "msh", mesh)

    def save(self) -> HirearchicalMap:
        out = HirearchicalMap()
        out.insert_array("positions", self.positions)
        out.insert_hirearchycal_map("mesh", mesh_to_serial(self.msh))
        out.insert_hirearchycal_map("reference_frame", rf_to_serial(self.reference_frame))
        return out

    @classmethod
    def load(cls, label: str, group: HirearchicalMap):
        return cls(label=label, reference_frame=rf_from_serial(group.get_hirearchical_map("reference_frame")),
                   mesh=mesh_from_serial(group.get_hirearchical_map("mesh")), positions=group.get_array("positions"))

    def __eq__(self, other) -> bool:
        return (isinstance(other, Geometry) and self.label == other.label and self.msh == other.msh
                and np.allclose(self.positions, other.positions))

    @property
    def normals(self) -> npt.NDArray[np.float64]:
        n = self.msh.surface_normal(self.positions)
        return self.reference_frame.from_parent_without_offset(n, n)

    @property
    def centers(self) -> npt.NDArray[np.float64]:
        c = self.msh.surface_average_vec3(self.positions)
        return self.reference_frame.from_parent_with_offset(c, c)


@dataclass(frozen=True, eq=False)
class GeometryInfo:
    """Where one body sits in the merged mesh (:361-385)."""

    rf: ReferenceFrame
    msh: Mesh
    pos: npt.NDArray[np.float64]
    closed: bool
    points: slice
    lines: slice
    surfaces: slice


@dataclass(frozen=True)
class SimulationGeometry(Mapping):
    """Bodies merged into one mesh (:388-731)."""

    _info: dict
    mesh: Mesh
    dual: Mesh
    n_surfaces: int
    n_lines: int
    n_points: int

    def __init__(self, *geometries: Geometry) -> None:
        info: dict[str, GeometryInfo] = {}
        meshes = []
        n_points = n_lines = n_surfaces = 0
        for g in geometries:
            if g.label in info:
                raise ValueError(f'Geometries with duplicated label "{g.label}" were found.')
            meshes.append(g.msh)
            dl = g.msh.compute_dual().line_data
            closed = bool(dl.shape[0] == 0 or not np.any(dl == INVALID_ID))
            c_p, c_l, c_s = g.msh.n_points, g.msh.n_lines, g.msh.n_surfaces
            info[g.label] = GeometryInfo(g.reference_frame, g.msh, g.positions, closed,
                                         slice(n_points, n_points + c_p), slice(n_lines, n_lines + c_l),
                                         slice(n_surfaces, n_surfaces + c_s))
            n_points += c_p
            n_lines += c_l
            n_surfaces += c_s
        mesh = Mesh.merge_meshes(*meshes)
        object.__setattr__(self, "_info", info)
        object.__setattr__(self, "mesh", mesh)
        object.__setattr__(self, "dual", mesh.compute_dual())
        object.__setattr__(self, "n_points", n_points)
        object.__setattr__(self, "n_lines", n_lines)
        object.__setattr__(self, "n_surfaces", n_surfaces)

    def __getitem__(self, key: str) -> GeometryInfo:
        return self._info[key]

    def __iter__(self) -> Iterator[str]:
        return iter(self._info)

    def __len__(self) -> int:
        return len(self._info)

    def positions_at_time(self, t: float) -> npt.NDArray[np.float64]:
        pos = np.empty((self.n_points, 3), np.float64)
        for name in self._info:
            info = self._info[name]
            pos[info.points] = info.rf.at_time(float(t)).to_global_with_offset(info.pos)
        return pos

    def velocity_at_time(self, t: float) -> npt.NDArray[np.float64]:
        vel = np.empty((self.n_points, 3), np.float64)
        for name in self._info:
            info = self._info[name]
            rf = info.rf.at_time(float(t))
            pos = np.array(info.pos)
            v = np.zeros_like(pos)
            while rf is not None:
                rf.add_velocity(pos, v)
                rf.to_parent_with_offset(pos, pos)
                rf.to_parent_without_offset(v, v)
                rf = rf.parent
            vel[info.points] = v
        return vel

    def te_normal_criterion(self, crit: float) -> npt.NDArray[np.uint32]:
        """Edges between rings whose normals have dot product < crit (:615-638)."""
        normals = np.empty((self.n_surfaces, 3), np.float64)
        for name in self._info:
            info = self._info[name]
            normals[info.surfaces] = info.msh.surface_normal(info.pos)
        return self.dual.dual_normal_criterion(crit, normals)

    def te_free_criterion(self) -> npt.NDArray[np.uint32]:
        """Edges with only one ring attached (:640-652)."""
        return self.dual.dual_free_edges()

    def line_adjecency_information(self, lines: Sequence[int] | npt.NDArray[np.integer]):
        """(bordering nodes, adjacent rings) of the given lines (:654-681)."""
        ids = np.asarray(lines, np.int64).reshape(-1)
        return (self.mesh.line_data[ids].astype(np.uint64), self.dual.line_data[ids].astype(np.uint64))

    def save(self) -> HirearchicalMap:
        out = HirearchicalMap()
        for name in self._info:
            info = self._info[name]
            out.insert_hirearchycal_map(name, Geometry(name, info.rf, info.msh, info.pos).save())
        return out

    @classmethod
    def load(cls, group: HirearchicalMap):
        return cls(*[Geometry.load(str(k), group.get_hirearchical_map(k)) for k in group])
