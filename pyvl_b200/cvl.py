"""The reference's C-level types, re-provided on top of libpvl_b200.

Mirrors python/pyvl/cvl.pyi:14-672 (types GeoID, Line, Surface, Mesh, ReferenceFrame and
the constant INVALID_ID).  Topology is built by the native host code of the C ABI; every
induction, normal and centroid computation runs as a CUDA kernel.  Arrays go in and come
out as numpy (the reference's contract); CUDA tensors are accepted too and then stay on
the device.
"""

from __future__ import annotations

import math
from collections.abc import Sequence

import numpy as np
import numpy.typing as npt
import torch

from . import _lib
from .device import Workspace, ptr, require_cuda, stream_ptr, to_device, to_device_u32

INVALID_ID: int = _lib.INVALID_ID


# --------------------------------------------------------------------------- small types
class GeoID:
    """Index with an orientation flag (src/geoidobject.c; src/core/common.h:46-50)."""

    __slots__ = ("_index", "_orientation")

    def __init__(self, index: int, orientation: object = False) -> None:
        self._index = int(index) & 0x7FFFFFFF
        self._orientation = bool(orientation)

    @property
    def index(self) -> int:
        return self._index

    @index.setter
    def index(self, v: int) -> None:
        self._index = int(v) & 0x7FFFFFFF

    @property
    def orientation(self) -> bool:
        return self._orientation

    @orientation.setter
    def orientation(self, o) -> None:
        self._orientation = bool(o)

    def __eq__(self, other) -> bool:
        return isinstance(other, GeoID) and other._index == self._index and other._orientation == self._orientation

    def __str__(self) -> str:
        return f"{'-' if self._orientation else '+'}{self._index}"

    def __repr__(self) -> str:
        return f"GeoID({self._index}, {self._orientation})"


class Line:
    """Connection between two points (src/lineobject.c)."""

    __slots__ = ("begin", "end")

    def __init__(self, begin: int | GeoID, end: int | GeoID) -> None:
        self.begin = begin.index if isinstance(begin, GeoID) else int(begin)
        self.end = end.index if isinstance(end, GeoID) else int(end)

    def __eq__(self, other) -> bool:
        return isinstance(other, Line) and other.begin == self.begin and other.end == self.end

    def __str__(self) -> str:
        return f"({self.begin} -> {self.end})"

    def __repr__(self) -> str:
        return f"Line({self.begin}, {self.end})"


class Surface:
    """Closed loop of lines (src/surfaceobject.c).  Consecutive lines must connect."""

    __slots__ = ("_lines",)

    def __init__(self, lines: Sequence[Line]) -> None:
        lines = tuple(lines)
        for i, ln in enumerate(lines):
            nxt = lines[(i + 1) % len(lines)]
            if ln.end != nxt.begin:
                raise ValueError(f"Line {i} ends at {ln.end}, but line {(i + 1) % len(lines)} begins at {nxt.begin}.")
        self._lines = lines

    @property
    def n_lines(self) -> int:
        return len(self._lines)

    @property
    def lines(self) -> tuple[Line, ...]:
        return self._lines

    def __str__(self) -> str:
        return "Surface(" + ", ".join(str(ln) for ln in self._lines) + ")"

    __repr__ = __str__


# --------------------------------------------------------------------------- helpers
def _is_tensor(a) -> bool:
    return isinstance(a, torch.Tensor)


def _check_array(a, shape: tuple, name: str, dtype=np.float64) -> None:
    """Shape/dtype validation with the reference's messages (src/common.h:8-66)."""
    if not isinstance(a, (np.ndarray, torch.Tensor)):
        raise TypeError(f"{name} was not an array, but was instead {type(a)}")
    if len(a.shape) != len(shape):
        raise ValueError(f"{name} did not have the expected number of axis ({len(shape)} required, {len(a.shape)} found).")
    for i, (want, got) in enumerate(zip(shape, a.shape)):
        if want and want != got:
            raise ValueError(f"{name} did not have the expected shape (axis {i} should have the size of {want}, "
                             f"but was instead {got}).")
    if isinstance(a, np.ndarray) and a.dtype != dtype:
        raise ValueError(f"{name} did not have the correct data type.")
    if isinstance(a, torch.Tensor) and a.dtype != torch.float64:
        raise ValueError(f"{name} did not have the correct data type.")


def _finish(result: torch.Tensor, like, out):
    """Return the result as numpy (writing into `out` when given) unless inputs were tensors."""
    if out is not None:
        if _is_tensor(out):
            out.copy_(result.reshape(out.shape))
            return out
        out[...] = result.cpu().numpy().reshape(out.shape)
        return out
    if _is_tensor(like):
        return result
    return result.cpu().numpy()


# --------------------------------------------------------------------------- Mesh
class Mesh:
    """Ring mesh in the reference's CSR form (src/core/mesh.h:130-139; src/meshobject.c).

    ``Mesh(n_points, connectivity)`` builds unique lines and the signed ring->line lists
    exactly as the reference's mesh_from_elements does (same line numbering and
    orientation bits), in linear time.
    """

    def __init__(self, n_points: int, connectivity) -> None:
        n_points = int(n_points)
        if n_points < 0:
            raise ValueError("n_points must be non-negative")
        try:
            elems = [np.asarray(e, dtype=np.int64).reshape(-1) for e in connectivity]
        except TypeError as e:
            raise TypeError("Second parameter must be a sequence of sequences") from e
        counts = np.array([e.size for e in elems], np.uint32)
        for i, e in enumerate(elems):
            if e.size < 3:
                raise ValueError(f"Element {i} had only {e.size} indices given (at least 3 are needed).")
            if e.size and (e.min() < 0 or e.max() > 0xFFFFFFFF):
                raise ValueError(f"Element {i} has an invalid point index.")
        flat = np.ascontiguousarray(np.concatenate(elems).astype(np.uint32) if elems else np.zeros(0, np.uint32))
        total = int(flat.size)
        lines = np.zeros((max(total, 1), 2), np.uint32)
        sl = np.zeros(max(total, 1), np.uint32)
        off = np.zeros(len(elems) + 1, np.uint32)
        n_lines = np.zeros(1, np.uint32)
        _lib.call("pvl_mesh_from_elements", n_points, len(elems), counts.ctypes.data, flat.ctypes.data,
                  lines.ctypes.data, sl.ctypes.data, off.ctypes.data, n_lines.ctypes.data)
        self._init(n_points, lines[: int(n_lines[0])].copy(), off, sl[:total].copy())

    @classmethod
    def _from_arrays(cls, n_points, lines, offsets, surface_lines) -> Mesh:
        self = cls.__new__(cls)
        self._init(int(n_points), np.ascontiguousarray(lines, np.uint32).reshape(-1, 2),
                   np.ascontiguousarray(offsets, np.uint32), np.ascontiguousarray(surface_lines, np.uint32))
        return self

    def _init(self, n_points, lines, offsets, surface_lines) -> None:
        self._n_points = n_points
        self._lines = lines
        self._offsets = offsets
        self._surface_lines = surface_lines
        self._dev: dict = {}
        self._ring_map = None

    # ------------------------------------------------------------------ properties
    @property
    def n_points(self) -> int:
        return self._n_points

    @property
    def n_lines(self) -> int:
        return int(self._lines.shape[0])

    @property
    def n_surfaces(self) -> int:
        return int(self._offsets.size - 1)

    @property
    def line_data(self) -> npt.NDArray[np.uint32]:
        v = self._lines.view()
        v.flags.writeable = False
        return v

    @property
    def surface_offsets(self) -> npt.NDArray[np.uint32]:
        return self._offsets

    @property
    def surface_lines(self) -> npt.NDArray[np.uint32]:
        return self._surface_lines

    def __str__(self) -> str:
        return f"Mesh({self.n_points} points, {self.n_lines} lines, {self.n_surfaces} surfaces)"

    __repr__ = __str__

    def __eq__(self, other) -> bool:
        if not isinstance(other, Mesh):
            return NotImplemented
        return (self.n_points == other.n_points and np.array_equal(self._lines, other._lines)
                and np.array_equal(self._offsets, other._offsets)
                and np.array_equal(self._surface_lines, other._surface_lines))

    # ------------------------------------------------------------------ topology
    def get_line(self, i: int) -> Line:
        i = int(i)
        if i >= self.n_lines or i < -self.n_lines:
            raise IndexError(f"Index {i} is our of bounds for a mesh with {self.n_lines} lines.")
        a, b = self._lines[i]
        return Line(int(a), int(b))

    def get_surface(self, i: int) -> Surface:
        """Surface i; lines come out in the reference's convention: a line stored forward is
        reported reversed (src/surfaceobject.c:215-236)."""
        i = int(i)
        if i >= self.n_surfaces or i < -self.n_surfaces:
            raise IndexError(f"Index {i} is our of bounds for a mesh with {self.n_surfaces} surfaces.")
        i %= self.n_surfaces
        out = []
        for g in self._surface_lines[self._offsets[i]: self._offsets[i + 1]]:
            a, b = self._lines[int(g) & 0x7FFFFFFF]
            out.append(Line(int(a), int(b)) if (int(g) >> 31) else Line(int(b), int(a)))
        s = Surface.__new__(Surface)
        s._lines = tuple(out)
        return s

    def to_element_connectivity(self) -> tuple[npt.NDArray[np.uint32], npt.NDArray[np.uint32]]:
        counts = np.zeros(self.n_surfaces, np.uint32)
        flat = np.zeros(max(int(self._offsets[-1]), 1), np.uint32)
        _lib.call("pvl_mesh_to_elements", self.n_surfaces, self._offsets.ctypes.data, self._surface_lines.ctypes.data,
                  self._lines.ctypes.data, counts.ctypes.data, flat.ctypes.data)
        return counts, flat[: int(self._offsets[-1])]

    def compute_dual(self) -> Mesh:
        """Dual mesh (src/core/mesh.c:70-173): rings become points, points become rings."""
        dl = np.zeros((max(self.n_lines, 1), 2), np.uint32)
        doff = np.zeros(self.n_points + 1, np.uint32)
        dsl = np.zeros(max(2 * self.n_lines, 1), np.uint32)
        _lib.call("pvl_mesh_dual", self.n_points, self.n_lines, self._lines.ctypes.data, self.n_surfaces,
                  self._offsets.ctypes.data, self._surface_lines.ctypes.data, dl.ctypes.data, doff.ctypes.data,
                  dsl.ctypes.data)
        return Mesh._from_arrays(self.n_surfaces, dl[: self.n_lines], doff, dsl[: int(doff[-1])])

    def copy(self) -> Mesh:
        return Mesh._from_arrays(self.n_points, self._lines.copy(), self._offsets.copy(), self._surface_lines.copy())

    @classmethod
    def merge_meshes(cls, *meshes: Mesh) -> Mesh:
        """Concatenate meshes, offsetting point and line ids (src/meshobject.c:779-860)."""
        for i, m in enumerate(meshes):
            if not isinstance(m, Mesh):
                raise TypeError(f"Element {i} in the input sequence was not a Mesh, but was instead {type(m)}")
        lines, offs, sls = [], [np.zeros(1, np.uint32)], []
        pts = lns = ent = 0
        for m in meshes:
            lines.append(m._lines.astype(np.uint64) + pts)
            offs.append(m._offsets[1:].astype(np.uint64) + ent)
            g = m._surface_lines.astype(np.uint64)
            sls.append(((g & 0x7FFFFFFF) + lns) | (g & 0x80000000))
            pts += m.n_points
            lns += m.n_lines
            ent += int(m._offsets[-1])
        return cls._from_arrays(pts, np.concatenate(lines).astype(np.uint32) if lines else np.zeros((0, 2), np.uint32),
                                np.concatenate(offs).astype(np.uint32),
                                np.concatenate(sls).astype(np.uint32) if sls else np.zeros(0, np.uint32))

    @classmethod
    def from_lines(cls, n_points: int, connectivity) -> Mesh:
        """Line-only mesh (src/meshobject.c:1159-1230)."""
        c = np.ascontiguousarray(connectivity, np.uint32)
        if c.ndim != 2 or c.shape[1] != 2:
            raise ValueError(f"Connectivity array must have the shape (N, 2), but instead its shape was {c.shape}.")
        if c.size and c.max() >= n_points:
            bad = int(np.nonzero((c >= n_points).any(axis=1))[0][0])
            raise ValueError(f"Line {bad} has points {tuple(c[bad])}, but there were only {n_points} points specified.")
        return cls._from_arrays(n_points, c, np.zeros(1, np.uint32), np.zeros(0, np.uint32))

    def dual_normal_criterion(self, crit: float, normals) -> npt.NDArray[np.uint32]:
        """Lines of this (dual) mesh whose end-point normals have dot < crit (meshobject.c:1064-1127)."""
        crit = float(crit)
        if crit > 1.0 or crit < -1.0:
            raise ValueError(f"Dot product criterion was {crit:g}, which is not inside the allowed range of -1.0 to +1.0.")
        _check_array(normals, (self.n_points, 3), "Normals array")
        n = np.asarray(normals.cpu().numpy() if _is_tensor(normals) else normals)
        ln = self._lines
        valid = (ln[:, 0] != INVALID_ID) & (ln[:, 1] != INVALID_ID)
        idx = np.nonzero(valid)[0]
        dp = np.einsum("ij,ij->i", n[ln[idx, 0]], n[ln[idx, 1]])
        return idx[dp < crit].astype(np.uint32)

    def dual_free_edges(self) -> npt.NDArray[np.uint32]:
        """Lines of this (dual) mesh with an INVALID end (meshobject.c:1129-1157)."""
        ln = self._lines
        return np.nonzero((ln[:, 0] == INVALID_ID) | (ln[:, 1] == INVALID_ID))[0].astype(np.uint32)

    def line_velocities_from_point_velocities(self, point_velocities, out) -> None:
        """Line velocity = mean of its end-point velocities (meshobject.c:739-778)."""
        _check_array(point_velocities, (self.n_points, 3), "Point velocities")
        _check_array(out, (self.n_lines, 3), "Output array")
        v = np.asarray(point_velocities)
        out[...] = 0.5 * (v[self._lines[:, 0]] + v[self._lines[:, 1]])

    def line_gradient(self, point_array, line_array=None):
        """Per-line difference of point values, end minus begin (meshobject.c:897-954)."""
        v = np.asarray(point_array, np.float64)
        if v.shape != (self.n_points,):
            raise ValueError("Point value array did not have the expected shape.")
        ln = self._lines.astype(np.int64)
        res = np.zeros(self.n_lines)
        ok1 = ln[:, 0] != INVALID_ID
        ok2 = ln[:, 1] != INVALID_ID
        res[ok1] -= v[ln[ok1, 0]]
        res[ok2] += v[ln[ok2, 1]]
        if line_array is not None:
            line_array[...] = res
            return line_array
        return res

    # ------------------------------------------------------------------ device data
    def device_arrays(self) -> dict:
        """Device copies of the topology (int32 tensors holding the uint32 bit patterns)."""
        dev = require_cuda()
        key = dev.index
        d = self._dev.get(key)
        if d is None:
            if self.n_lines and int(self._lines.max()) >= self.n_points:
                raise ValueError(f"The mesh references point {int(self._lines.max())}, but has only "
                                 f"{self.n_points} points.")
            offs, ents = self.ring_map()
            d = {
                "lines": to_device_u32(self._lines if self.n_lines else np.zeros((1, 2), np.uint32), dev),
                "offsets": to_device_u32(self._offsets, dev),
                "surface_lines": to_device_u32(self._surface_lines if self._surface_lines.size
                                               else np.zeros(1, np.uint32), dev),
                "map_offsets": to_device_u32(offs, dev),
                "map_entries": to_device_u32(ents if ents.size else np.zeros(1, np.uint32), dev),
            }
            t_off, t_lines, sl_local, max_nl = self.ring_tiles()
            d["tile_offsets"] = to_device_u32(t_off, dev)
            d["tile_lines"] = to_device_u32(t_lines if t_lines.size else np.zeros(1, np.uint32), dev)
            d["sl_local"] = to_device_u32(sl_local if sl_local.size else np.zeros(1, np.uint32), dev)
            d["tile_max"] = max_nl
            self._dev[key] = d
        return d

    RING_TILE = 128  # rings per tile of pvl_induction_normal_tiled

    def ring_tiles(self):
        """Per tile of RING_TILE consecutive rings: its distinct lines, and for every CSR entry
        its position in its tile's list (inputs of pvl_induction_normal_tiled)."""
        if getattr(self, "_ring_tiles", None) is None:
            off = self._offsets.astype(np.int64)
            ids = (self._surface_lines & np.uint32(0x7FFFFFFF)).astype(np.int64)
            n_t = -(-self.n_surfaces // self.RING_TILE)
            tile_off, tile_lines = [0], []
            local = np.zeros(ids.size, np.uint32)
            for t in range(n_t):
                a = off[t * self.RING_TILE]
                b = off[min((t + 1) * self.RING_TILE, self.n_surfaces)]
                uniq, inv = np.unique(ids[a:b], return_inverse=True)
                tile_lines.append(uniq)
                local[a:b] = inv
                tile_off.append(tile_off[-1] + uniq.size)
            tl = np.concatenate(tile_lines) if tile_lines else np.zeros(1, np.int64)
            max_nl = int(max((x.size for x in tile_lines), default=1))
            self._ring_tiles = (np.array(tile_off, np.uint32), tl.astype(np.uint32), local, max_nl)
        return self._ring_tiles

    def ring_map(self):
        """Line -> signed ring ids (transpose of the ring CSR)."""
        if self._ring_map is None:
            offs = np.zeros(self.n_lines + 1, np.uint32)
            ents = np.zeros(max(int(self._offsets[-1]), 1), np.uint32)
            _lib.call("pvl_line_ring_map", self.n_lines, self.n_surfaces, self._offsets.ctypes.data,
                      self._surface_lines.ctypes.data, offs.ctypes.data, ents.ctypes.data)
            self._ring_map = (offs, ents[: int(self._offsets[-1])])
        return self._ring_map

    # ------------------------------------------------------------------ geometry on GPU
    def _vec3_op(self, fn: str, values, out, name: str):
        _check_array(values, (self.n_points, 3), name)
        d = self.device_arrays()
        x = to_device(values)
        res = torch.empty((self.n_surfaces, 3), dtype=torch.float64, device=x.device)
        _lib.call(fn, self.n_surfaces, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]), ptr(x), ptr(res),
                  stream_ptr())
        if out is not None:
            _check_array(out, (self.n_surfaces, 3), "Output array")
        return _finish(res, values, out)

    def surface_normal(self, positions, out=None, /):
        """Unit ring normals (src/meshobject.c:956-1008 -> src/core/mesh.c:48-68)."""
        if not _is_tensor(positions):
            positions = np.ascontiguousarray(positions, np.float64)
        return self._vec3_op("pvl_surface_normal", positions, out, "Input array")

    def surface_average_vec3(self, vectors, out=None, /):
        """Per-ring mean of point vectors (src/meshobject.c:1010-1062 -> mesh.c:24-46)."""
        if not _is_tensor(vectors):
            vectors = np.ascontiguousarray(vectors, np.float64)
        return self._vec3_op("pvl_surface_average", vectors, out, "Input array")

    # ------------------------------------------------------------------ induction on GPU
    def _prep(self, tol, positions, control_points):
        tol = float(tol)
        _check_array(positions, (self.n_points, 3), "Position array")
        _check_array(control_points, (0, 3), "Control point array")
        return tol, to_device(positions), to_device(control_points)

    def induction_matrix3(self, tol, positions, control_points, normals, out=None, line_buffer=None, /):
        """(n_cp, n_surfaces) normal induction, fused pair + ring sum (src/meshobject.c:384-473).

        ``line_buffer`` is accepted for signature compatibility and ignored: no line buffer
        exists on this path."""
        tol, pos, cps = self._prep(tol, positions, control_points)
        _check_array(normals, tuple(control_points.shape), "Normal array")
        nrm = to_device(normals)
        n_cp = cps.shape[0]
        if out is not None:
            _check_array(out, (n_cp, self.n_surfaces), "Output array")
        d = self.device_arrays()
        res = torch.empty((n_cp, self.n_surfaces), dtype=torch.float64, device=pos.device)
        ws, nb = Workspace.get(_lib.query("pvl_segments_workspace", self.n_lines, _lib.PVL_F64))
        _lib.call("pvl_induction_normal", _lib.PVL_F64, self.n_points, self.n_lines, ptr(d["lines"]), ptr(pos),
                  self.n_surfaces, ptr(d["offsets"]), ptr(d["surface_lines"]), n_cp, ptr(cps), ptr(nrm), tol,
                  ptr(res), self.n_surfaces, ws, nb, stream_ptr())
        return _finish(res, positions, out)

    def induction_matrix(self, tol, positions, control_points, out=None, line_buffer=None, /):
        """(n_cp, n_surfaces, 3) ring induction, fused pair + ring sum (src/meshobject.c:475-556)."""
        tol, pos, cps = self._prep(tol, positions, control_points)
        n_cp = cps.shape[0]
        if out is not None:
            _check_array(out, (n_cp, self.n_surfaces, 3), "Output tensor")
        d = self.device_arrays()
        res = torch.empty((n_cp, self.n_surfaces, 3), dtype=torch.float64, device=pos.device)
        ws, nb = Workspace.get(_lib.query("pvl_segments_workspace", self.n_lines, _lib.PVL_F64))
        _lib.call("pvl_induction_matrix", self.n_points, self.n_lines, ptr(d["lines"]), ptr(pos), self.n_surfaces,
                  ptr(d["offsets"]), ptr(d["surface_lines"]), n_cp, ptr(cps), tol, ptr(res), ws, nb, stream_ptr())
        return _finish(res, positions, out)

    def line_induction_matrix(self, tol, positions, control_points, out=None, /):
        """(n_cp, n_lines, 3) per-segment induction (src/meshobject.c:1232-1286)."""
        tol, pos, cps = self._prep(tol, positions, control_points)
        n_cp = cps.shape[0]
        if out is not None:
            _check_array(out, (n_cp, self.n_lines, 3), "Output tensor")
        d = self.device_arrays()
        res = torch.empty((n_cp, self.n_lines, 3), dtype=torch.float64, device=pos.device)
        ws, nb = Workspace.get(_lib.query("pvl_segments_workspace", self.n_lines, _lib.PVL_F64))
        _lib.call("pvl_line_induction", self.n_points, self.n_lines, ptr(d["lines"]), ptr(pos), n_cp, ptr(cps), tol,
                  ptr(res), ws, nb, stream_ptr())
        return _finish(res, positions, out)

    def induced_velocity(self, tol, positions, points, circulation, precision: int = _lib.PVL_F64):
        """sum_j K_ij Gamma_j: velocity at points induced by the rings carrying `circulation`.

        Equals ``np.vecdot(self.induction_matrix(tol, positions, points), circulation[None, :, None],
        axis=1)`` (the reference's pattern, python/pyvl/solver.py:274-279) without
        materialising the matrix."""
        tol, pos, pts = self._prep(tol, positions, points)
        gam = to_device(circulation).reshape(-1)
        if gam.numel() != self.n_surfaces:
            raise ValueError("circulation must have one value per surface")
        d = self.device_arrays()
        lg = torch.empty(max(self.n_lines, 1), dtype=torch.float64, device=pos.device)
        _lib.call("pvl_line_circulation", self.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]), ptr(gam), 0,
                  ptr(lg), stream_ptr())
        res = torch.empty((pts.shape[0], 3), dtype=torch.float64, device=pos.device)
        ws, nb = Workspace.get(_lib.query("pvl_line_velocity_workspace", self.n_lines, pts.shape[0], precision))
        _lib.call("pvl_line_velocity", precision, self.n_points, self.n_lines, ptr(d["lines"]), ptr(pos), ptr(lg),
                  pts.shape[0], ptr(pts), None, tol, 1.0, 0.0, ptr(res), ws, nb, stream_ptr())
        return _finish(res, points, None)

    @staticmethod
    def line_forces(primal: Mesh, dual: Mesh, circulation, positions, freestream, out=None):
        """Kutta-Joukowski line forces (src/meshobject.c:1288-1396); circulation is Gamma / 2 pi."""
        if not isinstance(primal, Mesh) or not isinstance(dual, Mesh):
            raise TypeError("primal and dual must be Mesh objects")
        if (primal.n_points != dual.n_surfaces or primal.n_lines != dual.n_lines
                or primal.n_surfaces != dual.n_points):
            raise ValueError(
                "Given meshes can not be dual to each other, since the number of points,lines, and surfaces don't "
                f"match as primal ({primal.n_points}, {primal.n_lines}, {primal.n_surfaces}) and dual "
                f"({dual.n_points}, {dual.n_lines}, {dual.n_surfaces}).")
        _check_array(circulation, (primal.n_surfaces,), "Circulation array")
        _check_array(positions, (primal.n_points, 3), "Positions array")
        _check_array(freestream, (primal.n_points, 3), "Velocity array")
        if out is not None:
            _check_array(out, (primal.n_lines, 3), "Output array")
        dev = require_cuda()
        pl = primal.device_arrays()["lines"]
        dl = to_device_u32(dual._lines if dual.n_lines else np.zeros((1, 2), np.uint32), dev)
        res = torch.empty((primal.n_lines, 3), dtype=torch.float64, device=dev)
        # keep the device copies referenced until the kernel has been enqueued
        circ_d, pos_d, vel_d = to_device(circulation), to_device(positions), to_device(freestream)
        _lib.call("pvl_line_forces", primal.n_lines, ptr(pl), ptr(dl), ptr(circ_d), ptr(pos_d), ptr(vel_d), ptr(res),
                  stream_ptr())
        return _finish(res, positions, out)


# --------------------------------------------------------------------------- ReferenceFrame
def _clamp_angle(a: float) -> float:
    """src/core/common.h:212-218 (IEEE remainder, then shift into [0, 2 pi))."""
    rem = math.remainder(float(a), 2 * math.pi)
    return 2 * math.pi + rem if rem < 0 else rem


def _mat_from_angles(a) -> np.ndarray:
    """real3x3_from_angles, src/core/common.h:165-185."""
    cx, sx = math.cos(a[0]), math.sin(a[0])
    cy, sy = math.cos(a[1]), math.sin(a[1])
    cz, sz = math.cos(a[2]), math.sin(a[2])
    return np.array([
        [cy * cz, sx * sy * cz - cx * sz, cx * sy * cz + sx * sz],
        [cy * sz, sx * sy * sz + cx * cz, cx * sy * sz - sx * cz],
        [-sy, sx * cy, cx * cy],
    ], np.float64)


def _prepare(r, out):
    """Input/output checks of the transformations (src/referenceframeobject.c:296-365)."""
    x = np.ascontiguousarray(r, np.float64)
    if x.ndim < 1 or x.shape[-1] != 3:
        raise ValueError(f"Input array does not have the last axis with 3 dimensions (shape is {x.shape}).")
    if out is not None:
        if not isinstance(out, np.ndarray):
            raise TypeError("Second argument must be an array.")
        if not out.flags.c_contiguous:
            raise ValueError("Output array is not C-contiguous.")
        if out.dtype != np.float64:
            raise ValueError("Output array is not of C double type.")
        if out.shape != x.shape:
            raise ValueError("Output array does not have the same exact shape as the input array.")
    return x


def _emit(res, out):
    if out is not None:
        out[...] = res
        return out
    return res


class ReferenceFrame:
    """Rigid frame: rotation by angles about x, y, z then an offset, relative to a parent.

    Mirrors src/referenceframeobject.c (transforms :367-615, at_time :700-730).  Host-side
    kinematics: a handful of 3 x 3 products per step, computed with numpy.
    """

    # Initialised in __new__ like the reference's C type, so that subclasses written for the
    # reference (``self = super().__new__(cls, offset=..., theta=..., parent=...)``) work.
    def __new__(cls, offset=(0, 0, 0), theta=(0, 0, 0), parent: ReferenceFrame | None = None, *args, **kwargs):
        if parent is not None and not isinstance(parent, ReferenceFrame):
            raise TypeError(f'Argument "parent" must be a ReferenceFrame object, but it was {type(parent)}')
        self = object.__new__(cls)
        self._offset = np.asarray(offset, np.float64).reshape(3).copy()
        self._angles = np.array([_clamp_angle(t) for t in np.asarray(theta, np.float64).reshape(3)])
        self._parent = parent
        return self

    def __init__(self, *args, **kwargs) -> None:
        pass

    @classmethod
    def _make(cls, offset, angles, parent) -> ReferenceFrame:
        new = object.__new__(ReferenceFrame)
        new._offset = np.asarray(offset, np.float64).reshape(3).copy()
        new._angles = np.asarray(angles, np.float64).reshape(3).copy()
        new._parent = parent
        return new

    @property
    def parent(self) -> ReferenceFrame | None:
        return self._parent

    @property
    def parents(self) -> tuple[ReferenceFrame, ...]:
        out = []
        p = self._parent
        while p is not None:
            out.append(p)
            p = p._parent
        return tuple(out)

    @property
    def offset(self) -> np.ndarray:
        return self._offset.copy()

    @property
    def angles(self) -> np.ndarray:
        return self._angles.copy()

    @property
    def rotation_matrix(self) -> np.ndarray:
        return _mat_from_angles(self._angles)

    @property
    def rotation_matrix_inverse(self) -> np.ndarray:
        return _mat_from_angles(self._angles).T.copy()

    def __repr__(self) -> str:
        a, o = self._angles, self._offset
        body = f"({a[0]:g}, {a[1]:g}, {a[2]:g}), ({o[0]:g}, {o[1]:g}, {o[2]:g})"
        if self._parent is not None:
            return f"ReferenceFrame({body}, parent={self._parent!r})"
        return f"ReferenceFrame({body})"

    def __eq__(self, other) -> bool:
        # src/referenceframeobject.c:247-290, including its comparison of squared
        # differences against 1e-10 as written there.
        if type(other) is not ReferenceFrame or type(self) is not ReferenceFrame:
            return False
        a, b = self, other
        result = True
        while a is not None and b is not None:
            d1 = a._offset - b._offset
            if float(d1 @ d1) < 1e-10:
                result = False
                break
            d2 = a._angles - b._angles
            if float(d2 @ d2) < 1e-10:
                result = False
                break
            a, b = a._parent, b._parent
        if a is not None or b is not None:
            result = False
        return result

    __hash__ = object.__hash__

    # ------------------------------------------------------------------ transforms
    def from_parent_with_offset(self, r, out=None, /):
        x = _prepare(r, out)
        return _emit(x @ self.rotation_matrix.T + self._offset, out)

    def from_parent_without_offset(self, r, out=None, /):
        x = _prepare(r, out)
        return _emit(x @ self.rotation_matrix.T, out)

    def to_parent_with_offset(self, r, out=None, /):
        x = _prepare(r, out)
        return _emit((x - self._offset) @ self.rotation_matrix, out)

    def to_parent_without_offset(self, r, out=None, /):
        x = _prepare(r, out)
        return _emit(x @ self.rotation_matrix, out)

    def _chain(self):
        # The reference merges the transformation of every frame that has a parent,
        # starting from this one (src/referenceframeobject.c:497-500, 547-550).
        p = self
        while p._parent is not None:
            yield p
            p = p._parent

    def from_global_with_offset(self, r, out=None, /):
        x = _prepare(r, out)
        mat, off = self.rotation_matrix, self._offset.copy()
        for p in self._chain():
            rp = p.rotation_matrix
            mat, off = rp @ mat, p._offset + rp @ off
        return _emit(x @ mat.T + off, out)

    def from_global_without_offset(self, r, out=None, /):
        x = _prepare(r, out)
        mat = self.rotation_matrix
        for p in self._chain():
            mat = p.rotation_matrix @ mat
        return _emit(x @ mat.T, out)

    def to_global_with_offset(self, r, out=None, /):
        x = _prepare(r, out)
        mat, off = self.rotation_matrix.T, self._offset.copy()
        for p in self._chain():
            ta = p.rotation_matrix.T
            mat, off = mat @ ta, ta @ (p._offset + mat @ off)
        return _emit(x @ mat.T - off, out)

    def to_global_without_offset(self, r, out=None, /):
        x = _prepare(r, out)
        mat = self.rotation_matrix.T
        for p in self._chain():
            mat = mat @ p.rotation_matrix.T
        return _emit(x @ mat.T, out)

    # ------------------------------------------------------------------ derived frames
    def _copy_with(self, offset=None, angles=None) -> ReferenceFrame:
        return ReferenceFrame._make(self._offset if offset is None else offset,
                                    self._angles if angles is None else angles, self._parent)

    def rotate_x(self, theta: float) -> ReferenceFrame:
        a = self._angles.copy()
        a[0] = _clamp_angle(a[0] + float(theta))
        return self._copy_with(angles=a)

    def rotate_y(self, theta: float) -> ReferenceFrame:
        a = self._angles.copy()
        a[1] = _clamp_angle(a[1] + float(theta))
        return self._copy_with(angles=a)

    def rotate_z(self, theta: float) -> ReferenceFrame:
        a = self._angles.copy()
        a[2] = _clamp_angle(a[2] + float(theta))
        return self._copy_with(angles=a)

    def with_offset(self, new_offset) -> ReferenceFrame:
        o = np.asarray(new_offset, np.float64)
        if o.shape != (3,):
            raise ValueError("Offset must be a 3-element vector.")
        return self._copy_with(offset=o)

    def at_time(self, t: float):
        """Same frame, parent evolved to time t (src/referenceframeobject.c:700-730)."""
        return ReferenceFrame._make(self._offset, self._angles,
                                    self._parent.at_time(t) if self._parent is not None else None)

    def add_velocity(self, positions, velocity, /) -> None:
        """A fixed frame adds nothing; only the arguments are checked (:939-956)."""
        p = np.asarray(positions)
        if p.ndim != 2 or p.shape[1] != 3:
            raise ValueError("Position array did not have the expected shape.")
        v = velocity
        if not isinstance(v, np.ndarray) or v.shape != p.shape:
            raise ValueError("Velocity array did not have the expected shape.")

    @staticmethod
    def angles_from_rotation(rotation_matrix) -> np.ndarray:
        """angles_from_real3x3, src/core/common.h:207-210."""
        m = np.asarray(rotation_matrix, np.float64)
        if m.shape != (3, 3):
            raise ValueError("Rotation matrix must be a (3, 3) array.")
        return np.array([math.atan2(m[2, 1], m[2, 2]), math.atan2(-m[2, 0], math.hypot(m[0, 0], m[1, 0])),
                         math.atan2(m[1, 0], m[0, 0])])

    def save(self, hmap, /) -> None:
        hmap["offset"] = self.offset
        hmap["angles"] = self.angles
        hmap["type"] = "pyvl.cvl.ReferenceFrame"

    @classmethod
    def load(cls, group, parent: ReferenceFrame | None = None):
        new = object.__new__(cls)
        new._offset = np.asarray(group["offset"], np.float64).reshape(3).copy()
        new._angles = np.asarray(group["angles"], np.float64).reshape(3).copy()
        new._parent = parent
        return new
