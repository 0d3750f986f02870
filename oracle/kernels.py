"""ctypes bindings to oracle.c (the plain-C restatement of the reference kernels).

Test infrastructure only.  ``build()`` compiles ``oracle/liboracle.so`` with gcc; the
file is git-ignored and travels with the tree to the GPU host prebuilt.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np
import numpy.typing as npt

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
INVALID_ID = 0x7FFFFFFF

_lib = None


def build(force: bool = False) -> Path:
    """Compile oracle.c into liboracle.so (gcc -O2 -fopenmp)."""
    src = HERE / "oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-fno-fast-math",
               "-ffp-contract=off", str(src), "-o", str(LIB_PATH), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        U = ctypes.c_uint
        L.orc_line_induction.argtypes = [U, P, P, U, P, P, ctypes.c_double]
        L.orc_ring_reduce.argtypes = [U, P, P, U, U, P, P, P]
        L.orc_surface_center.argtypes = [U, P, P, P, P, P]
        L.orc_surface_normal.argtypes = [U, P, P, P, P, P]
        L.orc_mesh_from_elements.argtypes = [U, P, P, P, P, P]
        L.orc_mesh_from_elements.restype = U
        L.orc_dual_lines.argtypes = [U, U, P, P, P]
        L.orc_line_forces.argtypes = [U, P, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleMesh:
    """Topology of a ring mesh, built exactly as mesh_from_elements builds it.

    ``lines`` (L, 2) uint32, ``offsets`` (P+1,) uint32, ``surface_lines`` (sum,) uint32
    with bit 31 = reversed (src/core/mesh.h:130-139, src/core/common.h:46-56).
    """

    def __init__(self, n_points: int, elements):
        elems = [np.asarray(e, np.uint32).reshape(-1) for e in elements]
        counts = np.array([e.size for e in elems], np.uint32)
        flat = np.ascontiguousarray(np.concatenate(elems) if elems else np.zeros(0, np.uint32))
        total = int(flat.size)
        lines = np.zeros((max(total, 1), 2), np.uint32)
        sl = np.zeros(max(total, 1), np.uint32)
        off = np.zeros(len(elems) + 1, np.uint32)
        n_lines = lib().orc_mesh_from_elements(len(elems), _p(counts), _p(flat), _p(lines), _p(sl), _p(off))
        self.n_points = int(n_points)
        self.lines = lines[:n_lines].copy()
        self.surface_lines = sl[:total].copy()
        self.offsets = off
        self._dual = None

    @property
    def n_lines(self) -> int:
        return int(self.lines.shape[0])

    @property
    def n_surfaces(self) -> int:
        return int(self.offsets.size - 1)

    def dual_lines(self) -> npt.NDArray[np.uint32]:
        if self._dual is None:
            out = np.zeros((self.n_lines, 2), np.uint32)
            lib().orc_dual_lines(self.n_lines, self.n_surfaces, _p(self.offsets),
                                 _p(self.surface_lines), _p(out))
            self._dual = out
        return self._dual

    def line_induction_matrix(self, tol: float, positions, cpts, chunk_bytes: int = 1 << 28):
        pos, cp = _f64(positions), _f64(cpts)
        out = np.empty((cp.shape[0], self.n_lines, 3), np.float64)
        step = max(1, chunk_bytes // max(1, self.n_lines * 24))
        for i0 in range(0, cp.shape[0], step):
            c = np.ascontiguousarray(cp[i0:i0 + step])
            o = np.empty((c.shape[0], self.n_lines, 3), np.float64)
            lib().orc_line_induction(self.n_lines, _p(self.lines), _p(pos), c.shape[0], _p(c), _p(o), tol)
            out[i0:i0 + step] = o
        return out

    def _reduce(self, tol, positions, cpts, normals, chunk_bytes=1 << 28):
        pos, cp = _f64(positions), _f64(cpts)
        nrm = _f64(normals) if normals is not None else None
        n_cp = cp.shape[0]
        shape = (n_cp, self.n_surfaces) if nrm is not None else (n_cp, self.n_surfaces, 3)
        out = np.empty(shape, np.float64)
        step = max(1, chunk_bytes // max(1, self.n_lines * 24))
        for i0 in range(0, n_cp, step):
            c = np.ascontiguousarray(cp[i0:i0 + step])
            n = np.ascontiguousarray(nrm[i0:i0 + step]) if nrm is not None else None
            buf = np.empty((c.shape[0], self.n_lines, 3), np.float64)
            lib().orc_line_induction(self.n_lines, _p(self.lines), _p(pos), c.shape[0], _p(c), _p(buf), tol)
            o = np.empty((c.shape[0],) + shape[1:], np.float64)
            lib().orc_ring_reduce(self.n_surfaces, _p(self.offsets), _p(self.surface_lines), self.n_lines,
                                  c.shape[0], _p(n), _p(buf), _p(o))
            out[i0:i0 + step] = o
        return out

    def induction_matrix(self, tol: float, positions, cpts):
        """(n_cp, P, 3): restates Mesh.induction_matrix, src/meshobject.c:475-556."""
        return self._reduce(tol, positions, cpts, None)

    def induction_matrix3(self, tol: float, positions, cpts, normals):
        """(n_cp, P): restates Mesh.induction_matrix3, src/meshobject.c:384-473."""
        return self._reduce(tol, positions, cpts, normals)

    def surface_normal(self, positions):
        out = np.empty((self.n_surfaces, 3), np.float64)
        lib().orc_surface_normal(self.n_surfaces, _p(self.offsets), _p(self.surface_lines),
                                 _p(self.lines), _p(_f64(positions)), _p(out))
        return out

    def surface_average_vec3(self, vectors):
        out = np.empty((self.n_surfaces, 3), np.float64)
        lib().orc_surface_center(self.n_surfaces, _p(self.offsets), _p(self.surface_lines),
                                 _p(self.lines), _p(_f64(vectors)), _p(out))
        return out


def line_forces(primal: OracleMesh, dual_lines, circulation, positions, velocity):
    """Restates Mesh.line_forces, src/meshobject.c:1288-1396 (circulation already / 2 pi)."""
    out = np.empty((primal.n_lines, 3), np.float64)
    dl = np.ascontiguousarray(dual_lines, np.uint32)
    lib().orc_line_forces(primal.n_lines, _p(primal.lines), _p(dl), _p(_f64(circulation)),
                          _p(_f64(positions)), _p(_f64(velocity)), _p(out))
    return out


def use_threads(n: int | None = None) -> None:
    """Set the OpenMP thread count used by later oracle calls (default: all cores)."""
    os.environ["OMP_NUM_THREADS"] = str(n or os.cpu_count() or 1)
