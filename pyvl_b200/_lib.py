"""ctypes binding of libpvl_b200.so (the C ABI declared in include/pvl_b200.h).

The library is built in-tree by ``python -m pyvl_b200.build``.  There is no fallback:
if the library is missing, every call raises.  Status codes are mapped onto the
exception types the reference raises for the same conditions (ValueError for bad
arguments, RuntimeError for topology and runtime failures).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpvl_b200.so"

PVL_OK = 0
PVL_ERR_ARG = -1
PVL_ERR_CUDA = -2
PVL_ERR_ALLOC = -3
PVL_ERR_SINGULAR = -4
PVL_ERR_NOT_CONVERGED = -5
PVL_ERR_TOPOLOGY = -6
PVL_ERR_TIMEOUT = -7
PVL_ERR_NONFINITE = -8
PVL_F64 = 0
PVL_F32 = 1
INVALID_ID = 0x7FFFFFFF

_P = ctypes.c_void_p
_U = ctypes.c_uint32
_D = ctypes.c_double
_I = ctypes.c_int
_Z = ctypes.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "pvl_last_error": (ctypes.c_char_p, []),
    "pvl_version": (_I, []),
    "pvl_mesh_from_elements": (_I, [_U, _U, _P, _P, _P, _P, _P, _P]),
    "pvl_mesh_dual": (_I, [_U, _U, _P, _U, _P, _P, _P, _P, _P]),
    "pvl_mesh_to_elements": (_I, [_U, _P, _P, _P, _P, _P]),
    "pvl_line_ring_map": (_I, [_U, _U, _P, _P, _P, _P]),
    "pvl_surface_normal": (_I, [_U, _P, _P, _P, _P, _P, _P]),
    "pvl_surface_average": (_I, [_U, _P, _P, _P, _P, _P, _P]),
    "pvl_rhs": (_I, [_U, _P, _P, _D, _D, _D, _P, _P, _P, _P]),
    "pvl_segments_workspace": (_Z, [_U, _I]),
    "pvl_line_induction": (_I, [_U, _U, _P, _P, _U, _P, _D, _P, _P, _Z, _P]),
    "pvl_induction_matrix": (_I, [_U, _U, _P, _P, _U, _P, _P, _U, _P, _D, _P, _P, _Z, _P]),
    "pvl_induction_normal_tiled": (_I, [_U, _U, _P, _P, _U, _P, _P, _P, _P, _P, _U, _U, _P, _P, _D, _P, _U, _P, _Z,
                                        _P]),
    "pvl_induction_normal": (_I, [_I, _U, _U, _P, _P, _U, _P, _P, _U, _P, _P, _D, _P, _U, _P, _Z, _P]),
    "pvl_line_velocity_workspace": (_Z, [_U, _U, _I]),
    "pvl_line_velocity": (_I, [_I, _U, _U, _P, _P, _P, _U, _P, _P, _D, _D, _D, _P, _P, _Z, _P]),
    "pvl_line_circulation": (_I, [_U, _P, _P, _P, _U, _P, _P]),
    "pvl_line_velocity_noalloc": (_I, [_I, _U, _U, _P, _P, _P, _U, _P, _P, _D, _D, _D, _P, _P]),
    "pvl_wake_node_velocity_workspace": (_Z, [_U, _U, _U, _I]),
    "pvl_wake_node_velocity": (_I, [_I, _U, _U, _P, _P, _P, _U, _U, _U, _P, _D, _D, _D, _D, _P, _P, _Z, _P]),
    "pvl_wake_node_velocity_cols": (_I, [_I, _U, _U, _P, _P, _P, _U, _U, _U, _U, _U, _U, _P, _P, _D, _D, _D, _D, _P,
                                         _P, _Z, _P]),
    "pvl_wake_node_velocity_rows": (_I, [_I, _U, _U, _P, _P, _P, _U, _U, _U, _U, _U, _U, _U, _P, _P, _D, _D, _D, _D,
                                         _P, _P, _Z, _P]),
    "pvl_wake_node_velocity_list": (_I, [_I, _U, _U, _P, _P, _P, _U, _U, _U, _U, _P, _U, _P, _P, _D, _D, _D, _D,
                                         _P, _P, _Z, _P]),
    "pvl_wake_interp_rows": (_I, [_U, _U, _U, _U, _P, _P]),
    "pvl_wake_interp_rows_spaced": (_I, [_U, _U, _U, _U, _U, _P, _P]),
    "pvl_wake_interp_cols": (_I, [_U, _U, _U, _U, _P, _U, _P, _P, _U, _P, _P, _P]),
    "pvl_gather_points": (_I, [_U, _P, _U, _P, _P, _P]),
    "pvl_stencil_normal_add": (_I, [_U, _P, _U, _P, _P, _U, _P, _P, _P, _P]),
    "pvl_wake_fold_implicit": (_I, [_U, _U, _P, _P, _P, _U, _P]),
    "pvl_wake_fold_implicit_distinct": (_I, [_U, _U, _P, _P, _P, _U, _P]),
    "pvl_wake_advect": (_I, [_U, _U, _U, _P, _P, _D, _P, _P, _P, _P]),
    "pvl_wake_advect_cols": (_I, [_U, _U, _U, _P, _P, _P, _U, _D, _P, _P, _P, _P]),
    "pvl_wake_shed": (_I, [_U, _U, _P, _P, _P, _P, _P]),
    "pvl_lu_workspace": (_Z, [_U]),
    "pvl_lu_solve_workspace": (_Z, [_U]),
    "pvl_lu_factor": (_I, [_U, _P, _U, _P, _P, _P, _Z, _P]),
    "pvl_lu_solve": (_I, [_U, _P, _U, _P, _P, _P, _P, _Z, _P]),
    "pvl_group_mean_remove": (_I, [_U, _P, _P, _P]),
    "pvl_border_groups": (_I, [_U, _U, _P, _P, _U, _P, _P]),
    "pvl_line_forces": (_I, [_U, _P, _P, _P, _P, _P, _P, _P]),
    "pvl_gemm_tf32": (_I, [_U, _U, _U, ctypes.c_float, _P, _U, _P, _U, ctypes.c_float, _P, _U, _P, _P]),
    "pvl_gemv_f64": (_I, [_U, _U, _D, _P, _U, _P, _D, _P, _P]),
    "pvl_gemv_f32mat": (_I, [_U, _U, _D, _P, _U, _P, _D, _P, _P]),
    "pvl_gemv_f32": (_I, [_U, _U, _D, _P, _U, _P, _D, _P, _P]),
    "pvl_lu_solve_blocked": (_I, [_U, _P, _U, _P, _P, _P, _Z, _P]),
    "pvl_gmres_ctl_bytes": (_Z, []),
    "pvl_gmres_max_iter": (_U, []),
    "pvl_gmres_graph_create": (_I, [_U, _P, _U, _P, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U, _D, _P, _P, _P, _Z,
                                    _P, _U, _U, _P, _P, _P]),
    "pvl_gmres_graph_launch": (_I, [ctypes.c_uint64, _P]),
    "pvl_gmres_graph_account": (_I, [ctypes.c_uint64, _U, _U]),
    "pvl_gmres_graph_destroy": (_I, [ctypes.c_uint64]),
    "pvl_axpy_f64": (_I, [_U, _D, _P, _P, _P]),
    "pvl_basis_project": (_I, [_U, _U, _P, _U, _P, _P, _P]),
    "pvl_normalize": (_I, [_U, _P, _P, _P, _P]),
    "pvl_combine": (_I, [_U, _U, _P, _U, _P, _P, _P]),
    "pvl_pad_convert_f32": (_I, [_U, _P, _U, _P, _U, _U, _P]),
    "pvl_lu32_workspace": (_Z, [_U]),
    "pvl_lu32_factor": (_I, [_U, _P, _U, _P, _P, _P, _P, _Z, _P]),
    "pvl_lu32_inverse": (_I, [_U, _P, _U, _P, _P, _U, _P, _U, _P, _P, _Z, _P]),
    "pvl_batch_ring_job_bytes": (_Z, []),
    "pvl_batch_sweep_job_bytes": (_Z, []),
    "pvl_batch_wake_case_bytes": (_Z, []),
    "pvl_batch_solve_case_bytes": (_Z, []),
    "pvl_batch_gmres_state_bytes": (_Z, []),
    "pvl_batch_gmres_max_iter": (_U, []),
    "pvl_prep_segments": (_I, [_I, _U, _U, _P, _P, _P, _D, _P, _P]),
    "pvl_batch_ring_matrix": (_I, [_I, _P, _P, _U, _U, _P, _P, _P, _U, _P, _P, _P, _D, _P, _U, _P]),
    "pvl_batch_ring_matrix_tiled": (_I, [_I, _P, _P, _U, _U, _P, _P, _P, _P, _P, _P, _P, _U, _U, _P, _P, _P, _D,
                                         _P, _P, _U, _P]),
    "pvl_batch_sweep": (_I, [_I, _I, _P, _P, _U, _U, _P, _P, _P, _U, _P, _P, _P, _D, _P, _U, _P]),
    "pvl_batch_sweep_reduce": (_I, [_P, _P, _U, _U, _P, _P, _P, _P, _P, _P]),
    "pvl_batch_fold_implicit": (_I, [_P, _P, _U, _P, _P, _P, _P]),
    "pvl_batch_wake_advect": (_I, [_P, _P, _U, _U, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pvl_batch_wake_shed": (_I, [_P, _P, _U, _U, _P, _P, _P, _P, _P]),
    "pvl_batch_increment": (_I, [_P, _P]),
    "pvl_batch_gmres_workspace": (_Z, [_U, _U, _U]),
    "pvl_batch_gmres": (_I, [_P, _P, _U, _U, _P, _P, _P, _U, _D, _P, _P, _P, _Z, _P]),
    "pvl_mlp_param_count": (_U, []),
    "pvl_mlp_input_count": (_U, []),
    "pvl_mlp_features": (_I, [_U, _P, _P, _P, _P, _P, _P, _P, _U, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pvl_mlp_forward": (_I, [_U, _P, _P, _D, _P, _P, _P, _P]),
    "pvl_mlp_train_workspace": (_Z, [_U]),
    "pvl_mlp_gradient": (_I, [_U, _P, _P, _P, _U, _P, _P, _P, _Z, _P]),
    "pvl_mlp_adam": (_I, [_P, _P, _P, _P, _P, _U, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                          _P]),
    "pvl_mlp_to_bf16": (_I, [_P, _P, _P]),
    "pvl_launch_count": (ctypes.c_ulonglong, []),
}

_lib = None


class PvlError(RuntimeError):
    """A C-ABI call failed; ``code`` is the PVL_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def lib() -> ctypes.CDLL:
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA extension with `python -m pyvl_b200.build` "
                "(pyvl_b200 has no CPU fallback)"
            )
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def call(name: str, *args) -> int:
    """Call an entry point and raise on a non-zero status."""
    rc = getattr(lib(), name)(*args)
    if rc != PVL_OK:
        msg = lib().pvl_last_error().decode(errors="replace")
        if rc == PVL_ERR_ARG:
            raise ValueError(msg)
        raise PvlError(rc, f"{name} failed ({rc}): {msg}")
    return rc


def query(name: str, *args) -> int:
    """Call a size query (returns its value)."""
    return int(getattr(lib(), name)(*args))
