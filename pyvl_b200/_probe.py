"""ctypes binding of libpvl_probe.so: measurement and test probes (pyvl_b200/probe/pvl_probe.h).

Benchmarks and tests load it beside the product library; nothing in the product path does.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

from . import _lib

LIB_PATH = Path(__file__).resolve().parent / "libpvl_probe.so"

_P, _U, _I, _D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_double
SIGNATURES = {
    "pvl_probe_last_error": (ctypes.c_char_p, []),
    "pvl_probe_fma": (_D, [_I, _U, _U, _P, _P]),
    "pvl_probe_far_series": (_I, [_U, _P, _P, _P, _P, _P]),
    "pvl_probe_trsv_timeout": (_I, [_U, _P, _U, _P, _P, _P, _P, ctypes.c_longlong, ctypes.c_int32, _I, _P]),
    "pvl_probe_gemm_timeout": (_I, [_U, _U, _U, _P, _U, _P, _U, _P, _U, _P, ctypes.c_longlong, _P]),
}

_lib_handle = None


def lib() -> ctypes.CDLL:
    global _lib_handle
    if _lib_handle is None:
        _lib.lib()  # the probe library links the product library (found beside it)
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build with `python -m pyvl_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib_handle = L
    return _lib_handle


def call(name: str, *args) -> int:
    rc = getattr(lib(), name)(*args)
    if rc != _lib.PVL_OK:
        msg = lib().pvl_probe_last_error().decode(errors="replace")
        if rc == _lib.PVL_ERR_ARG:
            raise ValueError(msg)
        raise _lib.PvlError(rc, f"{name} failed ({rc}): {msg}")
    return rc
