"""JSON form of a HirearchicalMap (python/pyvl/fio/io_json.py:15-49): arrays keep dtype and shape."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from .io_common import HirearchicalMap


def _encode(hmap: HirearchicalMap) -> dict:
    out = {}
    for k in hmap:
        v = hmap[k]
        if isinstance(v, HirearchicalMap):
            out[k] = {"__map__": _encode(v)}
        elif isinstance(v, np.ndarray):
            out[k] = {"__array__": v.tolist(), "dtype": str(v.dtype), "shape": list(v.shape)}
        else:
            out[k] = v
    return out


def _decode(d: dict) -> HirearchicalMap:
    hm = HirearchicalMap()
    for k, v in d.items():
        if isinstance(v, dict) and "__map__" in v:
            hm[k] = _decode(v["__map__"])
        elif isinstance(v, dict) and "__array__" in v:
            hm[k] = np.array(v["__array__"], dtype=v["dtype"]).reshape(v["shape"])
        else:
            hm[k] = v
    return hm


def serialize_json(hmap: HirearchicalMap, path: Path | str) -> None:
    Path(path).write_text(json.dumps(_encode(hmap)))


def deserialize_json(path: Path | str) -> HirearchicalMap:
    return _decode(json.loads(Path(path).read_text()))
