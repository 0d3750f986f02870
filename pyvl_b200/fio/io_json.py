"""JSON form of a HirearchicalMap, in the reference's own file format
(python/pyvl/fio/io_json.py:15-49): nested maps are JSON objects, arrays nested lists, scalars
and strings as they are; reading turns every list back into a numpy array.  Files written by
either package load in the other."""

from __future__ import annotations

import json
from collections.abc import Sequence
from pathlib import Path
from typing import Any

import numpy as np

from .io_common import HirearchicalMap


def _plain(value: Any) -> Any:
    """JSON-ready form of one value (maps -> dicts, arrays -> lists, numpy scalars -> Python)."""
    if isinstance(value, HirearchicalMap):
        return {k: _plain(value[k]) for k in value}
    if isinstance(value, np.ndarray):
        return value.tolist()
    if isinstance(value, np.generic):
        return value.item()
    return value


def _to_map(obj: dict) -> HirearchicalMap:
    hm = HirearchicalMap()
    for key, value in obj.items():
        if isinstance(value, Sequence) and not isinstance(value, str):
            hm[key] = np.array(value)
        else:
            hm[key] = value
    return hm


def serialize_json(hmap: HirearchicalMap, path: Path | str) -> None:
    """Save a HirearchicalMap into a JSON file."""
    Path(path).write_text(json.dumps(_plain(hmap)))


def deserialize_json(path: Path | str) -> HirearchicalMap:
    """Load a HirearchicalMap from a JSON file."""
    return json.loads(Path(path).read_text(), object_hook=_to_map)
