"""Nested key -> value mapping used to save and load solver objects.

Mirrors python/pyvl/fio/io_common.py:13-157 (same typed insert/get methods, same
"module.Name" encoding of types).
"""

from __future__ import annotations

import importlib
from collections.abc import MutableMapping
from typing import Any, Callable

import numpy as np
import numpy.typing as npt


_PKG = __name__.split(".")[0]  # this package's top-level name


class HirearchicalMap(MutableMapping):
    """Mapping that holds values and nested HirearchicalMaps under unique keys."""

    def __init__(self) -> None:
        self._map: dict[str, Any] = {}

    def __getitem__(self, key: str) -> Any:
        return self._map[key]

    def __setitem__(self, key: str, value: Any) -> None:
        self._map[key] = value

    def __delitem__(self, key: str) -> None:
        del self._map[key]

    def __iter__(self):
        return iter(self._map)

    def __len__(self) -> int:
        return len(self._map)

    def __contains__(self, key: object) -> bool:
        return key in self._map

    def _insert(self, key: str, value: Any) -> None:
        if key in self._map:
            raise KeyError(f'The key "{key}" is already in the mapping.')
        self._map[key] = value

    def insert_type(self, key: str, t: type) -> None:
        """Stored as "module.Name"; this package's classes are written under the reference's
        module names (pyvl.*), so that the files are the reference's format."""
        if not isinstance(t, type):
            raise TypeError(f"The value was not a type but {type(t).__name__}")
        mod = t.__module__
        if mod == _PKG or mod.startswith(_PKG + "."):
            mod = "pyvl" + mod[len(_PKG):]
        self._insert(key, mod + "." + t.__name__)

    def insert_array(self, key: str, value: npt.ArrayLike) -> None:
        self._insert(key, np.array(value))

    def insert_string(self, key: str, value: str) -> None:
        if not isinstance(value, str):
            raise TypeError(f"The value was not a string but {type(value).__name__}")
        self._insert(key, np.array(value))

    def insert_scalar(self, key: str, value: int | float) -> None:
        if not isinstance(value, (int, float)):
            raise TypeError(f"The value was not an int or float but {type(value).__name__}")
        self._insert(key, value)

    def insert_int(self, key: str, value: int) -> None:
        if not isinstance(value, int):
            raise TypeError(f"The value was not an int but {type(value).__name__}")
        self._insert(key, value)

    def insert_hirearchycal_map(self, key: str, value: HirearchicalMap) -> None:
        if not isinstance(value, HirearchicalMap):
            raise TypeError(f"The value was not a HirearchicalMap but {type(value).__name__}")
        if value is self:
            raise ValueError("A map can not contain itself.")
        self._insert(key, value)

    def get_type(self, key: str) -> type:
        """The class named "module.Name"; the reference's pyvl.* names resolve to this
        package's classes of the same module path and name."""
        name = str(self._map[key])
        mod, _, attr = name.rpartition(".")
        if mod == "pyvl" or mod.startswith("pyvl."):
            mod = _PKG + mod[len("pyvl"):]
        return getattr(importlib.import_module(mod), attr)

    def get_array(self, key: str) -> npt.NDArray:
        return np.asarray(self._map[key])

    def get_string(self, key: str) -> str:
        return str(self._map[key])

    def get_scalar(self, key: str) -> float:
        return float(self._map[key])

    def get_int(self, key: str) -> int:
        return int(self._map[key])

    def get_hirearchical_map(self, key: str) -> HirearchicalMap:
        v = self._map[key]
        if not isinstance(v, HirearchicalMap):
            raise TypeError(f'Key "{key}" does not hold a HirearchicalMap.')
        return v


SerializationFunction = Callable[[HirearchicalMap, Any], None]
