"""Serialisation of solver state (python/pyvl/fio): HirearchicalMap and its JSON form."""

from .io_common import HirearchicalMap as HirearchicalMap
from .io_json import deserialize_json as deserialize_json
from .io_json import serialize_json as serialize_json
