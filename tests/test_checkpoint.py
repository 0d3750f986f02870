"""Checkpoint files in the reference's own format (python/pyvl/fio/io_json.py, solver.py:70-108,
wake_models.py:233-291): a solver-state snapshot written by the reference's run_solver loads
into this package, and this package writes it back in the same format.  No GPU."""

import json
from pathlib import Path

import numpy as np

GOLD = Path(__file__).resolve().parent / "golden"


def test_reference_snapshot_loads():
    from pyvl_b200.fio import deserialize_json
    from pyvl_b200.solver import SolverState
    from pyvl_b200.wake_models import WakeModelLineExplicitUnsteady

    gold = np.load(GOLD / "checkpoint_flat.npz")
    hmap = deserialize_json(GOLD / "checkpoint_flat.json")
    state = SolverState.load(hmap)
    assert np.array_equal(state.circulation, gold["circulation"])
    assert isinstance(state.wake_model, WakeModelLineExplicitUnsteady)
    assert np.array_equal(state.wake_model.wake_positions, gold["wake_positions"])
    assert np.array_equal(state.wake_model.circulation, gold["wake_circulation"])
    assert state.iteration == 2


def test_snapshot_round_trip_in_reference_format(tmp_path):
    from pyvl_b200.fio import deserialize_json, serialize_json
    from pyvl_b200.solver import SolverState

    state = SolverState.load(deserialize_json(GOLD / "checkpoint_flat.json"))
    out = tmp_path / "again.json"
    serialize_json(state.save(), out)
    ours = json.loads(out.read_text())
    ref = json.loads((GOLD / "checkpoint_flat.json").read_text())

    def same(a, b, path=""):
        assert type(a) is type(b) or (isinstance(a, (int, float)) and isinstance(b, (int, float))), path
        if isinstance(a, dict):
            assert set(a) == set(b), (path, set(a) ^ set(b))
            for k in a:
                same(a[k], b[k], f"{path}/{k}")
        elif isinstance(a, list):
            assert np.array_equal(np.array(a), np.array(b)), path
        else:
            assert a == b, (path, a, b)

    same(ours, ref)
