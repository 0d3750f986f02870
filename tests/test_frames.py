"""ReferenceFrame and its subclasses vs the reference's own frames (golden vectors)."""

from pathlib import Path

import numpy as np
import pytest

from pyvl_b200 import ReferenceFrame, RotorReferenceFrame, TranslatingReferenceFrame

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "frames.npz")
FNS = ("from_parent_with_offset", "from_parent_without_offset", "to_parent_with_offset", "to_parent_without_offset",
       "from_global_with_offset", "from_global_without_offset", "to_global_with_offset", "to_global_without_offset")


def frames():
    f0 = ReferenceFrame(GOLD["f0/offset"], GOLD["f0/angles"])
    f1 = ReferenceFrame(GOLD["f1/offset"], GOLD["f1/angles"], f0)
    f2 = ReferenceFrame(GOLD["f2/offset"], GOLD["f2/angles"], f1)
    return {"f0": f0, "f1": f1, "f2": f2}


@pytest.mark.parametrize("name", ["f0", "f1", "f2"])
def test_transforms_match_reference(name):
    f = frames()[name]
    x = GOLD["x"]
    assert np.allclose(f.rotation_matrix, GOLD[f"{name}/rot"], rtol=0, atol=1e-15)
    assert np.allclose(f.rotation_matrix_inverse, GOLD[f"{name}/rot_inv"], rtol=0, atol=1e-15)
    for fn in FNS:
        assert np.allclose(getattr(f, fn)(x), GOLD[f"{name}/{fn}"], rtol=1e-14, atol=1e-14), fn
    assert np.allclose(f.rotate_x(2.1).angles, GOLD[f"{name}/rot_x"], atol=1e-15)
    assert np.allclose(f.rotate_y(-1.1).angles, GOLD[f"{name}/rot_y"], atol=1e-15)
    assert np.allclose(f.rotate_z(7.5).angles, GOLD[f"{name}/rot_z"], atol=1e-15)


def test_angles_from_rotation():
    m = frames()["f2"].rotation_matrix
    assert np.allclose(ReferenceFrame.angles_from_rotation(m), GOLD["angles_from_rotation"], atol=1e-14)


def test_subclass_frames_match_reference():
    f0 = frames()["f0"]
    tr = TranslatingReferenceFrame((1, 2, 3), (0.1, 0.2, 0.3), (0.5, -1, 2), f0, 0.5).at_time(2.25)
    assert np.allclose(tr.offset, GOLD["translating/offset"], atol=1e-15)
    assert np.allclose(tr.angles, GOLD["translating/angles"], atol=1e-15)
    v = np.zeros((7, 3))
    tr.add_velocity(GOLD["translating/p"], v)
    assert np.allclose(v, GOLD["translating/velocity"], atol=1e-15)
    rr = RotorReferenceFrame((0, 1, 0), (0.3, 0.0, 0.2), None, (0.1, 0.2, 2.0), 0.0).at_time(1.7)
    assert np.allclose(rr.offset, GOLD["rotor/offset"], atol=1e-15)
    assert np.allclose(rr.angles, GOLD["rotor/angles"], atol=1e-13)
    v = np.zeros((7, 3))
    rr.add_velocity(GOLD["translating/p"], v)
    assert np.allclose(v, GOLD["rotor/velocity"], atol=1e-15)


def test_reference_frame_behaviour():
    """test/pytests/test_reference_frame.py: wrapping, parents, rotations, inverses, out args."""
    rf0 = ReferenceFrame(theta=(0.2, 0.3, -2), offset=(3, 2, 0))
    assert np.sin(rf0.angles) == pytest.approx(np.sin([0.2, 0.3, -2]))
    assert all(rf0.offset == (3, 2, 0))
    rng = np.random.default_rng(0)
    rf_0 = ReferenceFrame(rng.random(3), rng.random(3))
    rf_1 = ReferenceFrame((102, 4.20, 1.4), (31.2, 33.0, -2), rf_0)
    rf_2 = ReferenceFrame((-102, -4.20, 1.4), (-31.2, 33.0, 2), rf_1)
    assert rf_2.parent is rf_1 and rf_2.parents == (rf_1, rf_0)
    rf_z = ReferenceFrame((31.2, 33.0, -2), (0, 0, 0), rf_0)
    r = rf_z.rotate_x(2.1)
    assert r.parent is rf_z.parent and r.angles[0] == rf_z.angles[0] + 2.1 and all(r.offset == rf_z.offset)
    assert all(rf_z.with_offset([0, 2, 3.0]).offset == [0, 2, 3.0])
    for _ in range(20):
        rf = ReferenceFrame(rng.random(3), rng.random(3))
        assert pytest.approx(rf.rotation_matrix @ rf.rotation_matrix.T) == np.eye(3)
        x = rng.random((12, 5, 2, 3))
        assert pytest.approx(x) == rf.to_parent_with_offset(rf.from_parent_with_offset(x))
    x_in = rng.random((3, 1, 4, 10, 3))
    with pytest.raises(TypeError):
        rf.to_parent_with_offset(x_in, "SOME random object")
    with pytest.raises(ValueError):
        rf.to_parent_with_offset(x_in, np.array([[0, 2, 3.0]]))
    with pytest.raises(ValueError):
        rf.to_parent_with_offset(x_in, np.empty_like(x_in, dtype=np.float32))
    x_out = np.empty_like(x_in)
    assert rf.to_parent_with_offset(x_in, x_out) is x_out
