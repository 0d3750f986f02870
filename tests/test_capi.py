"""The C-ABI library: it loads, exports every symbol include/pvl_b200.h declares, and its
host-side topology matches the reference's (golden vectors).  No GPU needed."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from pyvl_b200 import _lib, _probe
from pyvl_b200.cvl import Mesh

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def declared_symbols():
    text = (ROOT / "include" / "pvl_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pvl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert not [n for n in names if n not in _lib.SIGNATURES], [n for n in names if n not in _lib.SIGNATURES]
    # measurement and test probes live in their own library, outside the product ABI
    assert not [n for n in names if "probe" in n]


def test_probe_library_exports_its_header():
    text = (ROOT / "pyvl_b200" / "probe" / "pvl_probe.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = sorted(set(re.findall(r"\b(pvl_[a-z0-9_]+)\s*\(", text)))
    lib = ctypes.CDLL(str(_probe.LIB_PATH))
    assert names and not [n for n in names if not hasattr(lib, n)]
    assert sorted(_probe.SIGNATURES) == names


def test_version_and_error_string():
    assert _lib.lib().pvl_version() >= 100
    with pytest.raises(ValueError):
        Mesh(3, [[0, 1]])


def _cases():
    d = np.load(GOLD / "kernels.npz")
    return d, sorted({k.split("/")[0] for k in d.files})


@pytest.mark.parametrize("name", _cases()[1])
def test_topology_matches_reference(name):
    d, _ = _cases()
    g = lambda k: d[f"{name}/{k}"]  # noqa: E731
    elems = np.split(g("elements_flat"), np.cumsum(g("elements_counts"))[:-1])
    m = Mesh(g("positions").shape[0], elems)
    assert np.array_equal(m.line_data, g("lines"))
    assert np.array_equal(m.surface_offsets, g("offsets"))
    assert np.array_equal(m.surface_lines, g("surface_lines"))
    dual = m.compute_dual()
    assert np.array_equal(dual.line_data, g("dual_lines"))
    counts, flat = m.to_element_connectivity()
    assert np.array_equal(counts, g("to_elem_counts"))
    assert np.array_equal(flat, g("to_elem_flat"))
    assert np.array_equal(dual.dual_free_edges(), g("free_edges"))
    if f"{name}/normal_crit" in d.files:
        # normals from the golden file (the GPU computes them in the GPU tests)
        from oracle.kernels import OracleMesh
        om = OracleMesh(g("positions").shape[0], elems)
        crit = dual.dual_normal_criterion(-0.5, om.surface_normal(g("positions")))
        assert np.array_equal(crit, g("normal_crit"))


def test_reference_mesh_tests():
    """test/pytests/test_mesh.py:8-16 and :71-102 (construction, merge)."""
    elements = [[0, 1, 2, 3], [2, 3, 4], [0, 1, 4], [2, 4, 5]]
    msh = Mesh(max(max(e) for e in elements), elements)
    counts, conn = msh.to_element_connectivity()
    assert np.all(counts == [len(e) for e in elements])
    assert np.all(conn == np.array(sum(elements, start=[])))
    msh1 = Mesh(6, [[0, 1, 2, 3], [2, 3, 4], [0, 1, 4], [2, 4, 5]])
    msh2 = Mesh(6, [[2, 1, 0], [1, 2, 3], [4, 1, 5]])
    msh3 = Mesh(6, [[4, 1, 0], [5, 2, 4]])
    merged = Mesh.merge_meshes(msh1, msh2, msh3)
    assert merged.n_surfaces == msh1.n_surfaces + msh2.n_surfaces + msh3.n_surfaces
    assert merged.n_lines == msh1.n_lines + msh2.n_lines + msh3.n_lines
    assert merged.n_points == msh1.n_points + msh2.n_points + msh3.n_points
    n_lines = n_surfaces = point_offset = 0
    for m in (msh1, msh2, msh3):
        for i_s in range(m.n_surfaces):
            sm, so = merged.get_surface(n_surfaces), m.get_surface(i_s)
            for l1, l2 in zip(sm.lines, so.lines, strict=True):
                assert l1.begin == l2.begin + point_offset
                assert l1.end == l2.end + point_offset
            n_surfaces += 1
        for i_l in range(m.n_lines):
            lm, lo = merged.get_line(n_lines), m.get_line(i_l)
            assert lm.begin == lo.begin + point_offset and lm.end == lo.end + point_offset
            n_lines += 1
        point_offset += m.n_points


def test_line_ring_map_is_transpose():
    m = Mesh(85, [list(map(int, e)) for e in __import__("pyvl_b200.workloads", fromlist=["x"]).flat_wing().elements])
    offs, ents = m.ring_map()
    seen = []
    for l in range(m.n_lines):
        for e in ents[offs[l]:offs[l + 1]]:
            seen.append((int(e) & 0x7FFFFFFF, l, int(e) >> 31))
    ref = []
    for s in range(m.n_surfaces):
        for g in m.surface_lines[m.surface_offsets[s]:m.surface_offsets[s + 1]]:
            ref.append((s, int(g) & 0x7FFFFFFF, int(g) >> 31))
    assert sorted(seen) == sorted(ref)


def test_wake_node_columns_merge_shared_trailing_edge_nodes():
    """Adjacent strips share a trailing-edge node: their node columns get one representative,
    and the merged wake mesh keeps one streamwise line per shared column."""
    import numpy as np

    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import wake_node_columns, wake_ring_connectivity

    bn = np.array([[0, 1], [1, 2], [2, 3], [7, 6]])  # strips 0-2 chained, strip 3 separate and reversed
    rep, cols, slot = wake_node_columns(bn)
    assert rep.tolist() == [0, 1, 1, 3, 3, 5, 6, 7]
    assert cols.tolist() == [0, 1, 3, 5, 6, 7]
    assert (cols[slot] == rep).all()
    R, S = 5, 4
    plain = Mesh(2 * (R + 1) * S, wake_ring_connectivity(R, S))
    merged = Mesh(2 * (R + 1) * S, wake_ring_connectivity(R, S, bn))
    # per strip: R + 1 spanwise and 2 R streamwise lines; two shared columns save 2 R lines
    assert plain.n_lines == S * (3 * R + 1)
    assert merged.n_lines == plain.n_lines - 2 * R


def test_argument_errors_are_reported_before_any_device_work():
    """Null pointers, bad sizes and short workspaces come back as the reference's exception
    types with a message, from the host-side checks that run before any CUDA call (so they
    hold without a GPU).  Fake device addresses stand in where a pointer must be non-null."""
    fake = 1 << 20  # 16-byte aligned, never dereferenced: every call below fails before use
    # the far-field evaluator of the probe library
    _probe.call("pvl_probe_far_series", 0, None, None, None, None, None)  # nothing to do
    with pytest.raises(ValueError, match="null pointer"):
        _probe.call("pvl_probe_far_series", 8, None, fake, fake, fake, None)
    # the segment-sum velocity
    with pytest.raises(ValueError, match="pts is NULL"):
        _lib.call("pvl_line_velocity", _lib.PVL_F64, 4, 2, fake, fake, fake, 5, None, None, 1e-6, 1.0, 0.0, fake,
                  fake, 1 << 20, None)
    with pytest.raises(ValueError, match="unknown precision"):
        _lib.call("pvl_line_velocity", 7, 4, 2, fake, fake, fake, 5, fake, None, 1e-6, 1.0, 0.0, fake, fake,
                  1 << 20, None)
    need = _lib.query("pvl_line_velocity_workspace", 2, 5, _lib.PVL_F64)
    with pytest.raises(_lib.PvlError, match="workspace"):
        _lib.call("pvl_line_velocity", _lib.PVL_F64, 4, 2, fake, fake, fake, 5, fake, None, 1e-6, 1.0, 0.0, fake,
                  fake, need - 1, None)
    # the device-driven GMRES graph
    n = 64
    args = dict(n=n, A=fake, lda=n, Minv=fake, ldm=n, b=fake, x=fake, V=fake, Z=fake, W=fake, r0=fake, w=fake,
                v32=fake, ctl=fake, max_iter=8, tol=1e-12, ipiv=fake, info=fake, ws=fake,
                ws_bytes=_lib.query("pvl_lu_workspace", n), gamma=None, n_gamma=0, n_groups=0, group_offsets=None,
                status=fake)
    h = ctypes.c_uint64(7)

    def create(**kw):
        a = dict(args, **kw)
        _lib.call("pvl_gmres_graph_create", *a.values(), ctypes.byref(h))

    with pytest.raises(ValueError, match="graph_out is NULL"):
        _lib.call("pvl_gmres_graph_create", *args.values(), None)
    with pytest.raises(ValueError, match="null pointer"):
        create(W=None)
    assert h.value == 0  # cleared before the checks
    with pytest.raises(ValueError, match="max_iter"):
        create(max_iter=_lib.query("pvl_gmres_max_iter") + 1)
    with pytest.raises(ValueError, match="inconsistent sizes"):
        create(lda=n - 1)
    with pytest.raises(ValueError, match="aligned"):
        create(v32=fake + 4)
    with pytest.raises(_lib.PvlError, match="workspace"):
        create(ws_bytes=args["ws_bytes"] - 1)
