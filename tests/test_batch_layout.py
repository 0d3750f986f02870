"""Host-side tables of the batched engine (pyvl_b200/batch.py), checked without a GPU: every
index a batched kernel reads stays inside its array, and the persistent kernels' work items
cover every (control point, ring) and (point, segment) pair of every case exactly once."""

import numpy as np
import pytest


@pytest.fixture(scope="module")
def layout():
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.workloads import batch_wings

    cases = batch_wings(n_cases=7, seed=5, steps=9, p_min=64, p_max=500)
    return BatchEngine(cases, host_only=True), cases


def _records(t, dtype):
    return np.frombuffer(t.numpy().tobytes(), dtype)


def test_ring_jobs_cover_each_block_once(layout):
    from pyvl_b200.batch import RING_JOB

    e, cases = layout
    cpb = e.tile["ring"]
    for name, n_cols, csr_rows, out_size in (("body", e.P, e.n_rings, e.A.numel()),
                                             ("implicit", e.S, len(e.row0_offsets) - 1, e.implicit.numel()),
                                             ("implicit_fold", e.S, len(e.row0_offsets) - 1, e.A.numel())):
        jobs_t, items_t, n_items = e.ring_tables[name]
        jobs = _records(jobs_t, RING_JOB)
        items = items_t.numpy().view(np.uint32)
        assert np.array_equal(items, jobs["item_begin"])
        seen = [np.zeros((int(j["n_cp"]), int(j["n_rings"])), np.int32) for j in jobs]
        for item in range(n_items):
            jb = int(np.searchsorted(items, item, side="right") - 1)
            J = jobs[jb]
            col_tiles = -(-int(J["n_rings"]) // 128)
            local = item - int(J["item_begin"])
            rb, ct = divmod(local, col_tiles)
            i0 = rb * cpb
            for q in range(cpb):
                if i0 + q >= J["n_cp"]:
                    break
                j0, j1 = ct * 128, min(ct * 128 + 128, int(J["n_rings"]))
                seen[jb][i0 + q, j0:j1] += 1
        for J, s in zip(jobs, seen):
            assert (s == 1).all()
            assert int(J["ring_begin"]) + int(J["n_rings"]) <= csr_rows
            assert int(J["cp_begin"]) + int(J["n_cp"]) <= e.n_rings
            assert int(J["out_begin"]) + int(J["n_cp"]) * int(J["ld"]) <= out_size


def _active(e, J, rows):
    """Segments a sweep job covers when the wake has `rows` rows (csrc/batch.cu, SweepJob)."""
    from pyvl_b200.batch import NO_ROWS

    if int(J["seg_rows"]) == NO_ROWS:
        return int(J["seg_count"])
    return min(int(J["seg_count"]), int(e.seg_upto[int(J["seg_rows"]) + min(rows, e.R)]))


def test_sweep_jobs_in_bounds_and_cover_pairs(layout):
    from pyvl_b200.batch import SWEEP_JOB

    e, cases = layout
    threads, ppt = e.tile["sweep"]
    kpts = threads * ppt
    n_part = e.partials.numel() // 3
    for name, n_seg, n_pts_arr, out_rows in (("wake", e.wake_mesh.n_lines, e.n_rings, e.n_rings),
                                             ("advect", e.body.n_lines, e.pidx.numel(), e.node_vel.shape[0])):
        jobs_t, items_t, n_items, pt_item_t, n_total = e.sweep_tables[name]
        jobs = _records(jobs_t, SWEEP_JOB)
        items = items_t.numpy().view(np.uint32)
        for rows in (1, 4, e.R):
            cover = [np.zeros(int(j["pt_max"]), np.int64) for j in jobs]
            for item in range(n_items):
                jb = int(np.searchsorted(items, item, side="right") - 1)
                J = jobs[jb]
                n_pts = int(J["pt_max"]) if not J["pt_per_row"] else int(J["pt_per_row"]) * min(
                    rows, int(J["pt_max"]) // int(J["pt_per_row"]))
                blocks = -(-int(J["pt_max"]) // kpts)
                split, pb = divmod(item - int(J["item_begin"]), blocks)
                assert split < J["n_split"]
                l0 = int(J["seg_begin"]) + split * int(J["per"])
                l1 = int(J["seg_begin"]) + min(_active(e, J, rows), (split + 1) * int(J["per"]))
                p0, p1 = pb * kpts, min(pb * kpts + kpts, n_pts)
                if p0 < p1:
                    cover[jb][p0:p1] += max(0, l1 - l0)
            for J, cv in zip(jobs, cover):
                n_pts = int(J["pt_max"]) if not J["pt_per_row"] else int(J["pt_per_row"]) * min(
                    rows, int(J["pt_max"]) // int(J["pt_per_row"]))
                assert (cv[:n_pts] == _active(e, J, rows)).all()  # every point meets every live segment once
                assert (cv[n_pts:] == 0).all()
        for J in jobs:
            assert int(J["seg_begin"]) + int(J["seg_count"]) <= n_seg
            assert int(J["pt_begin"]) + int(J["pt_max"]) <= n_pts_arr
            assert int(J["part_begin"]) + int(J["n_split"]) * int(J["pt_max"]) <= n_part
            assert int(J["out_begin"]) + int(J["pt_max"]) <= out_rows


def test_wake_tables_in_bounds(layout):
    e, cases = layout
    pidx = e.pidx.numpy().view(np.uint32)
    assert pidx.max() < e.n_wake_pts
    bn = e.bn.numpy().view(np.uint32)
    assert bn.max() < e.n_points
    slot = e.col_slot.numpy().view(np.uint32).reshape(-1)
    adj = e.adj.numpy().view(np.uint32).reshape(-1)
    o = 0
    for k in range(e.B):
        S = int(e.S[k])
        assert slot[2 * o:2 * (o + S)].max() < e.NC[k]
        a = adj[2 * o:2 * (o + S)]
        assert ((a == 0x7FFFFFFF) | (a < e.P[k])).all()
        o += S
    # first-row rings of the implicit blocks are the merged wake mesh's rings s*R (row 0), with
    # their lines renumbered into the row order of the sweep (same node pairs, same orientation)
    off, sl = e.wake_mesh.surface_offsets, e.wake_mesh.surface_lines
    old_lines = np.asarray(e.wake_mesh._lines, np.uint32).reshape(-1, 2)
    shed0 = 0
    for k in range(e.B):
        for s in range(int(e.S[k])):
            r = (shed0 + s) * e.R
            a0, a1 = e.row0_offsets[shed0 + s], e.row0_offsets[shed0 + s + 1]
            new, old = e.row0_lines[a0:a1], sl[off[r]:off[r + 1]]
            assert np.array_equal(new & 0x80000000, old & 0x80000000)
            assert np.array_equal(e.wake_lines_rm[new & 0x7FFFFFFF], old_lines[old & 0x7FFFFFFF])
        shed0 += int(e.S[k])


def test_row_ordered_wake_lines(layout):
    """The wake's lines in row order per case: a permutation of the merged wake mesh's lines,
    the line -> ring map and the row-0 rings follow it, and the lines of rows < k of a case
    are exactly its first seg_upto[k] lines (so a sweep over that prefix misses no live line)."""
    e, cases = layout
    wl, R = e.wake_mesh, e.R
    old_lines = np.asarray(wl._lines, np.uint32).reshape(-1, 2)
    new_lines = e.wake_lines_rm
    key = lambda a: set(map(tuple, a.tolist()))
    assert len(new_lines) == len(old_lines) and key(new_lines) == key(old_lines)
    # recover the permutation from the unique (start, end) node pairs
    pos = {tuple(v): i for i, v in enumerate(old_lines.tolist())}
    order = np.array([pos[tuple(v)] for v in new_lines.tolist()])
    m_off, m_ent = wl.ring_map()
    for i in range(0, len(order), max(1, len(order) // 300)):
        o = order[i]
        a = e.wake_map_entries_rm[e.wake_map_offsets_rm[i]:e.wake_map_offsets_rm[i + 1]]
        assert np.array_equal(a, m_ent[m_off[o]:m_off[o + 1]])
    # row-0 rings reference the same node pairs as before the renumbering
    for g_new, g_old in zip(e.row0_lines[:200], np.concatenate(
            [((wl.surface_lines[wl.surface_offsets[s * R]:wl.surface_offsets[s * R + 1]]))
             for s in range(int(np.sum(e.S)))])[:200]):
        assert (g_new & 0x80000000) == (g_old & 0x80000000)
        assert tuple(new_lines[g_new & 0x7FFFFFFF]) == tuple(old_lines[g_old & 0x7FFFFFFF])
    # prefix property per case
    off, ids = wl.surface_offsets.astype(np.int64), (wl.surface_lines & 0x7FFFFFFF).astype(np.int64)
    inv = np.empty_like(order)
    inv[order] = np.arange(order.size)
    per_case = e.seg_upto.reshape(e.B, R + 1)[:, R].astype(np.int64)  # every line has a row < R
    assert per_case.sum() == wl.n_lines
    line_off = np.concatenate([[0], np.cumsum(per_case)])
    ring0 = 0
    for c in range(e.B):
        S = int(e.S[c])
        up = e.seg_upto[c * (R + 1):(c + 1) * (R + 1)]
        assert up[0] == 0 and np.all(np.diff(up.astype(np.int64)) >= 0)
        for k in (1, 2, R):
            rings = [ring0 + s * R + r for s in range(S) for r in range(k)]
            used = np.unique(np.concatenate([ids[off[j]:off[j + 1]] for j in rings]))
            new = inv[used] - line_off[c]
            assert new.min() >= 0 and new.max() < up[k] and used.size == up[k]
        ring0 += S * R


def test_ring_tile_tables(layout):
    """Column tiles of the tiled ring kernel: every tile lists exactly the distinct lines of its
    (up to) 128 rings, every CSR entry points at its own line in its tile's list, and the
    shared-memory stride covers the longest list."""
    e, cases = layout
    for name, off, sl, n_rings in (("body", e.body.surface_offsets, e.body.surface_lines, e.P),
                                   ("implicit", e.row0_offsets, e.row0_lines, e.S)):
        t = e.ring_tiles[name]
        off = np.asarray(off, np.int64)
        ids = np.asarray(sl, np.uint32) & 0x7FFFFFFF
        toff, tl, sll = t["tile_offsets"].astype(np.int64), t["tile_lines"], t["sl_local"]
        assert len(sll) == len(ids) and t["max"] == int(np.diff(toff).max())
        r0 = 0
        for j, n in enumerate(np.asarray(n_rings, np.int64)):
            for ct in range(-(-int(n) // 128)):
                tile = int(t["job_tile"][j]) + ct
                a, b = off[r0 + ct * 128], off[r0 + min(ct * 128 + 128, int(n))]
                lines = tl[toff[tile]:toff[tile + 1]]
                assert np.array_equal(lines, np.unique(ids[a:b]))
                assert np.array_equal(lines[sll[a:b]], ids[a:b])
            r0 += int(n)
        assert r0 == len(off) - 1
