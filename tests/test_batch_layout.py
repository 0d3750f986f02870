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
                                             ("implicit", e.S, len(e.row0_offsets) - 1, e.implicit.numel())):
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
                l1 = int(J["seg_begin"]) + min(int(J["seg_count"]), (split + 1) * int(J["per"]))
                p0, p1 = pb * kpts, min(pb * kpts + kpts, n_pts)
                if p0 < p1:
                    cover[jb][p0:p1] += l1 - l0
            for J, cv in zip(jobs, cover):
                n_pts = int(J["pt_max"]) if not J["pt_per_row"] else int(J["pt_per_row"]) * min(
                    rows, int(J["pt_max"]) // int(J["pt_per_row"]))
                assert (cv[:n_pts] == int(J["seg_count"])).all()  # every point meets every segment once
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
    # first-row rings of the implicit blocks are the merged wake mesh's rings s*R (row 0)
    off, sl = e.wake_mesh.surface_offsets, e.wake_mesh.surface_lines
    shed0 = 0
    for k in range(e.B):
        for s in range(int(e.S[k])):
            r = (shed0 + s) * e.R
            a0, a1 = e.row0_offsets[shed0 + s], e.row0_offsets[shed0 + s + 1]
            assert np.array_equal(e.row0_lines[a0:a1], sl[off[r]:off[r + 1]])
        shed0 += int(e.S[k])
