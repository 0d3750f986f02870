"""Batched stepping of many independent wings (or bodies) of uneven size.

``BatchEngine(cases)`` steps every case of a list of workload ``Case`` objects together, one
launch per kernel over the whole batch (csrc/batch.cu), with the same per-case arithmetic as
``SolverEngine``: control points, normals and RHS, the body matrix, the implicit first wake row
folded into it, the explicit wake rows in the RHS, the solve, the wake advection by freestream
plus body induction, and the shedding of the trailing-edge circulation (python/pyvl/solver.py:175-263,
python/pyvl/wake_models.py:83-223 per case).  The solve is the device-resident Jacobi-preconditioned
GMRES with FP64 residuals (tolerance ``solve_tol``, relative residual), so a whole step runs without
host synchronisation and, from the second step on, is captured once as a CUDA graph and replayed.
``tune()`` is the autotuner: it times every tile shape of the persistent sweep and ring kernels on
this batch and keeps the fastest.

The reference steps one geometry per solver loop and has no batched form; a per-case loop of
``SolverEngine`` is the comparison (bench.py --workload batch).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .cvl import Mesh
from .device import ptr, require_cuda, stream_ptr, to_device_u32
from .engine import wake_node_columns, wake_ring_connectivity, wake_row0_mesh, wake_spec_from_te

RING_JOB = np.dtype([("cp_begin", "<u4"), ("n_cp", "<u4"), ("ring_begin", "<u4"), ("n_rings", "<u4"),
                     ("out_begin", "<u8"), ("ld", "<u4"), ("item_begin", "<u4")])
SWEEP_JOB = np.dtype([(k, "<u4") for k in ("seg_begin", "seg_count", "pt_begin", "pt_max", "pt_per_row",
                                          "out_begin", "n_split", "per", "part_begin", "item_begin", "mode",
                                          "case_id", "seg_rows")])
NO_ROWS = 0xFFFFFFFF  # SweepJob.seg_rows of a job swept over all its segments
WAKE_CASE = np.dtype({"names": ["P", "S", "n_cols", "ring_begin", "mat_begin", "imp_begin", "shed_begin",
                                "pos_begin", "circ_begin", "vel_begin", "dt"],
                      "formats": ["<u4", "<u4", "<u4", "<u4", "<u8", "<u4", "<u4", "<u4", "<u4", "<u4", "<f8"],
                      "offsets": [0, 4, 8, 12, 16, 24, 28, 32, 36, 40, 48], "itemsize": 56})
SOLVE_CASE = np.dtype([("row_begin", "<u4"), ("n", "<u4"), ("mat_begin", "<u8")])

SWEEP_TILES = [(128, 1), (128, 2), (128, 4), (256, 1), (256, 2)]
RING_TILES = [8, 16, 32]


def _check_layouts() -> None:
    for name, dt in (("ring_job", RING_JOB), ("sweep_job", SWEEP_JOB), ("wake_case", WAKE_CASE),
                     ("solve_case", SOLVE_CASE)):
        n = int(_lib.query(f"pvl_batch_{name}_bytes"))
        if n != dt.itemsize:
            raise RuntimeError(f"batch record {name}: library has {n} bytes, host layout {dt.itemsize}")


def ring_tile_tables(offsets, surface_lines, n_rings, tile: int = 128):
    """Column tiles of the ring jobs for pvl_batch_ring_matrix_tiled.  The CSR rows (rings) are
    the jobs' rings back to back (job j owns n_rings[j] of them); each job's rings are cut into
    tiles of `tile`.  Returns job_tile (first tile of each job), tile_offsets and tile_lines (the
    distinct lines of every tile, ascending), sl_local (each CSR entry's position in its tile's
    list) and the longest list."""
    off = np.asarray(offsets, np.int64)
    ids = (np.asarray(surface_lines, np.uint32) & np.uint32(0x7FFFFFFF)).astype(np.int64)
    n_rings = np.asarray(n_rings, np.int64)
    per_job = -(-n_rings // tile)
    job_tile = np.concatenate([[0], np.cumsum(per_job)[:-1]]).astype(np.int64)
    ring_job = np.repeat(np.arange(n_rings.size), n_rings)
    ring_begin = np.concatenate([[0], np.cumsum(n_rings)[:-1]])
    ring_tile = job_tile[ring_job] + (np.arange(ring_job.size) - ring_begin[ring_job]) // tile
    entry_tile = np.repeat(ring_tile, np.diff(off))
    base = int(ids.max()) + 1 if ids.size else 1
    uniq, inv = np.unique(entry_tile * base + ids, return_inverse=True)
    counts = np.bincount(uniq // base, minlength=int(per_job.sum()))
    tile_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    sl_local = inv.reshape(-1) - tile_off[entry_tile]
    return (job_tile.astype(np.uint32), tile_off.astype(np.uint32), (uniq % base).astype(np.uint32),
            sl_local.astype(np.uint32), int(counts.max()) if counts.size else 1)


def _dev_records(arr: np.ndarray, dev) -> torch.Tensor:
    return torch.as_tensor(np.frombuffer(arr.tobytes(), np.uint8).copy(), device=dev)


def _splits(n_segments: int, n_points: int, pts_per_cta: int, target_ctas: int = 148 * 8) -> tuple[int, int]:
    """Segment ranges of one sweep job: enough work items for the GPU, >= 2 tiles per range."""
    blocks = max(1, -(-n_points // pts_per_cta))
    s = max(1, -(-target_ctas // blocks))
    s = min(s, max(1, -(-n_segments // 256)))
    per = -(-n_segments // s)
    return -(-n_segments // per), per


# weights of (gamma, g0, g1, g2, g3) by the number of stored solutions: keep gamma, the last
# solution, then the linear, quadratic and cubic extrapolations through 2, 3 and 4 of them
_EXTRAP = [[1.0, 0.0, 0.0, 0.0, 0.0],
           [0.0, 1.0, 0.0, 0.0, 0.0],
           [0.0, 2.0, -1.0, 0.0, 0.0],
           [0.0, 3.0, -3.0, 1.0, 0.0],
           [0.0, 4.0, -6.0, 4.0, -1.0]]


class BatchEngine:
    """Every case of ``cases`` stepped together on the device (see the module docstring)."""

    def __init__(self, cases, solve_tol: float = 1e-12, max_iter: int = 8, tile: dict | None = None,
                 host_only: bool = False, reuse_static_bodies: bool = False):
        self.host_only = host_only  # build the tables on the host only (layout checks without a GPU)
        self.dev = torch.device("cpu") if host_only else require_cuda()
        _check_layouts()
        self.cases = list(cases)
        B = self.B = len(self.cases)
        if B == 0:
            raise ValueError("empty batch")
        R = {int(c.line_rows) for c in self.cases}
        if len(R) != 1:
            raise ValueError("every case of a batch needs the same number of wake rows")
        self.R = R = R.pop()
        tols = {float(c.tol) for c in self.cases}
        if len(tols) != 1:
            raise ValueError("every case of a batch needs the same vortex tolerance")
        self.tol = tols.pop()
        self.solve_tol = float(solve_tol)
        self.max_iter = int(max_iter)
        # rigid, motionless bodies: their matrix is the same every step, so it can be built once
        from .workloads import Static

        self.static = bool(reuse_static_bodies) and all(isinstance(c.kinematics, Static) for c in self.cases)
        self.A_body = None
        self.tile = dict(tile or {"sweep": (128, 1), "ring": 16})
        dev = self.dev
        f64 = dict(dtype=torch.float64, device=dev)

        # ---------------- topology, per case and concatenated
        meshes, wmeshes, row0s, specs = [], [], [], []
        P, S, NC, NP, L, WL = [], [], [], [], [], []
        cols_all, slot_all, bn_all, adj_all = [], [], [], []
        for c in self.cases:
            m = Mesh(c.n_points, c.elements)
            spec = wake_spec_from_te(m, c.te_node_pairs, R, c.t0)
            s_ = int(spec.shedding_lines.size)
            bn = np.asarray(spec.bordering_nodes, np.int64).reshape(s_, 2)
            wm = Mesh(2 * (R + 1) * s_, wake_ring_connectivity(R, s_, bn))
            _, cols, slot = wake_node_columns(bn)
            meshes.append(m)
            wmeshes.append(wm)
            row0s.append(wake_row0_mesh(wm, s_, R))
            specs.append(spec)
            P.append(m.n_surfaces)
            S.append(s_)
            NC.append(int(cols.size))
            NP.append(m.n_points)
            L.append(m.n_lines)
            WL.append(wm.n_lines)
            cols_all.append(cols)
            slot_all.append(slot)
            bn_all.append(bn)
            adj_all.append(np.asarray(spec.adjacent_surfaces, np.int64).reshape(s_, 2))
        self.P, self.S, self.NC = np.array(P), np.array(S), np.array(NC)
        ring_off = np.concatenate([[0], np.cumsum(P)]).astype(np.int64)
        pt_off = np.concatenate([[0], np.cumsum(NP)]).astype(np.int64)
        line_off = np.concatenate([[0], np.cumsum(L)]).astype(np.int64)
        wline_off = np.concatenate([[0], np.cumsum(WL)]).astype(np.int64)
        shed_off = np.concatenate([[0], np.cumsum(S)]).astype(np.int64)
        wpt_off = 2 * (R + 1) * shed_off
        mat_off = np.concatenate([[0], np.cumsum(np.asarray(P, np.int64) ** 2)]).astype(np.int64)
        imp_off = np.concatenate([[0], np.cumsum(np.asarray(P, np.int64) * np.asarray(S))]).astype(np.int64)
        vel_off = np.concatenate([[0], np.cumsum(np.asarray(NC, np.int64) * R)]).astype(np.int64)
        self.ring_off, self.pt_off, self.mat_off = ring_off, pt_off, mat_off
        self.n_rings, self.n_points = int(ring_off[-1]), int(pt_off[-1])
        self.body = Mesh.merge_meshes(*meshes)
        self.wake_mesh = Mesh.merge_meshes(*wmeshes)
        # row-0 rings reference the wake lines: rebase them onto the merged wake mesh's lines
        sl0 = []
        for k, r0 in enumerate(row0s):
            g = r0.surface_lines.astype(np.uint64)
            sl0.append(((g & np.uint64(0x7FFFFFFF)) + np.uint64(wline_off[k])) | (g & np.uint64(0x80000000)))
        off0 = np.concatenate([[0], np.cumsum([r.n_surfaces and int(r.surface_offsets[-1]) for r in row0s])])
        self.row0_offsets = np.concatenate(
            [[0]] + [r.surface_offsets[1:].astype(np.int64) + off0[k] for k, r in enumerate(row0s)]).astype(np.uint32)
        self.row0_lines = np.concatenate(sl0).astype(np.uint32)
        # The wake's lines in row order within each case (lines first used by row 0, then row 1,
        # ...), so that the explicit wake term of a wake that has shed k rows sweeps a prefix of
        # each case's lines: seg_upto[c * (R + 1) + k] of them.  The segment table, the line
        # circulations (a permuted line -> ring map) and the row-0 rings all use this order.
        wl = self.wake_mesh
        w_off = wl.surface_offsets.astype(np.int64)
        w_ids = (wl.surface_lines & np.uint32(0x7FFFFFFF)).astype(np.int64)
        ring_row = np.arange(wl.n_surfaces, dtype=np.int64) % R  # rings s * R + r within each case
        min_row = np.full(wl.n_lines, R, np.int64)
        np.minimum.at(min_row, w_ids, np.repeat(ring_row, np.diff(w_off)))
        line_case = np.repeat(np.arange(B), WL)
        order = np.lexsort((np.arange(wl.n_lines), min_row, line_case))
        inv = np.empty_like(order)
        inv[order] = np.arange(order.size)
        self.wake_lines_rm = np.asarray(wl._lines, np.uint32).reshape(-1, 2)[order]
        m_off, m_ent = wl.ring_map()
        m_off = m_off.astype(np.int64)
        cnt = np.diff(m_off)[order]
        self.wake_map_offsets_rm = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
        src = np.repeat(m_off[order] - self.wake_map_offsets_rm[:-1].astype(np.int64), cnt) + np.arange(int(cnt.sum()))
        self.wake_map_entries_rm = np.asarray(m_ent, np.uint32)[src]
        r0 = self.row0_lines.astype(np.int64)
        self.row0_lines = ((inv[r0 & 0x7FFFFFFF]) | (r0 & 0x80000000)).astype(np.uint32)
        self.seg_upto = np.zeros(B * (R + 1), np.uint32)
        for k in range(B):
            rows_k = np.sort(min_row[wline_off[k]:wline_off[k + 1]])
            self.seg_upto[k * (R + 1):(k + 1) * (R + 1)] = np.searchsorted(rows_k, np.arange(R + 1), side="left")
        # segment-point pairs of the two sweeps once every wake has all R rows: the explicit wake
        # term (each case's wake lines at its control points) and the advection (each case's body
        # lines at its distinct wake node columns, every row)
        full = self.seg_upto.reshape(B, R + 1)[:, R].astype(np.int64)
        self.sweep_pairs_full = {"wake": int(np.sum(full * np.asarray(P, np.int64))),
                                 "advect": int(np.sum(np.asarray(L, np.int64) * np.asarray(NC, np.int64) * R))}
        self.d_body = None if host_only else self.body.device_arrays()
        self.d_wake = None if host_only else {
            "lines": to_device_u32(self.wake_lines_rm, dev),
            "map_offsets": to_device_u32(self.wake_map_offsets_rm, dev),
            "map_entries": to_device_u32(self.wake_map_entries_rm, dev),
        }
        self.d_seg_upto = to_device_u32(self.seg_upto, dev)
        self.d_row0 = {"offsets": to_device_u32(self.row0_offsets, dev), "lines": to_device_u32(self.row0_lines, dev)}
        n_wake_pts = int(wpt_off[-1])
        self.n_wake_pts = n_wake_pts

        # ---------------- per-case tables
        uinf = np.stack([np.asarray(c.freestream, np.float64) for c in self.cases])
        self.uinf = torch.as_tensor(uinf, device=dev)
        self.flow = torch.as_tensor(np.repeat(uinf, P, axis=0), device=dev)
        wc = np.zeros(B, WAKE_CASE)
        wc["P"], wc["S"], wc["n_cols"] = P, S, NC
        wc["ring_begin"], wc["mat_begin"], wc["imp_begin"] = ring_off[:-1], mat_off[:-1], imp_off[:-1]
        wc["shed_begin"], wc["pos_begin"], wc["circ_begin"] = shed_off[:-1], wpt_off[:-1], R * shed_off[:-1]
        wc["vel_begin"] = vel_off[:-1]
        wc["dt"] = [float(c.dt) for c in self.cases]
        self.wake_cases = _dev_records(wc, dev)
        sc = np.zeros(B, SOLVE_CASE)
        sc["row_begin"], sc["n"], sc["mat_begin"] = ring_off[:-1], P, mat_off[:-1]
        self.solve_cases = _dev_records(sc, dev)
        self.row_case = to_device_u32(np.repeat(np.arange(B), P).astype(np.uint32), dev)
        self.node_case = to_device_u32(np.repeat(np.arange(B), 2 * (R + 1) * np.asarray(S)).astype(np.uint32), dev)
        self.circ_case = to_device_u32(np.repeat(np.arange(B), R * np.asarray(S)).astype(np.uint32), dev)
        self.bn = to_device_u32(np.concatenate([b + pt_off[k] for k, b in enumerate(bn_all)]).astype(np.uint32), dev)
        adj = np.concatenate(adj_all)
        self.adj = to_device_u32(np.where(adj == 0x7FFFFFFF, 0x7FFFFFFF, adj).astype(np.uint32), dev)
        self.col_slot = to_device_u32(np.concatenate(slot_all).astype(np.uint32), dev)

        # ring jobs: body blocks and implicit (first wake row) blocks, one job per case
        self._ring_job_args = {
            "body": (P, ring_off[:-1], mat_off[:-1], P),
            "implicit": (S, shed_off[:-1], imp_off[:-1], S),
            "implicit_fold": (S, shed_off[:-1], mat_off[:-1], P),  # folded straight into the matrices
        }
        # the implicit blocks can be folded by the ring kernel itself when no ring of a case is
        # adjacent to two shedding-line sides (no two threads then update one matrix entry)
        self.fold_in_ring = all(np.unique(a[a != 0x7FFFFFFF]).size == int((a != 0x7FFFFFFF).sum())
                                for a in adj_all)
        self.ring_tables: dict = {}
        self.ring_tiles = {}  # per ring-job kind: column-tile tables (ring_tile_tables), host and device
        for name, off_, sl_, n_ in (("body", self.body.surface_offsets, self.body.surface_lines, P),
                                    ("implicit", self.row0_offsets, self.row0_lines, S)):
            jt, toff, tl, sll, mx = ring_tile_tables(off_, sl_, n_)
            self.ring_tiles[name] = {"job_tile": jt, "tile_offsets": toff, "tile_lines": tl, "sl_local": sll,
                                     "max": mx}
            if not host_only:
                self.ring_tiles[name]["dev"] = {k: to_device_u32(v if v.size else np.zeros(1, np.uint32), dev)
                                                for k, v in (("job_tile", jt), ("tile_offsets", toff),
                                                             ("tile_lines", tl), ("sl_local", sll))}

        # sweep jobs: explicit wake term (points = control points, segments = the case's wake
        # lines) and advection (points = the case's distinct wake node columns, row by row)
        pidx = []
        for k in range(B):
            base = wpt_off[k]
            cols = cols_all[k].astype(np.int64)
            rows = np.arange(R, dtype=np.int64)[:, None]
            pidx.append((base + cols[None, :] * (R + 1) + rows).reshape(-1))  # row-major: (row, column)
        self.pidx = to_device_u32(np.concatenate(pidx).astype(np.uint32), dev)
        self._sweep_specs = {
            "wake": dict(seg_begin=wline_off[:-1], seg_count=WL, pt_begin=ring_off[:-1], pt_max=P,
                         pt_per_row=[0] * B, out_begin=ring_off[:-1], mode=0, seg_rows=(R + 1) * np.arange(B)),
            "advect": dict(seg_begin=line_off[:-1], seg_count=L, pt_begin=R * np.concatenate([[0], np.cumsum(NC)[:-1]]),
                           pt_max=np.asarray(NC) * R, pt_per_row=NC, out_begin=vel_off[:-1], mode=1,
                           seg_rows=[NO_ROWS] * B),
        }
        self.sweep_tables: dict = {}

        # ---------------- state
        NR, NL, NWL = self.n_rings, self.body.n_lines, self.wake_mesh.n_lines
        self.pos = torch.zeros((self.n_points, 3), **f64)
        self.vel = torch.zeros((self.n_points, 3), **f64)
        self.cps = torch.zeros((NR, 3), **f64)
        self.cpv = torch.zeros((NR, 3), **f64)
        self.nrm = torch.zeros((NR, 3), **f64)
        self.rhs = torch.zeros(NR, **f64)
        self.gamma = torch.zeros(NR, **f64)
        # the GMRES start: the circulation extrapolated from the last solutions by the polynomial
        # through up to four of them (equal steps within a case); row k of _EXTRAP holds the
        # weights of (gamma, g0, g1, g2, g3) with k solutions stored, picked on the device so
        # that the captured step graph ramps up by itself
        self.ghist = torch.zeros((4, NR), **f64)
        self.ghist_count = torch.zeros((), dtype=torch.int64, device=dev)
        self.extrap_w = torch.tensor(_EXTRAP, **f64)
        self.A = torch.zeros(int(mat_off[-1]), **f64)
        self.implicit = torch.zeros(int(imp_off[-1]), **f64)
        self.seg_body = torch.empty(int(_lib.query("pvl_segments_workspace", max(NL, 1), _lib.PVL_F64)),
                                    dtype=torch.uint8, device=dev)
        self.seg_wake = torch.empty(int(_lib.query("pvl_segments_workspace", max(NWL, 1), _lib.PVL_F64)),
                                    dtype=torch.uint8, device=dev)
        self.body_line_gamma = torch.zeros(max(NL, 1), **f64)
        self.wake_line_gamma = torch.zeros(max(NWL, 1), **f64)
        # fixed buffers (a step writes the new wake into the scratch copies and copies it back), so
        # that one captured graph serves every step
        self.wpos = torch.zeros((n_wake_pts, 3), **f64)
        self.wpos_new = torch.zeros((n_wake_pts, 3), **f64)
        self.wcirc = torch.zeros(R * int(shed_off[-1]), **f64)
        self.wcirc_new = torch.zeros(R * int(shed_off[-1]), **f64)
        self.node_vel = torch.zeros((int(vel_off[-1]), 3), **f64)
        self.rows = torch.zeros(1, dtype=torch.int32, device=dev)  # device step counter of the wake
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self.fail_flags = torch.zeros(B, dtype=torch.uint8, device=dev)
        self.fail_count = torch.zeros(1, dtype=torch.int32, device=dev)
        nb = int(_lib.query("pvl_batch_gmres_workspace", NR, B, self.max_iter))
        self.gws = torch.empty(nb, dtype=torch.uint8, device=dev)
        self.partials = None
        self._build_tables()
        self.iteration = 0
        self.graph = None
        self.h_gamma = torch.empty(NR, dtype=torch.float64, pin_memory=not host_only)

    # ------------------------------------------------------------------ tables for the current tiles
    def _build_tables(self) -> None:
        B, dev = self.B, self.dev
        cpb = int(self.tile["ring"])
        for name, (ncols, rbeg, obeg, ld) in self._ring_job_args.items():
            jobs = np.zeros(B, RING_JOB)
            jobs["cp_begin"], jobs["n_cp"] = self.ring_off[:-1], self.P
            jobs["ring_begin"], jobs["n_rings"] = rbeg, ncols
            jobs["out_begin"], jobs["ld"] = obeg, ld
            items = -(-np.asarray(self.P) // cpb) * (-(-np.asarray(ncols) // 128))
            jobs["item_begin"] = np.concatenate([[0], np.cumsum(items)[:-1]])
            self.ring_tables[name] = (_dev_records(jobs, dev), to_device_u32(jobs["item_begin"].astype(np.uint32), dev),
                                      int(items.sum()))
        threads, ppt = self.tile["sweep"]
        kpts = threads * ppt
        part_total = 0
        for name, sp in self._sweep_specs.items():
            jobs = np.zeros(B, SWEEP_JOB)
            for k in ("seg_begin", "seg_count", "pt_begin", "pt_max", "pt_per_row", "out_begin", "seg_rows"):
                jobs[k] = sp[k]
            jobs["mode"] = sp["mode"]
            jobs["case_id"] = np.arange(B)
            items = np.zeros(B, np.int64)
            for c in range(B):
                ns, per = _splits(int(jobs["seg_count"][c]), int(jobs["pt_max"][c]), kpts)
                jobs["n_split"][c], jobs["per"][c] = ns, per
                jobs["part_begin"][c] = part_total
                part_total += ns * int(jobs["pt_max"][c])
                items[c] = -(-int(jobs["pt_max"][c]) // kpts) * ns
            jobs["item_begin"] = np.concatenate([[0], np.cumsum(items)[:-1]])
            pt_item = np.concatenate([[0], np.cumsum(jobs["pt_max"].astype(np.int64))[:-1]]).astype(np.uint32)
            self.sweep_tables[name] = (_dev_records(jobs, dev), to_device_u32(jobs["item_begin"].astype(np.uint32), dev),
                                       int(items.sum()), to_device_u32(pt_item, dev),
                                       int(jobs["pt_max"].astype(np.int64).sum()))
        if self.partials is None or self.partials.numel() < 3 * part_total:
            self.partials = torch.zeros(3 * max(part_total, 1), dtype=torch.float64, device=dev)

    # ------------------------------------------------------------------ pieces of a step
    def _ring(self, which: str, segs, off, sl, n_lines: int, out) -> None:
        jobs, items, n_items = self.ring_tables[which]
        t = self.ring_tiles["implicit" if which == "implicit_fold" else which]
        td = t["dev"]
        _lib.call("pvl_batch_ring_matrix_tiled", int(self.tile["ring"]), ptr(jobs), ptr(items), self.B, n_items,
                  ptr(self.counter), ptr(off), ptr(sl), ptr(td["sl_local"]), ptr(td["job_tile"]),
                  ptr(td["tile_offsets"]), ptr(td["tile_lines"]), t["max"], n_lines, ptr(segs), ptr(self.cps),
                  ptr(self.nrm), self.tol, ptr(self.adj) if which == "implicit_fold" else None, ptr(out), 0,
                  stream_ptr())

    def _sweep(self, which: str, segs, pts, pidx, out) -> None:
        jobs, items, n_items, pt_item, n_total = self.sweep_tables[which]
        s = stream_ptr()
        threads, ppt = self.tile["sweep"]
        _lib.call("pvl_batch_sweep", threads, ppt, ptr(jobs), ptr(items), self.B, n_items, ptr(self.counter),
                  ptr(self.rows), ptr(self.d_seg_upto), self.R, ptr(segs), ptr(pts),
                  ptr(pidx) if pidx is not None else None, self.tol, ptr(self.partials), 0, s)
        _lib.call("pvl_batch_sweep_reduce", ptr(jobs), ptr(pt_item), self.B, n_total, ptr(self.rows),
                  ptr(self.partials), ptr(self.nrm), ptr(self.uinf), ptr(out), s)

    def _assemble(self, with_wake: bool) -> None:
        s = stream_ptr()
        d, NR = self.d_body, self.n_rings
        _lib.call("pvl_surface_average", NR, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.pos), ptr(self.cps), s)
        _lib.call("pvl_surface_average", NR, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.vel), ptr(self.cpv), s)
        _lib.call("pvl_surface_normal", NR, ptr(d["offsets"]), ptr(d["surface_lines"]), ptr(d["lines"]),
                  ptr(self.pos), ptr(self.nrm), s)
        _lib.call("pvl_rhs", NR, ptr(self.nrm), ptr(self.flow), 0.0, 0.0, 0.0, ptr(self.cpv), ptr(self.rhs), None, s)
        if self.static and self.A_body is not None:
            self.A.copy_(self.A_body)
        else:
            _lib.call("pvl_prep_segments", _lib.PVL_F64, self.n_points, self.body.n_lines, ptr(d["lines"]),
                      ptr(self.pos), None, self.tol, ptr(self.seg_body), s)
            self._ring("body", self.seg_body, d["offsets"], d["surface_lines"], self.body.n_lines, self.A)
            if self.static:
                self.A_body = self.A.clone()
        if not with_wake:
            return
        w, wpos = self.d_wake, self.wpos
        _lib.call("pvl_line_circulation", self.wake_mesh.n_lines, ptr(w["map_offsets"]), ptr(w["map_entries"]),
                  ptr(self.wcirc), self.R, ptr(self.wake_line_gamma), s)
        _lib.call("pvl_prep_segments", _lib.PVL_F64, self.n_wake_pts, self.wake_mesh.n_lines, ptr(w["lines"]),
                  ptr(wpos), ptr(self.wake_line_gamma), self.tol, ptr(self.seg_wake), s)
        if self.fold_in_ring:
            self._ring("implicit_fold", self.seg_wake, self.d_row0["offsets"], self.d_row0["lines"],
                       self.wake_mesh.n_lines, self.A)
        else:
            self._ring("implicit", self.seg_wake, self.d_row0["offsets"], self.d_row0["lines"],
                       self.wake_mesh.n_lines, self.implicit)
            _lib.call("pvl_batch_fold_implicit", ptr(self.wake_cases), ptr(self.row_case), self.n_rings,
                      ptr(self.implicit), ptr(self.adj), ptr(self.A), s)
        self._sweep("wake", self.seg_wake, self.cps, None, self.rhs)

    def _solve(self) -> None:
        _lib.call("pvl_batch_gmres", ptr(self.solve_cases), ptr(self.row_case), self.n_rings, self.B, ptr(self.A),
                  ptr(self.rhs), ptr(self.gamma), self.max_iter, self.solve_tol, ptr(self.fail_flags),
                  ptr(self.fail_count), ptr(self.gws), self.gws.numel(), stream_ptr())

    def _advect(self) -> None:
        s = stream_ptr()
        _lib.call("pvl_batch_wake_advect", ptr(self.wake_cases), ptr(self.node_case), self.n_wake_pts, self.R,
                  ptr(self.rows), ptr(self.wpos), ptr(self.node_vel), ptr(self.col_slot), ptr(self.pos),
                  ptr(self.bn), ptr(self.wpos_new), s)
        self.wpos.copy_(self.wpos_new)

    def _wake_update(self) -> None:
        s = stream_ptr()
        d = self.d_body
        _lib.call("pvl_line_circulation", self.body.n_lines, ptr(d["map_offsets"]), ptr(d["map_entries"]),
                  ptr(self.gamma), 0, ptr(self.body_line_gamma), s)
        _lib.call("pvl_prep_segments", _lib.PVL_F64, self.n_points, self.body.n_lines, ptr(d["lines"]), ptr(self.pos),
                  ptr(self.body_line_gamma), self.tol, ptr(self.seg_body), s)
        self._sweep("advect", self.seg_body, self.wpos, self.pidx, self.node_vel)
        self._advect()
        _lib.call("pvl_batch_wake_shed", ptr(self.wake_cases), ptr(self.circ_case), self.wcirc.numel(), self.R,
                  ptr(self.wcirc), ptr(self.adj), ptr(self.gamma), ptr(self.wcirc_new), s)
        self.wcirc.copy_(self.wcirc_new)
        _lib.call("pvl_batch_increment", ptr(self.rows), s)

    # ------------------------------------------------------------------ public stepping
    def load_positions(self, positions: list) -> None:
        """Body node positions of every case (list of (n_points_c, 3) arrays)."""
        self.pos.copy_(torch.as_tensor(np.concatenate([np.asarray(p, np.float64) for p in positions]),
                                       device=self.dev))

    def load_positions_host(self, flat: torch.Tensor) -> None:
        """All cases' node positions, concatenated ((n_points, 3) FP64, pinned host memory), copied
        in asynchronously on the current stream; the captured step reads them from there."""
        self.pos.copy_(flat.reshape(self.pos.shape), non_blocking=True)

    def gamma_host_async(self):
        """Start copying every case's circulations (concatenated in case order) to pinned host
        memory; the returned object's result() waits for that copy only."""
        from .engine import HostResult

        if not hasattr(self, "_h_ring"):
            self._h_ring = [torch.empty(self.gamma.shape, dtype=torch.float64, pin_memory=True) for _ in range(4)]
            self._h_next = 0
        buf = self._h_ring[self._h_next]
        self._h_next = (self._h_next + 1) % len(self._h_ring)
        buf.copy_(self.gamma, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        return HostResult(buf, ev)

    def start(self, time: float = 0.0) -> None:
        """Positions at ``time`` and the wake pinned to the trailing edges (first wake update)."""
        self.load_positions([c.positions_at(time) for c in self.cases])
        self.A_body = None
        self.vel.copy_(torch.as_tensor(np.concatenate([c.velocities_at(time) for c in self.cases]), device=self.dev))
        self.rows.zero_()
        self._advect()  # rows = 0: every row collapses onto the trailing edge
        self.rows.fill_(1)
        self.ghist_count.zero_()
        self.iteration = 0

    def _step_body(self, with_wake: bool) -> None:
        self._assemble(with_wake)
        self._seed()
        self._solve()
        self._record_solution()
        self._wake_update()

    def _seed(self) -> None:
        """gamma <- the start of this step's GMRES: the previous solutions extrapolated."""
        w = torch.index_select(self.extrap_w, 0, self.ghist_count.clamp(max=4).reshape(1))[0]
        self.gamma.mul_(w[0])
        for i in range(4):
            self.gamma.addcmul_(self.ghist[i], w[i + 1])

    def _record_solution(self) -> None:
        for i in (3, 2, 1):
            self.ghist[i].copy_(self.ghist[i - 1])
        self.ghist[0].copy_(self.gamma)
        self.ghist_count.add_(1).clamp_(max=4)

    def step(self) -> None:
        """One solver iteration of every case (static bodies: positions stay as loaded)."""
        if self.iteration == 0:
            self._step_body(with_wake=False)
        elif self.graph is not None:
            self.graph.replay()
        else:
            self._step_body(with_wake=True)
        self.iteration += 1

    def capture(self) -> None:
        """Capture one steady step (iteration >= 1) as a CUDA graph; later steps replay it.
        Capturing records the step without running it."""
        if self.iteration == 0:
            raise RuntimeError("capture after the first step")
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        n0 = _lib.lib().pvl_launch_count()
        with torch.cuda.graph(g):
            self._step_body(with_wake=True)
        self.graph = g
        self.graph_kernels = int(_lib.lib().pvl_launch_count() - n0)  # kernels each replay runs

    def failures(self) -> int:
        """Cases whose GMRES missed 10x its tolerance since the last call (host read)."""
        n = int(self.fail_count.item())
        self.fail_count.zero_()
        return n

    # ------------------------------------------------------------------ autotuner
    def tune(self, reps: int = 3) -> dict:
        """Time every tile shape of the two persistent kernels on this batch (with a full wake
        row count) and keep the fastest; returns the timings in ms."""
        saved_rows = self.rows.clone()
        self.rows.fill_(self.R)
        timings: dict = {"sweep": {}, "ring": {}}
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = dict(self.tile)
        for tile in SWEEP_TILES:
            self.tile["sweep"] = tile
            self._build_tables()
            t = 0.0
            for r in range(reps + 1):
                torch.cuda.synchronize()
                ev0.record()
                self._sweep("advect", self.seg_body, self.wpos, self.pidx, self.node_vel)
                self._sweep("wake", self.seg_wake, self.cps, None, self.rhs)
                ev1.record()
                torch.cuda.synchronize()
                if r:
                    t += ev0.elapsed_time(ev1) / reps
            timings["sweep"][f"{tile[0]}x{tile[1]}"] = t
        best["sweep"] = min(SWEEP_TILES, key=lambda tl: timings["sweep"][f"{tl[0]}x{tl[1]}"])
        self.tile["sweep"] = best["sweep"]
        d = self.d_body
        for cpb in RING_TILES:
            self.tile["ring"] = cpb
            self._build_tables()
            t = 0.0
            for r in range(reps + 1):
                torch.cuda.synchronize()
                ev0.record()
                self._ring("body", self.seg_body, d["offsets"], d["surface_lines"], self.body.n_lines, self.A)
                ev1.record()
                torch.cuda.synchronize()
                if r:
                    t += ev0.elapsed_time(ev1) / reps
            timings["ring"][str(cpb)] = t
        best["ring"] = min(RING_TILES, key=lambda c: timings["ring"][str(c)])
        self.tile = best
        self._build_tables()
        self.rows.copy_(saved_rows)
        self.graph = None  # tables changed: recapture
        return {"chosen": {"sweep": list(best["sweep"]), "ring": best["ring"]}, "ms": timings}

    # ------------------------------------------------------------------ results
    def gamma_of(self, k: int) -> np.ndarray:
        a, b = int(self.ring_off[k]), int(self.ring_off[k + 1])
        return self.gamma[a:b].cpu().numpy()

    def wake_positions_of(self, k: int) -> np.ndarray:
        S = int(self.S[k])
        a = 2 * (self.R + 1) * int(np.sum(self.S[:k]))
        return self.wpos[a:a + 2 * (self.R + 1) * S].cpu().numpy().reshape(S, 2, self.R + 1, 3)
