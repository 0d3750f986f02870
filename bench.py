#!/usr/bin/env python
"""UVLM time steps per second on one B200: flapping 128 x 32 wing, 2000 free-wake steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--path mixed|plain]

Workload: the flapping, deforming wing (4096 vortex rings, 8352 body segments, heave 0.2 c,
+-10 deg twist, bending ~ y^2, k = 0.2) flown from t = 0 for 2000 steps: the wake grows by a
row per step to 400 rows (51,200 wake rings) and is truncated from then on.  A step is one
iteration of the solver loop: body assembly, implicit + explicit wake corrections, the 4096^2
solve and the advection of the wake.

Both paths fly the whole run (plain FP64 first, then mixed + learned):
* plain: FP64 assembly, FP64 LU every step (FP64 tensor-core trailing updates).
* mixed (+ learned): FP64 assembly and wake terms, GMRES with FP64 residuals preconditioned by
  the inverse of an FP32 tensor-core LU rebuilt when it goes stale (engine.RefreshPolicy),
  seeded by the per-panel MLP, FP32 far-row advection.  The network is trained on the GPU,
  between the two runs, on plain steps 440..943 (full wake, one flapping cycle).

Timed (K steps each, from step 1000 + W on, after 1000 + W untimed steps of the same run):
* ``value``: steps/s with each step's body positions/velocities already in HBM.
* ``e2e``: the next K steps through the public stepping API with positions/velocities copied
  from pinned host memory and the circulations copied back every step (gamma_host_async:
  step k+1 is enqueued before step k's circulations are read, every copy inside the window).
  Each window ends with the current stream joined to the side stream on which preconditioner
  rebuilds run, so a rebuild started in a window is inside it (``refreshes_in_window``).
* ``trajectory``: every step's circulation of the mixed run against the plain run's, CL every
  10 steps, steps/s over the whole run for both; ``accuracy``: three steps after the windows
  judged against the all-FP64 step of the same state.
* ``warm_start``: the same mixed engine seeded by the previous circulation, by the Jacobi
  correction the network starts from, and by the network, over the same timed window.
* ``roofline``: the dominant kernel (the FP64 segment sweep of the explicit wake term) timed
  live with CUDA events over the step's three row bands, as the mixed step launches it; 45 FLOP
  per segment-point pair (the reference kernel's arithmetic) against the FP64 FMA throughput
  measured live by pvl_probe_fma on the same GPU.  One sweep of every row at every point is
  ``rooflines_secondary.wake_term_full_sweep``.
* ``cpu_baseline``: the reference's own compiled kernels + LAPACK on the host cores, one whole
  full-wake step (oracle/refbench.py); ``--impl reference`` times K whole steps the same way.
With --gpus N > 1 each rank flies an independent replica (the headline case does not shard)
at its own phase of the cycle; value is the sum over ranks, timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "UVLM steps/s, mixed+learned vs plain FP64 on B200, at Γ rel err ≤1e-10"
WORKLOAD = ("flapping 128x32 wing, 4096 rings, 2000 free-wake steps from t = 0, wake truncated at 400 rows "
            "(51,200 wake rings)")
PAIR_FLOPS = 45  # arithmetic of one segment-point pair in the reference kernel (flow_solver.c:113-135)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["mixed", "plain"], default="mixed")
    ap.add_argument("--trajectory-steps", type=int, default=2000,
                    help="length of the run from t = 0 (config: 2000 free-wake steps) that both paths fly")
    ap.add_argument("--workload", choices=["flapping", "batch", "swept", "sphere"], default="flapping",
                    help="flapping: the deforming wing (headline); batch: 256 ragged wings x 50 steps; "
                         "swept: pitching swept wing, 200 steps; sphere: closed 5120-ring sphere")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-cases summary (bench.py --workload batch, run after the headline)")
    ap.add_argument("--profile-kernel", choices=["line_sum", "advect_f32", "wake_term", "wake_bands", "body", "gemv",
                                                 "lu", "lu32",
                                                 "mixed_step", "plain_step", "batch_step", "mlp", "gemm4096"],
                    default=None,
                    help="set up the workload, launch only that kernel family twice and exit (for ncu captures)")
    ap.add_argument("--fraction", type=int, default=16,
                    help="reference arm: warm-up steps sample 1/F of the wake points; whole steps run the "
                         "wake phases in F interleaved calls")
    return ap.parse_args()


def workload():
    from pyvl_b200 import workloads

    return workloads.flapping()


T_START_STEPS = 100  # the reference arm and the kernel timings use a seeded full wake at t = 100 dt
T_TIMED = 1000       # our arm times steps from 1000 + W on of the run from t = 0 (wake full from step 400)
TRAIN_STEPS = (440, 944)  # plain FP64 steps (full wake, one flapping cycle) whose inputs and circulations train the warm start
TRAIN_ITERS = 3000  # Adam iterations on 16 k-sample batches (2 M samples)
REF_TIMED_BUDGET_S = 150.0  # the reference arm's timed whole CPU steps stop once they would exceed this


def wake_setup(case, mesh=None):
    """Our arm: topology, wake spec and the seeded full-wake state (product code)."""
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import synthetic_full_wake, wake_spec_from_te

    mesh = Mesh(case.n_points, case.elements) if mesh is None else mesh
    t_start = T_START_STEPS * case.dt
    spec = wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, t_start - case.dt)
    pos, circ = synthetic_full_wake(case.positions_at(t_start - case.dt), spec, case.freestream, case.dt, seed=7)
    return mesh, spec, pos, circ, t_start


def wake_setup_reference(case):
    """Reference arm (no torch, no CUDA): the same spec and state from the oracle topology."""
    from oracle.kernels import OracleMesh
    from oracle.solver import shedding_setup
    from pyvl_b200.workloads import synthetic_full_wake

    shed, nodes, adj = shedding_setup(OracleMesh(case.n_points, case.elements), case.te_node_pairs)
    t_start = T_START_STEPS * case.dt
    te = case.positions_at(t_start - case.dt)[nodes.astype(np.int64)]
    pos, circ = synthetic_full_wake(te, case.line_rows, case.freestream, case.dt, seed=7)
    return nodes, adj, pos, circ, t_start


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference arm
def run_reference(args) -> None:
    """The reference's CPU path (compiled reference kernels + LAPACK) on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.refbench import ReferenceStep

    case = workload()
    nodes, adj, wpos, wcirc, t0 = wake_setup_reference(case)
    rs = ReferenceStep(case, wpos, wcirc, nodes, adj, fraction=args.fraction)
    # warm-up: sampled steps (the wake phases on 1/F of their points, scaled by F); timed: whole
    # steps on every control point and wake node -- K of them, or as many as fit in
    # REF_TIMED_BUDGET_S (at least one), so that the arm ends within a few minutes; `steps`
    # reports how many were timed
    est = [rs.step(t0 + k * case.dt)["step_estimate"] for k in range(args.warmup)]
    phases, spent = [], 0.0
    for k in range(args.steps):
        phases.append(rs.step(t0 + (args.warmup + k) * case.dt, whole=True))
        spent += phases[-1]["step_estimate"]
        if spent + phases[-1]["step_estimate"] > REF_TIMED_BUDGET_S:
            break
    times = [p["step_estimate"] for p in phases]
    sps = 1.0 / float(np.mean(times))
    sample = (f"each timed step: one whole full-wake step at 4096 rings and 400 wake rows (body geometry, body matrix, "
              f"wake corrections on every control point, LU solve, advection of every wake node; the wake phases in "
              f"{rs.F} interleaved calls to bound the reference's line buffers); wake mesh built once in "
              f"{rs.wake_mesh_seconds:.1f} s")
    detail = {"phases_s": {k: float(np.mean([p[k] for p in phases])) for k in ("body", "corrections", "solve",
                                                                                "advection")},
              "sampled_estimate_s_per_step": float(np.mean(est)) if est else None,
              # run_solver as shipped also rebuilds the wake mesh at every snapshot
              # (python/pyvl/solver.py:251: type(wm).load(wm.save()))
              "as_shipped_s_per_step": float(np.mean(times)) + rs.wake_mesh_seconds,
              "how": "warm-up steps sampled (1/F of the wake points, scaled by F: sampled_estimate); timed steps whole; "
                     "as shipped adds the per-snapshot wake-mesh rebuild of run_solver"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": len(phases), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rings": 4096, "wake_rows": 400,
                   "timed_steps": "full-wake steps (400 wake rows), as every step after step 400 of the run",
                   "parallelism": "host cores (OpenMP + LAPACK threads)"},
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": rs.threads, "kind": "reference", "sample": sample},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_step": detail,
    }), flush=True)


def batch_summary() -> dict:
    """Run the batched workload (256 ragged wings x 50 steps, bench.py --workload batch) in a
    subprocess after the headline measurement and quote its main figures."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--workload", "batch"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200, env=env)
        d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        keys = ("metric", "value", "unit", "ms_per_step", "config", "e2e", "roofline", "cpu_baseline",
                "per_case_loop", "speedup_vs_per_case_loop", "accuracy", "gmres_failures", "cuda_graph", "clocks")
        return {k: d.get(k) for k in keys}
    except Exception as e:  # reported, never fatal for the headline
        return {"failed": f"{type(e).__name__}: {e}"}


def cpu_baseline() -> dict | None:
    """Run the reference arm in a torch-free subprocess (one whole step after one sampled
    warm-up step) and quote it."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        return json.loads(line)["cpu_baseline"]
    except Exception as e:  # reported, never fatal for the GPU measurement
        return {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {type(e).__name__}: {e}"}


# ------------------------------------------------------------------ our arm
def wake_band_calls(eng, tol: float):
    """The argument tuples of the mixed step's three FP64 sweeps of the explicit wake term on the
    engine's current wake (every row shed), as MixedSolverEngine._far_wake_term issues them, and
    their pair count; the stencil's points are gathered first."""
    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    w, f = eng.wake, eng._far
    rm, d = w["rm"], w["rm_d"]
    up, n = w["lines_upto"], rm.n_lines
    a = up[f["chord_row"]]
    b = n if f["span_row"] is None else up[f["span_row"]]
    n_c, n_s = f["n_chord_eval"], f["n_span_eval"]
    wpos, lg, lines = eng.wake_positions.reshape(-1, 3), w["rm_line_gamma"], d["lines"]
    s = stream_ptr()
    _lib.call("pvl_gather_points", n_c, ptr(f["index"]), eng.P, ptr(eng.cps), ptr(f["pts"]), s)
    ws = (ptr(eng.ws), eng._ws_bytes, s)
    calls = [
        (_lib.PVL_F64, rm.n_points, a, ptr(lines), ptr(wpos), ptr(lg), eng.P, ptr(eng.cps), ptr(eng.nrm), tol, 1.0,
         1.0, ptr(eng.rhs)) + ws,
        (_lib.PVL_F64, rm.n_points, b - a, lines.data_ptr() + 8 * a, ptr(wpos), lg.data_ptr() + 8 * a, n_c,
         ptr(f["pts"]), None, tol, 1.0, 0.0, ptr(f["vals"])) + ws,
        (_lib.PVL_F64, rm.n_points, n - b, lines.data_ptr() + 8 * b, ptr(wpos), lg.data_ptr() + 8 * b, n_s,
         ptr(f["pts"]), None, tol, 1.0, 0.0, f["vals"].data_ptr() + 24 * n_c) + ws,
    ]
    return calls, a * eng.P + (b - a) * n_c + (n - b) * n_s


def profile_kernel(args) -> None:
    """Two launches of one kernel family on the benchmark state, nothing else (ncu target);
    mixed_step / batch_step: a few whole steps (launch lists)."""
    import torch

    if args.profile_kernel == "gemm4096":  # the TF32 tensor-core GEMM on a compute-bound 4096^3 product
        from pyvl_b200 import _lib
        from pyvl_b200.device import ptr, stream_ptr

        n = 4096
        g = torch.Generator(device="cuda").manual_seed(0)
        A = torch.randn(n, n, device="cuda", generator=g)
        Bt = torch.randn(n, n, device="cuda", generator=g)
        C = torch.zeros(n, n, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        ms = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.call("pvl_gemm_tf32", n, n, n, 1.0, ptr(A), n, ptr(Bt), n, 0.0, ptr(C), n, ptr(err), stream_ptr())
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        want = A.double() @ Bt.double().t()
        rel = float((torch.linalg.norm(C.double() - want) / torch.linalg.norm(want)).item())
        print(f"profile-kernel done gemm4096 ms={min(ms[1:]):.4f} tflops={2 * n ** 3 / (min(ms[1:]) * 1e-3) / 1e12:.1f} "
              f"rel_err={rel:.2e} err={int(err.item())}")
        return
    if args.profile_kernel == "batch_step":
        from pyvl_b200.batch import BatchEngine
        from pyvl_b200.workloads import batch_wings

        beng = BatchEngine(batch_wings(n_cases=256, seed=3, steps=50), solve_tol=1e-12, max_iter=8)
        beng.start(0.0)
        for _ in range(4):
            beng.step()
        torch.cuda.synchronize()
        print("profile-kernel done batch_step failures", beng.failures())
        return

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.engine import MixedSolverEngine

    case = workload()
    mesh, spec, wpos, wcirc, t0 = wake_setup(case)
    eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec, cp_patches=case.smooth_patches,
                            wake_col_runs=case.wake_col_runs)
    eng.set_wake_state(wpos, wcirc, step_count=case.line_rows + 1, time=t0 - case.dt)
    eng.load_inputs(case.positions_at(t0), case.velocities_at(t0))
    eng.iteration = 1
    eng.assemble_body_only()
    w = eng.wake
    if args.profile_kernel in ("line_sum", "advect_f32"):  # advection sweep of the distinct wake node columns
        S, R, L = spec.shedding_lines.size, case.line_rows, mesh.n_lines
        d = eng.d_body
        prec, r0 = (_lib.PVL_F64, 0) if args.profile_kernel == "line_sum" else (_lib.PVL_F32, 8)
        eng.body_line_gamma.fill_(1e-2)
        for _ in range(2):
            _lib.call("pvl_wake_node_velocity_cols", prec, mesh.n_points, L, ptr(d["lines"]), ptr(eng.pos),
                      ptr(eng.body_line_gamma), S, R, R, r0, R, w["n_cols"], ptr(w["cols"]), ptr(eng.wake_positions),
                      1.0, 0.0, 0.0, case.tol, ptr(w["node_vel"]), ptr(eng.ws), eng._ws_bytes, stream_ptr())
    elif args.profile_kernel == "wake_term":  # FP64 sweep of the explicit wake term
        rm, d = w["rm"], w["rm_d"]
        lg = w["rm_line_gamma"]
        lg.fill_(1e-3)
        for _ in range(2):
            _lib.call("pvl_line_velocity", _lib.PVL_F64, rm.n_points, rm.n_lines, ptr(d["lines"]),
                      ptr(eng.wake_positions.reshape(-1, 3)), ptr(lg), eng.P, ptr(eng.cps), ptr(eng.nrm), case.tol,
                      1.0, 0.0, ptr(eng.rhs), ptr(eng.ws), eng._ws_bytes, stream_ptr())
    elif args.profile_kernel == "wake_bands":  # the mixed step's three FP64 wake-term sweeps, twice
        w["rm_line_gamma"].fill_(1e-3)
        calls, _ = wake_band_calls(eng, case.tol)
        for _ in range(2):
            for c in calls:
                _lib.call("pvl_line_velocity", *c)
    elif args.profile_kernel == "body":  # the body matrix (tiled ring kernel)
        for _ in range(2):
            eng.assemble_body_only()
    elif args.profile_kernel == "gemv":  # the solve's matrix-vector products on the benchmark system
        eng.assemble()
        n = eng.N
        x = torch.randn(n, dtype=torch.float64, device="cuda")
        x32 = x.float()
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        M32 = eng.A.float()
        for _ in range(2):
            _lib.call("pvl_gemv_f64", n, n, 1.0, ptr(eng.A), n, ptr(x), 0.0, ptr(y), stream_ptr())
            _lib.call("pvl_gemv_f32", n, n, 1.0, ptr(M32), n, ptr(x32), 0.0, ptr(y), stream_ptr())
    elif args.profile_kernel == "lu":
        eng.assemble()
        A0 = eng.A.clone()
        for _ in range(2):
            eng.A.copy_(A0)
            _lib.call("pvl_lu_factor", eng.N, ptr(eng.A), eng.N, ptr(eng.ipiv), ptr(eng.info), ptr(eng.ws),
                      eng._ws_bytes, stream_ptr())
    elif args.profile_kernel == "mixed_step":  # 3 + 2 whole mixed steps (no warm start)
        for k in range(5):
            t = t0 + k * case.dt
            eng.step(t, case.positions_at(t), case.velocities_at(t))
    elif args.profile_kernel == "plain_step":  # 3 + 2 whole plain FP64 steps
        from pyvl_b200.engine import SolverEngine

        plain = SolverEngine(mesh, case.freestream, case.tol, spec)
        plain.set_wake_state(wpos, wcirc, step_count=case.line_rows + 1, time=t0 - case.dt)
        plain.iteration = 1
        for k in range(5):
            t = t0 + k * case.dt
            plain.step(t, case.positions_at(t), case.velocities_at(t))
        plain.check_status()
    elif args.profile_kernel == "mlp":  # warm-start network: two inference launches, two gradient launches
        from pyvl_b200.learned import WarmStartMLP

        mlp = WarmStartMLP(torch.device("cuda"), seed=0)
        g = torch.Generator(device="cuda").manual_seed(0)
        X = torch.randn(16384, 12, device="cuda", generator=g)
        T = torch.randn(16384, device="cuda", generator=g)
        base = torch.zeros(eng.P, dtype=torch.float64, device="cuda")
        out = torch.zeros_like(base)
        for _ in range(2):
            mlp.predict(X[: eng.P], base, out)
            mlp.gradient(X, T)
    else:  # the mixed path's preconditioner refresh (FP32 LU + inverse on the tensor cores)
        eng.assemble()
        for _ in range(2):
            eng.refresh_preconditioner()
    torch.cuda.synchronize()
    eng.check_status()
    print("profile-kernel done", args.profile_kernel)


def reduce_max_over_ranks(x: float, dist, device: str) -> float:
    """The largest of the ranks' values (every rank gets it); x itself without a process group.
    Each rank's timed region is measured on its own device, and the job's time is the slowest
    rank's."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps: int, ms_max: float, world: int) -> float:
    """Whole-job steps/s of ``world`` independent replicas that each ran ``steps`` steps, the
    slowest in ``ms_max`` milliseconds (weak scaling: the work grows with the ranks)."""
    return world * steps / (ms_max * 1e-3)


class LiftEvaluator:
    """CL of a state: circulatory_forces (python/pyvl/postprocess/forces.py:10-42) -- line
    forces with the freestream, the body's and the wake's induced velocity at the nodes minus
    the motion, then the wake's trailing-edge correction (wake_models.py:293-330) -- and the
    lift coefficient, all through the package's public API on the GPU.  One wake model object
    and one dual mesh serve every call."""

    def __init__(self, case, mesh, spec):
        from types import SimpleNamespace

        from pyvl_b200.wake_models import WakeModelLineExplicitUnsteady

        self.case, self.mesh = case, mesh
        self.dual = mesh.compute_dual()
        self.wm = WakeModelLineExplicitUnsteady(spec.bordering_nodes, spec.shedding_lines, spec.adjacent_surfaces,
                                                case.tol, 0.0, spec.line_rows)
        u = np.asarray(case.freestream, np.float64)
        self.u = u
        self.flow = SimpleNamespace(get_velocity=lambda t, p: np.tile(u, (np.asarray(p).reshape(-1, 3).shape[0], 1)))
        self.geo = SimpleNamespace(mesh=mesh)

    def __call__(self, eng, pos, vel, gamma) -> float:
        """CL of ring circulations ``gamma`` at the engine's wake state before its wake update."""
        from pyvl_b200.cvl import Mesh
        from pyvl_b200.postprocess import lift_coefficient

        wm, mesh = self.wm, self.mesh
        wm.wake_positions[...] = eng.wake_positions.cpu().numpy()
        wm.circulation[...] = eng.wake_circulation.cpu().numpy()
        wm.current_time = eng.wake["time"]
        pos = np.ascontiguousarray(pos, np.float64)
        gamma = np.asarray(gamma, np.float64)
        induced = mesh.induced_velocity(self.case.tol, pos, pos, gamma) + wm.get_velocity(pos)
        forces = Mesh.line_forces(mesh, self.dual, gamma / (2 * np.pi), pos,
                                  self.flow.get_velocity(0.0, pos) + induced - np.asarray(vel, np.float64))
        wm.correct_forces(forces, self.geo, pos, gamma, self.flow)
        return lift_coefficient(forces, self.u, self.case.s_ref)


def train_warm_start(X, T, seed: int = 0):
    """The learned warm start, trained on the GPU on recorded plain FP64 steps."""
    import torch

    from pyvl_b200.learned import WarmStartMLP

    mlp = WarmStartMLP(torch.device("cuda"), seed=seed)
    Xn, Tn = mlp.fit_statistics(X, T)
    losses = mlp.train(Xn, Tn, iters=TRAIN_ITERS, batch=16384, lr=2e-3, seed=seed)
    return mlp, {"samples": int(X.shape[0]), "loss_first": losses[0], "loss_last": losses[-1]}


def run_precision_case(args) -> None:
    """Plain FP64 vs the mixed path on the pitching swept wing (1024 rings, 200 steps, wake
    growing to 200 rows) or the closed sphere (5120 rings, bordered): time per step, the error
    of every mixed step against the all-FP64 step of the same state, the divergence of whole
    trajectories, and on the sphere the surface velocity."""
    import torch

    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine, wake_spec_from_te
    from pyvl_b200 import workloads

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    case = workloads.swept_pitching() if args.workload == "swept" else workloads.icosphere()
    mesh = Mesh(case.n_points, case.elements)
    groups = [(0, case.n_surfaces)] if case.closed else None

    def spec():
        if case.line_rows <= 0 or not len(case.te_node_pairs):
            return None
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    steps = case.nt if case.nt > 1 else max(args.steps, 5)
    times = [k * case.dt for k in range(steps)]
    runs = {}
    for kind in ("plain", "mixed"):
        eng = (SolverEngine(mesh, case.freestream, case.tol, spec(), groups) if kind == "plain" else
               MixedSolverEngine(mesh, case.freestream, case.tol, spec(), groups,
                                 gmres_tol=1e-13 if case.closed else 1e-12))
        hist, ms = [], 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for k, t in enumerate(times):
            p, v = case.positions_at(t), case.velocities_at(t)
            torch.cuda.synchronize()
            e0.record()
            eng.step(t, p, v)
            e1.record()
            torch.cuda.synchronize()
            if k >= 2:
                ms += e0.elapsed_time(e1)
            hist.append(eng.gamma_host())
        rec = {"ms_per_step": ms / max(1, steps - 2), "gamma": np.array(hist), "eng": eng}
        runs[kind] = rec
    mixed = runs["mixed"]["eng"]
    # per-step error of the mixed path: a fresh mixed engine judged at every step of the same run
    judge_eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec(), groups,
                                  gmres_tol=1e-13 if case.closed else 1e-12)
    judged = [judge_eng.step_judged(t, case.positions_at(t), case.velocities_at(t)) for t in times]
    gp, gm = runs["plain"]["gamma"], runs["mixed"]["gamma"]
    traj = [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(gm, gp)]
    extra = {}
    if case.closed:  # surface velocity at the control points: freestream + induced, both paths
        t = times[-1]
        pos = case.positions_at(t)
        cps = mesh.surface_average_vec3(pos)
        vel = {}
        for kind in ("plain", "mixed"):
            g = runs[kind]["gamma"][-1]
            vel[kind] = np.asarray(mesh.induced_velocity(case.tol, pos, cps, g)) + case.freestream
        extra["surface_velocity_rel_err"] = float(np.linalg.norm(vel["mixed"] - vel["plain"])
                                                  / np.linalg.norm(vel["plain"]))
    st = mixed.stats
    print(json.dumps({
        "metric": "UVLM steps/s, mixed vs plain FP64", "workload": args.workload,
        "value": 1000.0 / runs["mixed"]["ms_per_step"], "unit": "steps/s", "n_gpus": 1, "steps": steps,
        "higher_is_better": True, "dtype": "f64 residuals / f32+tf32 preconditioner", "data": "synthetic",
        "config": {"workload": case.name, "rings": case.n_surfaces, "wake_rows": case.line_rows,
                   "closed": bool(case.closed)},
        "plain_fp64": {"steps_per_s": 1000.0 / runs["plain"]["ms_per_step"], "ms_per_step": runs["plain"]["ms_per_step"]},
        "mixed": {"steps_per_s": 1000.0 / runs["mixed"]["ms_per_step"], "ms_per_step": runs["mixed"]["ms_per_step"],
                  "gmres_iters_mean": float(np.mean(st["gmres_iters"])), "fallbacks": st["fallbacks"],
                  "refreshes": st["refreshes"]},
        "speedup_mixed_over_plain": runs["plain"]["ms_per_step"] / runs["mixed"]["ms_per_step"],
        "accuracy": {"gamma_rel_err_per_step_max": max(judged), "trajectory_gamma_rel_diff_max": max(traj),
                     "tolerance": 1e-10, **extra,
                     "how": "every step judged against the all-FP64 step of the same state; trajectories of "
                            "the two engines compared step by step"},
    }), flush=True)


def batch_cpu_baseline(steps: int) -> dict:
    """The reference's kernels (oracle/_ref) + LAPACK on the host cores, per case, on every 32nd
    case of the batch for all its steps (a torch-free subprocess: the reference's extension is
    never loaded next to torch)."""
    code = ("import json, sys; sys.path.insert(0, %r)\n"
            "from oracle.refbench import reference_case_steps, _threads\n"
            "from pyvl_b200.workloads import batch_wings\n"
            "s, n = reference_case_steps(batch_wings(n_cases=256, seed=3, steps=%d)[::32], %d)\n"
            "print(json.dumps({'seconds': s, 'case_steps': n, 'cores': _threads()}))\n") % (str(ROOT), steps, steps)
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900, env=env)
        d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        return {"value": d["case_steps"] / d["seconds"], "unit": "case-steps/s", "cores": d["cores"],
                "kind": "reference", "sample": f"every 32nd case ({d['case_steps'] // steps} cases), all {steps} "
                                               "steps each, the reference's kernels + LAPACK, one case at a time"}
    except Exception as e:  # reported, never fatal for the GPU measurement
        return {"value": None, "unit": "case-steps/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {type(e).__name__}: {e}"}


def run_batch(args) -> None:
    """256 independent wings (ragged 128..2048 rings) x 50 free-wake steps: the batched engine
    (persistent launches, autotuned tiles, CUDA graph) against a per-case loop of the plain
    single-case engine on a sample of the same cases."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.batch import BatchEngine
    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import SolverEngine, wake_spec_from_te
    from pyvl_b200.workloads import batch_wings

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    steps = 50
    first = 2
    timed = steps - first
    cases = batch_wings(n_cases=256, seed=3, steps=steps)

    def run(reuse: bool):
        eng = BatchEngine(cases, solve_tol=1e-12, max_iter=8, reuse_static_bodies=reuse)
        eng.start(0.0)
        eng.step()
        eng.step()
        tuning = eng.tune(reps=2)
        eng.capture()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(first, steps):
            eng.step()
        e1.record()
        torch.cuda.synchronize()
        return eng, tuning, e0.elapsed_time(e1)

    def run_e2e():
        """The same steps through the public API with host data: every step copies all cases'
        node positions in from pinned memory and every case's circulations out (step k + 1 is
        enqueued before step k's are read)."""
        eng = BatchEngine(cases, solve_tol=1e-12, max_iter=8, tile=tuning["chosen_tiles"])
        eng.start(0.0)
        eng.step()
        eng.step()
        eng.capture()
        h_pos = torch.as_tensor(np.concatenate([c.positions_at(0.0) for c in cases]), dtype=torch.float64).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        pending = None
        for _ in range(first, steps):
            eng.load_positions_host(h_pos)
            eng.step()
            res = eng.gamma_host_async()
            if pending is not None:
                pending.result()
            pending = res
        pending.result()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), int(h_pos.numel() * 8), int(eng.gamma.numel() * 8)

    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    eng, tuning, ms = run(False)
    tuning["chosen_tiles"] = {"sweep": tuple(tuning["chosen"]["sweep"]), "ring": tuning["chosen"]["ring"]}
    ms_e2e, h2d, d2h = run_e2e()
    clocks = sampler.stop()
    fails = eng.failures()
    case_steps = len(cases) * timed
    # dominant kernels: the two persistent sweeps at full wake rows, against the FP64 FMA peak
    from pyvl_b200 import _probe
    from pyvl_b200.device import ptr, stream_ptr

    sweep_ms = tuning["ms"]["sweep"]["%dx%d" % tuning["chosen_tiles"]["sweep"]]
    sweep_pairs = eng.sweep_pairs_full["wake"] + eng.sweep_pairs_full["advect"]
    sink = torch.zeros(148 * 8, dtype=torch.float64, device="cuda")
    _probe.lib().pvl_probe_fma(_lib.PVL_F64, 148 * 8, 2000, ptr(sink), stream_ptr())
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    p0.record()
    flops = _probe.lib().pvl_probe_fma(_lib.PVL_F64, 148 * 8, 20000, ptr(sink), stream_ptr())
    p1.record()
    torch.cuda.synchronize()
    peak = flops / (p0.elapsed_time(p1) * 1e-3) / 1e12
    achieved = sweep_pairs * PAIR_FLOPS / (sweep_ms * 1e-3) / 1e12
    tuning.pop("chosen_tiles")
    eng_static, _, ms_static = run(True)
    fails += eng_static.failures()
    del eng_static
    # the reference's per-case loop (its compiled kernels + LAPACK on the host cores) on every
    # 32nd case, all 50 steps, in a torch-free subprocess
    base = batch_cpu_baseline(steps)
    # per-case loop of the plain single-case engine on every 8th case, same step range
    sample = cases[::8]
    t_loop = 0.0
    for c in sample:
        m = Mesh(c.n_points, c.elements)
        e = SolverEngine(m, c.freestream, c.tol, wake_spec_from_te(m, c.te_node_pairs, c.line_rows, c.t0))
        pos, vel = c.positions_at(0.0), c.velocities_at(0.0)
        for it in range(first):
            e.step(it * c.dt, pos, vel)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for it in range(first, steps):
            e.step(it * c.dt, pos, vel)
        torch.cuda.synchronize()
        t_loop += time.perf_counter() - t0
    loop_rate = len(sample) * timed / t_loop
    # accuracy: every 16th case of the batch against the per-case FP64 engine after all steps
    errs = []
    for k in range(0, len(cases), 16):
        c = cases[k]
        m = Mesh(c.n_points, c.elements)
        e = SolverEngine(m, c.freestream, c.tol, wake_spec_from_te(m, c.te_node_pairs, c.line_rows, c.t0))
        pos, vel = c.positions_at(0.0), c.velocities_at(0.0)
        for it in range(steps):
            e.step(it * c.dt, pos, vel)
        ref = e.gamma_host()
        errs.append(float(np.linalg.norm(eng.gamma_of(k) - ref) / np.linalg.norm(ref)))
    rate = case_steps / (ms * 1e-3)
    print(json.dumps({
        "metric": "batched UVLM case-steps/s", "value": rate, "unit": "case-steps/s", "n_gpus": 1,
        "steps": timed, "warmup": first, "ms_per_step": ms / timed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "256 independent swept/tapered wings, rings log-uniform in [128, 2048], 50 free-wake "
                               "steps each (wake up to 50 rows)",
                   "rings_total": int(eng.n_rings), "timed_steps": f"{first}..{steps - 1} of every case",
                   "solve": "device GMRES, Jacobi preconditioner, FP64 residual <= 1e-12"},
        "per_case_loop": {"value": loop_rate, "unit": "case-steps/s", "engine": "SolverEngine (FP64 LU) per case",
                          "sample": f"every 8th case ({len(sample)} cases), same steps"},
        "speedup_vs_per_case_loop": rate / loop_rate,
        "static_body_reuse": {"value": case_steps / (ms_static * 1e-3), "unit": "case-steps/s",
                              "note": "the same batch with each motionless body's matrix built once and copied per "
                                      "step (reuse_static_bodies=True); the per-case loop has no such reuse"},
        "accuracy": {"gamma_rel_err_vs_per_case_fp64_max": max(errs), "cases_checked": len(errs)},
        "e2e": {"value": case_steps / (ms_e2e * 1e-3), "unit": "case-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "fp64", "kernel": "batched_sweep_kernel (explicit wake term + advection, full wake rows)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "ms_per_launch_pair": sweep_ms, "pairs": sweep_pairs,
                     "peak_source": "FP64 FMA throughput measured live (pvl_probe_fma); 45 FLOP per pair"},
        "cpu_baseline": base,
        "gmres_failures": fails,
        "autotune": tuning,
        "gpu_launches": int(eng.graph_kernels * timed),
        "cuda_graph": {"kernels_per_step": eng.graph_kernels, "replays": timed},
        "clocks": clocks,
    }), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_kernel:
        return profile_kernel(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload in ("swept", "sphere"):
        return run_precision_case(args)
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr
    from pyvl_b200.engine import MixedSolverEngine, SolverEngine
    from pyvl_b200.learned import WarmStart, drive_step

    from pyvl_b200.cvl import Mesh
    from pyvl_b200.engine import wake_spec_from_te

    case = workload()
    if rank:
        case.meta["replica"] = rank
    mesh = Mesh(case.n_points, case.elements)
    W, K = args.warmup, args.steps
    t_first = T_TIMED + W                   # first timed step (the wake is full from step 400 on)
    t_e2e = t_first + K                     # first step of the end-to-end window
    t_judge = t_e2e + K                     # three judged steps follow
    n_steps = max(args.trajectory_steps, t_judge + 3)
    phase = 0.37 * rank                     # replicas fly at different phases of the cycle
    times = [(k + phase) * case.dt for k in range(n_steps)]
    # inputs of the timed steps prepared beforehand: resident on the device for the first window,
    # in host memory for the end-to-end window; every other step computes its own
    win = range(t_first, t_judge + 3)
    hpos = {k: case.positions_at(times[k]) for k in win}
    hvel = {k: case.velocities_at(times[k]) for k in win}
    dpos = torch.tensor(np.stack([hpos[k] for k in win]), device="cuda")
    dvel = torch.tensor(np.stack([hvel[k] for k in win]), device="cuda")

    def inputs(k):
        if k in hpos:
            return hpos[k], hvel[k]
        return case.positions_at(times[k]), case.velocities_at(times[k])
    lift = LiftEvaluator(case, mesh, wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0))
    cl_every = 10

    def spec():
        return wake_spec_from_te(mesh, case.te_node_pairs, case.line_rows, case.t0)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_max_over_ranks(x, dist, "cuda")

    def run_arm(kind: str, mlp=None, record=None, seed_mode="learned", last: int | None = None) -> dict:
        """One engine over the run from t = 0: untimed steps up to t_first, the device-resident
        timed window (K steps), the end-to-end window (K steps, host inputs and outputs), three
        judged steps (mixed only), then on to the end of the trajectory.  Every step's
        circulations are kept on the device (a 32 KB copy per step, inside the timed windows
        too) and CL is evaluated every ``cl_every`` steps outside them."""
        if kind == "plain":
            eng, warm = SolverEngine(mesh, case.freestream, case.tol, spec()), None
            if record is not None:
                warm = WarmStart(eng, None, record=True)
        else:
            eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec(), cp_patches=case.smooth_patches,
                                    wake_col_runs=case.wake_col_runs)
            warm = {"learned": lambda: WarmStart(eng, mlp), "jacobi": lambda: WarmStart(eng, jacobi=True),
                    "previous": lambda: None}[seed_mode]()
        end = n_steps if last is None else last
        G = torch.zeros((end, eng.P), dtype=torch.float64, device="cuda")
        cls, rec = {}, {}
        ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        run0, run1 = ev(), ev()
        run_ms, pending = 0.0, None
        torch.cuda.synchronize()
        run0.record()
        for k in range(end):
            if k == t_first or k == t_e2e:  # open a timed window
                if hasattr(eng, "wait_refresh"):  # a rebuild started before the window ends before it
                    eng.wait_refresh()
                run1.record()
                barrier()
                run_ms += run0.elapsed_time(run1)
                if k == t_first:
                    eng.check_status()
                    launches0 = _lib.lib().pvl_launch_count() + eng.replayed_kernels
                    n_solves0 = len(getattr(eng, "stats", {}).get("gmres_iters", []))
                    refresh0 = getattr(eng, "stats", {}).get("refreshes", 0)
                w0, w1 = ev(), ev()
                w0.record()
            host_window = t_e2e <= k < t_judge
            if t_first <= k < t_e2e:
                i = k - t_first
                pos, vel = dpos[i], dvel[i]
            else:
                pos, vel = inputs(k)
            hp, hv = (pos, vel) if k not in hpos else (hpos[k], hvel[k])  # host copies for CL
            # the plain run records the warm start's training data over `record` (steps it sees
            # with three steps of history); the mixed runs seed every solve
            use_warm = warm is not None and (record is None or record[0] <= k < record[1])
            eng.load_inputs(pos, vel)
            eng.assemble()
            x0 = warm.prepare() if use_warm else None
            eng.solve(x0) if x0 is not None else eng.solve()
            if use_warm:
                warm.finish()
            elif warm is not None:
                warm.n_hist = 0
            if kind != "plain" and t_judge <= k < t_judge + 3:  # judged against the all-FP64 step
                rec.setdefault("judge", []).append(eng.judge())
                rec.setdefault("judge_cl", []).append(
                    [lift(eng, hp, hv, g.cpu().numpy()) for g in (eng.gamma, eng.last_judge_ref)])
            G[k].copy_(eng.gamma)
            if host_window:  # the step's circulations to the host; step k+1 is enqueued before k is read
                res = eng.gamma_host_async()
                if pending is not None:
                    pending.result()
                pending = res
            in_window = t_first <= k < t_judge
            if not in_window and k % cl_every == cl_every - 1:
                run1.record()
                torch.cuda.synchronize()
                run_ms += run0.elapsed_time(run1)
                cls[k] = lift(eng, hp, hv, eng.gamma.cpu().numpy())
                run0.record()
            eng.wake_update(times[k])
            eng.iteration += 1
            if k + 1 == t_e2e or k + 1 == t_judge:  # close a timed window
                if pending is not None:
                    pending.result()
                    pending = None
                if hasattr(eng, "join_side_stream"):  # work on the side stream counts too
                    eng.join_side_stream()
                w1.record()
                barrier()
                ms = max_over_ranks(w0.elapsed_time(w1))
                run_ms += w0.elapsed_time(w1)
                if k + 1 == t_e2e:
                    getattr(eng, "stats", None)  # the mixed engine takes its solves' status records
                    rec["ms"] = ms
                    rec["launches"] = _lib.lib().pvl_launch_count() + eng.replayed_kernels - launches0
                    if kind != "plain":
                        st = eng.stats
                        rec["gmres_iters"] = [int(i) for i in st["gmres_iters"][n_solves0:n_solves0 + K]]
                        rec["initial_rel_residual_median"] = float(
                            np.median(st["initial_rel_residual"][n_solves0:n_solves0 + K]))
                        rec["refreshes_in_window"] = st["refreshes"] - refresh0
                else:
                    rec["ms_e2e"] = ms
                    if kind != "plain":
                        st = eng.stats
                        rec["gmres_iters_e2e"] = [int(i) for i in st["gmres_iters"][n_solves0 + K:n_solves0 + 2 * K]]
                    eng.check_status()
                run0.record()
        run1.record()
        torch.cuda.synchronize()
        run_ms += run0.elapsed_time(run1)
        eng.check_status()
        rec.update({"G": G, "cl": cls, "run_ms": run_ms, "steps": end})
        if kind != "plain":
            st = eng.stats
            rec.update({"fallbacks": st["fallbacks"], "refreshes": st["refreshes"],
                        "refresh_failures": st["refresh_failures"]})
        if record is not None:
            rec["train"] = warm.training_data()
        del eng, warm
        torch.cuda.empty_cache()
        return rec

    sampler = ClockSampler(local)
    results = {"plain": run_arm("plain", record=TRAIN_STEPS)}
    X, T = results["plain"].pop("train")
    mlp, train_info = train_warm_start(X, T, seed=rank)
    results["mixed"] = run_arm("mixed", mlp=mlp)
    # what the network buys: the same mixed solve seeded without it, up to the end of the timed window
    seeds = {"learned": results["mixed"]}
    for mode in ("jacobi", "previous"):
        seeds[mode] = run_arm("mixed", seed_mode=mode, last=t_e2e)
    clocks = sampler.stop()
    # whole-trajectory comparison of the mixed + learned run with the plain FP64 run
    Gp, Gm = results["plain"]["G"], results["mixed"]["G"]
    n_cmp = min(Gp.shape[0], Gm.shape[0])
    rel = (torch.linalg.vector_norm(Gm[:n_cmp] - Gp[:n_cmp], dim=1) /
           torch.linalg.vector_norm(Gp[:n_cmp], dim=1)).cpu().numpy()
    cl_p, cl_m = results["plain"]["cl"], results["mixed"]["cl"]
    cl_rel = {k: abs(cl_m[k] - cl_p[k]) / abs(cl_p[k]) for k in cl_p if k in cl_m}
    trajectory = {
        "steps": int(n_cmp), "start": "t = 0, empty wake (grows to 400 rows by step 400, then truncated)",
        "gamma_rel_max": float(rel.max()), "gamma_rel_max_at_step": int(rel.argmax()),
        "gamma_rel_last": float(rel[-1]),
        "cl_rel_max": max(cl_rel.values()), "cl_steps_compared": len(cl_rel),
        "cl_last": [cl_m[max(cl_m)], cl_p[max(cl_p)]],
        "tolerance": 1e-10,
        "plain_steps_per_s": 1000.0 * results["plain"]["steps"] / results["plain"]["run_ms"],
        "mixed_steps_per_s": 1000.0 * results["mixed"]["steps"] / results["mixed"]["run_ms"],
        "how": "both engines run the whole workload from t = 0; every step's circulation of the mixed + learned run "
               "vs the plain FP64 run's (relative 2-norm), CL every 10 steps through the line-force path; steps/s "
               "over the whole run (CL evaluations excluded)",
    }
    trajectory["speedup_mixed_over_plain"] = trajectory["mixed_steps_per_s"] / trajectory["plain_steps_per_s"]
    seed_arms = {m: {"ms_per_step": r["ms"] / K, "steps_per_s": replica_throughput(K, r["ms"], world),
                     "gmres_iters_mean": float(np.mean(r["gmres_iters"])),
                     "initial_rel_residual_median": r["initial_rel_residual_median"],
                     "refreshes_in_window": r["refreshes_in_window"]} for m, r in seeds.items()}
    del Gp, Gm, seeds
    results["plain"].pop("G")
    results["mixed"].pop("G")
    # ---------------- dominant kernel: the FP64 sweeps of the explicit wake term, timed alone on a
    # full-wake state (the seeded full wake that the kernel captures under ncu use as well): the
    # headline's three row bands (wake_bands), and one sweep of every row at every point
    _, spec_full, wpos, wcirc, t0 = wake_setup(case, mesh)
    eng = MixedSolverEngine(mesh, case.freestream, case.tol, spec_full, cp_patches=case.smooth_patches,
                            wake_col_runs=case.wake_col_runs)
    eng.set_wake_state(wpos, wcirc, step_count=case.line_rows + 1, time=t0 - case.dt)
    eng.iteration = 1
    eng.load_inputs(case.positions_at(t0), case.velocities_at(t0))
    eng.assemble_body_only()
    w = eng.wake
    rm, d = w["rm"], w["rm_d"]
    wpos_d = eng.wake_positions.reshape(-1, 3)
    lg = w["rm_line_gamma"]
    lg.fill_(1e-3)
    kargs = (_lib.PVL_F64, rm.n_points, rm.n_lines, ptr(d["lines"]), ptr(wpos_d), ptr(lg), eng.P, ptr(eng.cps),
             ptr(eng.nrm), case.tol, 1.0, 0.0, ptr(eng.rhs), ptr(eng.ws), eng._ws_bytes, stream_ptr())
    for _ in range(2):
        _lib.call("pvl_line_velocity", *kargs)
    reps = 5
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    k0.record()
    for _ in range(reps):
        _lib.call("pvl_line_velocity", *kargs)
    k1.record()
    torch.cuda.synchronize()
    full_ms = k0.elapsed_time(k1) / reps
    full_pairs = rm.n_lines * eng.P
    band_calls, pairs = wake_band_calls(eng, case.tol)
    for _ in range(2):
        for bc in band_calls:
            _lib.call("pvl_line_velocity", *bc)
    torch.cuda.synchronize()
    k0.record()
    for _ in range(reps):
        for bc in band_calls:
            _lib.call("pvl_line_velocity", *bc)
    k1.record()
    torch.cuda.synchronize()
    kms = k0.elapsed_time(k1) / reps
    achieved = pairs * PAIR_FLOPS / (kms * 1e-3) / 1e12
    from pyvl_b200 import _probe

    sink = torch.zeros(148 * 8, dtype=torch.float64, device="cuda")
    _probe.lib().pvl_probe_fma(_lib.PVL_F64, 148 * 8, 2000, ptr(sink), stream_ptr())
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    p0.record()
    flops = _probe.lib().pvl_probe_fma(_lib.PVL_F64, 148 * 8, 20000, ptr(sink), stream_ptr())
    p1.record()
    torch.cuda.synchronize()
    peak = flops / (p0.elapsed_time(p1) * 1e-3) / 1e12

    def time_call(name, args, reps=5):
        for _ in range(2):
            _lib.call(name, *args)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            _lib.call(name, *args)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # secondary rooflines: the FP32x2 advection sweep against the FP32 FMA peak, the body
    # matrix against the FP64 peak and the HBM write bandwidth
    S, R, L = w["S"], w["R"], mesh.n_lines
    r_near = eng.advect_near_rows
    eng.body_line_gamma.fill_(1e-2)
    ams = time_call("pvl_wake_node_velocity_cols", (
        _lib.PVL_F32, mesh.n_points, L, ptr(eng.d_body["lines"]), ptr(eng.pos), ptr(eng.body_line_gamma), S, R, R,
        r_near, R, w["n_cols"], ptr(w["cols"]), ptr(eng.wake_positions), 1.0, 0.0, 0.0, case.tol,
        ptr(w["node_vel"]), ptr(eng.ws), eng._ws_bytes, stream_ptr()))
    a_pairs = L * w["n_cols"] * (R - r_near)
    sink32 = torch.zeros(148 * 8, dtype=torch.float32, device="cuda")
    _probe.lib().pvl_probe_fma(_lib.PVL_F32, 148 * 8, 2000, ptr(sink32), stream_ptr())
    torch.cuda.synchronize()
    p0.record()
    flops32 = _probe.lib().pvl_probe_fma(_lib.PVL_F32, 148 * 8, 20000, ptr(sink32), stream_ptr())
    p1.record()
    torch.cuda.synchronize()
    peak32 = flops32 / (p0.elapsed_time(p1) * 1e-3) / 1e12
    db = eng.d_body
    bms = time_call("pvl_induction_normal_tiled", (
        mesh.n_points, L, ptr(db["lines"]), ptr(eng.pos), eng.P, ptr(db["offsets"]), ptr(db["surface_lines"]),
        ptr(db["tile_offsets"]), ptr(db["tile_lines"]), ptr(db["sl_local"]), db["tile_max"], eng.P, ptr(eng.cps),
        ptr(eng.nrm), case.tol, ptr(eng.A), eng.N, ptr(eng.ws), eng._ws_bytes, stream_ptr()))
    b_pairs = eng.P * int(mesh.ring_tiles()[1].size)  # (control point, distinct tile line) pairs
    hbm_peak = None
    mp = ROOT / "MEASURED_PEAKS.json"
    if mp.exists():
        hbm_peak = json.loads(mp.read_text()).get("hbm_gbs")
    traffic = traffic_full = None
    prof = ROOT / "profiles" / "line_sum_f64_flapping_wake_term.md"
    if prof.exists():
        for line in prof.read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch:"):
                traffic_full = float(line.split(":", 1)[1].split()[0])
            if line.startswith("band_traffic_bytes_per_step:"):
                traffic = float(line.split(":", 1)[1].split()[0])
    secondary = {
        "wake_term_full_sweep": {"kernel": "line_sum_f64_kernel (every wake row at every control point)",
                                 "ms_per_call": full_ms, "pairs": full_pairs,
                                 "achieved": full_pairs * PAIR_FLOPS / (full_ms * 1e-3) / 1e12, "peak": peak,
                                 "unit": "TFLOP/s",
                                 "frac": full_pairs * PAIR_FLOPS / (full_ms * 1e-3) / 1e12 / peak,
                                 "traffic": traffic_full},
        "advection_fp32x2": {"kernel": "line_sum_f32x2_kernel (wake rows %d..%d)" % (r_near, R - 1),
                             "ms_per_call": ams, "pairs": a_pairs,
                             "achieved": a_pairs * PAIR_FLOPS / (ams * 1e-3) / 1e12, "peak": peak32,
                             "unit": "TFLOP/s", "frac": a_pairs * PAIR_FLOPS / (ams * 1e-3) / 1e12 / peak32,
                             "peak_source": "FP32 FMA throughput measured live (pvl_probe_fma)"},
        "body_matrix": {"kernel": "ring_tile_kernel", "ms_per_call": bms, "pairs": b_pairs,
                        "achieved": b_pairs * PAIR_FLOPS / (bms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                        "frac": b_pairs * PAIR_FLOPS / (bms * 1e-3) / 1e12 / peak,
                        "hbm_write_gbs": 8.0 * eng.P * eng.P / (bms * 1e-3) / 1e9, "hbm_peak_gbs": hbm_peak},
    }
    del eng
    head = results[args.path]
    sps = replica_throughput(K, head["ms"], world)
    sps_e2e = replica_throughput(K, head["ms_e2e"], world)
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline()
    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        torch.cuda.empty_cache()
        batch = batch_summary()
    if rank == 0:
        h2d = 2 * mesh.n_points * 3 * 8
        d2h = mesh.n_surfaces * 8
        mx = results["mixed"]
        print(json.dumps({
            "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": head["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.path == "plain" else "f64 (residuals, assembly) / f32+tf32 (preconditioner) / "
                                                        "bf16 (warm-start network)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "rings": 4096, "wake_rows": 400, "path": args.path,
                       "timed_steps": f"{t_first}..{t_e2e - 1} (device-resident inputs), {t_e2e}..{t_judge - 1} "
                                      f"(end to end) of the run, after {t_first} untimed steps",
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "per-step working set (134 MB matrix + wake) exceeds the 126 MB L2"},
            "paths": {
                "plain_fp64": {"steps_per_s": replica_throughput(K, results["plain"]["ms"], world),
                               "ms_per_step": results["plain"]["ms"] / K,
                               "e2e_steps_per_s": replica_throughput(K, results["plain"]["ms_e2e"], world)},
                "mixed_learned": {"steps_per_s": replica_throughput(K, mx["ms"], world), "ms_per_step": mx["ms"] / K,
                                  "e2e_steps_per_s": replica_throughput(K, mx["ms_e2e"], world),
                                  "gmres_iters_mean": float(np.mean(mx["gmres_iters"])),
                                  "gmres_iters_mean_e2e": float(np.mean(mx["gmres_iters_e2e"])),
                                  "fallbacks": mx["fallbacks"], "preconditioner_refreshes": mx["refreshes"],
                                  "refreshes_in_window": mx["refreshes_in_window"],
                                  "refresh_failures": mx["refresh_failures"],
                                  "initial_rel_residual_median": mx["initial_rel_residual_median"],
                                  "warm_start_training": train_info,
                                  "far_wake": "explicit wake term of rows >= 64 at every other chordwise control "
                                              "point, of rows >= 192 every other spanwise too (quintic midpoint "
                                              "rule within each half wing); advection FP32 from row 8, every other "
                                              "node column from row 64 (quintic midpoint rule within each half "
                                              "wing), every other row from row 128 (cubic midpoint); error: "
                                              "trajectory"},
                "speedup_mixed_over_plain": results["plain"]["ms"] / mx["ms"],
            },
            "warm_start": {**seed_arms,
                           "how": "the same mixed engine over the same steps seeded by the previous circulation, by "
                                  "one Jacobi correction of it (the network's base), or by the network; timed window "
                                  "as the headline's"},
            "trajectory": trajectory,
            "accuracy": {"gamma_rel_err_vs_fp64_max": max(mx["judge"]), "judged_steps": len(mx["judge"]),
                         "cl_rel_err_vs_fp64_max": max(abs(a - b) / abs(b) for a, b in mx["judge_cl"]),
                         "cl_mixed_fp64_last": mx["judge_cl"][-1],
                         "tolerance": 1e-10,
                         "how": "after the timed steps, each judged step's mixed circulation vs the same state "
                                "assembled in FP64 and solved by FP64 LU; CL of both circulations at that state "
                                "through the line-force path (body + wake velocity at the nodes, trailing-edge "
                                "correction)"},
            "e2e": {"value": sps_e2e, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp64", "kernel": "line_sum_f64_kernel (explicit wake term)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic, "ms_per_step": kms, "pairs_per_step": pairs, "launches_per_step": 3,
                         "peak_source": "FP64 FMA throughput measured live (pvl_probe_fma); 45 FLOP per pair",
                         "timed": "the step's three pvl_line_velocity calls of the explicit wake term (rows 1-63 "
                                  "at every control point, 64-191 and 192-399 at the stencils' points): segment "
                                  "tables, sweeps and partial-sum reductions; traffic: their three sweeps"},
            "rooflines_secondary": secondary,
            "cpu_baseline": base,
            "batched_cases": batch,
            "gpu_launches": int(head["launches"]),
            "clocks": clocks,
        }), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    sys.path.insert(0, str(ROOT))
    main()
