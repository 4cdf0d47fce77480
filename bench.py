"""Benchmark of the B200 flux pass (one JSON line on rank 0).

Default workload (--workload serve): the serving request stream, whole --
Poisson arrivals at 200 requests/s for 60 s (seed 5, 12,058 requests), 70%
2D / 30% 3D static Voronoi meshes (periodic unit box) with generator counts
log-uniform in [1e3, 1e6] served from a pre-tessellated pool (10 log-size
bins per dimension), random-field states, U{10..200} steps, exact or HLLC
50/50.  The unit of work is the face-step (one nonzero-area face processed
in one time step, with its share of the gradient and update work).

  value  the whole stream's requests with their states resident in HBM,
         co-batched per (dimension, solver) class in launch groups, rounds
         of --chunk steps, CUDA events on the device (FP32/FP64 split pass).
         The requests form --steps consecutive segments of arrivals, one
         bench step each (states loaded before each segment's timed region).
  e2e    the whole stream served by the request server (sfx_server_*) from
         host memory at the arrival times: face-steps of completed requests
         over the makespan, p50/p99 request latency.
  served_speedup_vs_fp64
         e2e over the plain FP64 pass's served throughput on every
         --fp64-every-th request (submitted at once, a saturated server;
         the FP64 pass over the whole stream would take about 50 minutes),
         with the per-field relative L1 and max error of the split results
         against FP64 on those requests.

Other workloads: --workload sedov3d (Sedov 3D blast, 262,144 generators,
HLLC, one mesh; --precision fp64|split), --workload random3d (3D supersonic
random field, 2,097,152 generators, exact solver) and --workload batch2d
(1,024 2D step-state meshes in one launch group vs one FP64 launch sequence
per mesh).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload serve|sedov3d|random3d|batch2d] [--precision fp64|split]

Timing: CUDA events on the library's streams, barrier + synchronize on both
sides, max over ranks; untimed warm-up before the timed region.  Working
sets are larger than the 126 MB L2, so no separate L2 flush is done.

N>1 (serve): the GPUs share the one stream, whole requests each, assigned in
arrival order to the GPU with the least face work so far (no data-path
collective); value and e2e are all GPUs' face-steps over the slowest GPU's
time.  Other workloads: every rank runs its own meshes (weak scaling).

--impl reference times the reference's own CPU flux pass (the unmodified
Shadowfax sources built into oracle/_ref) on the host cores: for the stream,
one process per request on its first requests, each stepping its request
--steps times; that process loads no GPU library (its meshes come from the
standalone sfx_meshgen builder and a numpy reader).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_GEN = 262_144
SEED = 2
METRIC = "faces/s (face-steps per second) of the flux pass"
METRIC_SERVE = ("faces/s (face-steps per second) on 1 B200, served+batched FP32/FP64 split vs "
                "plain FP64 at <=1e-6 rel L1; p50/p99 latency")
UNIT = "face-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (sedov3d 50, batch2d 20); serve: the whole stream is "
                         "timed, its resident replay in this many consecutive segments of "
                         "arrivals (default 20), one step each")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    ap.add_argument("--n", type=int, default=None,
                    help="generators of sedov3d / random3d (default: 262,144 / 2,097,152)")
    ap.add_argument("--solver", default=None, choices=["Exact", "HLLC"],
                    help="sedov3d / random3d solver (default: HLLC / Exact)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="serve",
                    choices=["serve", "sod2d", "sedov3d", "random3d", "random2d", "batch2d"],
                    help="serve: the request stream (default); sedov3d: Sedov 3D blast "
                         "on one mesh; sod2d: 2D Sod tube, 10,000 generators, exact "
                         "solver, dt 1e-4; random3d: periodic 3D random field, exact solver; "
                         "batch2d: 1,024 2D meshes")
    ap.add_argument("--meshes", type=int, default=1024, help="batch2d: number of meshes")
    ap.add_argument("--duration", type=float, default=60.0,
                    help="serve: seconds of the stream (default: the whole 60 s)")
    ap.add_argument("--requests", type=int, default=None,
                    help="serve: only the stream's first N arrivals (quick runs)")
    ap.add_argument("--fp64-every", type=int, default=48,
                    help="serve: every N-th request is also served by the plain FP64 pass "
                         "(0: none)")
    ap.add_argument("--chunk", type=int, default=4, help="serve: steps per scheduling round")
    ap.add_argument("--pool-dir", default=None,
                    help="serve: read the pool meshes from mesh files in this directory, "
                         "writing the ones not there yet (sfx_meshfile_*)")
    a = ap.parse_args()
    if a.steps is None:
        a.steps = {"serve": 20, "sod2d": 100, "sedov3d": 50, "random3d": 10, "random2d": 10,
                   "batch2d": 20}[a.workload]
    if a.n is None:
        a.n = {"random3d": 2_097_152, "random2d": 2_097_152, "sod2d": 10_000}.get(a.workload,
                                                                                  N_GEN)
    if a.solver is None:
        a.solver = "Exact" if a.workload in ("random3d", "random2d", "sod2d") else "HLLC"
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region"""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["stdbuf", "-oL", "nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which: str):
        setattr(self, which, time.time())

    def wait_first_sample(self, timeout: float = 3.0):
        """nvidia-smi needs a moment to start: wait for its first line so the
        (short) timed region is covered"""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        """samples read between the marks t0 and t1 (widened by 0.25 s on each
        side when the timed region is shorter than the sampling period)"""
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", 1e300)
        pad = 0.0 if t1 - t0 > 0.5 else 0.25
        for ts, ln in self.lines:
            if not (t0 - pad <= ts <= t1 + pad):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window_s": round(t1 - t0, 4), "pad_s": pad}


def reduce_over_ranks(ms: float, work: float, device, world: int):
    """whole-job throughput over ranks: the work of all ranks (SUM) divided by
    the slowest rank's device time (MAX); returns (value, ms_max, work_total).
    Every rank makes the same two collective calls."""
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    w = torch.tensor([float(work)], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.SUM)
    ms_max, work_total = float(t.item()), float(w.item())
    return work_total / (ms_max / 1e3), ms_max, work_total


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(dim: int, n_cells: int, n_faces: int, nnz: int, precision: str):
    """bytes each kernel of one step must move at least once (FP64 plain):
    gradients: read W, pos, centroid, volume, CSR (offsets + entries) per
    cell; per face area, midpoint, left, right, kind, right generator
    position; write the gradient (dim*S) per cell.
    faces: read the face record, per cell W, gradient, centroid, pos, Q.m,
    total area; write dQ (S) per face.
    update: read Q, volume, CSR, dQ per face; write Q and W per cell."""
    S = dim + 2
    face_rec = 8 + 8 * dim + 4 + 4 + 4 + 8 * dim
    cell_grad_in = 8 * S + 8 * dim + 8 * dim + 8 + 4
    grad = n_cells * (cell_grad_in + 8 * dim * S) + nnz * 4 + n_faces * face_rec
    faces = n_faces * (face_rec + 8 * S) + n_cells * (8 * S + 8 * dim * S + 8 * dim + 8 * dim + 8 + 8)
    update = n_cells * (8 * S + 8 + 4 + 8 * S * 2) + nnz * 4 + n_faces * (8 * S + 8)
    return {"gradients": grad, "faces": faces, "update": update}


def split_kernel_bytes(dim: int, n_cells: int, n_faces: int, nnz: int):
    """bytes each split-pass kernel must move at least once per launch, in
    its device layout: face record fg (2 float4) + fi (int2) + shift code
    (1 B) + FP64 area vector (8 dim); cell record cw (2 float4), cx
    (float4), gradients cg (G float4, G = 4 in 3D, 2 in 2D); per-face dQ
    {mass, energy} float2 + FP64 momentum (8 dim); Q FP64 (8 S).
    gradients: cw, cx, offset, CSR entry, face fg + fi; write cg.
    faces: face record, dQ write, and per cell cw, cx, cg.
    update: offset, CSR entry, per-face dQ, Q read+write, volume, total
    area (FP64), write cw."""
    S = dim + 2
    G = 16 * (4 if dim == 3 else 2)
    grad = n_cells * (32 + 16 + 4 + G) + n_faces * (32 + 8) + nnz * 4
    faces = n_faces * (32 + 8 + 1 + 8 * dim + 8 + 8 * dim) + n_cells * (32 + 16 + G)
    update = n_cells * (4 + 16 * S + 8 + 8 + 32) + nnz * 4 + n_faces * (8 + 8 * dim)
    return {"gradients": grad, "faces": faces, "update": update}


# bytes per face-step of the whole step, fixed for this workload's roofline:
# face record + per-cell data / faces per cell (2D F ~ 3N, 3D F ~ 7.8N)
L2_BYTES = 126 << 20   # B200 L2
STEP_BYTES = {("fp64", 2): 144, ("fp64", 3): 120, ("split", 2): 92, ("split", 3): 70}


def build_problem(args):
    """Sedov 3D (reflective cube, seed 2) or the 3D random field (periodic
    cube, seed 3) with the chosen solver"""
    from shadowfax_b200 import workloads as wl
    if args.workload == "random3d":
        return wl.random_field3d(n=args.n, seed=3, solver=args.solver)
    if args.workload == "random2d":
        return wl.random_field2d(n=args.n, seed=3, solver=args.solver)
    if args.workload == "sod2d":
        return wl.sod2d(n=args.n, seed=1, solver=args.solver)
    return wl.sedov3d(n=args.n, seed=SEED, solver=args.solver)


def problem_text(args, pr):
    m = pr.mesh
    if args.workload in ("random3d", "random2d"):
        box = "cube" if m.dim == 3 else "square"
        return (f"{args.workload} {pr.solver}, {m.n_cells} generators (seed 3), "
                f"{m.n_active_faces} faces, periodic unit {box}, log-normal density, Gaussian "
                f"velocities, CFL-0.4 dt")
    if args.workload == "sod2d":
        return (f"sod2d {pr.solver}, {m.n_cells} generators (seed 1), {m.n_active_faces} faces, "
                f"reflective unit square, rho/p 1/1 | 0.125/0.1 at x = 0.5, dt 1e-4")
    return (f"sedov3d {pr.solver}, {m.n_cells} generators (seed {SEED}), {m.n_active_faces} "
            f"faces, reflective unit cube, CFL-0.4 dt")


def cpu_baseline(pr, steps: int | None = None):
    """reference CPU pass (oracle/_ref, unmodified Shadowfax sources), one
    core, on the same mesh for a bounded number of steps (about 3e7
    face-steps, at least 3 steps and at most 100)"""
    from oracle.oracle import Params, ref_binary, run_reference
    if steps is None:
        steps = max(3, min(100, int(3e7 // max(pr.mesh.n_active_faces, 1))))
    exe = ref_binary(pr.mesh.dim, "libm")
    if not exe.exists():
        return None
    p = Params(solver=pr.solver, gamma=pr.gamma, use_libm_pow=True)
    r = run_reference(pr.mesh, p, pr.dt, steps + 1, pr.W0, pow_kind="libm")
    secs = float(np.sum(r["step_seconds"][1:]))
    value = pr.mesh.n_active_faces * steps / secs
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{steps} timed steps (+1 warm-up) of the full {pr.mesh.n_cells}-cell "
                      f"mesh, reference VorCell/VorFace/HLLC loops, 1 MPI rank (single thread)"}


def cpu_baseline_many(probs, steps: int = 2, warmup: int = 1):
    """reference CPU pass on a sample of the batch: one mesh per process, as
    many processes as host cores, run concurrently (the reference has no
    threads; independent meshes are its best case)"""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle import Params, ref_binary, run_reference
    if not ref_binary(2, "libm").exists():
        return None
    P = min(os.cpu_count() or 1, len(probs))
    sample = probs[:P]

    def one(pr):
        p = Params(solver=pr.solver, gamma=pr.gamma, use_libm_pow=True)
        r = run_reference(pr.mesh, p, pr.dt, steps + warmup, pr.W0, pow_kind="libm")
        # a request that fails inside the sample (the reference's exceptions)
        # counts the steps it completed
        done = min(int(r["steps"]), steps + warmup) - warmup
        if done <= 0:
            return 0, 0.0
        return pr.mesh.n_active_faces * done, float(np.sum(r["step_seconds"][warmup:warmup + done]))

    with ThreadPoolExecutor(max_workers=P) as ex:
        res = list(ex.map(one, sample))
    # sum of the per-process rates: every core kept busy (the makespan of
    # unequal meshes would leave cores idle and understate the CPU)
    value = sum(w / s for w, s in res if s > 0)
    return {"value": value, "unit": UNIT, "cores": P, "kind": "reference",
            "sample": f"{len(sample)} meshes of the batch ({sum(p.mesh.n_cells for p in sample)} "
                      f"cells), {warmup} warm-up + {steps} timed steps each, one reference "
                      f"process per mesh on {P} host cores concurrently (P processes, not an "
                      f"MPI run; value = sum of the per-process rates)"}


def bench_batch(args, rank, world, local, torch):
    """batch2d: many independent 2D meshes, HLLC, each at its own CFL dt.
    Ours: FP32/FP64-split pass, all meshes in one launch group (one launch per
    phase per step, the steps captured in a CUDA graph, lanes per cell tuned).
    Baseline on the same GPU: the plain-FP64 pass launched mesh by mesh."""
    from shadowfax_b200 import _lib as L
    from shadowfax_b200 import workloads as wl
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    t_build = time.time()
    probs = wl.batch2d(count=args.meshes, seed=4 + 1000 * rank)
    t_build = time.time() - t_build
    faces = sum(pr.mesh.n_active_faces for pr in probs)
    solver = RiemannSolverFactory.generate("HLLC")
    stream = torch.cuda.Stream(device=local)
    ctx = Context(2, solver, L.PREC_SPLIT, device=local)
    ctx.set_stream(stream.cuda_stream)
    members = []
    for pr in probs:
        fp = FluxPass(ctx, pr.mesh)
        fp.set_primitive(pr.W0)
        members.append(fp)
    grp = Group(ctx, members, [pr.dt for pr in probs])
    lanes = grp.tune(3)
    face_variant = grp.tune_faces(3)
    for fp, pr in zip(members, probs):   # tuning reads the states only; reset anyway
        fp.set_primitive(pr.W0)
    with torch.cuda.stream(stream), ClockSampler(local) as clk:
        clk.wait_first_sample()
        st = grp.step(args.warmup, graph=True)
        assert np.all(st == 0), st
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        grp.step(args.steps, graph=True, status=False)   # capture the K-step graph
        torch.cuda.synchronize()
        clk.mark("t0")
        n_launch0 = L.lib().sfx_launch_count()
        e0.record(stream)
        grp.step(args.steps, graph=True, status=False)
        e1.record(stream)
        n_launches = L.lib().sfx_launch_count() - n_launch0
        torch.cuda.synchronize()
        clk.mark("t1")
        time.sleep(0.3)
        ms = e0.elapsed_time(e1)
        st = grp.step(1, graph=False)
        assert np.all(st == 0), st
    value, ms_max, _ = reduce_over_ranks(ms, faces * args.steps, f"cuda:{local}", world)
    # end to end through the public API with host buffers: per step every
    # mesh's W and Q uploaded from host memory, one group step, W and Q read back
    saved = [fp.state() for fp in members]
    host = saved
    e2e_steps = max(1, min(args.steps, 5))
    nbytes = sum(W.nbytes + Q.nbytes for W, Q in host)
    with torch.cuda.stream(stream):
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for fp, (W, Q) in zip(members, host):
                fp.set_state(W, Q)
            grp.step(1, graph=True, status=False)
            host = [fp.state() for fp in members]
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1e3
    for fp, (W, Q) in zip(members, saved):   # back to the state the accuracy check expects
        fp.set_state(W, Q)
    e2e_val, _, _ = reduce_over_ranks(e2e_ms, faces * e2e_steps, f"cuda:{local}", world)
    # FP64 baseline: one launch sequence per mesh
    ctx64 = Context(2, solver, L.PREC_FP64, device=local)
    ctx64.set_stream(stream.cuda_stream)
    m64 = []
    for pr in probs:
        fp = FluxPass(ctx64, pr.mesh)
        fp.set_primitive(pr.W0)
        m64.append(fp)
    base_steps = max(1, min(args.steps, 5))
    with torch.cuda.stream(stream):
        for fp, pr in zip(m64, probs):
            fp.step(pr.dt, 1, stats=False)
        torch.cuda.synchronize()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(base_steps):
            for fp, pr in zip(m64, probs):
                fp.step(pr.dt, 1, stats=False)
        b1.record(stream)
        torch.cuda.synchronize()
    fp64_value = faces * base_steps / (b0.elapsed_time(b1) / 1e3)
    for fp in m64:
        fp.close()
    ctx64.close()
    # accuracy of the split group against the plain-FP64 pass (sample)
    acc = []
    for j in range(0, len(probs), max(1, len(probs) // 16)):
        pr = probs[j]
        ca = Context(2, solver, L.PREC_FP64, device=local)
        a = FluxPass(ca, pr.mesh)
        a.set_primitive(pr.W0)
        a.step(pr.dt, args.warmup + 2 * args.steps + 1)
        Qa = a.state()[1]
        Qb = members[j].state()[1]
        acc.append(float(np.max(np.abs(Qb - Qa).sum(0)[[0, -1]] / np.abs(Qa).sum(0)[[0, -1]])))
        a.close()
        ca.close()
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_many(probs)
    peak, peak_kind = peaks()
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"batch2d: {len(probs)} independent 2D meshes, generators "
                                   f"log-uniform in [1e3, 1e5] (total {sum(p.mesh.n_cells for p in probs)}"
                                   f" cells, {faces} faces), step states, HLLC, own CFL dt each",
                       "precision": "split", "launch": "one launch group, CUDA graph of K steps",
                       "lanes_per_cell": lanes, "face_variant": face_variant,
                       "l2": "working set > L2 (no flush)",
                       "parallelism": f"replicas x{world}", "mesh_build_s": round(t_build, 1)},
            "clocks": clk.summary(),
            "fp64_per_mesh": {"value": fp64_value, "unit": UNIT, "steps": base_steps,
                              "launch": "4 launches per mesh per step, plain FP64"},
            "speedup_vs_fp64_per_mesh": value / fp64_value,
            "split_vs_fp64_max_rel_l1_mass_energy": max(acc) if acc else None,
            "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s",
                         "peak_source": f"hbm_gbs {peak_kind}",
                         "step_bytes_per_face": 92,
                         "achieved": 92 * value / 1e9, "frac": 92 * value / 1e9 / peak,
                         "note": "bytes per face-step of the split pass, 2D (algorithmic)"},
            "cpu_baseline": cb,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
                    "note": "wall clock: per step every mesh's W and Q from host memory, one "
                            "group step, W and Q back (sfx_state_upload_WQ / "
                            "sfx_group_step / sfx_state_download)"},
            "gpu_launches": int(n_launches),
        }
    grp.close()
    for fp in members:
        fp.close()
    ctx.close()
    return line


SERVE_BUDGET = 150 << 30
# reference processes of the CPU sample at most (each holds a whole mesh of
# up to 7e5 cells in the reference's per-cell objects)
SERVE_CPU_PROCS = 48


def serve_requests(args):
    """the request stream: every arrival of --duration seconds (default the
    whole 60 s), or the first --requests arrivals (quick runs)"""
    from shadowfax_b200 import workloads as wl
    if args.requests:
        return wl.serve_stream(count=args.requests, seed=5)
    return wl.serve_stream(duration=args.duration, seed=5)


def shard_requests(reqs, world: int, k: int = 10) -> np.ndarray:
    """The rank serving each request of one stream shared by `world` GPUs:
    whole requests, no data-path collective.  In arrival order each request
    goes to the rank with the least face work assigned so far (the lowest
    rank on ties), the face work of a request being its pool mesh's cells x
    faces per cell (3 in 2D, 7.8 in 3D, Poisson-Voronoi averages) x its steps.
    Every rank computes the same assignment from the stream alone."""
    from shadowfax_b200 import workloads as wl
    sizes = wl.serve_pool_sizes(k)
    load = np.zeros(world)
    owner = np.empty(len(reqs), np.int64)
    for j, r in enumerate(reqs):
        dim, n = 2 + r.mesh // k, float(sizes[r.mesh % k])
        q = int(np.argmin(load))
        owner[j] = q
        load[q] += n * (3.0 if dim == 2 else 7.8) * r.nsteps
    return owner


def l1_rel_fields(a, b):
    """relative L1 error per conserved field (mass, momentum, energy); the
    momentum components share the L1 norm of the momentum magnitude"""
    D = b.shape[1] - 2
    den = np.abs(b).sum(0)
    den[1:D + 1] = np.sqrt((b[:, 1:D + 1] ** 2).sum(1)).sum()
    e = np.abs(a - b).sum(0) / den
    return np.array([e[0], e[1:D + 1].max(), e[D + 1]])


def max_rel_fields(a, b):
    """largest per-cell error per conserved field relative to the field's
    largest magnitude (momentum: the largest momentum magnitude)"""
    D = b.shape[1] - 2
    den = np.abs(b).max(0)
    den[1:D + 1] = np.sqrt((b[:, 1:D + 1] ** 2).sum(1)).max()
    e = np.abs(a - b).max(0) / np.maximum(den, 1e-300)
    return np.array([e[0], e[1:D + 1].max(), e[D + 1]])


def run_served(pool, reqs, precision, chunk, keep_states=False, device=0, at_once=False,
               tuning=None):
    """serve requests through the request server (C ABI, host states in and
    out): submitted at their arrival times from a feeder thread (at_once:
    all at time 0, a saturated server), completions collected concurrently;
    returns per-request results (with states when keep_states), launches and
    server stats.  tuning: {(dim, solver): the tuners' choices} for the split
    server's launch groups"""
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.serve import Server
    srv = Server(precision=precision, memory_budget=SERVE_BUDGET, chunk_steps=chunk,
                 device=device)
    try:
        if precision == L.PREC_SPLIT:
            for (d, solver), t in (tuning or {}).items():
                srv.set_tuning(d, solver, t["lanes_per_cell"], t["face_variant"])
        ids = {j: srv.add_mesh(m) for j, m in enumerate(pool.meshes) if m is not None}
        # warm-up: a short request per class on the smallest meshes present
        warm = []
        for d in (2, 3):
            js = [j for j in ids if (j >= pool.k) == (d == 3)]
            for solver in ("Exact", "HLLC"):
                if js:
                    j0 = min(js)
                    warm.append(srv.submit(ids[j0], pool.states[j0][0], solver,
                                           pool.dts[j0][0], 3))
        srv.drain(600.0)
        for r in warm:
            srv.poll(r, want_state=False)
        lock = threading.Lock()
        pending = {}
        results = {}
        n0 = L.lib().sfx_launch_count()
        t_base = time.perf_counter()

        def feeder():
            for j, r in enumerate(reqs):
                delay = t_base + r.t - time.perf_counter()
                if delay > 0 and not at_once:
                    time.sleep(delay)
                rid = srv.submit(ids[r.mesh], pool.states[r.mesh][r.state], r.solver,
                                 pool.dts[r.mesh][r.state], r.nsteps)
                with lock:
                    pending[rid] = j

        th = threading.Thread(target=feeder, daemon=True)
        th.start()
        # collect results only when the server reports new completions: one
        # poll per pending request every millisecond would contend with the
        # worker thread for the server's lock (latencies are the server's
        # timestamps, so the collection rate does not enter them)
        seen, last = -1, 0.0
        while len(results) < len(reqs):
            st = srv.stats()
            done = st.completed + st.failed
            now = time.perf_counter()
            # (and every 50 ms: a request may finish before the feeder has
            # recorded its id)
            if done != seen or now - last > 0.05:
                seen, last = done, now
                with lock:
                    items = list(pending.items())
                for rid, j in items:
                    res = srv.poll(rid, want_state=keep_states)
                    if res is not None:
                        results[j] = res
                        with lock:
                            del pending[rid]
            time.sleep(0.002)
        th.join()
        launches = L.lib().sfx_launch_count() - n0
        st = srv.stats()
    finally:
        srv.shutdown()
    return [results[j] for j in range(len(reqs))], launches, st


def served_summary(res, st=None):
    ok = [r for r in res if r.status == 0]
    lat = np.array([r.t_done - r.t_submit for r in ok]) if ok else np.zeros(1)
    t0 = min(r.t_submit for r in res)
    t1 = max(r.t_done for r in res)
    fs = sum(r.face_steps for r in ok)
    return {"value": fs / (t1 - t0), "unit": UNIT, "requests": len(res), "completed": len(ok),
            "failed": len(res) - len(ok), "face_steps": int(fs), "makespan_s": t1 - t0,
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()),
            "rounds": int(st.rounds) if st is not None else None,
            "worker_s": {k: round(float(v), 3) for k, v in
                         zip(("admit", "launch", "finish", "collect"), st.worker_s)}
            if st is not None else None}


def _budget_waves(idx, nbytes):
    """consecutive runs of requests whose instances fit the device budget"""
    waves, cur, used = [], [], 0
    for j in idx:
        b = nbytes(j)
        if cur and used + b > SERVE_BUDGET:
            waves.append(cur)
            cur, used = [], 0
        cur.append(j)
        used += b
    if cur:
        waves.append(cur)
    return waves


def run_resident(pool, reqs, nseg, warmup, chunk, torch, local):
    """The requests with every state resident in HBM before each timed
    region, co-batched per (dimension, solver) class: one launch group per
    class on its own stream, rounds of `chunk` steps with device step
    counters, finished requests dropped between rounds (the server's
    schedule without arrivals and host transfers).  The requests, in arrival
    order, form `nseg` consecutive segments, one bench step each; a segment
    larger than the 150 GB budget runs in waves.  Before the first timed
    segment: the per-kernel roofline on the first wave and `warmup` untimed
    rounds of every class, then the states are loaded again.  Returns a dict
    (face_steps, ms, segment_ms, launches, roofline, waves, failed)."""
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    pool_ctx = {d: Context(d, RiemannSolverFactory.generate("HLLC"), L.PREC_SPLIT, device=local)
                for d in (2, 3)}
    bases = {j: FluxPass(pool_ctx[m.dim], m) for j, m in enumerate(pool.meshes) if m is not None}
    classes = [(d, sv) for d in (2, 3) for sv in ("Exact", "HLLC")]
    cctx, cstream = {}, {}
    for c in classes:
        cctx[c] = Context(c[0], RiemannSolverFactory.generate(c[1]), L.PREC_SPLIT, device=local)
        cstream[c] = torch.cuda.Stream(device=local)
        cctx[c].set_stream(cstream[c].cuda_stream)
    main = torch.cuda.current_stream(local)
    segments = [s for s in np.array_split(np.arange(len(reqs)), nseg) if len(s)]
    nbytes = lambda j: bases[reqs[j].mesh].clone_bytes(L.PREC_SPLIT)  # noqa: E731
    seg_ms, face_steps, launches, roof, nwaves = [], 0, 0, None, 0
    tuning = {}
    failed = set()
    first = True
    for seg in segments:
        ms_seg = 0.0
        for wave in _budget_waves(seg, nbytes):
            nwaves += 1
            inst = {}
            for j in wave:
                r = reqs[j]
                c = (pool.meshes[r.mesh].dim, r.solver)
                fp = bases[r.mesh].clone(cctx[c])
                fp.set_primitive(pool.states[r.mesh][r.state])
                inst[j] = (c, fp)
            if first:
                roof = resident_roofline(pool, reqs, inst, classes, cctx)
                # what the tuners kept for each class
                tuning = {c: roof["classes"][f"{c[0]}D {c[1]}"]["tuned"]
                          for c in classes if f"{c[0]}D {c[1]}" in roof["classes"]}
                for c in classes:
                    js = [j for j in wave if inst[j][0] == c]
                    if js and warmup:
                        g = Group(cctx[c], [inst[j][1] for j in js],
                                  [pool.dts[reqs[j].mesh][reqs[j].state] for j in js])
                        for _ in range(warmup):
                            g.step(chunk, graph=False, status=False)
                        g.close()
                torch.cuda.synchronize()
                for j, (c, fp) in inst.items():      # back to the initial states
                    fp.set_primitive(pool.states[reqs[j].mesh][reqs[j].state])
                first = False
            torch.cuda.synchronize()
            live = {c: [j for j in wave if inst[j][0] == c] for c in classes}
            left = {j: reqs[j].nsteps for j in wave}
            groups = {c: None for c in classes}
            reused = {c: 0 for c in classes}
            n0 = L.lib().sfx_launch_count()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("resident")  # the timed region, for profilers
            e0.record(main)
            for c in classes:
                cstream[c].wait_event(e0)
            while any(live.values()):
                for c in classes:
                    if groups[c] is None and live[c]:
                        groups[c] = Group(cctx[c], [inst[j][1] for j in live[c]],
                                          [pool.dts[reqs[j].mesh][reqs[j].state]
                                           for j in live[c]])
                        groups[c].set_steps([left[j] for j in live[c]])
                        t = tuning.get(c)
                        if t:
                            groups[c].set_lanes(t["lanes_per_cell"])
                            groups[c].set_face_variant(t["face_variant"])
                        reused[c] = 0
                for c in classes:
                    if groups[c] is not None:
                        groups[c].step(chunk, graph=reused[c] > 0, status=False)
                for c in classes:
                    g = groups[c]
                    if g is None:
                        continue
                    steps_left = g.get_steps()
                    st = g.status()
                    for j, k, e in zip(live[c], steps_left, st):
                        left[j] = 0 if e else int(k)
                        if e:
                            failed.add(j)
                    keep = [j for j in live[c] if left[j] > 0]
                    if len(keep) != len(live[c]):
                        g.close()
                        groups[c] = None
                        live[c] = keep
                    else:
                        reused[c] += 1
            for c in classes:
                ev = torch.cuda.Event()
                ev.record(cstream[c])
                main.wait_event(ev)
            e1.record(main)
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
            ms_seg += e0.elapsed_time(e1)
            launches += L.lib().sfx_launch_count() - n0
            face_steps += sum(pool.meshes[reqs[j].mesh].n_active_faces * reqs[j].nsteps
                              for j in wave if j not in failed)
            for c in classes:
                if groups[c] is not None:
                    groups[c].close()
            for c, fp in inst.values():
                fp.close()
        seg_ms.append(ms_seg)
    for fp in bases.values():
        fp.close()
    for c in classes:
        cctx[c].close()
    for c in pool_ctx.values():
        c.close()
    return {"face_steps": face_steps, "ms": float(sum(seg_ms)), "segment_ms": seg_ms,
            "launches": launches, "roofline": roof, "waves": nwaves, "failed": len(failed),
            "tuning": tuning}


# DRAM bytes (read + write) per active face of one launch of each split
# kernel, from one-kernel ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum) of a 300,000-cell periodic random-field mesh in 3D
# (2,396,113 faces) and a 700,000-cell one in 2D; the gathers and the per-face
# records scale with the faces, so a launch over F faces moves about F times
# these
TRAFFIC_B_PER_FACE = {("faces", 3, "Exact"): 106.8, ("faces", 3, "HLLC"): 102.0,
                      ("gradients", 3): 61.4, ("update", 3): 52.8,
                      ("faces", 2, "Exact"): 104.8, ("faces", 2, "HLLC"): 98.6,
                      ("gradients", 2): 73.3, ("update", 2): 54.2}


def split_kernel_name(role: str, solver: str) -> str:
    if role == "faces":
        return "k_group_sfaces_exact" if solver == "Exact" else "k_group_sfaces"
    return {"gradients": "k_group_sgrad", "update": "k_group_sapply"}[role]


def split_traffic(role: str, dim: int, solver: str, faces: int):
    """DRAM bytes of one launch over ``faces`` active faces, or None where no
    capture of that kernel exists"""
    key = (role, dim, solver) if role == "faces" else (role, dim)
    return TRAFFIC_B_PER_FACE[key] * faces if key in TRAFFIC_B_PER_FACE else None


def resident_roofline(pool, reqs, inst, classes, cctx):
    """per-kernel device times of every class (all of its requests in one
    launch group, CUDA events around each launch): the dominant kernel of the
    class with the most face work, and each class's figures"""
    from shadowfax_b200.hydro import Group
    peak, peak_kind = peaks()
    names = ["gradients", "faces", "update"]
    work = {c: 0 for c in classes}
    for j, (c, fp) in inst.items():
        work[c] += pool.meshes[reqs[j].mesh].n_active_faces * reqs[j].nsteps
    per_class = {}
    for c in classes:
        js = [j for j, (cc, _) in inst.items() if cc == c]
        if not js:
            continue
        g = Group(cctx[c], [inst[j][1] for j in js],
                  [pool.dts[reqs[j].mesh][reqs[j].state] for j in js])
        # the timing tuners on this class's meshes (the states are read, not
        # changed): lanes per cell of the gradient/update kernels, the face
        # kernel's variant; the kernels are then timed as tuned
        tuned = {"lanes_per_cell": int(g.tune(2)), "face_variant": int(g.tune_faces(2))}
        g.step_timed(1)
        steps = 3
        ms, nl = g.step_timed(steps)
        g.close()
        per_launch = ms / steps
        alg = {k: 0 for k in names}
        faces = 0
        for j in js:
            m = pool.meshes[reqs[j].mesh]
            b = split_kernel_bytes(m.dim, m.n_cells, m.n_faces, m.nnz)
            for k in names:
                alg[k] += b[k]
            faces += m.n_active_faces
        D = c[0]
        per_class[c] = {
            "requests": len(js), "faces": faces, "face_work_share": work[c] / sum(work.values()),
            "kernel_ms": {k: float(v) for k, v in zip(names, per_launch)},
            "achieved_gbs": {k: alg[k] / (per_launch[i] / 1e3) / 1e9 for i, k in enumerate(names)},
            "algorithmic_bytes": alg,
            "step_face_steps_per_s": faces / (per_launch.sum() / 1e3),
            "step_frac": STEP_BYTES[("split", D)] * faces / (per_launch.sum() / 1e3) / 1e9 / peak,
            "tuned": tuned}
    top_c = max(per_class, key=lambda c: work[c])
    pc = per_class[top_c]
    kms = pc["kernel_ms"]
    top = max(names, key=lambda k: kms[k])
    kname = split_kernel_name(top, top_c[1])
    D = top_c[0]
    traffic = split_traffic(top, D, top_c[1], pc["faces"])
    roof = {"bound": "hbm", "kernel": kname,
            "class": f"{D}D {top_c[1]}, {pc['requests']} requests, {pc['faces']} faces",
            "achieved": pc["achieved_gbs"][top], "peak": peak, "unit": "GB/s",
            "frac": pc["achieved_gbs"][top] / peak, "traffic": traffic,
            "traffic_note": "DRAM bytes per face from a one-kernel ncu capture of a "
                            "300,000-cell mesh of the same dimension and solver, times the "
                            "faces of this launch",
            "peak_source": f"hbm_gbs {peak_kind} (of measured)",
            "algorithmic_bytes_per_launch": pc["algorithmic_bytes"][top],
            "kernel_ms": kms,
            "note": "the exact-solver face kernel is bound by instruction issue and FP64 "
                    "latency (divergent solver paths), not by HBM",
            "step_bytes_per_face": STEP_BYTES[("split", D)],
            "step_frac": pc["step_frac"],
            "classes": {f"{c[0]}D {c[1]}": v for c, v in per_class.items()}}
    hllc = per_class.get((3, "HLLC")) or per_class.get((2, "HLLC"))
    if hllc is not None:
        roof["hllc_pass"] = {"faces_kernel_achieved_gbs": hllc["achieved_gbs"]["faces"],
                             "faces_kernel_frac": hllc["achieved_gbs"]["faces"] / peak,
                             "step_frac": hllc["step_frac"]}
    return roof


def serve_cpu_sample(pool, reqs, steps: int = 2, warmup: int = 1):
    """the reference CPU pass on the stream's first P requests (P = host
    cores, at most 48), one process per request, concurrently"""
    from shadowfax_b200.workloads import Problem
    P = min(os.cpu_count() or 1, SERVE_CPU_PROCS)
    probs = []
    for r in reqs[:P]:
        m = pool.meshes[r.mesh]
        probs.append(Problem(f"req{len(probs)}", m, pool.states[r.mesh][r.state], r.solver,
                             pool.dts[r.mesh][r.state], steps))
    cb = cpu_baseline_many(probs, steps, warmup)
    if cb is not None:
        cb["sample"] = (f"the stream's first {len(probs)} requests ({sum(p.mesh.n_cells for p in probs)}"
                        f" cells, both solvers, 2D and 3D), {warmup} warm-up + {steps} timed "
                        f"steps each, one reference process per request on {len(probs)} host cores "
                        f"concurrently (P processes, not an MPI run; value = sum of the "
                        f"per-process rates)")
    return cb


def serve_config(args, reqs, world):
    """the workload description both arms print (no GPU or pool needed)"""
    from shadowfax_b200 import workloads as wl
    n2 = sum(1 for r in reqs if r.mesh < 10)
    whole = not args.requests and args.duration >= 60.0
    span = "the whole 60 s stream" if whole else f"{reqs[-1].t:.1f} s of the 60 s stream"
    return {"workload": f"serve: request stream of {len(reqs)} Poisson arrivals at 200/s "
                        f"({span}, seed 5), {n2} 2D / {len(reqs) - n2} 3D periodic static "
                        f"meshes, N log-uniform in [1e3, 1e6] from a pool of 20 pre-tessellated "
                        f"meshes (10 log bins per dimension), random-field states, steps "
                        f"U{{10..200}}, exact/HLLC 50/50, gamma 5/3, 150 GB device budget",
            "step": f"one of {args.steps} consecutive segments of the stream's arrivals",
            "l2": "working set > L2 (no flush)",
            "parallelism": (f"{world} GPUs, whole requests per GPU by least face work"
                            if world > 1 else "1 GPU"),
            "pool_sizes": [int(x) for x in wl.serve_pool_sizes()]}


def bench_serve(args, rank, world, local, torch):
    """The request stream on this rank's GPU: the resident replay (value),
    the stream served from host memory at its arrival times (e2e, p50/p99),
    and a sample of it served by the plain FP64 pass and by the split pass
    with every request submitted at once (the split-vs-FP64 throughput ratio
    of a saturated server, and the accuracy of the split results)."""
    from shadowfax_b200 import _lib as L
    from shadowfax_b200 import workloads as wl
    all_reqs = serve_requests(args)
    owner = shard_requests(all_reqs, world)
    reqs = [r for r, o in zip(all_reqs, owner) if o == rank]
    t_build = time.time()
    used = sorted({r.mesh for r in all_reqs})
    pool = wl.serve_pool(only=set(used), cache_dir=args.pool_dir)
    t_build = time.time() - t_build
    offered = sum(pool.meshes[r.mesh].n_active_faces * r.nsteps for r in all_reqs)
    log = (lambda *a: print(*a, file=sys.stderr, flush=True)) if rank == 0 else (lambda *a: None)
    log(f"[bench] {len(all_reqs)} requests, {offered:.3e} face-steps offered; pool "
        f"{t_build:.0f} s")
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clk:
        clk.wait_first_sample()
        clk.mark("t0")
        t0 = time.time()
        res = run_resident(pool, reqs, args.steps, args.warmup, args.chunk, torch, local)
        log(f"[bench] resident {res['face_steps'] / res['ms'] * 1e3:.3e} face-steps/s "
            f"({time.time() - t0:.0f} s)")
        t0 = time.time()
        res32, launches, st32 = run_served(pool, reqs, L.PREC_SPLIT, args.chunk, False, local,
                                           tuning=res["tuning"])
        clk.mark("t1")
        log(f"[bench] served ({time.time() - t0:.0f} s)")
        time.sleep(0.3)
    split = served_summary(res32, st32)
    e2e_value, _, _ = reduce_over_ranks(1e3 * split["makespan_s"], split["face_steps"],
                                        f"cuda:{local}", world)
    # a sample served by both passes, every request submitted at once
    sub = reqs[::args.fp64_every] if args.fp64_every > 0 else []
    fp64s = splits = None
    errs, maxe, drift = [], [], []
    if sub:
        t0 = time.time()
        res64, _, st64 = run_served(pool, sub, L.PREC_FP64, args.chunk, True, local, at_once=True)
        sub32, _, sts = run_served(pool, sub, L.PREC_SPLIT, args.chunk, True, local, at_once=True,
                                   tuning=res["tuning"])
        log(f"[bench] fp64 sample {len(sub)} requests ({time.time() - t0:.0f} s)")
        fp64s, splits = served_summary(res64, st64), served_summary(sub32, sts)
        for j, (a, b) in enumerate(zip(sub32, res64)):
            if a.status or b.status:
                continue
            errs.append(l1_rel_fields(a.Q, b.Q))
            maxe.append(max_rel_fields(a.Q, b.Q))
            m = pool.meshes[sub[j].mesh]
            W0 = pool.states[sub[j].mesh][sub[j].state]
            D = m.dim
            V = m.cell_volume
            mass0 = float((W0[:, 0] * V).sum())
            en0 = float(((W0[:, D + 1] / (wl.GAMMA - 1) + 0.5 * W0[:, 0] *
                          (W0[:, 1:D + 1] ** 2).sum(1)) * V).sum())
            drift.append([abs(a.Q[:, 0].sum() - mass0) / mass0,
                          abs(a.Q[:, D + 1].sum() - en0) / en0,
                          abs(b.Q[:, 0].sum() - mass0) / mass0,
                          abs(b.Q[:, D + 1].sum() - en0) / en0])
    fp64_val, _, _ = reduce_over_ranks(1e3 * (fp64s["makespan_s"] if fp64s else 1.0),
                                       fp64s["face_steps"] if fp64s else 0, f"cuda:{local}", world)
    split_sub_val, _, _ = reduce_over_ranks(1e3 * (splits["makespan_s"] if splits else 1.0),
                                            splits["face_steps"] if splits else 0,
                                            f"cuda:{local}", world)
    # every rank's worst error (MAX over ranks of the per-field maxima)
    ev = torch.tensor([*(np.max(errs, 0) if errs else [-1.0] * 3),
                       *(np.max(maxe, 0) if maxe else [-1.0] * 3),
                       *(np.max(drift, 0) if drift else [-1.0] * 4)],
                      dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(ev, op=torch.distributed.ReduceOp.MAX)
    ev = [float(x) if x >= 0 else None for x in ev.tolist()]
    value, ms_max, fs_total = reduce_over_ranks(res["ms"], res["face_steps"], f"cuda:{local}",
                                                world)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = serve_cpu_sample(pool, all_reqs)
    h2d = sum(pool.states[r.mesh][r.state].nbytes for r in reqs)
    d2h = 2 * h2d
    if rank != 0:
        return None
    cfg = serve_config(args, all_reqs, world)
    fields = ("mass", "momentum", "energy")
    speedup = e2e_value / fp64_val if fp64s and fp64_val > 0 else None
    return {
        "metric": METRIC_SERVE, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": cfg,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "note": "the whole stream served by the request server at its arrival "
                        "times: request states from host memory, results (W and Q) to host "
                        "memory, completed face-steps over the makespan (first arrival to "
                        "last completion)"},
        "served_speedup_vs_fp64": speedup,
        "served_speedup_vs_fp64_same_sample": (split_sub_val / fp64_val
                                               if fp64s and fp64_val > 0 else None),
        "p50_latency_s": split["p50_latency_s"], "p99_latency_s": split["p99_latency_s"],
        "split_vs_fp64_error": {
            "rel_l1": dict(zip(fields, ev[0:3])), "max_rel": dict(zip(fields, ev[3:6])),
            "requests": len(errs),
            "sample": f"every {args.fp64_every}th request of the stream, run to completion "
                      f"by both passes; max over requests; max_rel = largest cell error / "
                      f"largest magnitude of the field"},
        "fp64_served": {"value": fp64_val, "unit": UNIT,
                        "sample": f"every {args.fp64_every}th request ({len(sub)} on rank 0), "
                                  f"all submitted at once to a plain-FP64 server (each request "
                                  f"stepped with its own launches)",
                        "detail": fp64s},
        "split_served_same_sample": {"value": split_sub_val, "unit": UNIT, "detail": splits},
        "conservation_max_rel_drift": {
            "split": {"mass": ev[6], "energy": ev[7]},
            "fp64": {"mass": ev[8], "energy": ev[9]},
            "note": "energy changes where get_W floors the pressure at 1e-30 and "
                    "rewrites the energy (the reference algorithm does the same)"},
        "served": split,
        "resident": {"face_steps": int(fs_total), "ms": ms_max, "waves": res["waves"],
                     "failed_requests": res["failed"],
                     "segment_ms": [round(x, 3) for x in res["segment_ms"]],
                     "chunk_steps": args.chunk,
                     "note": "value: states resident in HBM, co-batched per (dimension, "
                             "solver) class in launch groups, CUDA events per segment"},
        "roofline": res["roofline"],
        "cpu_baseline": cb,
        "gpu_launches": int(res["launches"]),
        "gpu_launches_served": int(launches),
        "pool_build_s": round(t_build, 1),
        "face_steps_offered": int(offered),
        "precision": "split: FP32 gradients/reconstruction/HLLC/p* Newton, FP64 final p* "
                     "step, exact-solver sampling, accumulation and get_W",
    }


def flux_error_by_branch(pr, device, face_variant=0):
    """one flux pass from the initial state in FP64 and in split precision
    (the benchmarked face-kernel variant): relative L1 error of the per-face
    dQ (mass, momentum, energy) over all faces and over the faces of each
    FP64 wave pattern (shock, rarefaction, near-vacuum), and the largest
    per-face error relative to the largest |dQ| of its field"""
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    out = {}
    for prec in (L.PREC_FP64, L.PREC_SPLIT):
        ctx = Context(pr.mesh.dim, RiemannSolverFactory.generate(pr.solver, pr.gamma), prec,
                      device=device)
        fp = FluxPass(ctx, pr.mesh)
        if prec == L.PREC_SPLIT:
            fp.set_face_variant(face_variant or 0)
        fp.set_primitive(pr.W0)
        grad, dQ, br, rc, _ = fp.flux_pass(pr.dt)
        fp.close()
        ctx.close()
        if rc:
            return {"status": int(rc)}
        out[prec] = (dQ, br)
    dQ64, br = out[L.PREC_FP64]
    dQ32 = out[L.PREC_SPLIT][0]
    D = pr.mesh.dim
    region = (br >> 5) & 15
    vac = ((br & 7) != 0) | (region == 11)
    masks = {"all": np.ones(len(br), bool)}
    if pr.solver == "Exact":
        masks.update({"shock": np.isin(region, [1, 2, 6, 7]) & ~vac,
                      "rarefaction": np.isin(region, [3, 4, 5, 8, 9, 10]) & ~vac,
                      "near_vacuum": vac})
    res = {}
    for name, m in masks.items():
        if not m.any():
            res[name] = {"faces": 0}
            continue
        a, b = dQ32[m], dQ64[m]
        den = np.abs(b).sum(0)
        den[1:D + 1] = np.sqrt((b[:, 1:D + 1] ** 2).sum(1)).sum()
        e = np.abs(a - b).sum(0) / np.maximum(den, 1e-300)
        mx = (np.abs(a - b) / np.maximum(np.abs(dQ64).max(0), 1e-300)).max(0)
        res[name] = {"faces": int(m.sum()), "rel_l1": {"mass": float(e[0]),
                                                       "momentum": float(e[1:D + 1].max()),
                                                       "energy": float(e[D + 1])},
                     "max_rel": float(mx.max())}
    return res


def run_reference_arm(args, rank, world):
    """--impl reference: the reference's own CPU pass on the host cores"""
    if rank != 0:
        return
    if args.workload == "serve":
        return run_reference_serve(args, world)
    pr = build_problem(args)
    # a bounded sample: 5 steps, or up to 3e6 face-steps on a small mesh
    steps = max(1, min(args.steps, max(5, int(3e6 // pr.mesh.n_active_faces))))
    from oracle.oracle import ref_binary
    if not ref_binary(pr.mesh.dim, "libm").exists():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref reference harness not built (needs the reference tree)"}))
        return
    cb = cpu_baseline(pr, steps)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * pr.mesh.n_active_faces / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": problem_text(args, pr), "solver": pr.solver,
                       "precision": "fp64"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_reference_serve(args, world=1):
    """--impl reference on the request stream: the reference CPU pass
    (oracle/_ref, the unmodified Shadowfax sources) on the host cores, one
    process per request for the stream's first P requests, each process
    --warmup untimed and --steps timed steps (a bounded sample: the reference
    has no request loop).  The meshes are made by the standalone sfx_meshgen
    program and read with numpy, so this process never loads the GPU library.
    Launched on N ranks, rank 0 alone runs it and its line carries N and the
    config the GPU arm prints at N."""
    from oracle.oracle import ref_binary
    from shadowfax_b200 import workloads as wl
    if not (ref_binary(2, "libm").exists() and ref_binary(3, "libm").exists()):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref reference harness not built (needs the reference tree)"}))
        return
    reqs = serve_requests(args)
    P = min(os.cpu_count() or 1, SERVE_CPU_PROCS)
    with tempfile.TemporaryDirectory() as td:
        pool = wl.serve_pool(only={r.mesh for r in reqs[:P]}, cache_dir=args.pool_dir or td,
                             library=False)
        cb = serve_cpu_sample(pool, reqs, args.steps, args.warmup)
    faces = sum(pool.meshes[r.mesh].n_active_faces for r in reqs[:P])
    line = {"metric": METRIC_SERVE, "value": cb["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * faces / cb["value"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": serve_config(args, reqs, world),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference's CPU flux pass on a bounded sample of the stream (its first "
                    "requests, one process each, every process stepping its request --steps "
                    "times); the meshes come from the standalone face-list builder "
                    "(sfx_meshgen), the same face lists the GPU pass gets"}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        # rank 0's host cores alone; the other ranks exit at once, so no
        # process group (and no timeout while rank 0 runs its sample)
        run_reference_arm(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    if args.workload in ("batch2d", "serve"):
        fn = bench_batch if args.workload == "batch2d" else bench_serve
        line = fn(args, rank, world, local, torch)
        if line is not None:
            print(json.dumps(line))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    pr = build_problem(args)
    mesh = pr.mesh
    prec = L.PREC_FP64 if args.precision == "fp64" else L.PREC_SPLIT
    D = mesh.dim
    ctx = Context(D, RiemannSolverFactory.generate(pr.solver, pr.gamma), prec, device=local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(pr.W0)
    faces = mesh.n_active_faces
    dt = pr.dt
    lanes = face_variant = None
    if args.precision == "split":
        # the timing tuners (they step the state; it is loaded again after):
        # lanes per cell of the gradient/update kernels, face-kernel variant
        lanes = fp.tune(dt, 3)
        face_variant = fp.tune_faces(dt, 3)
        fp.set_primitive(pr.W0)

    # a mesh whose device data fit in the L2 is timed step by step, with a
    # 256 MB write between the steps outside the timed events, so that no
    # step starts from a warm L2
    dev_bytes = L.lib().sfx_mesh_device_bytes(D, mesh.n_cells, mesh.n_faces, mesh.nnz, prec)
    flush = (torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
             if dev_bytes < L2_BYTES else None)
    with torch.cuda.stream(stream), ClockSampler(local) as clk:
        clk.wait_first_sample()
        for _ in range(args.warmup):
            fp.step(dt, 1, stats=False)
        # every measured segment starts from the initial state (the supersonic
        # random field reaches negative energies after some tens of steps)
        fp.set_primitive(pr.W0)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(1 if flush is None else args.steps)]
        clk.mark("t0")
        n_launch0 = L.lib().sfx_launch_count()
        if flush is None:
            events[0][0].record(stream)
            for _ in range(args.steps):
                fp.step(dt, 1, stats=False)
            events[0][1].record(stream)
        else:
            for e0, e1 in events:
                flush.fill_(1)
                e0.record(stream)
                fp.step(dt, 1, stats=False)
                e1.record(stream)
        n_launches = L.lib().sfx_launch_count() - n_launch0
        torch.cuda.synchronize()
        clk.mark("t1")
        time.sleep(0.3)
        ms = sum(e0.elapsed_time(e1) for e0, e1 in events)
        if world > 1:
            dist.barrier()
        st = fp.step(dt, 1)  # status check after the timed region
        assert st.status == 0, st.status
    value, ms_max, _ = reduce_over_ranks(ms, faces * args.steps, f"cuda:{local}", world)

    # per-kernel device times (events around every launch) for the roofline
    fp.set_primitive(pr.W0)
    kms, launches = fp.step_timed(dt, args.steps)
    names = ["gradients", "faces", "update"]
    per_launch = kms / args.steps
    top = int(np.argmax(per_launch))
    if args.precision == "split":
        alg = split_kernel_bytes(D, mesh.n_cells, mesh.n_faces, mesh.nnz)
        kname = split_kernel_name(names[top], pr.solver)
        traffic = split_traffic(names[top], D, pr.solver, mesh.n_active_faces)
    else:
        alg = algorithmic_bytes(D, mesh.n_cells, mesh.n_faces, mesh.nnz, args.precision)
        kname = {"gradients": "k_grad_terms + k_grad_sum", "faces": "k_faces",
                 "update": "k_apply"}[names[top]]
        traffic = None
    peak, peak_kind = peaks()
    achieved = alg[names[top]] / (per_launch[top] / 1e3) / 1e9
    step_bytes = sum(alg.values())
    roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "peak_source": f"hbm_gbs {peak_kind}",
            "algorithmic_bytes_per_launch": alg[names[top]],
            "kernel_ms": {n: float(v) for n, v in zip(names, per_launch)},
            "step_achieved_gbs": step_bytes / (ms_max / args.steps / 1e3) / 1e9,
            "step_bytes_per_face": STEP_BYTES[(args.precision, D)],
            "step_frac": STEP_BYTES[(args.precision, D)] * value / 1e9 / peak}

    # end to end through the C ABI with host buffers: per step upload W and Q
    # from host memory, one step, download W and Q
    fp.set_primitive(pr.W0)
    W0, Q0 = fp.state()
    W = W0.copy()
    Q = Q0.copy()
    nbytes = W.nbytes + Q.nbytes
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fp.set_state(W, Q)
        fp.step(dt, 1, stats=False)
        W, Q = fp.state()
    e3.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max(e2.elapsed_time(e3), wall * 1e3)
    e2e_val = faces * args.steps * world / (e2e_ms / 1e3)

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(pr)
    flux_err = (flux_error_by_branch(pr, local, face_variant)
                if args.precision == "split" and rank == 0 else None)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32/f64",
            "data": "synthetic",
            "config": {"workload": problem_text(args, pr),
                       "solver": pr.solver, "precision": args.precision,
                       "lanes_per_cell": lanes, "face_variant": face_variant,
                       "l2": ("working set > L2 (no flush)" if flush is None else
                              "L2 flushed between steps (256 MB write outside the timed "
                              "events; step times summed)"),
                       "parallelism": f"replicas x{world}"},
            "clocks": clk.summary(),
            "roofline": roof,
            "cpu_baseline": cb,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": int(n_launches),
            "split_vs_fp64_face_flux_error": flux_err,
        }
        print(json.dumps(line))
    fp.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
