"""Benchmark of the B200 flux pass (one JSON line on rank 0).

Workload (N=1): the 3D Sedov-type blast on a static Voronoi mesh of 262,144
generators uniform in the reflective unit cube (seed 2), gamma 5/3, HLLC
solver, global CFL-0.4 time step; a "step" is one full pass of the hot path
(gradients -> face fluxes -> update_Q/get_W) over the mesh.  The metric is
face-steps per second (one nonzero-area face processed in one time step,
with its share of the gradient and update work).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|split]

Timing: CUDA events on the stream the library launches on, barrier +
synchronize on both sides, max over ranks; W untimed warm-up steps.  The
step's working set (about 300 MB: faces, cells, gradients, per-face fluxes)
is larger than the 126 MB L2, so no separate L2 flush is done.

N>1: every rank runs its own replica of the mesh (independent meshes, no
data-path collective): weak scaling.

--impl reference times the reference's own CPU flux pass (the unmodified
Shadowfax sources built into oracle/_ref) on the host cores on the same mesh.
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
UNIT = "face-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    ap.add_argument("--n", type=int, default=N_GEN, help="generators (default: config size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="sedov3d", choices=["sedov3d", "batch2d"],
                    help="sedov3d: config 2 on one mesh; batch2d: config 4, 1,024 meshes")
    ap.add_argument("--meshes", type=int, default=1024, help="batch2d: number of meshes")
    return ap.parse_args()


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


def build_problem(n: int):
    from shadowfax_b200 import workloads as wl
    return wl.sedov3d(n=n, seed=SEED, solver="HLLC")


def cpu_baseline(pr, steps: int = 3):
    """reference CPU pass (oracle/_ref, unmodified Shadowfax sources), one
    core, on the same mesh for a bounded number of steps"""
    from oracle.oracle import Params, ref_binary, run_reference
    exe = ref_binary(3, "libm")
    if not exe.exists():
        return None
    p = Params(solver=pr.solver, gamma=pr.gamma, use_libm_pow=True)
    r = run_reference(pr.mesh, p, pr.dt, steps + 1, pr.W0, pow_kind="libm")
    secs = float(np.sum(r["step_seconds"][1:]))
    value = pr.mesh.n_active_faces * steps / secs
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{steps} timed steps (+1 warm-up) of the full {pr.mesh.n_cells}-cell "
                      f"mesh, reference VorCell/VorFace/HLLC loops, 1 MPI rank (single thread)"}


def cpu_baseline_many(probs, steps: int = 2):
    """reference CPU pass on a sample of the batch: one mesh per process, as
    many processes as host cores, run concurrently (the reference has no
    threads; independent meshes are its best case)"""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle import Params, ref_binary, run_reference
    if not ref_binary(2, "libm").exists():
        return None
    P = os.cpu_count() or 1
    sample = probs[:P]

    def one(pr):
        p = Params(solver=pr.solver, gamma=pr.gamma, use_libm_pow=True)
        r = run_reference(pr.mesh, p, pr.dt, steps + 1, pr.W0, pow_kind="libm")
        return pr.mesh.n_active_faces * steps, float(np.sum(r["step_seconds"][1:]))

    with ThreadPoolExecutor(max_workers=P) as ex:
        res = list(ex.map(one, sample))
    work = sum(w for w, _ in res)
    secs = max(s for _, s in res)
    return {"value": work / secs, "unit": UNIT, "cores": P, "kind": "reference",
            "sample": f"{len(sample)} meshes of the batch ({sum(p.mesh.n_cells for p in sample)} "
                      f"cells), {steps} timed steps each, one reference process per mesh on "
                      f"{P} host cores concurrently (P processes, not an MPI run)"}


def bench_batch(args, rank, world, local, torch):
    """config 4: many independent 2D meshes, HLLC, each at its own CFL dt.
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
        e0.record(stream)
        grp.step(args.steps, graph=True, status=False)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark("t1")
        time.sleep(0.3)
        ms = e0.elapsed_time(e1)
        st = grp.step(1, graph=False)
        assert np.all(st == 0), st
    t = torch.tensor([ms], device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    value = faces * args.steps * world / (ms_max / 1e3)
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
                       "lanes_per_cell": lanes, "l2": "working set > L2 (no flush)",
                       "parallelism": f"replicas x{world}", "mesh_build_s": round(t_build, 1)},
            "clocks": clk.summary(),
            "fp64_per_mesh": {"value": fp64_value, "unit": UNIT, "steps": base_steps,
                              "launch": "3 launches per mesh per step, plain FP64"},
            "speedup_vs_fp64_per_mesh": value / fp64_value,
            "split_vs_fp64_max_rel_l1_mass_energy": max(acc) if acc else None,
            "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s",
                         "peak_source": f"hbm_gbs {peak_kind}",
                         "step_bytes_per_face": 92,
                         "achieved": 92 * value / 1e9, "frac": 92 * value / 1e9 / peak,
                         "note": "bytes per face-step of the split pass, 2D (algorithmic)"},
            "cpu_baseline": cb,
            "gpu_launches": 3 * args.steps,
        }
    grp.close()
    for fp in members:
        fp.close()
    ctx.close()
    return line


def run_reference_arm(args, rank, world):
    """--impl reference: the reference's own CPU pass on the host cores"""
    if rank != 0:
        return
    pr = build_problem(args.n)
    steps = max(1, min(args.steps, 5))
    from oracle.oracle import ref_binary
    if not ref_binary(3, "libm").exists():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref reference harness not built (needs the reference tree)"}))
        return
    cb = cpu_baseline(pr, steps)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * pr.mesh.n_active_faces / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"sedov3d HLLC, {pr.mesh.n_cells} generators, "
                                   f"{pr.mesh.n_active_faces} faces, reflective unit cube",
                       "solver": "HLLC", "precision": "fp64"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_env()
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    torch.cuda.set_device(local)
    if args.workload == "batch2d":
        line = bench_batch(args, rank, world, local, torch)
        if line is not None:
            print(json.dumps(line))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    pr = build_problem(args.n)
    mesh = pr.mesh
    prec = L.PREC_FP64 if args.precision == "fp64" else L.PREC_SPLIT
    ctx = Context(3, RiemannSolverFactory.generate(pr.solver, pr.gamma), prec, device=local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(pr.W0)
    faces = mesh.n_active_faces
    dt = pr.dt
    lanes = None
    if args.precision == "split":
        lanes = fp.tune(dt, 3)     # lanes per cell for the gradient/update kernels
        fp.set_primitive(pr.W0)

    with torch.cuda.stream(stream), ClockSampler(local) as clk:
        clk.wait_first_sample()
        for _ in range(args.warmup):
            fp.step(dt, 1, stats=False)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clk.mark("t0")
        e0.record(stream)
        for _ in range(args.steps):
            fp.step(dt, 1, stats=False)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark("t1")
        time.sleep(0.3)
        ms = e0.elapsed_time(e1)
        if world > 1:
            dist.barrier()
        st = fp.step(dt, 1)  # status check after the timed region
        assert st.status == 0, st.status
    t = torch.tensor([ms], device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = faces * args.steps * world / (ms_max / 1e3)

    # per-kernel device times (events around every launch) for the roofline
    kms, launches = fp.step_timed(dt, args.steps)
    names = ["gradients", "faces", "update"]
    per_launch = kms / args.steps
    top = int(np.argmax(per_launch))
    alg = algorithmic_bytes(3, mesh.n_cells, mesh.n_faces, mesh.nnz, args.precision)
    peak, peak_kind = peaks()
    achieved = alg[names[top]] / (per_launch[top] / 1e3) / 1e9
    step_bytes = sum(alg.values())
    roof = {"bound": "hbm", "kernel": f"k_{names[top]}", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "traffic": None,
            "peak_source": f"hbm_gbs {peak_kind}",
            "algorithmic_bytes_per_launch": alg[names[top]],
            "kernel_ms": {n: float(v) for n, v in zip(names, per_launch)},
            "step_achieved_gbs": step_bytes / (ms_max / args.steps / 1e3) / 1e9}

    # end to end through the C ABI with host buffers: per step upload W and Q
    # from host memory, one step, download W and Q
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
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32/f64",
            "data": "synthetic",
            "config": {"workload": f"sedov3d HLLC, {mesh.n_cells} generators (seed {SEED}), "
                                   f"{faces} faces, reflective unit cube, CFL-0.4 dt",
                       "solver": pr.solver, "precision": args.precision,
                       "lanes_per_cell": lanes,
                       "l2": "working set > L2 (no flush)",
                       "parallelism": f"replicas x{world}"},
            "clocks": clk.summary(),
            "roofline": roof,
            "cpu_baseline": cb,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": 3 * args.steps,
        }
        print(json.dumps(line))
    fp.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
