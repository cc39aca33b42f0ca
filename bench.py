#!/usr/bin/env python
"""Benchmark of the B200 LBM step on the 256^3 gravity-down scene.

Workload (one "step" = one worker tick of src/worker.js:96-100: Sim.step,
absorbDeadCells, RigidSphere.step): 256x256x256 grid, FP32, walls on every
face, liquid below a seeded +-0.5-cell sinusoidal interface at y = 96, tau 0.6,
tauPhi 0.8, sigma 1e-3, W 4, rhoL/rhoG = 10, g = -1e-5, a density-2 sphere of
radius 24 at (128, 200, 128).  Synthetic data; the state (5.3 GB) is far larger
than L2, so no flush is needed between steps.

Metric: MLUPS counting every cell of the grid each step (test/bench.mjs:28-29).
  value  -- K device-resident steps (lbm_run_coupled), CUDA events on the
            library's stream, max over ranks, all ranks' cells summed.
  e2e    -- the public Python API as src/worker.js drives it: per step
            sim.step / absorbDeadCells / RigidSphere.step (sphere state and plan
            up, impulses down), and the RG8 volume read back every 2 steps.

`python bench.py --impl reference` times the CPU restatement of the reference's
step (oracle/, OpenMP over the host's cores) on the same scene.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "claude-vibe-code-raytracing_b200")
for _p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "D3Q27+D3Q7 MLUPS (all cells per step), 256^3 plain FP32"
UNIT = "MLUPS"
BYTES_PER_CELL = {"f32": 313, "f16": 177, "bf16": 177, "f64": 626}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f64"])
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--rows", type=int, default=0)
    ap.add_argument("--zchunk", type=int, default=0)
    ap.add_argument("--workload", default="scene",
                    choices=["scene", "batch", "serve", "precision", "render", "phases"],
                    help="scene: the 256^3 line (default); batch: 64 seeded scenes stepped together; "
                         "serve: a Poisson request stream through the continuous-batching server; "
                         "precision: FP32/FP16/BF16 storage against an FP64 run; "
                         "render: the raymarcher, 1920x1080 frames of the 256^3 scene; "
                         "phases: test/bench_phases.mjs, the seven Sim phases timed one by one")
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without its fp16 / batch / served objects")
    return ap.parse_args()


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def max_over_ranks(v, ws, local):
    if ws == 1:
        return v
    from b200lbm import placement
    return placement.max_over_ranks(v)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        sm = [num(r[1]) for r in rows]
        mx = max(num(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(size, storage):
    """DRAM bytes per fused-kernel launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(p))
        return d.get(f"{storage}_{size}")
    except Exception:
        return None


def scene_config(size, storage, ws):
    """The workload description both arms (this library and --impl reference) print."""
    return {"workload": f"gravity-down pool {size}^3 with a density-2 sphere r={24 * size // 256}",
            "grid": [size] * 3, "storage": storage, "parallelism": f"replicas x{ws}",
            "l2": "state > 126 MB L2, no flush needed"}


def cpu_baseline(size, steps, threads=None):
    """The oracle (CPU restatement of src/sim.js + src/solid.js) on the same scene,
    OpenMP over the host's cores; `steps` timed steps after one warm-up."""
    import scenes
    from oracle import oracle
    threads = threads or os.cpu_count()
    sim, sol = scenes.cfg2(oracle.OracleSim, oracle.OracleSphere, n=size)
    sim.set_threads(threads)
    scenes.substep(sim, sol)
    t0 = time.perf_counter()
    for _ in range(steps):
        scenes.substep(sim, sol)
    dt = (time.perf_counter() - t0) / steps
    n = size ** 3
    return {"value": n / dt * 1e-6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} timed steps (+1 warm-up) of the {size}^3 scene, "
                      f"{dt * 1e3:.0f} ms/step, oracle/lbm_oracle.c with OpenMP"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    size = args.size
    budget_s = 150.0
    import scenes
    from oracle import oracle
    threads = os.cpu_count()
    sim, sol = scenes.cfg2(oracle.OracleSim, oracle.OracleSphere, n=size)
    sim.set_threads(threads)
    # the requested warm-up steps (a CPU step of the full scene takes seconds:
    # past 3 steps the warm-up stops after about a minute; the line reports
    # how many ran)
    warm, tw = 0, time.perf_counter()
    while warm < args.warmup:
        scenes.substep(sim, sol)
        warm += 1
        if warm >= 3 and time.perf_counter() - tw > 60.0:
            break
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        scenes.substep(sim, sol)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = (time.perf_counter() - t0) / done
    v = size ** 3 / dt * 1e-6
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": done, "warmup": warm, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 math, f32 storage",
        "data": "synthetic",
        "config": scene_config(size, "f32", args.gpus),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{done} of {args.steps} steps of the {size}^3 scene "
                                   f"(bounded to ~{budget_s:.0f} s), CPU restatement of the "
                                   "reference with OpenMP; the reference JS needs Node, absent here"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _shape_name(rows, zchunk):
    """'4x32' for the plain form; a suffix names the compact-ring forms:
    'c' register loads, 'a' per-thread async copies, 's' bulk-staged rows,
    't' tensor-map (TMA) staged rows, 'p' register loads behind tensor
    prefetches into L2."""
    form = "s" if rows & 0x100 else "c" if rows & 0x400 else "a" if rows & 0x800 else \
        "t" if rows & 0x1000 else "p" if rows & 0x2000 else ""
    return f"{rows & 0xff}{form}x{zchunk}"


def batch_result(args, dev, ws=1, rank=0, steps=100):
    """64 seeded scenes of mixed sizes (FP16 storage) stepped together: one
    persistent fused launch per step, the steps replayed as a CUDA graph, tile
    shape from the autotuner; beside it the same scenes one after another.
    With N ranks each GPU takes whole scenes (placement.shard by cells); the
    result counts all ranks' cells over the slowest rank's time.  The batched
    fused kernel's roofline: 177 B per interior cell of every scene over its
    CUDA-event time (lbm_batch_time_fused)."""
    import torch

    from b200lbm import Batch, autotune, placement, workloads
    torch.cuda.set_device(dev)
    storage = "f16" if args.storage == "f32" else args.storage
    specs = workloads.scene_specs(args.scenes, seed=0)
    specs = placement.shard(specs, ws, workloads.cells)[rank]
    scenes = [workloads.build(sp, storage, dev) for sp in specs]
    cells = sum(sim.n for sim, _ in scenes)
    interior = sum((sim.nx - 2) * (sim.ny - 2) * (sim.nz - 2) for sim, _ in scenes)
    K = steps
    with Batch(scenes) as batch:
        batch.run(2)
        rows, zchunk, timings = autotune.tune(batch, [sp["dims"] for sp in specs], storage, force=True)
        # an even count: the timed run then starts at the ping-pong parity the
        # 2-step graph was captured at, so it is not recaptured while timed
        batch.run(max(2, args.warmup + args.warmup % 2))
        torch.cuda.synchronize(dev)
        clocks = Clocks(dev)
        clocks.start()
        l0 = batch.launch_count()
        t0 = time.perf_counter()
        batch.run(K, use_graph=True)
        dt_graph = time.perf_counter() - t0
        clk = clocks.stop()
        t0 = time.perf_counter()
        batch.run(K, use_graph=False)
        dt_eager = time.perf_counter() - t0
        fused = batch.launch_count() - l0
        fused_ms = batch.time_fused(rows, zchunk, reps=10)
    t0 = time.perf_counter()
    for sim, solid in scenes:
        sim.run_coupled(solid, K)
    dt_seq = time.perf_counter() - t0
    for sim, _ in scenes:
        sim.close()
    if ws > 1:
        cells = placement.sum_over_ranks(cells)
        dt_graph, dt_eager, dt_seq = (placement.max_over_ranks(v) for v in (dt_graph, dt_eager, dt_seq))
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL[storage] * interior / (fused_ms * 1e-3) / 1e9
    return {
        "mlups": cells * K / dt_graph / 1e6, "unit": UNIT, "steps": K, "storage": storage,
        "ms_per_step": dt_graph / K * 1e3, "cells": cells, "scenes": args.scenes,
        "eager_mlups": cells * K / dt_eager / 1e6,
        "sequential_mlups": cells * K / dt_seq / 1e6,
        "batched_fused_launches": fused,
        "tile": _shape_name(rows, zchunk),
        "timings_ms": {_shape_name(r, z): t for (r, z), t in timings.items()},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "kernel": kernel_name(rows, batch=True),
                     "kernel_ms": fused_ms, "bytes_per_cell": BYTES_PER_CELL[storage],
                     "cells_per_launch": interior},
        "timing": "wall clock around whole runs (host work included), after a synchronize; "
                  "kernel_ms by CUDA events (rank 0's scenes)",
        "clocks": clk,
    }


def run_batch(args, dev, ws=1, rank=0):
    r = batch_result(args, dev, ws, rank, steps=args.steps if args.steps != 2000 else 100)
    if rank != 0:
        return
    line = {
        "metric": f"batched MLUPS, {args.scenes} seeded scenes of mixed sizes", "value": r["mlups"],
        "unit": UNIT, "n_gpus": ws, "steps": r["steps"], "higher_is_better": True, "dtype": r["storage"],
        "data": "synthetic", "scaling": "strong",
        "config": {"workload": f"{args.scenes} scenes, edges U[32,160], pool 30-60% of ny, 1-3 spheres",
                   "parallelism": f"whole scenes per GPU x{ws}", "cells": r["cells"], "storage": r["storage"],
                   "tile": r["tile"], "timings_ms": r["timings_ms"]},
        **{k: r[k] for k in ("ms_per_step", "eager_mlups", "sequential_mlups", "batched_fused_launches",
                             "roofline", "timing", "clocks")},
    }
    print(json.dumps(line), flush=True)


def serve_result(args, dev, ws=1, rank=0):
    """A seeded Poisson request stream (20/s, mixed sizes, 10% at 256^3,
    500-5000 steps, a frame every 20 steps) through the continuous-batching
    server (FP16 storage), and the same requests one at a time with plain
    FP32 per-scene launches."""
    import torch

    from b200lbm import placement, serve, workloads
    torch.cuda.set_device(dev)
    reqs = workloads.request_stream(args.requests, seed=0)
    storage = "f16" if args.storage == "f32" else args.storage
    clocks = Clocks(dev)
    clocks.start()
    if ws > 1:
        # one stream shared by every rank's server: each GPU claims the next
        # request when it has room (placement.ClaimQueue over the group's store)
        claims = placement.ClaimQueue(reqs, store=placement.default_store(), key="bench-serve")
        barrier(ws)
        rep = serve.Server(storage=storage, device=dev).run(None, realtime=True, claims=claims)
        mine = set(rep["claimed"])
        reqs = [r for r in reqs if r["rid"] in mine]
    else:
        rep = serve.Server(storage=storage, device=dev).run(reqs, realtime=True)
    clk = clocks.stop()
    seq = serve.sequential(reqs, storage="f32", device=dev)
    if ws > 1:
        for r in (rep, seq):
            r["scene_steps"] = placement.sum_over_ranks(r["scene_steps"])
            r["wall_s"] = placement.max_over_ranks(r["wall_s"])
            r["scene_steps_per_s"] = r["scene_steps"] / r["wall_s"]
    return {
        "scene_steps_per_s": rep["scene_steps_per_s"], "unit": "scene-steps/s", "storage": storage,
        "frame_interval_s": rep["frame_interval_s"], "ttff_s": rep["ttff_s"],
        "workload": f"{args.requests} requests, Poisson 20/s, sizes U[32,160]^3 + 10% 256^3, "
                    "500-5000 steps, RG8 frame every 20 steps",
        "served": rep, "sequential_plain_f32": seq,
        "speedup_vs_sequential": rep["scene_steps_per_s"] / seq["scene_steps_per_s"],
        "clocks": clk,
    }


def run_serve(args, dev, ws=1, rank=0):
    r = serve_result(args, dev, ws, rank)
    if rank != 0:
        return
    line = {
        "metric": "served scene-steps/s, Poisson request stream of mixed-size scenes",
        "value": r["scene_steps_per_s"], "unit": "scene-steps/s", "n_gpus": ws,
        "higher_is_better": True, "dtype": r["storage"], "data": "synthetic",
        "config": {"workload": r["workload"], "storage": r["storage"]},
        **{k: r[k] for k in ("served", "sequential_plain_f32", "speedup_vs_sequential", "clocks")},
    }
    print(json.dumps(line), flush=True)


def run_precision(args, dev):
    """The 256^3 scene in FP64 storage (the GPU error reference) and in FP32,
    FP16 and BF16 storage from the same initial state: field errors, sphere
    drift and the FP64 sums of mass and phase after the same steps."""
    import torch

    import scenes
    from b200lbm import RigidSphere, Sim
    torch.cuda.set_device(dev)
    size = args.size
    steps = args.steps if args.steps != 2000 else 1000
    out = {}

    def run(storage):
        sim, sol = scenes.cfg2(lambda *a: Sim(*a, storage=storage, device=dev), RigidSphere, n=size)
        m0 = (float(np.sum(sim.field64("rho"))), float(np.sum(sim.field64("phi"))))
        t0 = time.perf_counter()
        sim.run_coupled(sol, steps)
        dt = time.perf_counter() - t0
        f = {k: sim.field64(k) for k in ("phi", "rho", "ux", "uy", "uz")}
        m1 = (float(np.sum(f["rho"])), float(np.sum(f["phi"])))
        c = np.array([sol.cx, sol.cy, sol.cz])
        sim.close()
        return f, c, m0, m1, dt

    ref, cref, m0r, m1r, _ = run("f64")
    u_ref = np.concatenate([ref["ux"], ref["uy"], ref["uz"]])
    for st in ("f32", "f16", "bf16"):
        f, c, m0, m1, dt = run(st)
        e = {}
        for k in ("phi", "rho"):
            d = f[k] - ref[k]
            e[k] = {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref[k])), "linf": float(np.abs(d).max())}
        u = np.concatenate([f["ux"], f["uy"], f["uz"]])
        d = u - u_ref
        e["u"] = {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(u_ref)),
                  "linf_over_umax": float(np.abs(d).max() / np.abs(u_ref).max())}
        e["sphere_drift_cells"] = float(np.abs(c - cref).max())
        e["mass_drift"] = (m1[0] - m0[0]) / m0[0]
        e["phase_drift"] = (m1[1] - m0[1]) / m0[1]
        e["mlups"] = size ** 3 * steps / dt / 1e6
        out[st] = e
    line = {
        "metric": f"storage-form error vs FP64 GPU run, {size}^3 gravity-down pool, {steps} steps",
        "value": out["f16"]["phi"]["rel_l2"], "unit": "rel-L2 of phi (FP16 storage)", "n_gpus": 1,
        "higher_is_better": False, "data": "synthetic", "steps": steps,
        "fp64_mass_drift": (m1r[0] - m0r[0]) / m0r[0], "fp64_phase_drift": (m1r[1] - m0r[1]) / m0r[1],
        "forms": out,
        "timing": "mlups here is wall clock of Sim.run_coupled incl. host set-up, not the bench figure",
    }
    print(json.dumps(line), flush=True)


def run_render(args, dev):
    """Frames of the reference's renderer (its fragment shader, one CUDA
    thread per pixel) over the 256^3 scene's RG8 volume: pack + render per
    frame, CUDA events on the library's stream; beside it the C restatement
    of the shader on one host core for one frame."""
    import torch

    import scenes
    from b200lbm import RigidSphere, Sim
    from b200lbm._capi import LbmCamera, LbmSphere, check, lib
    torch.cuda.set_device(dev)
    size, W, H = args.size, 1920, 1080
    sim, sol = scenes.cfg2(lambda *a: Sim(*a, storage=args.storage, device=dev), RigidSphere, n=size)
    sim.run_coupled(sol, 20)
    L = lib()
    cam = LbmCamera()
    L.lbm_camera_default(C.byref(cam))
    sph = (LbmSphere * 1)()
    sol.to_c(sph[0])
    vol = torch.empty(2 * sim.n, dtype=torch.uint8, device=f"cuda:{dev}")
    img = torch.empty((H, W, 4), dtype=torch.uint8, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(L.lbm_stream(sim.handle), device=dev)
    h = sim.handle

    def frame():
        check(h, L.lbm_pack_volume_device(h, C.c_void_p(vol.data_ptr())))
        rc = L.lbm_render_volume(C.c_void_p(vol.data_ptr()), sim.nx, sim.ny, sim.nz, sph, C.byref(cam), W, H,
                                 C.c_void_p(img.data_ptr()), L.lbm_stream(h))
        assert rc == 0

    for _ in range(3):
        frame()
    K = args.steps if args.steps != 2000 else 50
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        frame()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / K
    from oracle import oracle
    host = sim.packVolume().copy()
    t0 = time.perf_counter()
    oracle.render(host, sim.nx, sim.ny, sim.nz, (sol.cx, sol.cy, sol.cz, sol.r), width=W, height=H)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    sim.close()
    line = {
        "metric": f"rendered frames/s, {W}x{H}, {size}^3 RG8 volume (pack + raymarch)", "value": 1e3 / ms,
        "unit": "frames/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic", "dtype": "f32",
        "ms_per_frame": ms, "steps": K,
        "config": {"workload": f"gravity-down pool {size}^3, reference start view, 48 march steps",
                   "width": W, "height": H},
        "cpu_baseline": {"value": 1e3 / cpu_ms, "unit": "frames/s", "cores": 1, "kind": "port",
                         "sample": "one frame of oracle/render_oracle.c (the shader restated in C)"},
    }
    print(json.dumps(line), flush=True)


PHASES = ("retagCells", "handleFreshCells", "computePhiGradients", "collidePhase", "streamPhase",
          "collideHydro", "streamHydroAndMacro")


def _call_phase(sim, sol, name):
    if name in ("retagCells", "streamHydroAndMacro"):
        getattr(sim, name)(sol)
    elif name == "handleFreshCells":
        sim.handleFreshCells(sol)
    else:
        getattr(sim, name)()


def run_phases(args, dev):
    """test/bench_phases.mjs on the device: the seven Sim phases called one by
    one through the public API (each timed with CUDA events on the handle's
    stream), after 20 coupled warm-up steps, at the harness's 40x28x40 and at
    256^3; beside them the fused step (Sim.step) on the same state and, at
    40x28x40, the oracle's phases on one host thread."""
    import torch

    import scenes
    from b200lbm import RigidSphere, Sim
    from b200lbm._capi import lib
    from oracle import oracle

    torch.cuda.set_device(dev)
    out = {}
    for label, build, reps in (("40x28x40", lambda S, R: scenes.bench(S, R), 80),
                               (f"{args.size}^3", lambda S, R: scenes.cfg2(S, R, n=args.size), 10)):
        sim, sol = build(Sim, RigidSphere)
        for _ in range(20):
            scenes.substep(sim, sol)
        for p in PHASES:  # one untimed round: the phase path's scratch is allocated on first use
            _call_phase(sim, sol, p)
        sim.synchronize()
        stream = torch.cuda.ExternalStream(lib().lbm_stream(sim.handle))
        ms = {p: 0.0 for p in PHASES + ("step (fused)",)}
        for _ in range(reps):
            for p in PHASES + ("step (fused)",):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if p == "step (fused)":
                    sim.step(sol)
                else:
                    _call_phase(sim, sol, p)
                e1.record(stream)
                e1.synchronize()
                ms[p] += e0.elapsed_time(e1)
        per = {p: v / reps for p, v in ms.items()}
        total = sum(per[p] for p in PHASES)
        out[label] = {"ms": per, "phases_total_ms": total,
                      "share": {p: per[p] / total for p in PHASES},
                      "mlups_phases": sim.n / (total * 1e-3) * 1e-6,
                      "mlups_fused": sim.n / (per["step (fused)"] * 1e-3) * 1e-6}
        sim.close()
    o, osol = scenes.bench(oracle.OracleSim, oracle.OracleSphere)
    for _ in range(20):
        scenes.substep(o, osol)
    cpu = {p: 0.0 for p in PHASES}
    reps = 10
    for _ in range(reps):
        for p in PHASES:
            t0 = time.perf_counter()
            _call_phase(o, osol, p)
            cpu[p] += (time.perf_counter() - t0) * 1e3
    cpu = {p: v / reps for p, v in cpu.items()}
    line = {
        "metric": "per-phase ms of one step (test/bench_phases.mjs breakdown)",
        "value": out[f"{args.size}^3"]["phases_total_ms"], "unit": "ms per step (seven phases)",
        "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "test/bench_phases.mjs scene (40x28x40) and the gravity-down pool "
                               f"{args.size}^3, 20 warm-up ticks, phases called one by one"},
        "gpu": out,
        "cpu_baseline": {"ms": cpu, "total_ms": sum(cpu.values()), "cores": 1, "kind": "port",
                         "sample": f"40x28x40, {reps} repetitions of the seven oracle phases"},
    }
    print(json.dumps(line), flush=True)


def kernel_name(rows, batch=False):
    """The fused kernel a tile shape launches."""
    pipe = bool(rows & (0x100 | 0x400 | 0x800 | 0x1000 | 0x2000))
    return ("k_fused_pipe" if pipe else "k_fused_step" if not batch else "k_fused_batch") + \
        ("_batch" if batch and pipe else "")


def scene_form(args, storage, steps, dev, ws, local):
    """The 256^3 scene in another storage form: `steps` device-resident steps
    after the warm-up, CUDA events on the library's stream (max over ranks),
    and the fused kernel's roofline."""
    import torch

    import scenes
    from b200lbm import RigidSphere, Sim
    from b200lbm._capi import LbmSphere, check, lib
    L = lib()
    size = args.size
    sim, sol = scenes.cfg2(lambda *a: Sim(*a, storage=storage, device=dev), RigidSphere, n=size)
    h = sim.handle
    if args.rows:
        check(h, L.lbm_set_fused_config(h, args.rows, args.zchunk or 32))
    rows, zchunk = sim.fused_config()
    sph = (LbmSphere * 1)()
    sol.to_c(sph[0])
    stream = torch.cuda.ExternalStream(L.lbm_stream(h), device=dev)
    check(h, L.lbm_run_coupled(h, sph, 1, args.warmup, 0, None))
    check(h, L.lbm_fused_timing(h, 1))
    barrier(ws)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    check(h, L.lbm_run_coupled(h, sph, 1, steps, 0, None))
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(ev0.elapsed_time(ev1), ws, local)
    fms, fn = C.c_double(), C.c_int64()
    check(h, L.lbm_fused_timing_query(h, C.byref(fms), C.byref(fn)))
    sim.close()
    per_launch = fms.value / max(1, fn.value)
    interior = (size - 2) ** 3
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL[storage] * interior / (per_launch * 1e-3) / 1e9
    return {"storage": storage, "mlups": ws * size ** 3 * steps / (ms * 1e-3) * 1e-6, "unit": UNIT,
            "steps": steps, "ms_per_step": ms / steps, "tile": _shape_name(rows, zchunk),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "kernel": kernel_name(rows),
                         "kernel_ms": per_launch, "bytes_per_cell": BYTES_PER_CELL[storage],
                         "cells_per_launch": interior}}


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.workload != "scene":
        if args.workload in ("precision", "render", "phases"):
            if rank == 0:
                {"precision": run_precision, "render": run_render,
                 "phases": run_phases}[args.workload](args, local)
        else:
            {"batch": run_batch, "serve": run_serve}[args.workload](args, local, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch

    import scenes
    from b200lbm import RigidSphere, Sim
    from b200lbm._capi import LbmSphere, check, lib

    dev = local
    torch.cuda.set_device(dev)
    size = args.size
    L = lib()

    sim, sol = scenes.cfg2(lambda *a: Sim(*a, storage=args.storage, device=dev), RigidSphere, n=size)
    h = sim.handle
    if args.rows:
        check(h, L.lbm_set_fused_config(h, args.rows, args.zchunk or 32))
    sim._sync()
    rows, zchunk = sim.fused_config()
    sph = (LbmSphere * 1)()
    sol.to_c(sph[0])
    stream = torch.cuda.ExternalStream(L.lbm_stream(h), device=dev)

    # warm-up through the device loop
    check(h, L.lbm_run_coupled(h, sph, 1, args.warmup, 0, None))

    # ---------------- timed region: K device-resident steps
    n_cells = size ** 3
    interior = (size - 2) ** 3
    clocks = Clocks(dev)
    c0 = C.c_int64()
    check(h, L.lbm_launch_count(h, C.byref(c0)))
    check(h, L.lbm_fused_timing(h, 1))
    barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    rc = L.lbm_run_coupled(h, sph, 1, args.steps, 0, None)
    if L.lbm_checked_build():
        rec = (C.c_int64 * 4)()
        L.lbm_fault_record(h, rec)
        print("fault record", list(rec), file=sys.stderr, flush=True)
    check(h, rc)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(ws)
    ms = ev0.elapsed_time(ev1)
    fused_ms = C.c_double()
    fused_n = C.c_int64()
    check(h, L.lbm_fused_timing_query(h, C.byref(fused_ms), C.byref(fused_n)))
    check(h, L.lbm_fused_timing(h, 0))
    c1 = C.c_int64()
    check(h, L.lbm_launch_count(h, C.byref(c1)))
    ms_max = max_over_ranks(ms, ws, local)
    value = ws * n_cells * args.steps / (ms_max * 1e-3) * 1e-6
    sol.from_c(sph[0])

    # roofline of the fused kernel
    peak, peak_kind = measured_peak()
    per_launch_ms = fused_ms.value / max(1, fused_n.value)
    bpc = BYTES_PER_CELL[args.storage]
    achieved = bpc * interior / (per_launch_ms * 1e-3) / 1e9
    traffic = ncu_traffic(size, args.storage)

    # ---------------- e2e through the public API (worker.js cadence)
    e2e_steps = min(args.e2e_steps, args.steps)
    # two page-locked frame buffers, filled alternately: on a frame step the
    # fused kernel packs the RG8 volume (stepFrame) and the copy runs while the
    # next steps do; every copy has landed before the clock stops
    frames = [sim.frameBuffer(), sim.frameBuffer()]
    nframe = 0
    substeps = 2
    torch.cuda.synchronize(dev)
    barrier(ws)
    x0 = (C.c_uint64(), C.c_uint64())
    check(h, L.lbm_transfer_bytes(h, C.byref(x0[0]), C.byref(x0[1])))
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        if (s + 1) % substeps == 0:
            if nframe >= 2:
                sim.waitFrameSlot()  # frames[nframe % 2] (two frames back) has landed: the consumer takes it
            sim.stepFrame(sol, frames[nframe % 2])
            nframe += 1
        else:
            sim.step(sol)
        sol.absorbDeadCells(sim)
        sol.step(1.0, sim.gravity)
    sim.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, ws, local)
    e2e_value = ws * n_cells * e2e_steps / e2e_s * 1e-6
    x1 = (C.c_uint64(), C.c_uint64())
    check(h, L.lbm_transfer_bytes(h, C.byref(x1[0]), C.byref(x1[1])))
    h2d = (x1[0].value - x0[0].value) / e2e_steps
    d2h = (x1[1].value - x0[1].value) / e2e_steps

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(size, args.cpu_steps)
    sphere_state = {"cx": sol.cx, "cy": sol.cy, "cz": sol.cz}
    sim.close()

    # the forms the metric names beside the plain line: FP16 storage on the
    # same scene, the 64-scene batch, and the served request stream
    extras = {}
    if not args.no_extras:
        if args.storage == "f32":
            f16 = scene_form(args, "f16", min(args.steps, 1000), dev, ws, local)
            f16["over_f32"] = f16["mlups"] / value
            extras["fp16"] = f16
        extras["batch"] = batch_result(args, dev, ws, rank, steps=100)
        extras["served"] = serve_result(args, dev, ws, rank)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
            "config": scene_config(size, args.storage, ws),
            "tile": _shape_name(rows, zchunk),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "kernel": kernel_name(rows), "kernel_ms": per_launch_ms,
                         "bytes_per_cell": bpc, "cells_per_launch": interior},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "path": "Sim.step + absorbDeadCells + RigidSphere.step; every 2nd step Sim.stepFrame (the step with packVolume fused into it) into alternating page-locked frame buffers (copy overlapped with the next steps; waitFrames before the clock stops)"},
            "gpu_launches": int(c1.value - c0.value),
            "clocks": clk,
            "cpu_baseline": cpu,
            "sphere": sphere_state,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
