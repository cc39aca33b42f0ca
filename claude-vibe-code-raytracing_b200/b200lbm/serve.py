"""Serving: a continuous-batching loop for scene-simulation requests.

The reference serves one interactive scene per browser tab (src/worker.js:
a Web Worker steps its Sim and posts an RG8 volume every few steps).  Server
runs many such scenes on one GPU at once:

  * a request names a scene (grid, pool level, spheres; see workloads.py), a
    number of steps and a frame cadence;
  * admission by device footprint (lbm_footprint_bytes plus the per-scene
    working buffers) against the memory budget, in arrival order, passing
    over a request that does not fit yet to admit later ones that do -- until
    the one passed over has waited AGE_LIMIT_S, after which nothing is
    admitted ahead of it, so a large request still runs when memory frees;
  * an admitted scene is built and initialised on a worker thread, on its
    own stream, while the running scenes keep stepping; it joins at the next
    tick after it is ready;
  * each scene's lattices stay on the device from admission to completion;
  * every tick the active scenes advance together as one Batch (one
    persistent fused launch per step, the step sequence replayed as a CUDA
    graph) by one frame interval, and every scene's RG8 volume is streamed
    back to the host;
  * between ticks finished scenes leave and newly arrived ones join, so work
    that arrives while others run overlaps with them on the device; the
    Batch object is kept and only told its new members (its stream, tables
    and frame buffer stay; the step graph is captured anew);
  * the tile shape is tuned incrementally (one candidate per tick) with the
    timings kept per batch signature, so a membership seen before reuses its
    shape.

Each scene's results do not depend on what it was batched with: the batch
gives every scene exactly the results of running it alone (tests/
test_batch_gpu.py and tests/test_serve_gpu.py check this bit for bit).

The report gives throughput (scene-steps/s and MLUPS over the whole run) and
latency: time to first frame (from arrival, including the wait for admission)
and the interval between consecutive frames of a request, as p50 / p99.
"""
from __future__ import annotations

import collections
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import autotune, workloads
from ._capi import STORAGE, lib
from .batch import Batch

# per-scene working buffers beyond lbm_footprint_bytes: compaction counts,
# impulse slots, the frame staging buffer and the device plan (generous)
_EXTRA_PER_CELL = 8
_EXTRA_FIXED = 32 << 20


def footprint(spec, storage):
    nx, ny, nz = spec["dims"]
    base = lib().lbm_footprint_bytes(nx, ny, nz, STORAGE[storage])
    return int(base + _EXTRA_PER_CELL * nx * ny * nz + _EXTRA_FIXED)


# a request passed over for lack of memory blocks later ones after this long
AGE_LIMIT_S = 2.0


def admit(queue, used, budget, now, fp, age_limit=AGE_LIMIT_S):
    """Requests to admit now, in arrival order, among those that have arrived
    by `now`: each that fits in budget - used is taken; one that does not fit
    is passed over while it has waited less than age_limit seconds (later,
    smaller requests may go ahead of it), and once it has waited longer
    nothing more is admitted ahead of it.  fp(req) -> bytes.  A request
    larger than the whole budget is admitted alone when nothing else is
    running, so it is not starved forever (it may then fail to allocate,
    which the caller reports)."""
    out = []
    for req in queue:
        if req["arrival"] > now:
            break
        need = fp(req)
        if used + need <= budget or (used == 0 and not out):
            out.append(req)
            used += need
        elif now - req["arrival"] >= age_limit:
            break
    return out


def percentiles(xs, ps=(50, 99)):
    if not xs:
        return {f"p{p}": None for p in ps}
    a = np.asarray(xs, dtype=np.float64)
    return {f"p{p}": float(np.percentile(a, p)) for p in ps}


class Server:
    def __init__(self, storage="f16", budget_bytes=None, tick=None, use_graph=True, tune=True, device=0,
                 prepare=True):
        self.storage = storage
        self.budget = budget_bytes if budget_bytes is not None else int(0.9 * 180e9)
        self.tick = tick
        self.use_graph = use_graph
        self.tune = tune
        self.device = device
        self.prepare = prepare
        self.prepared = None

    def start(self):
        """Server start-up (once, before the first run; run calls it): load
        the storage form's fused kernels and grow the device's memory pool to
        the budget (at most the free memory less 4 GB), so that neither a
        first launch nor a new scene's allocation stalls a tick.  Records the
        reserved bytes (0 when the reserve did not fit)."""
        if self.prepared is not None or not self.prepare:
            return
        import torch
        free, _ = torch.cuda.mem_get_info(self.device)
        want = max(0, min(self.budget, free - 4 * 2**30))
        rc = lib().lbm_prepare_device(self.device, STORAGE[self.storage], want)
        self.prepared = want if rc == 0 else 0

    def run(self, requests, realtime=True, on_frame=None, on_finish=None, claims=None):
        """Serve `requests` (dicts with rid, arrival, spec, steps, frame_every;
        frame_every must be the same for all and divide every steps).
        realtime: a request becomes visible at its arrival time (seconds after
        the start); otherwise all are visible at once.  on_frame(rid, index,
        volume) gets every RG8 volume; on_finish(rid, sim, solid) runs before a
        finished scene is released.  claims: a placement.ClaimQueue shared
        with the other serving processes of the job (one per GPU); requests
        are then claimed from it whenever this GPU has room for the next one
        (`requests` is not used).  Returns the report dict."""
        if claims is not None:
            requests = claims.requests
        reqs = sorted(requests, key=lambda r: (r["arrival"], r["rid"]))
        every = {r["frame_every"] for r in reqs}
        if len(every) != 1:
            raise ValueError("all requests of one run share the frame cadence")
        every = every.pop()
        tick = self.tick or every
        if tick % every or any(r["steps"] % tick for r in reqs):
            raise ValueError("the tick must be a multiple of the frame cadence and divide every request")
        self.start()
        queue = collections.deque(reqs if claims is None else ())
        claimed = []
        fpr = lambda r: footprint(r["spec"], self.storage)  # noqa: E731
        active = []  # dicts: req, sim, solid, done, fp, frames, last
        used = 0
        batch = None
        members = None
        tuner = None
        ttff, interval, done_at = [], [], {}
        tick_run, tick_tune = [], []  # seconds per tick: the batch's steps + frames, the tuner
        # the rest of a loop iteration: admission and collecting built scenes,
        # telling the batch its members, retiring finished scenes
        seg = {"admit": [], "members": [], "retire": []}
        changes = 0  # membership changes of the batch
        slow = []  # per tick: (batch run s, membership changed, active, building, cells)
        scene_steps = cell_steps = 0
        max_active = 0
        ticks = 0
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: float("inf"))
        pool = ThreadPoolExecutor(max_workers=2, thread_name_prefix="lbm-build")
        building = []  # (req, fp, future) admitted, not yet built
        try:
            while queue or active or building or (claims is not None and not claims.exhausted()):
                tl0 = time.perf_counter()
                now = clock()
                if claims is not None:
                    # claim arrived requests while this GPU has room for them
                    pending = used + sum(fpr(r) for r in queue)
                    while True:
                        nxt = claims.peek()
                        if nxt is None or nxt["arrival"] > now:
                            break
                        if pending + fpr(nxt) > self.budget and (active or building or queue):
                            break
                        got = claims.claim()
                        if got is None:
                            break
                        queue.append(got)
                        claimed.append(got["rid"])
                        pending += fpr(got)
                for req in admit(list(queue), used, self.budget, now, fpr):
                    queue.remove(req)
                    fp = footprint(req["spec"], self.storage)
                    used += fp
                    building.append((req, fp, pool.submit(workloads.build, req["spec"], self.storage,
                                                          self.device)))
                if building and not active:
                    building[0][2].result()  # nothing to step meanwhile
                still_building = []
                for req, fp, fut in building:
                    if fut.done():
                        sim, solid = fut.result()
                        active.append(dict(req=req, sim=sim, solid=solid, done=0, fp=fp, frames=0, last=None))
                    else:
                        still_building.append((req, fp, fut))
                building = still_building
                if not active:
                    # idle until the next arrival
                    nxt = queue[0] if queue else (claims.peek() if claims is not None else None)
                    if nxt is not None:
                        wait = nxt["arrival"] - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait if queue else min(wait, 0.01))
                    continue
                max_active = max(max_active, len(active))
                ids = [a["req"]["rid"] for a in active]
                tk0 = time.perf_counter()
                seg["admit"].append(tk0 - tl0)
                changed = ids != members
                if changed:
                    pairs = [(a["sim"], a["solid"]) for a in active]
                    if batch is None:
                        batch = Batch(pairs)
                    else:
                        batch.set_scenes(pairs)
                    members = ids
                    changes += 1
                    tuner = None
                tkm = time.perf_counter()
                seg["members"].append(tkm - tk0)
                frames = batch.run(tick, frame_every=every, use_graph=self.use_graph)
                tk1 = time.perf_counter()
                ticks += 1
                if self.tune:
                    # one candidate tile shape per tick: no tick waits for the whole list
                    if tuner is None:
                        tuner = autotune.Incremental(
                            batch, [(a["sim"].nx, a["sim"].ny, a["sim"].nz) for a in active], self.storage)
                    tuner.step()
                t = time.perf_counter() - t0
                tick_run.append(tk1 - tkm)
                slow.append((tk1 - tkm, changed, len(active), len(building),
                             sum(a["sim"].n for a in active)))
                tick_tune.append(t + t0 - tk1)
                for a, fr in zip(active, frames):
                    for j in range(fr.shape[0]):
                        if a["frames"] == 0:
                            ttff.append(t - a["req"]["arrival"] if realtime else t)
                        else:
                            interval.append(t - a["last"])
                        a["last"] = t
                        if on_frame is not None:
                            on_frame(a["req"]["rid"], a["frames"], fr[j])
                        a["frames"] += 1
                    a["done"] += tick
                    scene_steps += tick
                    cell_steps += tick * a["sim"].n
                still = []
                for a in active:
                    if a["done"] >= a["req"]["steps"]:
                        if on_finish is not None:
                            on_finish(a["req"]["rid"], a["sim"], a["solid"])
                        done_at[a["req"]["rid"]] = t
                        used -= a["fp"]
                        a["sim"].close()
                    else:
                        still.append(a)
                if len(still) != len(active):
                    active = still
                seg["retire"].append(time.perf_counter() - t - t0)
        finally:
            if batch is not None:
                batch.close()
            for a in active:
                a["sim"].close()
            for _, _, fut in building:
                try:
                    fut.result()[0].close()
                except Exception:
                    pass
            pool.shutdown(wait=True)
        wall = time.perf_counter() - t0
        return {
            "requests": len(reqs) if claims is None else len(claimed),
            "wall_s": wall,
            "ticks": ticks,
            "scene_steps": scene_steps,
            "scene_steps_per_s": scene_steps / wall if wall > 0 else None,
            "mlups": cell_steps / wall / 1e6 if wall > 0 else None,
            "ttff_s": percentiles(ttff),
            "frame_interval_s": percentiles(interval),
            "frames": len(ttff) + len(interval),
            "max_active": max_active,
            "membership_changes": changes,
            "tick_run_s": percentiles(tick_run, (50, 99, 100)),
            "tick_tune_s": percentiles(tick_tune, (50, 99, 100)),
            "slowest_ticks": [dict(run_s=r, membership_changed=c, active=a, building=b, cells=n)
                              for r, c, a, b, n in sorted(slow, key=lambda t: -t[0])[:5]],
            "reserved_bytes": self.prepared,
            "claimed": claimed if claims is not None else None,
            **{f"{k}_s": percentiles(v, (50, 99, 100)) for k, v in seg.items()},
            "storage": self.storage,
            "budget_bytes": self.budget,
        }


def sequential(requests, storage="f32", device=0, on_finish=None):
    """Baseline: the same requests one at a time in arrival order, each on
    its own with Sim.run_coupled (per-scene launches, no batching)."""
    reqs = sorted(requests, key=lambda r: (r["arrival"], r["rid"]))
    t0 = time.perf_counter()
    scene_steps = cell_steps = 0
    for req in reqs:
        sim, solid = workloads.build(req["spec"], storage, device)
        sim.run_coupled(solid, req["steps"], frame_every=req["frame_every"])
        scene_steps += req["steps"]
        cell_steps += req["steps"] * sim.n
        if on_finish is not None:
            on_finish(req["rid"], sim, solid)
        sim.close()
    wall = time.perf_counter() - t0
    return {"requests": len(reqs), "wall_s": wall, "scene_steps": scene_steps,
            "scene_steps_per_s": scene_steps / wall, "mlups": cell_steps / wall / 1e6,
            "storage": storage}
