"""Batch -- many independent scenes advanced together on one GPU.

The reference runs one scene per Web Worker (src/worker.js:94-115).  A Batch
advances many Sim scenes of any sizes with one persistent fused launch per
step over every scene's tiles, the per-scene plan / retag / fresh-cell /
impulse / RigidSphere.step kernels as parallel branches around it, and the
step sequence captured as a CUDA graph and replayed (lbm_batch_* in
include/lbm_b200.h).  Each scene's results equal Sim.run_coupled on that
scene alone.

    batch = Batch([(sim_a, solid_a), (sim_b, None)])
    frames = batch.run(200, frame_every=20)   # list of (frames, 2*n) arrays
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import LbmError, LbmSphere, check, lib
from .solid import spheres_of, to_c_array


class Batch:
    def __init__(self, scenes, rows=None, zchunk=None):
        """scenes: list of (Sim, solid) pairs; solid is a RigidSphere, a
        CompositeSolid or None.  All Sims on one device with one storage."""
        self.scenes = list(scenes)
        if not self.scenes:
            raise ValueError("a batch needs at least one scene")
        self._b = None
        n = len(self.scenes)
        handles = (C.c_void_p * n)(*[sim.handle for sim, _ in self.scenes])
        out = C.c_void_p()
        rc = lib().lbm_batch_create(handles, n, C.byref(out))
        if rc != 0:
            raise LbmError(rc, "lbm_batch_create: the scenes must be distinct, on one device, one storage form")
        self._b = out
        if rows is not None or zchunk is not None:
            self.set_config(rows or 4, zchunk or 32)

    def set_scenes(self, scenes):
        """Replace the scenes (a list of (Sim, solid) pairs on the same device
        and storage form) and keep the batch's stream, tables and frame
        buffer; the step graph is captured anew at the next run."""
        scenes = list(scenes)
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        n = len(scenes)
        handles = (C.c_void_p * n)(*[sim.handle for sim, _ in scenes])
        self._check(lib().lbm_batch_set_scenes(self._b, handles, n))
        self.scenes = scenes

    def _check(self, rc):
        if rc != 0:
            raise LbmError(rc, (lib().lbm_batch_last_error(self._b) or b"").decode(errors="replace"))

    def set_config(self, rows, zchunk):
        """Fused tile shape: rows per CTA (2, 4, 8, or 4 | autotune.STAGED for the
        staged FP16/BF16 form) and z planes per CTA."""
        self._check(lib().lbm_batch_set_config(self._b, int(rows), int(zchunk)))

    def run(self, nsteps, frame_every=0, use_graph=True):
        """nsteps coupled steps of every scene.  Returns, per scene, the RG8
        volumes after every frame_every-th step (array (frames, 2*n)), or None."""
        n = len(self.scenes)
        arrays, counts, solids = [], [], []
        for sim, solid in self.scenes:
            sim._sync()
            sp = spheres_of(solid)
            arrays.append(to_c_array(sp))
            counts.append(len(sp))
            solids.append(sp)
        sph = (C.POINTER(LbmSphere) * n)(*[C.cast(a, C.POINTER(LbmSphere)) for a in arrays])
        cnt = (C.c_int * n)(*counts)
        nfr = nsteps // frame_every if frame_every > 0 else 0
        frames = [np.empty((nfr, 2 * sim.n), dtype=np.uint8) for sim, _ in self.scenes] if nfr else None
        fptr = (C.POINTER(C.c_uint8) * n)(*[f.ctypes.data_as(C.POINTER(C.c_uint8)) for f in frames]) \
            if nfr else None
        rc = lib().lbm_batch_run(self._b, sph, cnt, int(nsteps), int(frame_every) if nfr else 0, fptr,
                                 1 if use_graph else 0)
        for (sim, _), sp, arr in zip(self.scenes, solids, arrays):
            sim._moved()
            for i, b in enumerate(sp):
                b.from_c(arr[i])
        self._check(rc)
        return frames

    def time_fused(self, rows, zchunk, reps=5):
        """Average ms of one batched fused launch with this tile shape (after a run)."""
        ms = C.c_double()
        self._check(lib().lbm_batch_time_fused(self._b, int(rows), int(zchunk), int(reps), C.byref(ms)))
        return ms.value

    def launch_count(self):
        v = C.c_int64()
        self._check(lib().lbm_batch_launch_count(self._b, C.byref(v)))
        return v.value

    def close(self):
        if self._b:
            lib().lbm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
