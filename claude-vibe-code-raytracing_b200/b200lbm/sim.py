"""Sim -- the reference's `class Sim` (src/sim.js:29-601) backed by the
sm_100a CUDA library through its C ABI.

Same constructor, methods, fields and parameter properties as the reference, so
its driver loop (src/worker.js:94-115) and test scripts read unchanged:

    sim = Sim(40, 28, 40); sim.initFlat(14); sim.tau = 0.7
    solid = RigidSphere(40, 28, 40, cx=20, cy=6, cz=20, r=4, density=1.6)
    sim.step(solid); solid.absorbDeadCells(sim); solid.step(1.0, sim.gravity)
    sim.phi[sim.idx(6, 6, 6)]

Field arrays (f, h, rho, phi, ux, ...) are host mirrors in the reference
layout.  Reading one downloads it if the device has moved on since the last
read; writing elements marks it dirty and it is uploaded before the next
device call -- the JS code's direct typed-array access (src/worker.js:58-69)
keeps working.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import FIELDS, LbmImpulse, LbmParams, check, lib
from .solid import evaluate_generic, impulse_array, is_generic, spheres_of, to_c_array


class _HostBlock:
    """Owns one lbm_host_alloc block; freed when the last array using it goes."""

    def __init__(self, nbytes):
        p = C.c_void_p()
        rc = lib().lbm_host_alloc(nbytes, C.byref(p))
        if rc != _capi.OK:
            raise _capi.LbmError(rc, f"lbm_host_alloc({nbytes}) failed")
        self.ptr = p.value

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().lbm_host_free(C.c_void_p(self.ptr))
            self.ptr = None


def pinned_empty(nbytes):
    """A uint8 numpy array of nbytes in page-locked host memory."""
    block = _HostBlock(nbytes)
    arr = np.ctypeslib.as_array((C.c_uint8 * nbytes).from_address(block.ptr))
    arr = arr.view(_PinnedArray)
    arr._block = block  # keeps the memory alive as long as the array (or a view of it)
    return arr


class _PinnedArray(np.ndarray):
    def __array_finalize__(self, obj):
        if obj is not None:
            self._block = getattr(obj, "_block", None)

# D3Q27 velocity set, rest first then opposite pairs (src/lattices.js:34-49)
_DIRS = ((0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1),
         (-1, 0, 1), (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1), (1, 1, 1), (-1, -1, -1),
         (1, 1, -1), (-1, -1, 1), (1, -1, 1), (-1, 1, -1), (-1, 1, 1), (1, -1, -1))

_PARAM_NAMES = ("tau", "tauPhi", "sigma", "gravity", "rhoL", "rhoG", "W", "mobility")
# upload order: phi before h (h may be stored relative to phi), tags last
_UPLOAD_ORDER = ("phi", "rho", "ux", "uy", "uz", "f", "f2", "h", "h2", "usx", "usy", "usz",
                 "gx", "gy", "gz", "lap", "bodyFx", "bodyFy", "bodyFz", "tag", "tagPrev",
                 "phiPrev")


class TrackedArray(np.ndarray):
    """numpy array that tells its Sim when elements are written, and refreshes
    itself from the device when read after the device state moved on."""

    def __array_finalize__(self, obj):
        self._sim = getattr(obj, "_sim", None)
        self._field = getattr(obj, "_field", None)

    def _fresh(self):
        sim = self._sim
        if sim is not None and self._field is not None:
            sim._refresh(self._field)

    def __getitem__(self, key):
        self._fresh()
        return super().__getitem__(key)

    def __setitem__(self, key, value):
        self._fresh()
        super().__setitem__(key, value)
        if self._sim is not None and self._field is not None:
            self._sim._dirty.add(self._field)

    def __array_wrap__(self, arr, context=None, return_scalar=False):
        # results of arithmetic on a field are plain arrays, not field mirrors
        arr = np.asarray(arr).view(np.ndarray)
        return arr[()] if return_scalar else arr

    def fill(self, value):
        super().fill(value)
        if self._sim is not None and self._field is not None:
            self._sim._dirty.add(self._field)

    def set(self, src, offset=0):  # TypedArray.prototype.set
        self[offset:offset + len(src)] = np.asarray(src)


def _np_dtype(field):
    return np.uint8 if field in ("tag", "tagPrev") else np.float32


class Sim:
    """class Sim (src/sim.js:29-601) on the GPU."""

    def __init__(self, nx, ny, nz, storage="f32", device=0):
        h = C.c_void_p()
        rc = lib().lbm_create(nx, ny, nz, _capi.STORAGE[storage], device, C.byref(h))
        if rc != _capi.OK:
            raise _capi.LbmError(rc, f"lbm_create({nx},{ny},{nz},{storage}) failed")
        object.__setattr__(self, "_h", h)
        object.__setattr__(self, "nx", nx)
        object.__setattr__(self, "ny", ny)
        object.__setattr__(self, "nz", nz)
        object.__setattr__(self, "n", nx * ny * nz)
        object.__setattr__(self, "storage", storage)
        # src/sim.js:88-95
        object.__setattr__(self, "_params", dict(tau=0.6, tauPhi=0.7, sigma=0.012, gravity=0.0010,
                                                 rhoL=1.0, rhoG=0.05, W=4.0, mobility=0.02))
        object.__setattr__(self, "_params_dirty", True)
        object.__setattr__(self, "_mirror", {})
        object.__setattr__(self, "_mirror_version", {})
        object.__setattr__(self, "_version", 0)
        object.__setattr__(self, "_dirty", set())
        # lattice offsets (src/sim.js:71-85), read-only views for callers
        nxny = nx * ny
        dirs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
                (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1),
                (-1, 0, 1), (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1), (1, 1, 1), (-1, -1, -1),
                (1, 1, -1), (-1, -1, 1), (1, -1, 1), (-1, 1, -1), (-1, 1, 1), (1, -1, -1)]
        off27 = np.array([-(ez * nxny + ey * nx + ex) for ex, ey, ez in dirs], dtype=np.int32)
        object.__setattr__(self, "neighOffset27", off27)
        object.__setattr__(self, "fOffset27", off27 * 27 + np.arange(27, dtype=np.int32))
        object.__setattr__(self, "neighOffset7", off27[:7].copy())
        object.__setattr__(self, "hOffset7", off27[:7] * 7 + np.arange(7, dtype=np.int32))

    # ------------------------------------------------------------ lifetime
    def close(self):
        h = self.__dict__.get("_h")
        if h:
            lib().lbm_destroy(h)
            self.__dict__["_h"] = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------ params
    def __getattr__(self, name):
        d = self.__dict__
        if name in _PARAM_NAMES:
            return d["_params"][name]
        if name in FIELDS:
            self._refresh(name)
            return d["_mirror"][name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _PARAM_NAMES:
            self._params[name] = float(value)
            self.__dict__["_params_dirty"] = True
        elif name in FIELDS:
            arr = getattr(self, name)
            arr[...] = value
        else:
            object.__setattr__(self, name, value)

    # ------------------------------------------------------------ mirrors
    def _count(self, field):
        if field in ("f", "f2"):
            return self.n * 27
        if field in ("h", "h2"):
            return self.n * 7
        return self.n

    def _refresh(self, field):
        d = self.__dict__
        mirror = d["_mirror"]
        if field in mirror and (d["_mirror_version"][field] == d["_version"] or field in d["_dirty"]):
            return
        arr = mirror.get(field)
        if arr is None:
            base = np.empty(self._count(field), dtype=_np_dtype(field))
            arr = base.view(TrackedArray)
            arr._sim = self
            arr._field = field
            mirror[field] = arr
        buf = np.asarray(arr).view(np.ndarray)
        check(self._h, lib().lbm_download_field(self._h, FIELDS[field], buf.ctypes.data_as(C.c_void_p),
                                                buf.size))
        d["_mirror_version"][field] = d["_version"]

    def _sync(self):
        """Push parameter changes and host-side field writes to the device."""
        d = self.__dict__
        if d["_params_dirty"]:
            p = LbmParams(**{k: d["_params"][k] for k in _PARAM_NAMES})
            check(self._h, lib().lbm_set_params(self._h, C.byref(p)))
            d["_params_dirty"] = False
        if d["_dirty"]:
            uploaded = set(d["_dirty"])
            for field in _UPLOAD_ORDER:
                if field in uploaded:
                    buf = np.ascontiguousarray(np.asarray(d["_mirror"][field]).view(np.ndarray))
                    check(self._h, lib().lbm_upload_field(self._h, FIELDS[field],
                                                          buf.ctypes.data_as(C.c_void_p), buf.size))
            d["_dirty"].clear()
            old = d["_version"]
            d["_version"] = old + 1
            # mirrors that matched the device still do; the uploaded ones now match
            for f in d["_mirror"]:
                if d["_mirror_version"][f] == old or f in uploaded:
                    d["_mirror_version"][f] = d["_version"]
            if "phiPrev" in uploaded:
                # phiPrev writes stay host-side until the next retag overwrites it
                d["_mirror_version"]["phiPrev"] = d["_version"]

    def _moved(self):
        self.__dict__["_version"] += 1

    def _completed(self, rc, apply):
        """After a call that steps: the device state moved; the results are
        applied when the steps completed (also when the NaN watchdog then
        reported a non-finite field), and a non-zero status raises."""
        self._moved()
        if rc in (_capi.OK, _capi.ERR_NAN):
            apply()
        check(self._h, rc)

    # ------------------------------------------------------------ reference API
    def idx(self, x, y, z):
        return ((z * self.ny) + y) * self.nx + x

    def rhoFromPhi(self, p):
        return self.rhoG + p * (self.rhoL - self.rhoG)

    def initFlat(self, waterlineY):
        """src/sim.js:112-134 (tanh profile, wall tags, f = w, h = w*phi, then seedHydrostatic)."""
        self.__dict__["_dirty"].clear()
        self._sync()
        check(self._h, lib().lbm_init_flat(self._h, float(waterlineY)))
        self._moved()

    def initProfile(self, phi_col):
        """initFlat with a column profile phi_col[y] (ny values) in place of
        the waterline's tanh (lbm_init_profile): what writing phi, phiPrev and
        h = w7 phi cell by cell after initFlat and then calling
        seedHydrostatic gives, with the fields kept on the device."""
        col = np.ascontiguousarray(phi_col, dtype=np.float64)
        if col.shape != (self.ny,):
            raise ValueError("phi_col needs ny values")
        self.__dict__["_dirty"].clear()
        self._sync()
        check(self._h, lib().lbm_init_profile(self._h, col.ctypes.data_as(C.POINTER(C.c_double)), self.ny))
        self._moved()

    def seedHydrostatic(self):
        """src/sim.js:144-173"""
        self._sync()
        check(self._h, lib().lbm_seed_hydrostatic(self._h))
        self._moved()

    def computePhiGradients(self):
        self._sync()
        check(self._h, lib().lbm_compute_phi_gradients(self._h))
        self._moved()

    def retagCells(self, solid):
        if is_generic(solid):
            return self._retag_generic(solid)
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        check(self._h, lib().lbm_retag_cells(self._h, arr, len(sp)))
        self._moved()

    # ------------------------------------------------------------ duck-typed solids
    # Any object with contains / surfaceVelocity / applyImpulseAtCell
    # (README.md:69-73) runs through the phase-by-phase kernels: its predicates
    # are evaluated here on the host and uploaded as a mask, and its
    # momentum exchange comes back as a scan-ordered list of links that is
    # replayed through its applyImpulseAtCell (src/sim.js:517-536).
    def _retag_generic(self, solid):
        if getattr(solid, "use_device", False) and hasattr(solid, "world_triangles"):
            # a mesh body (b200lbm.MeshSolid): voxelised on the device
            tri = np.ascontiguousarray(solid.world_triangles(), dtype=np.float64)
            m = solid.motion()
            self._sync()
            check(self._h, lib().lbm_retag_cells_mesh(self._h, tri.ctypes.data_as(C.c_void_p), len(tri),
                                                      C.byref(m)))
            self._moved()
            return
        mask, us = evaluate_generic(solid, self.nx, self.ny, self.nz)
        self._sync()
        check(self._h, lib().lbm_retag_cells_mask(self._h, mask.ctypes.data_as(C.c_void_p),
                                                  us.ctypes.data_as(C.c_void_p)))
        self._moved()

    def _links_generic(self, solid):
        L = lib()
        cnt = C.c_int()
        check(self._h, L.lbm_solid_links(self._h, None, None, None, 0, C.byref(cnt)))
        n = cnt.value
        if n == 0:
            return
        cells = np.empty(n, dtype=np.int32)
        dirs = np.empty(n, dtype=np.int8)
        mom = np.empty(n, dtype=np.float64)
        check(self._h, L.lbm_solid_links(self._h, cells.ctypes.data_as(C.c_void_p), dirs.ctypes.data_as(C.c_void_p),
                                         mom.ctypes.data_as(C.c_void_p), n, C.byref(cnt)))
        nx, nxny = self.nx, self.nx * self.ny
        apply = solid.applyImpulseAtCell
        for i, k, m in zip(cells.tolist(), dirs.tolist(), mom.tolist()):
            ex, ey, ez = _DIRS[k]
            z, r = divmod(i, nxny)
            y, x = divmod(r, nx)
            apply(x - ex, y - ey, z - ez, -m * ex, -m * ey, -m * ez)

    def _step_generic(self, solid):
        """src/sim.js:202-210 for a duck-typed solid, phase by phase."""
        self._retag_generic(solid)
        self.handleFreshCells(solid)
        self.computePhiGradients()
        self.collidePhase()
        self.streamPhase()
        self.collideHydro()
        self.streamHydroAndMacro(solid)

    def handleFreshCells(self, solid=None):
        self._sync()
        check(self._h, lib().lbm_handle_fresh_cells(self._h))
        self._moved()

    def collidePhase(self):
        self._sync()
        check(self._h, lib().lbm_collide_phase(self._h))
        self._moved()

    def streamPhase(self):
        self._sync()
        check(self._h, lib().lbm_stream_phase(self._h))
        self._moved()

    def collideHydro(self):
        self._sync()
        check(self._h, lib().lbm_collide_hydro(self._h))
        self._moved()

    def streamHydroAndMacro(self, solid):
        if is_generic(solid):
            self._sync()
            rc = lib().lbm_stream_hydro_and_macro(self._h, None, 0, None)
            self._completed(rc, lambda: None)
            self._links_generic(solid)
            return
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        out = impulse_array(len(sp))
        rc = lib().lbm_stream_hydro_and_macro(self._h, arr, len(sp), out)
        self._completed(rc, lambda: [b.add_impulse(out[i]) for i, b in enumerate(sp)])

    def step(self, solid):
        """src/sim.js:202-210, as one fused device step (phase by phase for a
        duck-typed solid that is not made of RigidSpheres)."""
        if is_generic(solid):
            return self._step_generic(solid)
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        out = impulse_array(len(sp))
        rc = lib().lbm_step(self._h, arr, len(sp), out)
        self._completed(rc, lambda: [b.add_impulse(out[i]) for i, b in enumerate(sp)])

    def stepFrame(self, solid, out):
        """step(solid) on a frame step: the fused kernel also writes the
        step's RG8 volume (packVolume, src/sim.js:586-600), which is copied
        into `out` (a frameBuffer) while the next steps run -- packVolumeAsync
        after step without its separate pass over the grid.  `out` holds the
        frame after waitFrames()."""
        if is_generic(solid):
            self.step(solid)
            return self.packVolumeAsync(out)
        buf = np.asarray(out).view(np.ndarray)
        if buf.dtype != np.uint8 or buf.size < self.n * 2 or not buf.flags.c_contiguous:
            raise ValueError("stepFrame needs a contiguous uint8 buffer of 2*n bytes")
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        res = impulse_array(len(sp))
        rc = lib().lbm_step_frame(self._h, arr, len(sp), res, buf.ctypes.data_as(C.c_void_p))
        self._completed(rc, lambda: [b.add_impulse(res[i]) for i, b in enumerate(sp)])
        return out

    def step_begin(self, solid):
        """The first half of step (retagCells + handleFreshCells,
        src/sim.js:203-204); step_end(solid) with the same solid completes it."""
        if is_generic(solid):
            raise TypeError("a split step takes spheres (RigidSphere / CompositeSolid)")
        sp = spheres_of(solid)
        self._sync()
        rc = lib().lbm_step_begin(self._h, to_c_array(sp), len(sp))
        self._moved()
        check(self._h, rc)

    def step_end(self, solid):
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        out = impulse_array(len(sp))
        rc = lib().lbm_step_end(self._h, arr, len(sp), out)
        self._completed(rc, lambda: [b.add_impulse(out[i]) for i, b in enumerate(sp)])

    def render(self, solid=None, width=640, height=480, camera=None):
        """Renderer.uploadVolume + draw (src/render.js:431-434, 484-513) without
        a canvas: the current state rendered by the reference's fragment shader
        on the GPU.  Returns an RGBA8 image, shape (height, width, 4), top row
        first.  camera: an LbmCamera (default: the reference's start view)."""
        from ._capi import LbmCamera
        cam = camera
        if cam is None:
            cam = LbmCamera()
            lib().lbm_camera_default(C.byref(cam))
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp[:1])
        img = np.empty((height, width, 4), dtype=np.uint8)
        check(self._h, lib().lbm_render(self._h, arr if sp else None, C.byref(cam), width, height,
                                        img.ctypes.data_as(C.c_void_p)))
        return img

    def run_coupled(self, solid, nsteps, frame_every=0):
        """nsteps worker ticks (src/worker.js:96-100: sim.step(solid);
        solid.absorbDeadCells(sim); solid.step(1.0, sim.gravity)) entirely on
        the device.  The solid's state is updated in place.  Returns the RG8
        volumes after every frame_every-th step, shape (frames, 2*n), or None."""
        sp = spheres_of(solid)
        self._sync()
        arr = to_c_array(sp)
        nfr = nsteps // frame_every if frame_every > 0 else 0
        frames = np.empty((nfr, 2 * self.n), dtype=np.uint8) if nfr else None
        ptr = frames.ctypes.data_as(C.POINTER(C.c_uint8)) if nfr else None
        rc = lib().lbm_run_coupled(self._h, arr, len(sp), nsteps, frame_every if nfr else 0, ptr)
        self._completed(rc, lambda: [b.from_c(arr[i]) for i, b in enumerate(sp)])
        return frames

    def _absorb_dead(self, spheres):
        """RigidSphere.absorbDeadCells(sim) (src/solid.js:87-101) on the device."""
        if not spheres:
            return
        self._sync()
        arr = to_c_array(spheres)
        out = impulse_array(len(spheres))
        check(self._h, lib().lbm_absorb_dead_cells(self._h, arr, len(spheres), out))
        for i, b in enumerate(spheres):
            b.add_impulse(out[i])

    def packVolume(self, out=None, solidContains=None):
        """src/sim.js:586-600 (second argument ignored, as in the reference)."""
        self._sync()
        if out is None:
            out = np.empty(self.n * 2, dtype=np.uint8)
        buf = np.asarray(out).view(np.ndarray)
        if buf.dtype != np.uint8 or buf.size < self.n * 2 or not buf.flags.c_contiguous:
            raise ValueError("packVolume needs a contiguous uint8 buffer of 2*n bytes")
        check(self._h, lib().lbm_pack_volume(self._h, buf.ctypes.data_as(C.c_void_p)))
        return out

    def packVolumeAsync(self, out):
        """packVolume that returns at once: the frame is copied into `out`
        (a frameBuffer) while the steps queued after this call run.  `out`
        holds the frame after waitFrames(); do not read or reuse it before."""
        self._sync()
        buf = np.asarray(out).view(np.ndarray)
        if buf.dtype != np.uint8 or buf.size < self.n * 2 or not buf.flags.c_contiguous:
            raise ValueError("packVolumeAsync needs a contiguous uint8 buffer of 2*n bytes")
        check(self._h, lib().lbm_pack_volume_async(self._h, buf.ctypes.data_as(C.c_void_p)))
        return out

    def waitFrames(self):
        """Wait until every packVolumeAsync copy has reached its buffer."""
        check(self._h, lib().lbm_wait_frames(self._h))

    def waitFrameSlot(self):
        """Wait only for the older of the two frames in flight: with two
        frame buffers used in turn, the one the next stepFrame /
        packVolumeAsync will fill holds its frame after this call."""
        check(self._h, lib().lbm_wait_frame_slot(self._h))

    def frameBuffer(self):
        """A page-locked uint8 buffer of 2*n bytes for packVolume: the
        device-to-host copy of each frame then runs at full link speed (a
        pageable numpy buffer goes through driver staging buffers)."""
        return pinned_empty(self.n * 2)

    # ------------------------------------------------------------ extras
    def field64(self, name):
        """A field as a float64 copy (exact for the FP64 storage form)."""
        self._sync()
        out = np.empty(self._count(name), dtype=np.float64)
        check(self._h, lib().lbm_download_field_f64(self._h, FIELDS[name],
                                                    out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def synchronize(self):
        check(self._h, lib().lbm_synchronize(self._h))

    def setNanWatchdog(self, every):
        """Scan phi, rho and u for NaN/Inf after every `every` completed steps and
        raise LbmError (code ERR_NAN) naming the first such cell; 0 (the
        default) turns the scan off, as in the reference, where a blow-up only
        shows as NaN in the fields."""
        check(self._h, lib().lbm_set_nan_watchdog(self._h, int(every)))

    def last_sets(self):
        """(fresh, dead) cell index arrays found at the last retag, scan order."""
        nf, nd = C.c_int(), C.c_int()
        check(self._h, lib().lbm_last_sets(self._h, C.byref(nf), C.byref(nd)))
        fr = np.zeros(max(1, nf.value), dtype=np.int32)
        de = np.zeros(max(1, nd.value), dtype=np.int32)
        check(self._h, lib().lbm_download_sets(
            self._h, fr.ctypes.data_as(C.POINTER(C.c_int32)), nf.value,
            de.ctypes.data_as(C.POINTER(C.c_int32)), nd.value))
        return fr[:nf.value], de[:nd.value]

    def fused_config(self):
        """(rows, zchunk): the fused step's launch shape as set."""
        r, z = C.c_int(), C.c_int()
        check(self._h, lib().lbm_get_fused_config(self._h, C.byref(r), C.byref(z)))
        return r.value, z.value

    def launch_shape(self):
        """The tile shape the fused launches use: the shape set, or
        6 | LBM_FUSED_COMPACT where 6 | LBM_FUSED_TMA or 6 | LBM_FUSED_L2PF
        was set on a scene whose nx is not a multiple of 16."""
        r = C.c_int()
        check(self._h, lib().lbm_get_launch_shape(self._h, C.byref(r)))
        return r.value

    def set_fused_config(self, rows, zchunk=32):
        """Fused step launch shape: rows per CTA (2, 4, 8; 4 or 6 | 0x400
        compact, | 0x800 async, | 0x100 staged; 6 | 0x1000 TMA-staged,
        6 | 0x2000 compact with tensor prefetches into L2) and z planes per
        CTA.  Every shape gives the same bits."""
        self._sync()
        check(self._h, lib().lbm_set_fused_config(self._h, int(rows), int(zchunk)))

    def launch_count(self):
        v = C.c_int64()
        check(self._h, lib().lbm_launch_count(self._h, C.byref(v)))
        return v.value

    def device_bytes(self):
        v = C.c_size_t()
        check(self._h, lib().lbm_device_bytes(self._h, C.byref(v)))
        return v.value
