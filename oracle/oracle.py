"""Python view of the C oracle -- TEST INFRASTRUCTURE ONLY.

Wraps the oracle libraries built by oracle/Makefile with the reference's own
names, so parity tests read like the reference's test/ scripts:

    sim = OracleSim(40, 28, 40); sim.initFlat(14); sim.tau = 0.7
    ball = OracleSphere(40, 28, 40, cx=20, cy=6, cz=20, r=4, density=1.6)
    sim.step(ball); ball.absorbDeadCells(sim); ball.step(1.0, sim.gravity)

Class Sim follows src/sim.js:29-601, RigidSphere follows src/solid.js:8-211.
Field arrays are zero-copy numpy views of the oracle's own memory, in the
reference layout (cell i = (z*ny + y)*nx + x; f[i*27 + k], h[i*7 + k]).
store='f32' (default) keeps fields in float32 exactly as the reference's
Float32Arrays; store='f64' keeps them in double (reference for the GPU's FP64
storage form).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATHS = {"f32": os.path.join(_HERE, "_build", "liblbm_oracle.so"),
              "f64": os.path.join(_HERE, "_build", "liblbm_oracle_f64.so")}
_libs = {}


class _Sphere(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double), ("r", C.c_double),
        ("vx", C.c_double), ("vy", C.c_double), ("vz", C.c_double),
        ("wx", C.c_double), ("wy", C.c_double), ("wz", C.c_double),
        ("density", C.c_double),
        ("dragging", C.c_int),
        ("dragTargetX", C.c_double), ("dragTargetY", C.c_double), ("dragTargetZ", C.c_double),
        ("Fx", C.c_double), ("Fy", C.c_double), ("Fz", C.c_double),
        ("Tx", C.c_double), ("Ty", C.c_double), ("Tz", C.c_double),
        ("volume", C.c_double), ("mass", C.c_double), ("I", C.c_double),
    ]


_U8 = C.POINTER(C.c_uint8)


def _sim_struct(real):
    FP = C.POINTER(real)

    class _Sim(C.Structure):
        _fields_ = [
            ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n", C.c_int),
            ("f", FP), ("f2", FP), ("h", FP), ("h2", FP),
            ("rho", FP), ("ux", FP), ("uy", FP), ("uz", FP), ("phi", FP), ("phiPrev", FP),
            ("tag", _U8), ("tagPrev", _U8),
            ("usx", FP), ("usy", FP), ("usz", FP),
            ("gx", FP), ("gy", FP), ("gz", FP), ("lap", FP),
            ("bodyFx", FP), ("bodyFy", FP), ("bodyFz", FP),
            ("neighOffset27", C.c_int32 * 27), ("fOffset27", C.c_int32 * 27),
            ("neighOffset7", C.c_int32 * 7), ("hOffset7", C.c_int32 * 7),
            ("tau", C.c_double), ("tauPhi", C.c_double), ("sigma", C.c_double),
            ("gravity", C.c_double), ("rhoL", C.c_double), ("rhoG", C.c_double),
            ("W", C.c_double), ("mobility", C.c_double),
            ("omp", C.c_int),
        ]
    return _Sim


_SIM_STRUCT = {"f32": _sim_struct(C.c_float), "f64": _sim_struct(C.c_double)}
_DTYPE = {"f32": np.float32, "f64": np.float64}


def build():
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(store="f32"):
    L = _libs.get(store)
    if L is None:
        path = _LIB_PATHS[store]
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        SP = C.POINTER(_SIM_STRUCT[store])
        BP = C.POINTER(_Sphere)
        L.or_store_bytes.restype = C.c_int
        assert L.or_store_bytes() == (8 if store == "f64" else 4)
        L.or_sim_create.restype = SP
        L.or_render.restype = None
        L.or_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.c_int, C.c_int, C.c_void_p]
        L.or_sim_create.argtypes = [C.c_int, C.c_int, C.c_int]
        L.or_sim_destroy.argtypes = [SP]
        L.or_sim_set_omp.argtypes = [SP, C.c_int]
        L.or_init_flat.argtypes = [SP, C.c_double]
        for name in ["or_seed_hydrostatic", "or_compute_phi_gradients", "or_handle_fresh_cells",
                     "or_collide_phase", "or_stream_phase", "or_collide_hydro"]:
            getattr(L, name).argtypes = [SP]
        for name in ["or_retag_cells", "or_stream_hydro_and_macro", "or_step", "or_worker_substep"]:
            getattr(L, name).argtypes = [SP, BP, C.c_int]
        L.or_pack_volume.argtypes = [SP, _U8]
        L.or_sphere_init.argtypes = [BP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double]
        L.or_sphere_recompute_mass.argtypes = [BP]
        L.or_sphere_contains.argtypes = [BP, C.c_int, C.c_int, C.c_int]
        L.or_sphere_contains.restype = C.c_int
        L.or_sphere_surface_velocity.argtypes = [BP, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.or_sphere_apply_impulse.argtypes = [BP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                              C.c_double]
        L.or_absorb_dead_cells.argtypes = [BP, C.c_int, SP]
        L.or_sphere_step.argtypes = [BP, C.c_double, C.c_double]
        _libs[store] = L
    return L


_SPHERE_FIELDS = {name for name, _ in _Sphere._fields_}


class OracleSphere:
    """RigidSphere (src/solid.js:8-211) backed by the oracle's C struct."""

    def __init__(self, nx, ny, nz, cx=None, cy=None, cz=None, r=None, density=None):
        object.__setattr__(self, "_s", _Sphere())
        cx = nx * 0.5 if cx is None else cx
        cy = ny * 0.3 if cy is None else cy
        cz = nz * 0.5 if cz is None else cz
        r = min(nx, ny, nz) * 0.10 if r is None else r
        density = 1.4 if density is None else density
        lib().or_sphere_init(C.byref(self._s), nx, ny, nz, cx, cy, cz, r, density)

    def __getattr__(self, name):
        if name in _SPHERE_FIELDS:
            v = getattr(self._s, name)
            return bool(v) if name == "dragging" else v
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _SPHERE_FIELDS:
            setattr(self._s, name, int(bool(value)) if name == "dragging" else value)
        else:
            object.__setattr__(self, name, value)

    def recomputeMass(self):
        lib().or_sphere_recompute_mass(C.byref(self._s))

    def setRadius(self, r):
        self._s.r = r
        self.recomputeMass()

    def setDensity(self, d):
        self._s.density = d
        self.recomputeMass()

    def contains(self, x, y, z):
        return bool(lib().or_sphere_contains(C.byref(self._s), x, y, z))

    def surfaceVelocity(self, x, y, z, out=None):
        buf = (C.c_double * 3)()
        lib().or_sphere_surface_velocity(C.byref(self._s), x, y, z, buf)
        out = out if out is not None else [0.0, 0.0, 0.0]
        out[0], out[1], out[2] = buf[0], buf[1], buf[2]
        return out

    def applyImpulseAtCell(self, x, y, z, px, py, pz):
        lib().or_sphere_apply_impulse(C.byref(self._s), x, y, z, px, py, pz)

    def absorbDeadCells(self, sim):
        sim._L.or_absorb_dead_cells(C.byref(self._s), 1, sim._p)

    def step(self, dt, gravity):
        lib().or_sphere_step(C.byref(self._s), dt, gravity)

    def state(self):
        return {name: getattr(self._s, name) for name, _ in _Sphere._fields_}


class OracleSpheres:
    """Composite solid: several spheres in one contiguous C array; the first
    sphere containing a cell owns it."""

    def __init__(self, spheres):
        self.arr = (_Sphere * len(spheres))()
        for b, s in enumerate(spheres):
            C.memmove(C.byref(self.arr[b]), C.byref(s._s), C.sizeof(_Sphere))
        self.count = len(spheres)

    def absorbDeadCells(self, sim):
        sim._L.or_absorb_dead_cells(self.arr, self.count, sim._p)

    def step(self, dt, gravity):
        for b in range(self.count):
            lib().or_sphere_step(C.byref(self.arr[b]), dt, gravity)

    def state(self, b):
        return {name: getattr(self.arr[b], name) for name, _ in _Sphere._fields_}


_PARAMS = ("tau", "tauPhi", "sigma", "gravity", "rhoL", "rhoG", "W", "mobility")
_FIELDS27 = ("f", "f2")
_FIELDS7 = ("h", "h2")
_FIELDS1 = ("rho", "ux", "uy", "uz", "phi", "phiPrev", "usx", "usy", "usz",
            "gx", "gy", "gz", "lap", "bodyFx", "bodyFy", "bodyFz")


def _solid_args(solid):
    if solid is None:
        return None, 0
    if isinstance(solid, OracleSpheres):
        return solid.arr, solid.count
    return C.byref(solid._s), 1


class OracleSim:
    """class Sim (src/sim.js:29-601) backed by the C oracle."""

    def __init__(self, nx, ny, nz, store="f32"):
        L = lib(store)
        p = L.or_sim_create(nx, ny, nz)
        object.__setattr__(self, "_L", L)
        object.__setattr__(self, "_p", p)
        object.__setattr__(self, "store", store)
        object.__setattr__(self, "nx", nx)
        object.__setattr__(self, "ny", ny)
        object.__setattr__(self, "nz", nz)
        object.__setattr__(self, "n", nx * ny * nz)
        s = p.contents
        n = nx * ny * nz
        views = {}
        for name in _FIELDS27:
            views[name] = np.ctypeslib.as_array(getattr(s, name), shape=(n * 27,))
        for name in _FIELDS7:
            views[name] = np.ctypeslib.as_array(getattr(s, name), shape=(n * 7,))
        for name in _FIELDS1:
            views[name] = np.ctypeslib.as_array(getattr(s, name), shape=(n,))
        views["tag"] = np.ctypeslib.as_array(s.tag, shape=(n,))
        views["tagPrev"] = np.ctypeslib.as_array(s.tagPrev, shape=(n,))
        object.__setattr__(self, "_views", views)

    def __del__(self):
        p = self.__dict__.get("_p")
        L = self.__dict__.get("_L")
        if p and L is not None:
            L.or_sim_destroy(p)
            self.__dict__["_p"] = None

    def __getattr__(self, name):
        if name in _PARAMS:
            return getattr(self._p.contents, name)
        views = self.__dict__.get("_views", {})
        if name in views:
            return views[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _PARAMS:
            setattr(self._p.contents, name, float(value))
        else:
            object.__setattr__(self, name, value)

    def set_threads(self, nthreads):
        self._L.or_sim_set_omp(self._p, int(nthreads))

    def idx(self, x, y, z):
        return ((z * self.ny) + y) * self.nx + x

    def rhoFromPhi(self, p):
        return self.rhoG + p * (self.rhoL - self.rhoG)

    def initFlat(self, waterlineY):
        self._L.or_init_flat(self._p, waterlineY)

    def seedHydrostatic(self):
        self._L.or_seed_hydrostatic(self._p)

    def computePhiGradients(self):
        self._L.or_compute_phi_gradients(self._p)

    def step(self, solid):
        self._L.or_step(self._p, *_solid_args(solid))

    def retagCells(self, solid):
        self._L.or_retag_cells(self._p, *_solid_args(solid))

    def handleFreshCells(self, solid=None):
        self._L.or_handle_fresh_cells(self._p)

    def collidePhase(self):
        self._L.or_collide_phase(self._p)

    def streamPhase(self):
        self._L.or_stream_phase(self._p)

    def collideHydro(self):
        self._L.or_collide_hydro(self._p)

    def streamHydroAndMacro(self, solid):
        self._L.or_stream_hydro_and_macro(self._p, *_solid_args(solid))

    def packVolume(self, out=None, solidContains=None):
        if out is None:
            out = np.zeros(self.n * 2, dtype=np.uint8)
        assert out.dtype == np.uint8 and out.size >= self.n * 2 and out.flags.c_contiguous
        self._L.or_pack_volume(self._p, out.ctypes.data_as(_U8))
        return out

    def worker_substep(self, solid):
        """sim.step(solid); solid.absorbDeadCells(sim); solid.step(1.0, g) (src/worker.js:96-100)."""
        self._L.or_worker_substep(self._p, *_solid_args(solid))


def render(volume, nx, ny, nz, sphere=None, camera=(math.pi * 0.25, -0.25, 2.4, 0.35, 0.75, 0.5),
           width=640, height=480):
    """The reference's renderer (src/render.js) restated in C: RGBA8 image of
    the RG8 `volume` (2*nx*ny*nz bytes), shape (height, width, 4), top row
    first.  sphere: (cx, cy, cz, r) in cells or None; camera: azimuth,
    elevation, distance, light direction."""
    L = lib()
    vol = np.ascontiguousarray(np.asarray(volume, dtype=np.uint8))
    assert vol.size == 2 * nx * ny * nz
    out = np.empty((height, width, 4), dtype=np.uint8)
    sp = (C.c_double * 4)(*sphere) if sphere is not None else None
    cam = (C.c_double * 6)(*camera)
    L.or_render(vol.ctypes.data_as(C.c_void_p), nx, ny, nz, sp, cam, width, height,
                out.ctypes.data_as(C.c_void_p))
    return out
