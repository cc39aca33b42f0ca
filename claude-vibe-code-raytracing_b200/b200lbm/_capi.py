"""ctypes binding of liblbm_b200.so (declared in include/lbm_b200.h).

The shared library is built in-tree by ``claude-vibe-code-raytracing_b200/csrc/Makefile``.
There is no fallback: if the library is missing or a CUDA device is absent the
calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# LBM_B200_CHECKED=1 selects the bounds-checked build (csrc/Makefile target `checked`)
LIB_PATH = os.path.join(_HERE, "liblbm_b200_checked.so" if os.environ.get("LBM_B200_CHECKED") == "1"
                        else "liblbm_b200.so")

OK = 0
ERR_ARG = -1
ERR_OOM = -2
ERR_CUDA = -3
ERR_TIMEOUT = -4
ERR_NAN = -5
ERR_STATE = -6
ERR_UNSUPPORTED = -7
ERR_CAPACITY = -8

STORE_F32, STORE_F16, STORE_BF16, STORE_F64 = 0, 1, 2, 3
STORAGE = {"f32": STORE_F32, "f16": STORE_F16, "bf16": STORE_BF16, "f64": STORE_F64}

FIELDS = {
    "f": 0, "f2": 1, "h": 2, "h2": 3, "rho": 4, "ux": 5, "uy": 6, "uz": 7, "phi": 8,
    "phiPrev": 9, "tag": 10, "tagPrev": 11, "usx": 12, "usy": 13, "usz": 14,
    "gx": 15, "gy": 16, "gz": 17, "lap": 18, "bodyFx": 19, "bodyFy": 20, "bodyFz": 21,
}
MAX_SPHERES = 8


class LbmParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in
                ("tau", "tauPhi", "sigma", "gravity", "rhoL", "rhoG", "W", "mobility")]


class LbmSphere(C.Structure):
    _fields_ = [(k, C.c_double) for k in
                ("cx", "cy", "cz", "r", "vx", "vy", "vz", "wx", "wy", "wz",
                 "density", "mass", "I", "dragTargetX", "dragTargetY", "dragTargetZ",
                 "Fx", "Fy", "Fz", "Tx", "Ty", "Tz")] + [("dragging", C.c_int32),
                                                          ("reserved", C.c_int32)]


class LbmImpulse(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("Fx", "Fy", "Fz", "Tx", "Ty", "Tz")]


class LbmRigidMotion(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz")]


class LbmCamera(C.Structure):
    _fields_ = [("azimuth", C.c_double), ("elev", C.c_double), ("dist", C.c_double),
                ("light", C.c_double * 3)]


class LbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lbm error {code}: {msg}")
        self.code = code


_lib = None

# (name, restype, argtypes)
_SIGS = [
    ("lbm_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("lbm_destroy", C.c_int, [C.c_void_p]),
    ("lbm_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_get_dims", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int)] * 4),
    ("lbm_device_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("lbm_footprint_bytes", C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ("lbm_set_params", C.c_int, [C.c_void_p, C.POINTER(LbmParams)]),
    ("lbm_get_params", C.c_int, [C.c_void_p, C.POINTER(LbmParams)]),
    ("lbm_upload_field", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("lbm_download_field", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("lbm_download_field_f64", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_size_t]),
    ("lbm_init_flat", C.c_int, [C.c_void_p, C.c_double]),
    ("lbm_init_profile", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int]),
    ("lbm_seed_hydrostatic", C.c_int, [C.c_void_p]),
    ("lbm_retag_cells", C.c_int, [C.c_void_p, C.POINTER(LbmSphere), C.c_int]),
    ("lbm_handle_fresh_cells", C.c_int, [C.c_void_p]),
    ("lbm_compute_phi_gradients", C.c_int, [C.c_void_p]),
    ("lbm_collide_phase", C.c_int, [C.c_void_p]),
    ("lbm_stream_phase", C.c_int, [C.c_void_p]),
    ("lbm_collide_hydro", C.c_int, [C.c_void_p]),
    ("lbm_stream_hydro_and_macro", C.c_int,
     [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.POINTER(LbmImpulse)]),
    ("lbm_step", C.c_int, [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.POINTER(LbmImpulse)]),
    ("lbm_step_begin", C.c_int, [C.c_void_p, C.POINTER(LbmSphere), C.c_int]),
    ("lbm_step_end", C.c_int, [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.POINTER(LbmImpulse)]),
    ("lbm_voxelize_mesh", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LbmRigidMotion), C.c_void_p,
                                     C.c_void_p]),
    ("lbm_retag_cells_mesh", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LbmRigidMotion)]),
    ("lbm_step_frame", C.c_int, [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.POINTER(LbmImpulse), C.c_void_p]),
    ("lbm_wait_frame_slot", C.c_int, [C.c_void_p]),
    ("lbm_absorb_dead_cells", C.c_int,
     [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.POINTER(LbmImpulse)]),
    ("lbm_pack_volume", C.c_int, [C.c_void_p, C.c_void_p]),
    ("lbm_pack_volume_device", C.c_int, [C.c_void_p, C.c_void_p]),
    ("lbm_host_alloc", C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    ("lbm_prepare_device", C.c_int, [C.c_int, C.c_int, C.c_uint64]),
    ("lbm_trim_device_memory", C.c_int, [C.c_int]),
    ("lbm_pack_volume_async", C.c_int, [C.c_void_p, C.c_void_p]),
    ("lbm_wait_frames", C.c_int, [C.c_void_p]),
    ("lbm_host_free", C.c_int, [C.c_void_p]),
    ("lbm_run_coupled", C.c_int,
     [C.c_void_p, C.POINTER(LbmSphere), C.c_int, C.c_int, C.c_int, C.c_void_p]),
    ("lbm_retag_cells_mask", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("lbm_solid_links", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    ("lbm_sphere_step_host", C.c_int,
     [C.POINTER(LbmSphere), C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
    ("lbm_synchronize", C.c_int, [C.c_void_p]),
    ("lbm_stream", C.c_void_p, [C.c_void_p]),
    ("lbm_last_sets", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("lbm_download_sets", C.c_int,
     [C.c_void_p, C.POINTER(C.c_int32), C.c_int, C.POINTER(C.c_int32), C.c_int]),
    ("lbm_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("lbm_checked_build", C.c_int, []),
    ("lbm_fault_record", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("lbm_test_withhold_stage_copy", C.c_int, [C.c_void_p, C.c_int]),
    ("lbm_test_sequential_fill", C.c_int, [C.c_void_p, C.c_int]),
    ("lbm_set_nan_watchdog", C.c_int, [C.c_void_p, C.c_int]),
    ("lbm_transfer_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("lbm_fused_timing", C.c_int, [C.c_void_p, C.c_int]),
    ("lbm_fused_timing_query", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("lbm_set_fused_config", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("lbm_get_fused_config", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("lbm_get_launch_shape", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("lbm_set_slab", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    ("lbm_slab_copy_planes", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int]),
    ("lbm_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("lbm_batch_destroy", C.c_int, [C.c_void_p]),
    ("lbm_batch_set_scenes", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("lbm_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_batch_set_config", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("lbm_batch_run", C.c_int,
     [C.c_void_p, C.POINTER(C.POINTER(LbmSphere)), C.POINTER(C.c_int), C.c_int, C.c_int,
      C.POINTER(C.POINTER(C.c_uint8)), C.c_int]),
    ("lbm_batch_time_fused", C.c_int,
     [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    ("lbm_batch_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("lbm_camera_default", None, [C.POINTER(LbmCamera)]),
    ("lbm_render_volume", C.c_int,
     [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(LbmSphere), C.POINTER(LbmCamera), C.c_int, C.c_int,
      C.c_void_p, C.c_void_p]),
    ("lbm_render", C.c_int,
     [C.c_void_p, C.POINTER(LbmSphere), C.POINTER(LbmCamera), C.c_int, C.c_int, C.c_void_p]),
    ("lbm_absorb_dead_cells_noalloc", C.c_int,
     [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double] + [C.c_void_p] * 6
     + [C.POINTER(LbmSphere), C.c_int, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
]

EXPORTED = [s[0] for s in _SIGS]


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C claude-vibe-code-raytracing_b200/csrc` "
                "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(handle, rc):
    if rc != OK:
        msg = lib().lbm_last_error(handle) if handle else b""
        raise LbmError(rc, (msg or b"").decode(errors="replace"))
    return rc
