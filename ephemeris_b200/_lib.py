"""ctypes binding of libeph_b200.so (the C ABI of include/eph_b200.h and include/eph_msystem.h).

The library is the only compute path: if it is missing or was built for another architecture, every
call fails loudly. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeph_b200.so")

NPLANES = 104
GP_TABLE_SIZE = 77
RING_MAX_DISKS = 64

STATUS = {0: "EPH_OK", 1: "EPH_ERR_ARG", 2: "EPH_ERR_CUDA", 3: "EPH_ERR_OOM", 4: "EPH_ERR_TIMEOUT",
          5: "EPH_ERR_STATE", 6: "EPH_ERR_LOAD", 7: "EPH_ERR_UNSUPPORTED", 8: "EPH_ERR_LIMIT",
          9: "EPH_ERR_STEP"}

# (name, restype, argtypes) of every exported entry point
_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.POINTER(ctypes.c_int32)
_VP = ctypes.c_void_p


class EphModels(ctypes.Structure):
    _fields_ = [("n_gp", ctypes.c_int32), ("gp_nz", _I32), ("gp_nt", _I32), ("gp_coef", _D),
                ("n_ring", ctypes.c_int32), ("ring_ndisk", _I32), ("ring_param", _D), ("ring_disk", _D)]


SIGNATURES = [
    ("eph_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_VP)]),
    ("eph_ctx_destroy", ctypes.c_int, [_VP]),
    ("eph_last_error", ctypes.c_char_p, [_VP]),
    ("eph_upload_system", ctypes.c_int, [_VP, ctypes.c_int64, _D, ctypes.POINTER(EphModels)]),
    ("eph_upload_planes_device", ctypes.c_int, [_VP, _VP]),
    ("eph_download_system", ctypes.c_int, [_VP, _D]),
    ("eph_device_planes", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("eph_rk12", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int64, ctypes.c_double, ctypes.c_double]),
    ("eph_integrate", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int64, _D, _D]),
    ("eph_accel", ctypes.c_int, [_VP]),
    ("eph_deform", ctypes.c_int, [_VP]),
    ("eph_set_stream", ctypes.c_int, [_VP, _VP]),
    ("eph_selftest_wait_timeout", ctypes.c_int, [_VP, ctypes.c_int64]),
    ("eph_set_launch", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    ("eph_get_launch", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("eph_launch_count", ctypes.c_int64, [_VP]),
    ("eph_set_body_costs", ctypes.c_int, [_VP, _D]),
    ("eph_autotune", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _D, _D]),
    ("eph_get_ownership", ctypes.c_int, [_VP, _I32, ctypes.POINTER(ctypes.c_int)]),
    ("eph_profile_phases", ctypes.c_int, [_VP, ctypes.c_int]),
    ("eph_phase_times", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    ("eph_batch_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_VP)]),
    ("eph_batch_destroy", ctypes.c_int, [_VP]),
    ("eph_batch_last_error", ctypes.c_char_p, [_VP]),
    ("eph_batch_upload", ctypes.c_int, [_VP, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_D),
                                        ctypes.POINTER(ctypes.POINTER(EphModels))]),
    ("eph_batch_integrate", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_int64), _D, _D]),
    ("eph_batch_download", ctypes.c_int, [_VP, ctypes.POINTER(_D)]),
    ("eph_batch_set_stream", ctypes.c_int, [_VP, _VP]),
    ("eph_batch_set_precision", ctypes.c_int, [_VP, ctypes.c_int]),
    ("eph_batch_set_coop_min", ctypes.c_int, [_VP, ctypes.c_int]),
    ("eph_batch_autotune", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_int64), ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_int), _D, _D]),
    ("eph_batch_info", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)]),
    ("eph_particles_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_VP)]),
    ("eph_particles_destroy", ctypes.c_int, [_VP]),
    ("eph_particles_last_error", ctypes.c_char_p, [_VP]),
    ("eph_particles_upload", ctypes.c_int, [_VP, ctypes.c_int64, _D, ctypes.POINTER(EphModels), ctypes.c_int64, _D]),
    ("eph_particles_integrate", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int64, _D, _D]),
    ("eph_particles_download", ctypes.c_int, [_VP, _D, _D]),
    ("eph_particles_set_stream", ctypes.c_int, [_VP, _VP]),
    ("eph_particles_set_precision", ctypes.c_int, [_VP, ctypes.c_int]),
    ("eph_particles_info", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]),
    ("eph_record_samples", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _D, _D, _D]),
    ("eph_serve_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _D, _D, ctypes.c_int, ctypes.c_int64,
                                         ctypes.c_double, ctypes.c_double, _D, ctypes.POINTER(_VP)]),
    ("eph_serve_destroy", ctypes.c_int, [_VP]),
    ("eph_serve_last_error", ctypes.c_char_p, [_VP]),
    ("eph_serve_set_budget", ctypes.c_int, [_VP, ctypes.c_int64]),
    ("eph_serve_set_step_log", ctypes.c_int, [_VP, ctypes.c_int64]),
    ("eph_serve_submit", ctypes.c_int, [_VP, ctypes.c_int64, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(ctypes.c_int64)]),
    ("eph_serve_poll", ctypes.c_int, [_VP, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]),
    ("eph_serve_result", ctypes.c_int, [_VP, ctypes.c_int64, _D, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64), _D, ctypes.POINTER(ctypes.c_int64)]),
    ("eph_serve_eval", ctypes.c_int, [_VP, ctypes.c_double, _D]),
    ("eph_serve_request_shape", ctypes.c_int, [_VP, ctypes.c_int64, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("eph_serve_info", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int64)]),
    ("eph_bspline_fit", ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, _D, _D]),
    ("eph_bspline_cheb_coef", ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("eph_bspline_fit_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                              ctypes.c_int64, _D, _D]),
    ("eph_ephem_open", ctypes.c_int, [_VP, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(_VP)]),
    ("eph_ephem_close", ctypes.c_int, [_VP]),
    ("eph_ephem_info", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int64), _D, _D]),
    ("eph_ephem_state", ctypes.c_int, [_VP, ctypes.c_double, _D, _D, _D]),
    ("eph_ephem_states", ctypes.c_int, [_VP, ctypes.c_int64, _D, _D]),
    ("eph_ephem_to_bspline", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, _D]),
    ("eph_ephem_rotation", ctypes.c_int, [_VP, ctypes.c_double, _D, _D, _D]),
    ("eph_ephem_set_orbital_state", ctypes.c_int, [_VP, _D, _D]),
    ("eph_geopotential_field", ctypes.c_int, [ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_int, ctypes.c_int64, _D, _D]),
    ("eph_fp64_fma_rate", ctypes.c_int, [ctypes.c_int, _D]),
    ("eph_integrate_noalloc", ctypes.c_int, [ctypes.c_int, _VP, ctypes.c_int64, _VP, ctypes.POINTER(EphModels),
                                             ctypes.c_double, ctypes.c_int64, _D, _D]),
    ("eph_msystem_load", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_VP)]),
    ("eph_msystem_free", ctypes.c_int, [_VP]),
    ("eph_msystem_size", ctypes.c_int64, [_VP]),
    ("eph_msystem_integrate", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int64, ctypes.c_int]),
    ("eph_msystem_accel", ctypes.c_int, [_VP, ctypes.c_int]),
    ("eph_msystem_get_planes", ctypes.c_int, [_VP, _D]),
    ("eph_msystem_set_planes", ctypes.c_int, [_VP, _D]),
    ("eph_msystem_t_eph", ctypes.c_int, [_VP, _D, _D]),
    ("eph_msystem_delta_t", ctypes.c_double, [_VP]),
    ("eph_msystem_integrator", ctypes.c_int, [_VP]),
    ("eph_msystem_models", ctypes.c_int, [_VP, ctypes.POINTER(EphModels)]),
    ("eph_msystem_sids", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint64)]),
    ("eph_msystem_ctx", _VP, [_VP]),
    ("eph_msystem_error", ctypes.c_char_p, [_VP]),
    ("eph_set_log_level", None, [ctypes.c_int]),
]

_lib = None


class EphError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"{STATUS.get(code, code)}: {msg}")


def load_library(path: str | None = None):
    """Load libeph_b200.so (building it first if the sources are newer) and bind every entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if path == LIB_PATH:
        from . import build as _build
        try:
            if _build.needs_build():
                _build.build()
        except Exception as exc:   # a stale library is still usable; a missing one is fatal below
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libeph_b200.so is missing and could not be built: {exc}") from exc
    if not os.path.exists(path):
        raise RuntimeError(f"libeph_b200.so not found at {path}: the CUDA path is required (no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def check(code: int, ctx=None, what: str = ""):
    if code != 0:
        msg = what
        lib = load_library()
        if ctx is not None:
            msg += ": " + (lib.eph_last_error(ctx) or b"").decode()
        raise EphError(code, msg)
