"""ctypes front-ends of the two CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle``    - the C restatement in oracle/eph_oracle.c (liboracle.so), always built.
* ``RefSystem`` - the reference's own CPU integrator compiled from its sources
                  (oracle/_ref/libephref.so, built by oracle/Makefile where the reference tree exists).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NPLANES = 104
GP_TABLE = 77
RING_MAX_DISKS = 64

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int32_p = ctypes.POINTER(ctypes.c_int32)


def _ptr(a, typ=_c_double_p):
    return a.ctypes.data_as(typ) if a is not None else None


@dataclass
class Models:
    """Geopotential and ring tables in body order (layout of include/eph_planes.h)."""
    gp_nz: np.ndarray
    gp_nt: np.ndarray
    gp_coef: np.ndarray       # [n_gp, 77]
    ring_ndisk: np.ndarray
    ring_param: np.ndarray    # [n_ring, 4]
    ring_disk: np.ndarray     # [n_ring, 64, 3]

    @staticmethod
    def empty():
        return Models(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, GP_TABLE)),
                      np.zeros(0, np.int32), np.zeros((0, 4)), np.zeros((0, RING_MAX_DISKS, 3)))


class _OrcModels(ctypes.Structure):
    _fields_ = [("n_gp", ctypes.c_int32), ("gp_nz", _c_int32_p), ("gp_nt", _c_int32_p),
                ("gp_coef", _c_double_p), ("n_ring", ctypes.c_int32), ("ring_ndisk", _c_int32_p),
                ("ring_param", _c_double_p), ("ring_disk", _c_double_p)]


def _orc_models(m: Models):
    keep = [np.ascontiguousarray(x) for x in (m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)]
    s = _OrcModels(len(keep[0]), _ptr(keep[0], _c_int32_p), _ptr(keep[1], _c_int32_p), _ptr(keep[2]),
                   len(keep[3]), _ptr(keep[3], _c_int32_p), _ptr(keep[4]), _ptr(keep[5]))
    return s, keep


def build_oracle():
    """Compile liboracle.so (and the reference library when its tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    """The C restatement (serial-branch order of the reference)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        L = ctypes.CDLL(path)
        L.orc_accel.argtypes = [ctypes.c_int64, _c_double_p, ctypes.POINTER(_OrcModels)]
        L.orc_deform.argtypes = [ctypes.c_int64, _c_double_p, ctypes.POINTER(_OrcModels)]
        L.orc_integrate.argtypes = [ctypes.c_int64, _c_double_p, ctypes.POINTER(_OrcModels), ctypes.c_double,
                                    ctypes.c_int64, _c_double_p, _c_double_p, _c_double_p]
        L.orc_integrate_stages.argtypes = [ctypes.c_int64, _c_double_p, ctypes.POINTER(_OrcModels), ctypes.c_double,
                                           ctypes.c_int64, _c_double_p, _c_double_p, _c_double_p, _c_double_p]
        L.orc_geopotential_sum.argtypes = [ctypes.POINTER(_OrcModels), ctypes.c_int32, ctypes.c_double,
                                           _c_double_p, _c_double_p]
        L.orc_ring_sum.argtypes = L.orc_geopotential_sum.argtypes
        self.L = L

    def accel(self, planes: np.ndarray, models: Models) -> np.ndarray:
        p = np.ascontiguousarray(planes, dtype=np.float64).copy()
        s, keep = _orc_models(models)
        self.L.orc_accel(p.shape[1], _ptr(p), ctypes.byref(s))
        return p

    def deform(self, planes: np.ndarray, models: Models) -> np.ndarray:
        p = np.ascontiguousarray(planes, dtype=np.float64).copy()
        s, keep = _orc_models(models)
        self.L.orc_deform(p.shape[1], _ptr(p), ctypes.byref(s))
        return p

    def integrate(self, planes, models, dt, n_step, t_eph=(0.0, 0.0), stage_acc=False):
        p = np.ascontiguousarray(planes, dtype=np.float64).copy()
        n = p.shape[1]
        s, keep = _orc_models(models)
        th = ctypes.c_double(t_eph[0])
        tl = ctypes.c_double(t_eph[1])
        acc = np.zeros((25 * abs(n_step), 3, n)) if stage_acc else None
        self.L.orc_integrate(n, _ptr(p), ctypes.byref(s), dt, n_step, ctypes.byref(th), ctypes.byref(tl), _ptr(acc))
        return p, (th.value, tl.value), acc

    def integrate_stages(self, planes, models, dt, n_step, t_eph=(0.0, 0.0)):
        """integrate() returning (planes, t_eph, stage_in, stage_out): the body planes right before
        and right after each of the 25*n_step accel() calls, each [stage][NPLANES][n]."""
        p = np.ascontiguousarray(planes, dtype=np.float64).copy()
        n = p.shape[1]
        s, keep = _orc_models(models)
        th = ctypes.c_double(t_eph[0])
        tl = ctypes.c_double(t_eph[1])
        # constants and model links are not rewritten per stage: start every stage from the input planes
        sin = np.repeat(p[None], 25 * n_step, axis=0)
        sout = sin.copy()
        self.L.orc_integrate_stages(n, _ptr(p), ctypes.byref(s), dt, n_step, ctypes.byref(th), ctypes.byref(tl),
                                    _ptr(sin), _ptr(sout))
        return p, (th.value, tl.value), sin, sout

    def geopotential_sum(self, models, k, R, r):
        s, keep = _orc_models(models)
        out = np.zeros(3)
        rr = np.ascontiguousarray(r, dtype=np.float64)
        self.L.orc_geopotential_sum(ctypes.byref(s), k, R, _ptr(rr), _ptr(out))
        return out

    def ring_sum(self, models, k, R, r):
        s, keep = _orc_models(models)
        out = np.zeros(3)
        rr = np.ascontiguousarray(r, dtype=np.float64)
        self.L.orc_ring_sum(ctypes.byref(s), k, R, _ptr(rr), _ptr(out))
        return out


REF_LIB = os.path.join(HERE, "_ref", "libephref.so")
BRIDGE_LIB = os.path.join(HERE, "_ref", "libephref_b200.so")
_REF_LIBS = {}


def ref_available(path: str = REF_LIB) -> bool:
    return os.path.exists(path)


def _ref_lib(path):
    if path not in _REF_LIBS:
        L = ctypes.CDLL(path)
        L.ref_load.restype = ctypes.c_void_p
        L.ref_load.argtypes = [ctypes.c_char_p]
        L.ref_free.argtypes = [ctypes.c_void_p]
        L.ref_clone.restype = ctypes.c_void_p
        L.ref_clone.argtypes = [ctypes.c_void_p]
        L.ref_size.restype = ctypes.c_int64
        L.ref_size.argtypes = [ctypes.c_void_p]
        L.ref_get_t_eph.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p]
        L.ref_delta_t.restype = ctypes.c_double
        L.ref_delta_t.argtypes = [ctypes.c_void_p]
        L.ref_set_log_level.argtypes = [ctypes.c_int]
        L.ref_thread_pool.argtypes = [ctypes.c_int]
        L.ref_integrate.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int64]
        L.ref_integrate_gpu.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int64]
        L.ref_accel.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_deform.argtypes = [ctypes.c_void_p]
        L.ref_get_planes.argtypes = [ctypes.c_void_p, _c_double_p, ctypes.POINTER(ctypes.c_uint64)]
        L.ref_set_planes.argtypes = [ctypes.c_void_p, _c_double_p]
        L.ref_get_models.restype = ctypes.c_int64
        L.ref_get_models.argtypes = [ctypes.c_void_p, _c_int32_p, _c_int32_p, _c_double_p, _c_int32_p,
                                     _c_double_p, _c_double_p]
        L.ref_capture.restype = ctypes.c_int64
        L.ref_capture.argtypes = [ctypes.c_void_p, _c_double_p, ctypes.c_int64]
        L.ref_set_log_level(40)   # LogLevel::ERROR: keep step-size warnings quiet
        _REF_LIBS[path] = L
    return _REF_LIBS[path]


class RefSystem:
    """One reference `msystem`, loaded by the reference's own loader from a config file.

    lib_path selects the build: libephref.so (CPU only) or libephref_b200.so (the reference with its
    GPU members served by the B200 bridge)."""
    _path = REF_LIB

    def __init__(self, config: str | None = None, handle=None, lib_path: str | None = None):
        if lib_path:
            self._path = lib_path
        L = self.lib()
        self.h = handle if handle is not None else L.ref_load(config.encode())
        if not self.h:
            raise RuntimeError(f"reference loader rejected {config}")

    def lib(self):
        return _ref_lib(self._path)

    def __del__(self):
        if getattr(self, "h", None):
            _ref_lib(self._path).ref_free(self.h)
            self.h = None

    def clone(self):
        return RefSystem(handle=self.lib().ref_clone(self.h), lib_path=self._path)

    @property
    def n(self) -> int:
        return int(self.lib().ref_size(self.h))

    @property
    def t_eph(self):
        hi, lo = ctypes.c_double(), ctypes.c_double()
        self.lib().ref_get_t_eph(self.h, ctypes.byref(hi), ctypes.byref(lo))
        return hi.value, lo.value

    def planes(self):
        p = np.zeros((NPLANES, self.n))
        sid = np.zeros(self.n, np.uint64)
        self.lib().ref_get_planes(self.h, _ptr(p), sid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return p

    def sids(self):
        p = np.zeros((NPLANES, self.n))
        sid = np.zeros(self.n, np.uint64)
        self.lib().ref_get_planes(self.h, _ptr(p), sid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return [int(s).to_bytes(8, "little").rstrip(b"\0").decode() for s in sid]

    def set_planes(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        self.lib().ref_set_planes(self.h, _ptr(p))

    def models(self) -> Models:
        L = self.lib()
        cnt = L.ref_get_models(self.h, None, None, None, None, None, None)
        ngp, nring = cnt & 0xFFFFFFFF, cnt >> 32
        m = Models(np.zeros(ngp, np.int32), np.zeros(ngp, np.int32), np.zeros((ngp, GP_TABLE)),
                   np.zeros(nring, np.int32), np.zeros((nring, 4)), np.zeros((nring, RING_MAX_DISKS, 3)))
        L.ref_get_models(self.h, _ptr(m.gp_nz, _c_int32_p), _ptr(m.gp_nt, _c_int32_p), _ptr(m.gp_coef),
                         _ptr(m.ring_ndisk, _c_int32_p), _ptr(m.ring_param), _ptr(m.ring_disk))
        return m

    def integrate(self, dt: float, n_step: int, use_gpu: int = 0):
        if use_gpu:
            self.lib().ref_integrate_gpu(self.h, dt, n_step)
        else:
            self.lib().ref_integrate(self.h, dt, n_step)

    def accel(self, option: int = -1):
        self.lib().ref_accel(self.h, option)

    def deform(self):
        self.lib().ref_deform(self.h)

    def integrate_capture(self, dt: float, n_step: int):
        """integrate() while capturing the body planes after each of the 25*n_step accel() calls."""
        L = self.lib()
        buf = np.zeros((25 * n_step, NPLANES, self.n))
        L.ref_capture(self.h, _ptr(buf), buf.shape[0])
        L.ref_integrate(self.h, dt, n_step)
        got = L.ref_capture(None, None, 0)
        return buf[:got]

    @staticmethod
    def thread_pool(enable: bool, lib_path: str = REF_LIB):
        _ref_lib(lib_path).ref_thread_pool(1 if enable else 0)
