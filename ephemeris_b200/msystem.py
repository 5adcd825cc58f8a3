"""Python mirror of the reference's msystem entry points for the RK12 path.

    ms = MSystem()
    ms.load("Config.txt")            # msystem::load           (src/modules/mass_loader.cpp:67-294)
    ms.integrate(dt, n_step, 1)      # msystem::integrate      (src/physics/mass.cpp:399-442)
    ms.accel(1)                      # msystem::accel(1)       (src/physics/mass.cpp:216-221)
    ms[i]                            # msystem::operator[]     (src/physics/mass.h:343,353) as a field dict

Every call goes through libeph_b200.so; the body state stays on the GPU between calls.

``Context`` is the lower-level C ABI (include/eph_b200.h): upload a plane array, integrate, download.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import NPLANES, EphModels, check, load_library

# plane offsets (include/eph_planes.h)
P = dict(R_HI=0, R_LO=3, V_HI=6, V_LO=9, GL_HI=12, GL_LO=15, S_HI=18, S_LO=27, W=36, GM=39, EXJ2=40, GM0=41,
         DGM=42, DJ2=43, RADIUS=44, INERTIA=45, K2=46, K2R=47, TIDE_DELAY=48, TIDE_DELAY_FACTOR=49, LUM=50,
         RECPT=51, A=52, R2=53, SR2=54, RR2G_4C=55, C_STATIC=56, PHI=65, BETA2=66, NACCEL=67, DACCEL=70,
         DTORQUE=73, GACCEL=76, BETA=79, GI=82, C_POTENTIAL=91, MIN_DISTANCE=100, MAX_INFLUENCE=101,
         GP_INDEX=102, RING_INDEX=103)
VEC3 = {"R_HI", "R_LO", "V_HI", "V_LO", "GL_HI", "GL_LO", "W", "NACCEL", "DACCEL", "DTORQUE", "GACCEL", "BETA"}
MAT9 = {"S_HI", "S_LO", "C_STATIC", "GI", "C_POTENTIAL"}

CPU_RK12, GPU_RK12, COMBINED_RK12 = 0, 1, 2


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Models:
    """Owned copies of the model tables plus the ctypes struct pointing at them."""

    def __init__(self, gp_nz, gp_nt, gp_coef, ring_ndisk, ring_param, ring_disk):
        self.gp_nz = np.ascontiguousarray(gp_nz, np.int32)
        self.gp_nt = np.ascontiguousarray(gp_nt, np.int32)
        self.gp_coef = np.ascontiguousarray(gp_coef, np.float64).reshape(len(self.gp_nz), 77)
        self.ring_ndisk = np.ascontiguousarray(ring_ndisk, np.int32)
        self.ring_param = np.ascontiguousarray(ring_param, np.float64).reshape(len(self.ring_ndisk), 4)
        self.ring_disk = np.ascontiguousarray(ring_disk, np.float64).reshape(len(self.ring_ndisk), 64, 3)

    @staticmethod
    def empty():
        return Models(np.zeros(0), np.zeros(0), np.zeros((0, 77)), np.zeros(0), np.zeros((0, 4)), np.zeros((0, 64, 3)))

    def struct(self) -> EphModels:
        i32 = ctypes.POINTER(ctypes.c_int32)
        return EphModels(len(self.gp_nz), self.gp_nz.ctypes.data_as(i32), self.gp_nt.ctypes.data_as(i32),
                         _dptr(self.gp_coef), len(self.ring_ndisk), self.ring_ndisk.ctypes.data_as(i32),
                         _dptr(self.ring_param), _dptr(self.ring_disk))


class Context:
    """One device context holding one system (include/eph_b200.h)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        check(self.lib.eph_ctx_create(device, ctypes.byref(h)), None, "eph_ctx_create")
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_ctx_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, planes: np.ndarray, models: Models | None = None):
        pl = np.ascontiguousarray(planes, np.float64)
        assert pl.shape[0] == NPLANES
        self._models = models or Models.empty()
        st = self._models.struct()
        check(self.lib.eph_upload_system(self.h, pl.shape[1], _dptr(pl), ctypes.byref(st)), self.h, "upload")
        self.n = pl.shape[1]

    def record_samples(self, dt: float, n_step: int, stride: int, t_eph=(0.0, 0.0)):
        """Integrate n_step steps, returning (samples [n_step/stride + 1][n][10], t_eph): position,
        velocity, Newtonian acceleration / c^2, potential / c^2 at the start and every stride steps."""
        out = np.empty((n_step // stride + 1, self.n, 10))
        hi, lo = ctypes.c_double(t_eph[0]), ctypes.c_double(t_eph[1])
        check(self.lib.eph_record_samples(self.h, dt, n_step, stride, ctypes.byref(hi), ctypes.byref(lo), _dptr(out)),
              self.h, "record_samples")
        return out, (hi.value, lo.value)

    def upload_device(self, d_ptr: int):
        check(self.lib.eph_upload_planes_device(self.h, ctypes.c_void_p(d_ptr)), self.h, "upload_device")

    def device_planes_ptr(self) -> int:
        p = ctypes.c_void_p()
        check(self.lib.eph_device_planes(self.h, ctypes.byref(p)), self.h, "device_planes")
        return p.value

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty((NPLANES, self.n)) if out is None else out
        check(self.lib.eph_download_system(self.h, _dptr(out)), self.h, "download")
        return out

    def rk12(self, dt: float, n_step: int, t_eph=(0.0, 0.0)):
        check(self.lib.eph_rk12(self.h, dt, n_step, t_eph[0], t_eph[1]), self.h, "rk12")

    def integrate(self, dt: float, n_step: int, t_eph=(0.0, 0.0)):
        hi, lo = ctypes.c_double(t_eph[0]), ctypes.c_double(t_eph[1])
        check(self.lib.eph_integrate(self.h, dt, n_step, ctypes.byref(hi), ctypes.byref(lo)), self.h, "integrate")
        return hi.value, lo.value

    def accel(self):
        check(self.lib.eph_accel(self.h), self.h, "accel")

    def deform(self):
        check(self.lib.eph_deform(self.h), self.h, "deform")

    def set_stream(self, stream_handle: int | None):
        check(self.lib.eph_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)), self.h, "set_stream")

    def set_launch(self, grid: int = 0, bodies_per_cta: int = 0):
        check(self.lib.eph_set_launch(self.h, grid, bodies_per_cta), self.h, "set_launch")

    def launch_shape(self):
        g, b = ctypes.c_int(), ctypes.c_int()
        check(self.lib.eph_get_launch(self.h, ctypes.byref(g), ctypes.byref(b)), self.h, "get_launch")
        return g.value, b.value

    def launches(self) -> int:
        return int(self.lib.eph_launch_count(self.h))

    def autotune(self, dt: float, n_step: int = 3, reps: int = 2, use_cache: bool = True):
        """Time candidate launch shapes / cost models on the uploaded system and keep the fastest.
        Returns (grid, bodies_per_cta, ms_per_step_tuned, ms_per_step_default)."""
        g, b = ctypes.c_int(), ctypes.c_int()
        t1, t0 = ctypes.c_double(), ctypes.c_double()
        check(self.lib.eph_autotune(self.h, dt, n_step, reps, 1 if use_cache else 0, ctypes.byref(g), ctypes.byref(b),
                                    ctypes.byref(t1), ctypes.byref(t0)), self.h, "autotune")
        return g.value, b.value, t1.value, t0.value

    def set_body_costs(self, cost=None):
        """Per-body work estimates (caller order) for the ownership split; None restores the built-in ones."""
        if cost is None:
            check(self.lib.eph_set_body_costs(self.h, None), self.h, "set_body_costs")
            return
        c = np.ascontiguousarray(cost, dtype=np.float64)
        check(self.lib.eph_set_body_costs(self.h, c.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), self.h,
              "set_body_costs")

    def ownership(self) -> np.ndarray:
        """[grid, 8] caller indices of the bodies each CTA owns (-1 padded)."""
        out = np.full(1024 * 8, -1, np.int32)
        g = ctypes.c_int()
        check(self.lib.eph_get_ownership(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                         ctypes.byref(g)), self.h, "get_ownership")
        return out[:g.value * 8].reshape(g.value, 8)

    PHASES = ("io", "rk", "barrier", "a_sweep", "a_update", "b_sweep", "b_ext", "b_final", "a_sweeps")

    def profile_phases(self, enable: bool = True):
        check(self.lib.eph_profile_phases(self.h, 1 if enable else 0), self.h, "profile_phases")

    def phase_times(self) -> np.ndarray:
        """[grid, 9] nanoseconds per phase of the last launch (profiling must be on); the last column counts
        the pass-A sweeps."""
        g, p = self.launch_shape()
        out = np.zeros(max(g, 1) * len(self.PHASES), np.uint64)
        gg, pp = ctypes.c_int(), ctypes.c_int()
        check(self.lib.eph_phase_times(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                       ctypes.byref(gg), ctypes.byref(pp)), self.h, "phase_times")
        return out[:gg.value * pp.value].reshape(gg.value, pp.value)


class Batch:
    """Many independent systems integrated together (eph_batch_* of include/eph_b200.h): the point-like
    (Newtonian + 1PN) ones in one persistent launch, one CTA per system; the others one by one."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        check(self.lib.eph_batch_create(device, ctypes.byref(h)), None, "eph_batch_create")
        self.h = h
        self.sizes = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc, what):
        if rc:
            from ._lib import EphError
            raise EphError(rc, f"{what}: {self.lib.eph_batch_last_error(self.h).decode()}")

    def upload(self, planes: list, models: list | None = None):
        pls = [np.ascontiguousarray(p, np.float64) for p in planes]
        mods = [m or Models.empty() for m in (models or [None] * len(pls))]
        self._keep = (pls, mods)
        n = (ctypes.c_int64 * len(pls))(*[p.shape[1] for p in pls])
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(pls))(*[_dptr(p) for p in pls])
        self._structs = [m.struct() for m in mods]
        mptrs = (ctypes.POINTER(EphModels) * len(pls))(*[ctypes.pointer(st) for st in self._structs])
        self._check(self.lib.eph_batch_upload(self.h, len(pls), n, ptrs, mptrs), "batch upload")
        self.sizes = [p.shape[1] for p in pls]

    def set_coop_min(self, bodies: int = 0):
        """Bodies from which a system is shared by a 4-CTA cluster (0: the default)."""
        self._check(self.lib.eph_batch_set_coop_min(self.h, bodies), "batch set_coop_min")

    def autotune(self, dt, n_step, step_frac: float = 0.05):
        """Time cluster-sharing thresholds on the uploaded batch; keeps the fastest.
        Returns (coop_min, ms_tuned, ms_default)."""
        k = len(self.sizes)
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (k,)))
        ns = (ctypes.c_int64 * k)(*np.broadcast_to(np.asarray(n_step, np.int64), (k,)).tolist())
        cm = ctypes.c_int()
        t1, t0 = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.eph_batch_autotune(self.h, _dptr(dts), ns, step_frac, ctypes.byref(cm), ctypes.byref(t1),
                                                ctypes.byref(t0)), "batch autotune")
        return cm.value, t1.value, t0.value

    def set_precision(self, mixed: bool):
        """FP32 EIH 1PN terms in the ensemble launch (True) or plain FP64 (False)."""
        self._check(self.lib.eph_batch_set_precision(self.h, 1 if mixed else 0), "batch set_precision")

    def integrate(self, dt, n_step, t_eph=None):
        k = len(self.sizes)
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (k,)))
        ns = (ctypes.c_int64 * k)(*np.broadcast_to(np.asarray(n_step, np.int64), (k,)).tolist())
        hi = np.zeros(k) if t_eph is None else np.ascontiguousarray(np.asarray(t_eph, np.float64)[:, 0])
        lo = np.zeros(k) if t_eph is None else np.ascontiguousarray(np.asarray(t_eph, np.float64)[:, 1])
        self._check(self.lib.eph_batch_integrate(self.h, _dptr(dts), ns, _dptr(hi), _dptr(lo)), "batch integrate")
        return np.stack([hi, lo], 1)

    def download(self) -> list:
        outs = [np.empty((NPLANES, n)) for n in self.sizes]
        ptrs = (ctypes.POINTER(ctypes.c_double) * len(outs))(*[_dptr(o) for o in outs])
        self._check(self.lib.eph_batch_download(self.h, ptrs), "batch download")
        return outs

    def set_stream(self, stream_handle: int | None):
        self._check(self.lib.eph_batch_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)), "batch set_stream")

    def info(self):
        k, l = ctypes.c_int32(), ctypes.c_int64()
        self._check(self.lib.eph_batch_info(self.h, ctypes.byref(k), ctypes.byref(l)), "batch info")
        return k.value, l.value


class Particles:
    """Massless test particles against perturbers (eph_particles_* of include/eph_b200.h)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        check(self.lib.eph_particles_create(device, ctypes.byref(h)), None, "eph_particles_create")
        self.h = h
        self.n_pert = self.n_part = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_particles_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc, what):
        if rc:
            from ._lib import EphError
            raise EphError(rc, f"{what}: {self.lib.eph_particles_last_error(self.h).decode()}")

    def upload(self, pert_planes: np.ndarray, models, particles: np.ndarray):
        """particles: [12][n] (position hi, lo; velocity hi, lo) or [6][n] (position, velocity)."""
        pl = np.ascontiguousarray(pert_planes, np.float64)
        pa = np.asarray(particles, np.float64)
        if pa.shape[0] == 6:
            z = np.zeros((3, pa.shape[1]))
            pa = np.concatenate([pa[0:3], z, pa[3:6], z])
        pa = np.ascontiguousarray(pa)
        self._models = models or Models.empty()
        st = self._models.struct()
        self._check(self.lib.eph_particles_upload(self.h, pl.shape[1], _dptr(pl), ctypes.byref(st), pa.shape[1], _dptr(pa)),
                    "particles upload")
        self.n_pert, self.n_part = pl.shape[1], pa.shape[1]

    def integrate(self, dt: float, n_step: int, t_eph=(0.0, 0.0)):
        hi, lo = ctypes.c_double(t_eph[0]), ctypes.c_double(t_eph[1])
        self._check(self.lib.eph_particles_integrate(self.h, dt, n_step, ctypes.byref(hi), ctypes.byref(lo)),
                    "particles integrate")
        return hi.value, lo.value

    def download(self, pert_out: np.ndarray | None = None, part_out: np.ndarray | None = None):
        """(perturber planes, particles [12][n]); optional output arrays (e.g. pinned buffers) are filled."""
        pl = np.empty((NPLANES, self.n_pert)) if pert_out is None else pert_out
        pa = np.empty((12, self.n_part)) if part_out is None else part_out
        assert pl.flags.c_contiguous and pa.flags.c_contiguous and pa.shape == (12, self.n_part)
        self._check(self.lib.eph_particles_download(self.h, _dptr(pl), _dptr(pa)), "particles download")
        return pl, pa

    def set_stream(self, stream: int | None):
        """Issue the work on a cudaStream_t (e.g. torch.cuda.Stream().cuda_stream); None: own stream."""
        self._check(self.lib.eph_particles_set_stream(self.h, ctypes.c_void_p(stream) if stream else None),
                    "particles set_stream")

    def set_precision(self, mixed: bool):
        """FP64 (default) or mixed precision (FP32 relativistic/deformation terms) for the particles."""
        self._check(self.lib.eph_particles_set_precision(self.h, 1 if mixed else 0), "particles set_precision")

    def info(self):
        """(kernels launched, summed particle-kernel device time in ms)."""
        n, ms = ctypes.c_int64(), ctypes.c_double()
        self._check(self.lib.eph_particles_info(self.h, ctypes.byref(n), ctypes.byref(ms)), "particles info")
        return n.value, ms.value


def bspline_fit(samples: np.ndarray, n: int, degree: int = 3) -> np.ndarray:
    """eph_bspline_fit: samples [mn + 1][channels] at uniform positions -> coefficients [n + degree][channels]."""
    sm = np.ascontiguousarray(samples, np.float64)
    if sm.ndim == 1:
        sm = sm[:, None]
    out = np.empty((n + degree, sm.shape[1]))
    check(load_library().eph_bspline_fit(degree, n, sm.shape[0] - 1, sm.shape[1], _dptr(sm), _dptr(out)), None,
          "bspline_fit")
    return out


def bspline_fit_batch(samples: np.ndarray, n: int, degree: int = 3, device: int = 0) -> np.ndarray:
    """eph_bspline_fit_batch: samples [series][mn + 1][channels] -> coefficients [series][n + degree][channels],
    solved on the GPU, bit-identical to bspline_fit per series."""
    sm = np.ascontiguousarray(samples, np.float64)
    out = np.empty((sm.shape[0], n + degree, sm.shape[2]))
    check(load_library().eph_bspline_fit_batch(device, degree, n, sm.shape[1] - 1, sm.shape[2], sm.shape[0], _dptr(sm),
                                               _dptr(out)), None, "bspline_fit_batch")
    return out


class Server:
    """Small-body serving against a device B-spline ephemeris (eph_serve_* of include/eph_b200.h)."""

    def __init__(self, coefs: np.ndarray, gm, knot: float, t0: float = 0.0, degree: int = 3, sr2=None,
                 device: int = 0):
        """coefs: [n_pert][n_intervals + degree][10] (bspline_fit per body of record_samples' channels)."""
        self.lib = load_library()
        c = np.ascontiguousarray(coefs, np.float64)
        g = np.ascontiguousarray(gm, np.float64)
        s2 = None if sr2 is None else np.ascontiguousarray(sr2, np.float64)
        self.n_intervals = c.shape[1] - degree
        self.n_pert = c.shape[0]
        self.span = (t0, t0 + self.n_intervals * knot)
        h = ctypes.c_void_p()
        rc = self.lib.eph_serve_create(device, c.shape[0], _dptr(g), None if s2 is None else _dptr(s2), degree,
                                       self.n_intervals, t0, knot, _dptr(c), ctypes.byref(h))
        check(rc, None, "eph_serve_create")
        self.h = h
        self.sizes = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_serve_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc, what):
        if rc:
            from ._lib import EphError
            raise EphError(rc, f"{what}: {self.lib.eph_serve_last_error(self.h).decode()}")

    def set_budget(self, nbytes: int):
        self._check(self.lib.eph_serve_set_budget(self.h, int(nbytes)), "set_budget")

    def set_step_log(self, cap: int):
        self._check(self.lib.eph_serve_set_step_log(self.h, int(cap)), "set_step_log")

    def submit(self, particles: np.ndarray, t_start: float, t_end: float, tol: float = 1e-13, h0: float = 86400.0) -> int:
        """particles: [12][n] (position hi, lo; velocity hi, lo) or [6][n]; returns the request id."""
        pa = np.asarray(particles, np.float64)
        if pa.shape[0] == 6:
            z = np.zeros((3, pa.shape[1]))
            pa = np.concatenate([pa[0:3], z, pa[3:6], z])
        pa = np.ascontiguousarray(pa)
        rid = ctypes.c_int64()
        self._check(self.lib.eph_serve_submit(self.h, pa.shape[1], _dptr(pa), t_start, t_end, tol, h0, ctypes.byref(rid)),
                    "submit")
        self.sizes[rid.value] = pa.shape[1]
        return rid.value

    def poll(self, rid: int) -> int:
        st = ctypes.c_int()
        self._check(self.lib.eph_serve_poll(self.h, rid, ctypes.byref(st)), "poll")
        return st.value

    def result(self, rid: int, log_cap: int = 0):
        """(particles [12][n], accepted, rejected[, step log]) of a launched request; releases it."""
        if rid not in self.sizes:
            from ._lib import EphError
            raise EphError(1, f"result: unknown request {rid}")
        out = np.empty((12, self.sizes[rid]))
        acc, rej, nl = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        log = np.empty(max(log_cap, 1))
        rc = self.lib.eph_serve_result(self.h, rid, _dptr(out), ctypes.byref(acc), ctypes.byref(rej),
                                       _dptr(log) if log_cap else None, ctypes.byref(nl) if log_cap else None)
        self._check(rc, "result")
        del self.sizes[rid]
        if log_cap:
            return out, acc.value, rej.value, log[:nl.value].copy()
        return out, acc.value, rej.value

    def shape(self, rid: int):
        """(lanes per particle, particles per block, blocks) of a request."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.eph_serve_request_shape(self.h, rid, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                    "shape")
        return a.value, b.value, c.value

    def eval(self, t: float) -> np.ndarray:
        """The device ephemeris at time t: [n_pert][10]."""
        out = np.empty((self.n_pert, 10))
        self._check(self.lib.eph_serve_eval(self.h, t, _dptr(out)), "eval")
        return out

    def info(self):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.eph_serve_info(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "info")
        return a.value, b.value, c.value


class MSystem:
    """A system of bodies loaded from the reference's initials files and integrated on the GPU."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.device = device
        self.h = None

    def load(self, fconfig: str) -> bool:
        self.close()
        h = ctypes.c_void_p()
        rc = self.lib.eph_msystem_load(fconfig.encode(), self.device, ctypes.byref(h))
        if rc != 0:
            return False
        self.h = h
        return True

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_msystem_free(self.h)
            self.h = None

    __del__ = close

    def _need(self):
        if not self.h:
            raise RuntimeError("no system loaded")

    def size(self) -> int:
        self._need()
        return int(self.lib.eph_msystem_size(self.h))

    __len__ = size

    def integrate(self, dt: float, n_step: int, USE_GPU: int = GPU_RK12):
        self._need()
        rc = self.lib.eph_msystem_integrate(self.h, dt, n_step, USE_GPU)
        check(rc, None, (self.lib.eph_msystem_error(self.h) or b"").decode())

    def accel(self, parallel_option: int = 1):
        self._need()
        rc = self.lib.eph_msystem_accel(self.h, parallel_option)
        check(rc, None, (self.lib.eph_msystem_error(self.h) or b"").decode())

    @property
    def t_eph(self):
        hi, lo = ctypes.c_double(), ctypes.c_double()
        self.lib.eph_msystem_t_eph(self.h, ctypes.byref(hi), ctypes.byref(lo))
        return hi.value, lo.value

    def ephemeris_time(self) -> int:
        hi, lo = self.t_eph
        return int(np.floor(hi + lo))

    @property
    def delta_t(self) -> float:
        return float(self.lib.eph_msystem_delta_t(self.h))

    @property
    def integrator(self) -> int:
        return int(self.lib.eph_msystem_integrator(self.h))

    def planes(self) -> np.ndarray:
        self._need()
        out = np.empty((NPLANES, self.size()))
        check(self.lib.eph_msystem_get_planes(self.h, _dptr(out)), None, "get_planes")
        return out

    def set_planes(self, planes: np.ndarray):
        self._need()
        pl = np.ascontiguousarray(planes, np.float64)
        check(self.lib.eph_msystem_set_planes(self.h, _dptr(pl)), None, "set_planes")

    def models(self) -> Models:
        st = EphModels()
        check(self.lib.eph_msystem_models(self.h, ctypes.byref(st)), None, "models")
        ng, nr = st.n_gp, st.n_ring
        take = lambda p, n, dt: np.ctypeslib.as_array(p, (n,)).astype(dt).copy() if n else np.zeros(0, dt)
        return Models(take(st.gp_nz, ng, np.int32), take(st.gp_nt, ng, np.int32), take(st.gp_coef, ng * 77, np.float64),
                      take(st.ring_ndisk, nr, np.int32), take(st.ring_param, nr * 4, np.float64),
                      take(st.ring_disk, nr * 64 * 3, np.float64))

    def sids(self):
        out = np.zeros(self.size(), np.uint64)
        self.lib.eph_msystem_sids(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return [int(s).to_bytes(8, "little").rstrip(b"\0").decode() for s in out]

    def __getitem__(self, i: int) -> dict:
        pl = self.planes()
        out = {}
        for name, p in P.items():
            w = 3 if name in VEC3 else 9 if name in MAT9 else 1
            out[name.lower()] = pl[p:p + w, i].copy() if w > 1 else float(pl[p, i])
        return out

    def context(self) -> ctypes.c_void_p:
        return self.lib.eph_msystem_ctx(self.h)


def set_log_level(level: int):
    load_library().eph_set_log_level(level)
