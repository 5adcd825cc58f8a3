"""Compressed ephemeris records of the reference, read through the library's host decoder.

`EphemerisInterpolator` mirrors the reference's `ephemeris_compressor::interpolator`
(src/modules/ephemeris_compressor.h:74-148): it takes one compressed record (the bytes that
`ephemeris_compressor::compress_orbital_data` / `compress_rotational_data` leave in their MFILE) and the
time span it covers. An orbital record returns position, velocity and the record's GM at a time in
[0, span] (`operator()(t, orbital_state_t*, keplerian&)`, ephemeris_compressor.cpp:1036-1053); a rotational
record returns the angular velocity and the surface frame's x and z axes (`operator()(t, rotational_state_t*)`,
ephemeris_compressor.cpp:1017-1034), a tidally locked one after `set_orbital_state` with the orbital state at
that time (ephemeris_compressor.cpp:1010-1015). `to_bspline` resamples an orbital record into the B-spline
table form of the device ephemeris used by `Server` (eph_serve_*) and `bspline_fit_batch`.
"""
import ctypes

import numpy as np

from ._lib import EphError, check, load_library

FORMAT_NAMES = {1: "STATE_VECTORS", 2: "KEPLERIAN_VECTORS", 3: "KEPLERIAN_CIRCULAR", 4: "KEPLERIAN_RAW",
                5: "AXIAL_OFFSET", 6: "QUATERNION", 7: "TIDAL_LOCK"}


class EphemerisInterpolator:
    """One compressed record over `span` seconds: orbital (formats 1-4) or rotational (formats 5-7)."""

    def __init__(self, record: bytes, span: float):
        self.lib = load_library()
        self._buf = np.frombuffer(bytes(record), np.uint8).copy()
        self.span = float(span)
        h = ctypes.c_void_p()
        check(self.lib.eph_ephem_open(self._buf.ctypes.data_as(ctypes.c_void_p), len(self._buf), self.span,
                                      ctypes.byref(h)), None, "eph_ephem_open")
        self.h = h
        f, d, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        rel, gm = ctypes.c_double(), ctypes.c_double()
        check(self.lib.eph_ephem_info(self.h, ctypes.byref(f), ctypes.byref(d), ctypes.byref(n), ctypes.byref(rel),
                                      ctypes.byref(gm)), None, "eph_ephem_info")
        self.format, self.degree, self.segments = f.value, d.value, n.value
        self.relative_error, self.gm = rel.value, gm.value

    def data_format(self) -> int:
        return self.format

    def format_name(self) -> str:
        return FORMAT_NAMES.get(self.format, "UNKNOWN")

    def is_orbital(self) -> bool:
        return 1 <= self.format <= 4

    def __call__(self, t: float):
        """(r[3], v[3], GM) at time t in [0, span]; GM is 0 for a state-vector record."""
        r, v, gm = np.zeros(3), np.zeros(3), ctypes.c_double()
        D = ctypes.POINTER(ctypes.c_double)
        check(self.lib.eph_ephem_state(self.h, float(t), r.ctypes.data_as(D), v.ctypes.data_as(D), ctypes.byref(gm)),
              None, "eph_ephem_state")
        return r, v, gm.value

    def states(self, times):
        """Positions and velocities [len(times)][6] at the given times."""
        t = np.ascontiguousarray(times, np.float64)
        out = np.empty((len(t), 6))
        D = ctypes.POINTER(ctypes.c_double)
        check(self.lib.eph_ephem_states(self.h, len(t), t.ctypes.data_as(D), out.ctypes.data_as(D)), None,
              "eph_ephem_states")
        return out

    def is_rotational(self) -> bool:
        return 5 <= self.format <= 7

    def set_orbital_state(self, r, v):
        """The orbital state at the next evaluation's time (needed by a tidally locked record)."""
        r = np.ascontiguousarray(r, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        D = ctypes.POINTER(ctypes.c_double)
        check(self.lib.eph_ephem_set_orbital_state(self.h, r.ctypes.data_as(D), v.ctypes.data_as(D)), None,
              "eph_ephem_set_orbital_state")

    def rotation(self, t: float):
        """(w[3], x[3], z[3]) of a rotational record at time t in [0, span]."""
        w, x, z = np.zeros(3), np.zeros(3), np.zeros(3)
        D = ctypes.POINTER(ctypes.c_double)
        check(self.lib.eph_ephem_rotation(self.h, float(t), w.ctypes.data_as(D), x.ctypes.data_as(D),
                                          z.ctypes.data_as(D)), None, "eph_ephem_rotation")
        return w, x, z

    def to_bspline(self, d: int, n: int, mn: int) -> np.ndarray:
        """Positions at mn + 1 uniform times over [0, span] fitted with n + d degree-d B-splines: [n + d][3]."""
        coefs = np.zeros((n + d, 3))
        check(self.lib.eph_ephem_to_bspline(self.h, int(d), int(n), int(mn),
                                            coefs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              None, "eph_ephem_to_bspline")
        return coefs

    def close(self):
        if getattr(self, "h", None):
            self.lib.eph_ephem_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["EphemerisInterpolator", "FORMAT_NAMES", "EphError"]
