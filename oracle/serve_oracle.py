"""CPU checker of the serving path (TEST INFRASTRUCTURE ONLY).

* ``RefSpline``  - the reference's own B-spline sampling (src/math/interp.h:263-345, compiled from its
                   sources into oracle/_ref/libephref.so through oracle/ref/ref_bspline.cpp): perturber
                   position, velocity, a_N/c^2 and phi/c^2 at any time from the fitted coefficients.
* ``replay``     - the particles' integration over a given sequence of accepted adaptive steps: each
                   accepted step h is two RK12 steps of h/2 (what the step-doubling controller keeps), in
                   the textbook form r_k = r0 + dt sum_j a_kj v_j, v_k = v0 + dt sum_j a_kj f_j
                   (src/integrators/RungeKutta.impl:148-186) in double precision; every stage acceleration
                   comes from the oracle's accel (oracle/eph_oracle.c, the reference's msystem::accel
                   restated) on the perturbers at the stage time plus the particles as GM = 1e-20 bodies.
                   The perturbers' a_N and phi there come from their positions, not from the fitted
                   channels the GPU reads (a difference far below the tolerances).

Only tests/ import this module.
"""
from __future__ import annotations

import ctypes
import os
import re
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libephref.so")
TABLE_H = os.path.join(HERE, "..", "include", "eph_rk12_table.h")
_D = ctypes.POINTER(ctypes.c_double)

R_HI, R_LO, V_HI, V_LO, GM = 0, 3, 6, 9, 39
NACC, DACC, GACC = 67, 70, 76


def rk12_table():
    """(a [26][26] double = hi + lo, c [26]) from the repository's coefficient table."""
    text = open(TABLE_H).read().split("EPH_RK12_COEF_BITS")[1]
    bits = [int(x, 16) for x in re.findall(r"0x[0-9a-fA-F]+", text)]
    vals = [struct.unpack("d", struct.pack("Q", b))[0] for b in bits]
    hi, lo = vals[0::2], vals[1::2]
    a = np.zeros((26, 26))
    for k in range(1, 26):
        for j in range(k):
            q = k * (k - 1) // 2 + j
            a[k, j] = hi[q] + lo[q]
    return a, a.sum(1)


class RefSpline:
    """The reference's bspline_fitter<double, 10> on each body's coefficients."""

    def __init__(self, coefs: np.ndarray, degree: int, knot: float, t0: float = 0.0, lib_path: str = REF_LIB):
        self.L = ctypes.CDLL(lib_path)
        self.L.ref_bspline_eval.argtypes = [ctypes.c_int, _D, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_int64, _D, _D, _D]
        self.c = np.ascontiguousarray(coefs, np.float64)
        self.d, self.knot, self.t0 = degree, knot, t0
        self.n = self.c.shape[1] - degree

    def __call__(self, t: float, expanded: bool = False) -> np.ndarray:
        """[M][10] at time t."""
        pos = np.array([(t - self.t0) / self.knot])
        out = np.empty((self.c.shape[0], 10))
        der = np.empty(10)
        for j in range(self.c.shape[0]):
            v = np.empty(10)
            rc = self.L.ref_bspline_eval(10, self.c[j].ctypes.data_as(_D), self.d, self.n, float(self.n),
                                         1 if expanded else 0, 1, pos.ctypes.data_as(_D), v.ctypes.data_as(_D),
                                         der.ctypes.data_as(_D))
            assert rc == 0
            out[j] = v
        return out


def _accel(oracle, tmpl, models, M, spline, t, r, v, mind=None):
    """Particle accelerations [3][P] at time t, positions/velocities [3][P]; mind (optional, [P]) is lowered
    to each particle's distance from the nearest perturber other than body 0."""
    pl = tmpl.copy()
    s = spline(t)
    if mind is not None:
        d = np.linalg.norm(s[1:, 0:3][:, :, None] - r[None, :, :], axis=1).min(axis=0)
        np.minimum(mind, d, out=mind)
    pl[R_HI:R_HI + 3, :M] = s[:, 0:3].T
    pl[R_LO:R_LO + 3, :M] = 0.0
    pl[V_HI:V_HI + 3, :M] = s[:, 3:6].T
    pl[V_LO:V_LO + 3, :M] = 0.0
    pl[R_HI:R_HI + 3, M:] = r
    pl[R_LO:R_LO + 3, M:] = 0.0
    pl[V_HI:V_HI + 3, M:] = v
    pl[V_LO:V_LO + 3, M:] = 0.0
    out = oracle.accel(pl, models)
    return ((out[GACC:GACC + 3] + out[DACC:DACC + 3]) + out[NACC:NACC + 3])[:, M:]


def replay(oracle, tmpl, models, M, spline, particles, t_start, steps):
    """particles: [12][P] (hi, lo); steps: accepted step sizes (signed). Returns positions, velocities [3][P]
    and each particle's closest approach to a perturber other than body 0 over the stage evaluations."""
    a, c = rk12_table()
    r = particles[0:3] + particles[3:6]
    v = particles[6:9] + particles[9:12]
    t = t_start
    mind = np.full(r.shape[1], np.inf)
    f0 = _accel(oracle, tmpl, models, M, spline, t, r, v, mind)
    for h in steps:
        for half in range(2):
            dt = h / 2
            fs, vs = [f0], [v]
            for k in range(1, 26):
                rk = r + dt * sum(a[k, j] * vs[j] for j in range(k) if a[k, j] != 0)
                vk = v + dt * sum(a[k, j] * fs[j] for j in range(k) if a[k, j] != 0)
                fk = _accel(oracle, tmpl, models, M, spline, t + c[k] * dt, rk, vk, mind)
                fs.append(fk)
                vs.append(vk)
            r, v, f0 = rk, vk, fk
            t = t + dt
    return r, v, mind
