"""Geopotential field known-answer tests.

The reference holds its geopotential evaluation to a known answer (src/tests/test_geopotential.cpp:78-140):
one coefficient at a time (every n = 2..8, m = 0..n, cosine and sine), 17 spheres of radius
1828.1828 * (-2.2)^k about a body of radius 1415.9265, 18 x 35 directions including both poles, relative
error below 1e-13 of the largest field on each sphere, and the field next to the polar axis continuous with
the value on it. The same grid and bound are used here against an independent exact evaluation
(tests/harmonics_ref.py: harmonic polynomials with rational coefficients, longdouble evaluation):

* the oracle's restatement of the reference's evaluation (CPU), and
* the device functions of the integration kernels (`eph_geopotential_field`, GPU: one point per thread as
  the particle kernels evaluate it, one point per 8 lanes and one point per lane as the step kernel does),
  which use Cunningham's Cartesian recursion, plus a comparison with the oracle on random full models.
"""
import ctypes

import numpy as np
import pytest

from tests import harmonics_ref as H


def _models(tab, nz, nt):
    from oracle.pyoracle import Models
    return Models(np.array([nz], np.int32), np.array([nt], np.int32), tab[None, :].copy(), np.zeros(0, np.int32),
                  np.zeros((0, 4)), np.zeros((0, 64, 3)))


def _rel(got, ref):
    ref = np.asarray(ref, dtype=float)
    return np.linalg.norm(got - ref, axis=1).max() / np.linalg.norm(ref, axis=1).max()


def test_oracle_geopotential_known_answer(oracle):
    spheres = list(H.kat_spheres())[::8]        # radii k = 1, 9, 17 of the 17 (CPU time)
    worst = 0.0
    for n, m, sine, tab, nz, nt in H.kat_cases():
        md = _models(tab, nz, nt)
        for pts in spheres:
            got = np.array([oracle.geopotential_sum(md, 0, H.KAT_R, p) for p in pts])
            worst = max(worst, _rel(got, H.model_field(tab, nz, nt, H.KAT_R, pts)))
    assert worst < H.KAT_EPS, worst


def _device_field(tab, nz, nt, R, pts, lanes=1):
    from ephemeris_b200 import load_library
    lib = load_library()
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    out = np.zeros_like(pts)
    D = ctypes.POINTER(ctypes.c_double)
    rc = lib.eph_geopotential_field(0, np.ascontiguousarray(tab).ctypes.data_as(D), nz, nt, R, lanes, len(pts),
                                    pts.ctypes.data_as(D), out.ctypes.data_as(D))
    assert rc == 0, rc
    return out


def test_geopotential_field_rejects_bad_arguments():
    from ephemeris_b200 import load_library
    lib = load_library()
    D = ctypes.POINTER(ctypes.c_double)
    tab = np.zeros(77)
    p = np.zeros(3)
    o = np.zeros(3)
    args = (tab.ctypes.data_as(D), 1.0, 1, 1, p.ctypes.data_as(D), o.ctypes.data_as(D))
    assert lib.eph_geopotential_field(0, args[0], 9, 0, *args[1:]) == 1       # degree above 8
    assert lib.eph_geopotential_field(0, args[0], 4, 5, *args[1:]) == 1       # tesseral above zonal
    assert lib.eph_geopotential_field(0, None, 4, 4, *args[1:]) == 1
    assert lib.eph_geopotential_field(0, args[0], 4, 4, 1.0, 4, 1, args[4], args[5]) == 1   # lanes not 0, 1 or 8


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [0, 1, 8])
def test_device_geopotential_known_answer(lanes):
    worst, worst_axis = 0.0, 0.0
    for n, m, sine, tab, nz, nt in H.kat_cases():
        for k, pts in enumerate(H.kat_spheres()):
            ref = H.model_field(tab, nz, nt, H.KAT_R, pts)
            got = _device_field(tab, nz, nt, H.KAT_R, pts, lanes)
            scale = np.linalg.norm(np.asarray(ref, dtype=float), axis=1).max()
            worst = max(worst, np.linalg.norm(got - np.asarray(ref, dtype=float), axis=1).max() / scale)
            rn = np.linalg.norm(pts[0])
            near = H.near_axis_points(k, rn)
            on = _device_field(tab, nz, nt, H.KAT_R, np.stack([np.zeros(len(near)), np.zeros(len(near)), near[:, 2]], 1),
                               lanes)
            got_near = _device_field(tab, nz, nt, H.KAT_R, near, lanes)
            worst_axis = max(worst_axis, np.linalg.norm(got_near - on, axis=1).max() / scale)
    assert worst < H.KAT_EPS, worst
    assert worst_axis < H.KAT_EPS, worst_axis


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [0, 1, 8])
def test_device_geopotential_matches_oracle(oracle, lanes):
    rng = np.random.default_rng(77)
    worst = 0.0
    for _ in range(40):
        nz = int(rng.integers(2, 9))
        nt = int(rng.integers(0, nz + 1))
        tab = np.zeros(77)
        for n in range(2, nz + 1):
            tab[n * n - 4] = rng.normal() * 1e-3 / n
            if n <= nt:
                tab[n * n - 4 + 1:n * n - 4 + 2 * n + 1] = rng.normal(size=2 * n) * 1e-3 / n
        R = 6.0e7
        pts = rng.normal(size=(256, 3))
        pts *= (R * rng.uniform(1.02, 40.0, size=256) / np.linalg.norm(pts, axis=1))[:, None]
        md = _models(tab, nz, nt)
        ref = np.array([oracle.geopotential_sum(md, 0, R, p) for p in pts])
        got = _device_field(tab, nz, nt, R, pts, lanes)
        err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        worst = max(worst, err.max())
    assert worst < 1e-13, worst
