"""The B-spline ephemeris fitter (eph_bspline_fit, host code of libeph_b200.so) against the reference's own
bspline_fitter (src/math/interp.h:68-150, compiled from its sources into oracle/_ref/libephref.so).

* The Chebyshev form of the basis, c(d, k, j), equals the reference's table bit for bit for the cubic
  (and lower) degree the ephemeris uses, and within 1.2e-16 up to degree 8.
* Fits of the reference test's own data (sin and cos of 0.1 i, src/tests/test_bspline.cpp:18-39, the
  cases with d <= 8) are bit-identical to the reference's coefficients for d <= 3, and for higher degrees
  within 1e-10 of them (the normal equations grow ill-conditioned with the degree) and within the
  reference test's own error bound of the fitted function.
"""
import ctypes
import os

import numpy as np
import pytest

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libephref.so")
_D = ctypes.POINTER(ctypes.c_double)
CASES = [(1, 1, 1, 1e-2), (1, 1, 2, 2e-2), (1, 20, 20, 1e-2), (2, 1, 2, 1e-3), (2, 19, 20, 2e-4), (2, 10, 20, 1e-3),
         (3, 1, 3, 5e-5), (3, 10, 20, 2e-5), (4, 1, 4, 5e-6), (4, 160, 1000, 5e-5), (5, 200, 1000, 2e-6),
         (6, 220, 1000, 2e-7), (7, 240, 1000, 5e-9), (8, 200, 1000, 3e-9)]


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    L = ctypes.CDLL(REF)
    L.ref_bspline_cheb_coef.restype = ctypes.c_double
    L.ref_bspline_cheb_coef.argtypes = [ctypes.c_int] * 3
    L.ref_bspline_fit.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, _D, _D]
    L.ref_bspline_eval.argtypes = [ctypes.c_int, _D, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int64, _D, _D, _D]
    return L


def test_chebyshev_table_matches_reference(ref):
    from ephemeris_b200._lib import load_library
    L = load_library()
    for d in range(0, 9):
        for k in range(d + 1):
            for j in range(d + 1):
                a, b = L.eph_bspline_cheb_coef(d, k, j), ref.ref_bspline_cheb_coef(d, k, j)
                if d <= 3:
                    assert a == b, (d, k, j)
                else:
                    assert abs(a - b) <= 1.2e-16, (d, k, j, a, b)


@pytest.mark.parametrize("d,n,mn,bound", CASES)
def test_fit_matches_reference(ref, d, n, mn, bound):
    from ephemeris_b200 import bspline_fit
    i = np.arange(mn + 1)
    xy = np.ascontiguousarray(np.stack([np.sin(i * 0.1), np.cos(i * 0.1)], 1))
    got = bspline_fit(xy, n, d)
    want = np.empty((n + d, 2))
    assert ref.ref_bspline_fit(2, d, n, mn, xy.ctypes.data_as(_D), want.ctypes.data_as(_D)) == 0
    if d <= 3:
        assert np.array_equal(got, want)
    else:
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    # the fitted function through the reference's own evaluator, against sin / cos
    x = np.linspace(0, mn, 4001)
    val, der = np.empty((len(x), 2)), np.empty((len(x), 2))
    assert ref.ref_bspline_eval(2, np.ascontiguousarray(got).ctypes.data_as(_D), d, n, float(mn), 0, len(x),
                                x.ctypes.data_as(_D), val.ctypes.data_as(_D), der.ctypes.data_as(_D)) == 0
    err = max(np.abs(val[:, 0] - np.sin(0.1 * x)).max(), np.abs(val[:, 1] - np.cos(0.1 * x)).max())
    assert err <= bound, err


def test_fit_rejects_bad_sizes():
    from ephemeris_b200 import bspline_fit, EphError
    with pytest.raises(EphError):
        bspline_fit(np.zeros((3, 2)), 5, 3)      # n + d > mn + 1
    with pytest.raises(EphError):
        bspline_fit(np.zeros((30, 2)), 5, 9)     # degree above the maximum
