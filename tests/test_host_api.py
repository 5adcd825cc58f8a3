"""Host-side behaviour of the particle, serving and B-spline entry points that needs no GPU: argument
checks happen before any device work and return the documented status codes."""
import ctypes

import numpy as np
import pytest

EPH_ERR_ARG, EPH_ERR_LIMIT = 1, 8


def _lib():
    from ephemeris_b200._lib import load_library
    return load_library()


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def test_bspline_fit_batch_rejects_bad_sizes_before_device_work():
    L = _lib()
    smp = np.zeros((2, 4, 10))
    out = np.zeros((2, 8, 10))
    assert L.eph_bspline_fit_batch(0, 3, 5, 3, 10, 2, _d(smp), _d(out)) == EPH_ERR_ARG   # n + d > mn + 1
    assert L.eph_bspline_fit_batch(0, 0, 1, 3, 10, 2, _d(smp), _d(out)) == EPH_ERR_ARG   # degree 0
    assert L.eph_bspline_fit_batch(0, 3, 1, 3, 0, 2, _d(smp), _d(out)) == EPH_ERR_ARG    # no channels
    assert L.eph_bspline_fit_batch(0, 3, 1, 3, 10, 2, None, _d(out)) == EPH_ERR_ARG


def test_serve_create_rejects_bad_arguments():
    L = _lib()
    h = ctypes.c_void_p()
    gm = np.ones(3)
    coef = np.zeros((3, 13, 10))
    assert L.eph_serve_create(0, 0, _d(gm), None, 3, 10, 0.0, 86400.0, _d(coef), ctypes.byref(h)) == EPH_ERR_ARG
    assert L.eph_serve_create(0, 3, _d(gm), None, 9, 10, 0.0, 86400.0, _d(coef), ctypes.byref(h)) == EPH_ERR_ARG
    assert L.eph_serve_create(0, 3, _d(gm), None, 3, 10, 0.0, 0.0, _d(coef), ctypes.byref(h)) == EPH_ERR_ARG
    assert L.eph_serve_create(0, 3, _d(gm), None, 3, 10, 0.0, 86400.0, None, ctypes.byref(h)) == EPH_ERR_ARG
    assert L.eph_serve_create(0, 2000, _d(gm), None, 3, 10, 0.0, 86400.0, _d(coef), ctypes.byref(h)) == EPH_ERR_ARG
    assert not h.value


def test_null_handles_are_rejected():
    L = _lib()
    z = ctypes.c_double()
    n = ctypes.c_int64()
    st = ctypes.c_int()
    assert L.eph_particles_upload(None, 1, None, None, 1, None) == EPH_ERR_ARG
    assert L.eph_particles_integrate(None, 1.0, 1, ctypes.byref(z), ctypes.byref(z)) == EPH_ERR_ARG
    assert L.eph_particles_set_precision(None, 0) == EPH_ERR_ARG
    assert L.eph_serve_submit(None, 1, None, 0.0, 1.0, 1e-13, 1.0, ctypes.byref(n)) == EPH_ERR_ARG
    assert L.eph_serve_poll(None, 1, ctypes.byref(st)) == EPH_ERR_ARG
    assert L.eph_serve_result(None, 1, None, None, None, None, None) == EPH_ERR_ARG
    assert L.eph_record_samples(None, 1.0, 2, 1, ctypes.byref(z), ctypes.byref(z), None) == EPH_ERR_ARG


def test_particle_and_serve_creation_without_a_device_fails_cleanly():
    """No GPU here: creation reports an error (and no handle) instead of crashing."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib()
    h = ctypes.c_void_p()
    assert L.eph_particles_create(0, ctypes.byref(h)) != 0 and not h.value
    gm = np.ones(3)
    coef = np.zeros((3, 13, 10))
    assert L.eph_serve_create(0, 3, _d(gm), None, 3, 10, 0.0, 86400.0, _d(coef), ctypes.byref(h)) != 0 and not h.value
