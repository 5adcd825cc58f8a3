"""eph_integrate_noalloc: the integration entry point that allocates nothing (its working memory is a fixed
array compiled into the library) against the context path eph_upload_system + eph_integrate.

Tolerances are the parity tests' own: position max_i |dr_i| / |r_i - r_star| <= 1e-12 and acceleration
max_i |da_i| / sum_j |GM_j/r_ij^2| <= 1e-14 (tests/test_gpu_parity.py).
"""
import ctypes

import numpy as np
import pytest

from tests.parity import accel_error, position_error

POS_TOL = 1e-12
ACC_TOL = 1e-14
MAX_BODIES = 1024          # EPH_NOALLOC_MAX_BODIES
MAX_GP = 16                # EPH_NOALLOC_MAX_GP
MAX_EXT = 16               # EPH_NOALLOC_MAX_EXT
EPH_ERR_ARG = 1
EPH_ERR_LIMIT = 8
P_GP_INDEX = 102           # EPH_P_GP_INDEX


def _lib():
    from ephemeris_b200._lib import load_library
    return load_library()


def _models(g):
    from ephemeris_b200 import Models
    m = g.models()
    return Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)


def _noalloc(lib, d_planes, n, models, dt, n_step, t):
    hi, lo = ctypes.c_double(t[0]), ctypes.c_double(t[1])
    st = models.struct()
    rc = lib.eph_integrate_noalloc(0, None, n, d_planes.data_ptr(), ctypes.byref(st), dt, n_step,
                                   ctypes.byref(hi), ctypes.byref(lo))
    return rc, (hi.value, lo.value)


def test_sizes_beyond_the_limit_are_rejected():
    """Checked on the host before any device work (no GPU needed); the planes pointer is never read."""
    from ephemeris_b200 import Models
    lib = _lib()
    hi, lo = ctypes.c_double(0.0), ctypes.c_double(0.0)
    fake = ctypes.c_void_p(256)
    st = Models.empty().struct()
    rc = lib.eph_integrate_noalloc(0, None, MAX_BODIES + 1, fake, ctypes.byref(st), 1.0, 1,
                                   ctypes.byref(hi), ctypes.byref(lo))
    assert rc == EPH_ERR_LIMIT
    nz = np.zeros(MAX_GP + 1, np.int32)
    coef = np.zeros((MAX_GP + 1, 77))
    big = Models(nz, nz.copy(), coef, np.zeros(0, np.int32), np.zeros((0, 4)), np.zeros((0, 64, 3)))
    st = big.struct()
    rc = lib.eph_integrate_noalloc(0, None, 8, fake, ctypes.byref(st), 1.0, 1, ctypes.byref(hi), ctypes.byref(lo))
    assert rc == EPH_ERR_LIMIT


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_full", "config2"])
def test_noalloc_matches_context_path_on_two_calls(golden, name):
    import torch
    from ephemeris_b200 import Context
    g = golden(name)
    lib = _lib()
    dt = float(g["dt"])
    n = g["load"].shape[1]
    models = _models(g)

    ctx = Context(0)
    ctx.upload(g["load"], models)
    d = torch.from_numpy(np.ascontiguousarray(g["load"])).to("cuda:0")
    torch.cuda.synchronize()
    t_ref = t_na = (0.0, 0.0)
    dev = torch.cuda.current_device()
    for n_step in (3, 2, -2):   # calls in a row, each from the previous one's output; the last one backwards
        t_ref = ctx.integrate(dt, n_step, t_ref)
        want = ctx.download()
        rc, t_na = _noalloc(lib, d, n, models, dt, n_step, t_na)
        assert rc == 0, rc
        assert torch.cuda.current_device() == dev
        got = d.cpu().numpy()
        assert np.isfinite(got[0:12]).all()
        assert position_error(got, want) <= POS_TOL
        assert accel_error(got, want) <= ACC_TOL
        assert t_na == t_ref
    ctx.close()


@pytest.mark.gpu
def test_limits_checked_after_reading_the_planes(golden):
    """The extended-body limit and the model indices are checked once the planes are read from the device:
    EPH_ERR_LIMIT for more than EPH_NOALLOC_MAX_EXT bodies with a model, EPH_ERR_ARG for an index beyond the
    models; the caller's planes are left untouched and the caller's device stays current."""
    import torch
    g = golden("small_full")
    lib = _lib()
    models = _models(g)
    pl = np.array(g["load"])
    n = pl.shape[1]
    assert n > MAX_EXT
    many = pl.copy()
    many[P_GP_INDEX, :MAX_EXT + 1] = 0            # 17 bodies share geopotential model 0
    bad = pl.copy()
    bad[P_GP_INDEX, 3] = len(models.gp_nz)        # one past the last model
    dev = torch.cuda.current_device()
    for planes, want in ((many, EPH_ERR_LIMIT), (bad, EPH_ERR_ARG)):
        d = torch.from_numpy(np.ascontiguousarray(planes)).to("cuda:0")
        torch.cuda.synchronize()
        rc, t = _noalloc(lib, d, n, models, float(g["dt"]), 1, (0.0, 0.0))
        assert rc == want, rc
        assert t == (0.0, 0.0)
        assert np.array_equal(d.cpu().numpy(), planes)
        assert torch.cuda.current_device() == dev
