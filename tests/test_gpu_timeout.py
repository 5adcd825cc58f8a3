"""The bounded device-side waits end, report EPH_ERR_TIMEOUT and leave the context usable.

Every wait of the step kernel (grid barrier, tile copy) has a time limit after which the kernel records a
status word and returns; it never traps or hangs. eph_selftest_wait_timeout makes one launch whose grid
barriers wait for one arrival more than the launch has, with a 1 ms limit: every CTA's wait runs out. No
GPU fault is involved: the kernel simply returns, and the next call on the same context runs normally.
"""
import ctypes
import time

import numpy as np
import pytest

EPH_ERR_ARG = 1
EPH_ERR_TIMEOUT = 4


def _lib():
    from ephemeris_b200 import load_library
    return load_library()


def test_selftest_rejects_bad_arguments():
    lib = _lib()
    assert lib.eph_selftest_wait_timeout(None, 1_000_000) == EPH_ERR_ARG


@pytest.mark.gpu
def test_bounded_wait_runs_out_and_context_stays_usable(golden):
    from ephemeris_b200 import Context, Models
    g = golden("small_full")
    m = g.models()
    models = Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)
    lib = _lib()
    ctx = Context(0)
    ctx.upload(g["load"], models)
    assert ctx.launch_shape()[0] > 1                       # a grid barrier exists
    assert lib.eph_selftest_wait_timeout(ctx.h, 10) == EPH_ERR_ARG           # limit below 0.1 ms
    assert lib.eph_selftest_wait_timeout(ctx.h, 5_000_000_000) == EPH_ERR_ARG  # limit above 2 s
    t0 = time.perf_counter()
    rc = lib.eph_selftest_wait_timeout(ctx.h, 1_000_000)
    elapsed = time.perf_counter() - t0
    assert rc == EPH_ERR_TIMEOUT, rc
    assert b"timed out" in lib.eph_last_error(ctx.h)
    assert elapsed < 2.0, elapsed
    assert np.array_equal(ctx.download(), g["load"])        # the planes were not written
    # the same context integrates normally afterwards, bit for bit like a fresh one
    dt = float(g["dt"])
    t = ctx.integrate(dt, 2)
    fresh = Context(0)
    fresh.upload(g["load"], models)
    t2 = fresh.integrate(dt, 2)
    assert tuple(t) == tuple(t2)
    assert np.array_equal(ctx.download(), fresh.download())
    ctx.close()
    fresh.close()
