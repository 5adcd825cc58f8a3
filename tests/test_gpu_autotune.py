"""The launch-shape autotuner (eph_autotune) on the full-physics systems (GPU).

It times candidate shapes and ownership cost models, keeps the fastest, and leaves the uploaded state as it
was. The chosen shape must not be slower than the built-in heuristic (re-timed independently here, with a
3 % allowance for timing noise), its results must stay within the parity tolerances, and a second context
of the same system must get the cached choice.
"""
import time

import numpy as np
import pytest

from tests.parity import position_error

pytestmark = pytest.mark.gpu


def _models(g):
    from ephemeris_b200 import Models
    m = g.models()
    return Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)


def _ms_per_step(ctx, planes, models, dt, steps=5, reps=3):
    import torch
    best = float("inf")
    for _ in range(reps):
        ctx.upload(planes, models)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.integrate(dt, steps)
        best = min(best, (time.perf_counter() - t0) / steps * 1e3)
    return best


@pytest.mark.parametrize("name", ["small_full", "config2"])
def test_autotuned_shape_not_slower_and_correct(golden, name):
    from ephemeris_b200 import Context
    g = golden(name)
    models = _models(g)
    dt = float(g["dt"])
    c = Context(0)
    c.upload(g["load"], models)
    grid, per, t_tuned, t_default = c.autotune(dt, n_step=3, reps=2, use_cache=False)
    print(f"{name}: tuned grid {grid} x {per} bodies/CTA {t_tuned:.3f} ms per RK12 step, heuristic {t_default:.3f}")
    assert t_tuned <= t_default
    assert np.array_equal(c.download(), g["load"])        # the uploaded state is left as it was
    assert c.launch_shape() == (grid, per)
    tuned = _ms_per_step(c, g["load"], models, dt)
    h = Context(0)
    h.upload(g["load"], models)
    heuristic = _ms_per_step(h, g["load"], models, dt)
    assert tuned <= 1.03 * heuristic, (tuned, heuristic)
    c.upload(g["load"], models)
    c.integrate(dt, 1)
    assert position_error(c.download(), g["step1"]) <= 1e-12
    # the cached choice for a second context of the same system
    d = Context(0)
    d.upload(g["load"], models)
    assert d.autotune(dt, n_step=1, reps=1, use_cache=True)[:2] == (grid, per)
    for x in (c, h, d):
        x.close()
