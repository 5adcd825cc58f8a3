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


def test_ensemble_autotune(tmp_path, oracle):
    """The ensemble launch's cluster-sharing threshold, tuned on a 48-member ensemble (5 % of each member's
    steps): never slower than the default, the uploaded state left as it was, and the members integrated
    with the chosen threshold still within the parity tolerances."""
    import os
    from ephemeris_b200 import Batch, MSystem, synth
    from oracle.pyoracle import Models as OModels
    ens = synth.make_ensemble(48, seed=3011)
    pls, mds, dts, ks = [], [], [], []
    for s, (m, k) in enumerate(ens):
        ms = MSystem(0)
        assert ms.load(synth.write_system(m, os.path.join(str(tmp_path), f"s{s}")))
        pls.append(ms.planes())
        mds.append(ms.models())
        dts.append(ms.delta_t)
        ks.append(k)
    b = Batch(0)
    b.upload(pls, mds)
    cm, t_tuned, t_default = b.autotune(dts, ks, step_frac=0.05)
    print(f"ensemble: cluster threshold {cm} bodies, {t_tuned:.1f} ms tuned, {t_default:.1f} ms default")
    assert t_tuned <= t_default
    for out, pl in zip(b.download(), pls):
        assert np.array_equal(out, pl)
    b.integrate(dts, [3] * len(pls))
    outs = b.download()
    big = int(np.argmax([p.shape[1] for p in pls]))
    for s in (0, big):
        md = mds[s]
        ref = oracle.integrate(pls[s], OModels(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param,
                                               md.ring_disk), dts[s], 3)[0]
        assert position_error(outs[s], ref) <= 1e-12
    b.close()
