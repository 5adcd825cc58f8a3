"""The C restatement oracle against the reference's own outputs (CPU only).

The oracle must reproduce the reference's serial CPU path bit for bit: the loaded state's
acceleration, every stage acceleration of the first step and the states after 1, 10, 100 and 1000 steps
(tests/golden/, recorded from the reference by tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from oracle.pyoracle import RefSystem, ref_available


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_accel_bit_exact(golden, oracle, name):
    g = golden(name)
    out = oracle.accel(g["load"], g.models())
    assert np.array_equal(out, g["accel"])


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_first_step_stage_accelerations_bit_exact(golden, oracle, name):
    g = golden(name)
    _, _, acc = oracle.integrate(g["load"], g.models(), float(g["dt"]), 1, stage_acc=True)
    assert np.array_equal(acc, g["stage_acc"])


def _chained(oracle, g, upto):
    """integrate() in the same calls as the recording (1, then up to each recorded step count):
    the per-pair maxima are reset at every call (src/physics/mass.cpp:406)."""
    pl, t, done = g["load"], (0.0, 0.0), 0
    for k in g.meta["steps"]:
        if k > upto:
            break
        pl, t, _ = oracle.integrate(pl, g.models(), float(g["dt"]), k - done, t_eph=t)
        done = k
    return pl, t


@pytest.mark.parametrize("name,steps", [("config1", 1), ("config1", 10), ("small_full", 10),
                                        ("small_full", 100), ("config2", 1)])
def test_steps_bit_exact(golden, oracle, name, steps):
    g = golden(name)
    out, t = _chained(oracle, g, steps)
    assert np.array_equal(out, g[f"step{steps}"])
    assert tuple(t) == tuple(g[f"t_eph{steps}"])


@pytest.mark.parametrize("name", ["config1", "small_full"])
def test_thousand_steps_bit_exact(golden, oracle, name):
    """1000 steps (with the recording's intermediate calls) of the Newtonian + 1PN system and of the
    full-physics test system (tides with lag, angular-velocity fixed point, geopotential, ring, rotation).
    The 504-body system's step 1000 is recorded too, for the GPU tests; the oracle's serial path takes
    minutes there, so it is checked at step 1 only."""
    g = golden(name)
    out, t = _chained(oracle, g, 1000)
    assert np.array_equal(out, g["step1000"])
    assert tuple(t) == tuple(g["t_eph1000"])


def test_deform_matches_reference_structure(golden, oracle):
    """deform() alone leaves C_potential/GI consistent with one pass of accel's harmonics update."""
    g = golden("small_full")
    d = oracle.deform(g["load"], g.models())
    assert np.all(np.isfinite(d[91:100])) and np.all(np.isfinite(d[82:91]))


def test_backward_integration_flips_dt(golden, oracle):
    g = golden("config1")
    fwd, t1, _ = oracle.integrate(g["load"], g.models(), float(g["dt"]), 2)
    back, t2, _ = oracle.integrate(fwd, g.models(), float(g["dt"]), -2, t_eph=t1)
    assert t2 == (0.0, 0.0)
    # RK12 is not time-symmetric, but two steps there and back return to the start closely
    from tests.parity import position_error
    assert position_error(back, g["load"]) < 1e-12


@pytest.mark.skipif(not ref_available(), reason="reference library oracle/_ref not built here")
@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_matches_live_reference(tmp_path, oracle, seed):
    """Fresh seeds of the full-physics recipe, reference vs restatement, 2 steps."""
    from ephemeris_b200 import synth
    cfg = synth.write_workload("small_full", str(tmp_path / f"s{seed}"), seed=seed, n_bodies=30)
    ref = RefSystem(cfg)
    RefSystem.thread_pool(False)
    p0, m = ref.planes(), ref.models()
    dt = ref.lib().ref_delta_t(ref.h)
    ref.integrate(dt, 2)
    out, _, _ = oracle.integrate(p0, m, dt, 2)
    assert np.array_equal(out, ref.planes())
