"""Parity of the CUDA RK12 path against the oracle and the reference's recorded outputs (GPU).

Tolerances (floating point; the GPU sums pairs in a different order and contracts products into FMAs):
  * per-stage acceleration: max_i |da_i| / sum_j |GM_j/r_ij^2| <= 1e-14
  * position after N steps: max_i |dr_i| / |r_i - r_star| <= 1e-12 (N = 1000 for the 33-body system)
  * after one step, the reference's own CPU-vs-GPU bounds of test_integrator
    (src/tests/test_integrator.cpp:15-20,22-45): r 1e-6 m, v 1e-8 m/s, w 1e-16, s.x/s.z 1e-13,
    scaled by 86400/t, and 1e-15 relative on min_distance / max_influence.
"""
import numpy as np
import pytest

from tests.parity import accel_error, position_error, rel_err

pytestmark = pytest.mark.gpu

ACC_TOL = 1e-14
POS_TOL = 1e-12


def _models(g):
    from ephemeris_b200 import Models
    m = g.models()
    return Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)


def _ctx(g, planes=None):
    from ephemeris_b200 import Context
    c = Context(0)
    c.upload(g["load"] if planes is None else planes, _models(g))
    return c


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_accel_matches_reference(golden, name):
    g = golden(name)
    c = _ctx(g)
    c.accel()
    out = c.download()
    assert accel_error(out, g["accel"]) <= ACC_TOL
    # torque and angular velocity of rotating bodies
    scale = np.abs(g["accel"][73:76]).max() or 1.0
    assert np.abs(out[73:76] - g["accel"][73:76]).max() <= 1e-12 * scale
    w = g["accel"][36:39]
    assert np.abs(out[36:39] - w).max() <= 1e-14 * (np.abs(w).max() or 1.0)


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_every_stage_acceleration(golden, oracle, name):
    """All 25 stage evaluations of a step, each from the oracle's own stage state."""
    g = golden(name)
    _, _, s_in, s_out = oracle.integrate_stages(g["load"], g.models(), float(g["dt"]), 1)
    c = _ctx(g)
    worst = 0.0
    for k in range(s_in.shape[0]):
        c.upload(s_in[k], _models(g))
        c.accel()
        worst = max(worst, accel_error(c.download(), s_out[k]))
    assert worst <= ACC_TOL, worst


def _test_integrator_bounds(out, ref, t_eph):
    """src/tests/test_integrator.cpp:22-45 with ref_cgpu_err (:16)."""
    f = 86400.0 / t_eph
    norm = lambda d: np.sqrt((d ** 2).sum(0)).max()
    dr = (out[0:3] - ref[0:3]) + (out[3:6] - ref[3:6])
    dv = (out[6:9] - ref[6:9]) + (out[9:12] - ref[9:12])
    errs = [norm(dr) * f / 1e-6, norm(dv) * f / 1e-8, norm(out[36:39] - ref[36:39]) * f / 1e-16,
            norm(out[18:21] - ref[18:21]) * f / 1e-13, norm(out[24:27] - ref[24:27]) * f / 1e-13]
    for p in (100, 101):
        errs.append(rel_err(out[p], ref[p]) / 1e-15)
    return max(errs)


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_one_step_within_reference_cpu_gpu_bounds(golden, name):
    g = golden(name)
    c = _ctx(g)
    t = c.integrate(float(g["dt"]), 1)
    out = c.download()
    assert tuple(t) == tuple(g["t_eph1"])
    assert position_error(out, g["step1"]) <= POS_TOL
    assert _test_integrator_bounds(out, g["step1"], t[0] + t[1]) < 1.0


def test_thousand_steps_position(golden):
    g = golden("config1")
    c = _ctx(g)
    t = (0.0, 0.0)
    done = 0
    for k in g.meta["steps"]:
        t = c.integrate(float(g["dt"]), k - done, t)
        done = k
        err = position_error(c.download(), g[f"step{k}"])
        assert err <= POS_TOL, (k, err)


def test_ten_steps_full_physics(golden):
    g = golden("small_full")
    c = _ctx(g)
    t = c.integrate(float(g["dt"]), 1)
    t = c.integrate(float(g["dt"]), 9, t)
    out = c.download()
    assert position_error(out, g["step10"]) <= POS_TOL
    assert rel_err(out[36:39], g["step10"][36:39], floor=np.abs(g["step10"][36:39]).max()) <= 1e-12


def test_rk12_entry_point_matches_integrate(golden):
    """eph_rk12 (Cuda_RungeKutta12 semantics) leaves the maxima to the caller; the state is the same."""
    g = golden("small_full")
    a, b = _ctx(g), _ctx(g)
    a.integrate(float(g["dt"]), 2)
    b.rk12(float(g["dt"]), 2)
    pa, pb = a.download(), b.download()
    assert np.array_equal(pa[:100], pb[:100])


@pytest.mark.parametrize("name", ["config1", "small_full"])
def test_launch_shapes_agree(golden, name):
    """Different CTA counts / bodies per CTA only reorder sums: same result within tolerance."""
    g = golden(name)
    outs = []
    for grid, per in [(0, 0), (0, 1), (0, 4), (0, 8)]:
        c = _ctx(g)
        c.set_launch(grid, per)
        c.integrate(float(g["dt"]), 2)
        outs.append(c.download())
    for o in outs[1:]:
        assert position_error(o, outs[0]) <= POS_TOL


def test_loader_matches_reference(golden):
    from ephemeris_b200 import MSystem
    g = golden("small_full")
    ms = MSystem(0)
    assert ms.load(g.config_path())
    pl = ms.planes()
    ref = g["load"]
    assert ms.sids() == list(g["sids"])
    # state and constants are parsed and built identically
    for p in list(range(0, 36)) + list(range(39, 56)) + [102, 103]:
        assert np.array_equal(pl[p], ref[p]), p
    # static harmonics corrected by the device deformation, relative to each body's matrix scale
    scale = np.abs(ref[56:65]).max(0)
    scale[scale == 0] = 1.0
    assert (np.abs(pl[56:65] - ref[56:65]) / scale).max() <= 1e-13
    assert accel_error(pl, ref) <= ACC_TOL


def test_msystem_integrate_and_errors(golden):
    from ephemeris_b200 import MSystem, EphError
    g = golden("config1")
    ms = MSystem(0)
    assert ms.load(g.config_path())
    ms.integrate(float(g["dt"]), 1, 1)
    assert ms.t_eph == tuple(g["t_eph1"])
    with pytest.raises(EphError):
        ms.integrate(float(g["dt"]), 1, 0)      # no CPU integrator in this library
    with pytest.raises(EphError):
        ms.accel(0)
    assert not MSystem(0).load("/nonexistent/Config.txt")


def test_c_abi_argument_errors(golden):
    from ephemeris_b200 import Context, EphError
    c = Context(0)
    with pytest.raises(EphError):
        c.accel()                                # nothing uploaded
    g = golden("config1")
    bad = g["load"].copy()
    bad[102, 0] = 5.0                            # geopotential index without a model
    with pytest.raises(EphError):
        c.upload(bad)
    with pytest.raises(EphError):
        c.set_launch(0, 99)
