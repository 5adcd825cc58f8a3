"""GPU code paths beyond the three fixture systems, each checked against the oracle or a known answer.

* A 1000-body full-physics system: more bodies than one shared-memory staging tile holds, so every
  sweep streams the bodies j through the tile in chunks (the fixtures all fit one tile).
* Systems of 1, 2 and 3 bodies (one CTA, empty or single-pair sweeps).
* The integrator order known-answer test of the reference (src/tests/test_order.cpp:10-99): a planet
  with a close moon integrated over the same span with eight step sizes; the order solved from
  successive differences of the moon's planet-relative position and velocity must exceed 11.375.

Tolerances are those of tests/test_gpu_parity.py: per-stage acceleration 1e-14 of sum_j |GM_j/r_ij^2|,
position 1e-12 of |r - r_star|.
"""
import math
import os

import numpy as np
import pytest

from tests.parity import accel_error, position_error

pytestmark = pytest.mark.gpu

ACC_TOL = 1e-14
POS_TOL = 1e-12


def _load(cfg):
    from ephemeris_b200 import MSystem
    ms = MSystem(0)
    assert ms.load(cfg)
    return ms


def _ctx(planes, models):
    from ephemeris_b200 import Context
    c = Context(0)
    c.upload(planes, models)
    return c


def test_streamed_tiles_system_matches_oracle(tmp_path, oracle):
    from ephemeris_b200 import synth
    from oracle.pyoracle import Models as OModels
    sysm = synth.make_config2(2002, n_asteroids=838)          # 1000 bodies
    cfg = synth.write_system(sysm, os.path.join(str(tmp_path), "big"))
    ms = _load(cfg)
    pl, md = ms.planes(), ms.models()
    assert pl.shape[1] == 1000
    om = OModels(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)
    c = _ctx(pl, md)
    c.accel()
    assert accel_error(c.download(), oracle.accel(pl, om)) <= ACC_TOL
    c = _ctx(pl, md)
    dt = ms.delta_t
    c.integrate(dt, 1)
    ref, _ = oracle.integrate(pl, om, dt, 1)[:2]
    out = c.download()
    assert position_error(out, ref) <= POS_TOL
    assert np.isfinite(out[0:12]).all()


@pytest.mark.parametrize("k", [1, 2, 3])
def test_tiny_systems_match_oracle(golden, oracle, k):
    g = golden("config1")
    pl = np.ascontiguousarray(g["load"][:, :k])
    md_o = g.models()
    from ephemeris_b200 import Models
    md = Models.empty()
    c = _ctx(pl, md)
    dt = float(g["dt"])
    c.integrate(dt, 20)
    out = c.download()
    ref = oracle.integrate(pl, md_o, dt, 20)[0]
    if k == 1:   # a lone body moves on a straight line: compare its state directly
        assert np.allclose(out[0:12], ref[0:12], rtol=1e-15, atol=0)
    else:
        assert position_error(out, ref) <= POS_TOL


def _order_solve(dratio, dt0, dt1, dt2):
    """Order p from dratio = (1 - b0^p) / (b1^p - 1), b0 = dt2/dt1, b1 = dt0/dt1, by Newton's method
    from the two-point estimate (the reference's solver, src/tests/test_order.cpp:10-35)."""
    b0, b1 = dt2 / dt1, dt0 / dt1
    lb0, lb1 = math.log(b0), math.log(b1)
    order = max(math.log(dratio) / (lb0 - lb1) * 2, 3.0)
    best, last, n_iter = math.nan, math.inf, 0
    while True:
        b1p, b0p = b1 ** order, b0 ** order
        diff = dratio * (b1p - 1) - (1 - b0p)
        if not abs(diff) < last:
            break
        best, last = order, abs(diff)
        order -= diff / (b0p * lb0 + b1p * dratio * lb1)
        n_iter += 1
    return best if n_iter >= 2 else math.nan


def test_integrator_order(tmp_path):
    """A star, a Mars-like planet and a Phobos-like moon (27 000 s period, 23 steps per orbit at the
    largest step), Newtonian + 1PN; eight step sizes dividing 950 400 s as in the reference test."""
    from ephemeris_b200 import synth
    gm_p, gm_m = 4.2828e13, 7.1e5
    rp, vp = synth._kepler_state(synth.GM_SUN + gm_p, 1.52 * synth.AU, 0.09, 0.03, 0.8, 5.0, 0.3)
    a_m = (gm_p * 27000.0 ** 2 / (4 * math.pi ** 2)) ** (1 / 3)
    rm, vm = synth._kepler_state(gm_p + gm_m, a_m, 0.015, 0.02, 0.3, 1.2, 2.0)
    bodies = [synth.Body("Star", "S0", synth.GM_SUN, 6.96e5),
              synth.Body("Planet", "P4", gm_p, 3390.0, r=tuple(rp), v=tuple(vp)),
              synth.Body("Moon", "M41", gm_m, 11.0, r=tuple(np.add(rp, rm)), v=tuple(np.add(vp, vm)))]
    synth._barycentric(bodies)
    cfg = synth.write_system(synth.System(bodies=bodies, delta_t=1200.0), os.path.join(str(tmp_path), "order"))
    ms = _load(cfg)
    pl, md = ms.planes(), ms.models()
    dts = [1200, 1080, 960, 880, 800, 720, 640, 600]
    span = 950400
    states = []
    for dt in dts:
        c = _ctx(pl, md)
        c.integrate(float(dt), span // dt)
        o = c.download()
        r = (o[0:3, 2] - o[0:3, 1]) + (o[3:6, 2] - o[3:6, 1])
        v = (o[6:9, 2] - o[6:9, 1]) + (o[9:12, 2] - o[9:12, 1])
        states.append((r, v))
    for i in range(1, len(dts) - 1):
        for q in range(2):
            d01 = np.linalg.norm(states[i - 1][q] - states[i][q])
            d12 = np.linalg.norm(states[i][q] - states[i + 1][q])
            dratio = d12 / d01
            assert 0 < dratio < 1, (i, q, dratio)
            order = _order_solve(dratio, dts[i - 1], dts[i], dts[i + 1])
            assert order > 11.375, (i, q, order)


def _momenta(pl, md):
    """Translational and angular momentum (times G), without and with the ring's share, as the
    reference's conservation test sums them (src/tests/test_conservation.cpp:25-86)."""
    r = pl[0:3] + pl[3:6]
    v = pl[6:9] + pl[9:12]
    gl = pl[12:15] + pl[15:18]
    gm = pl[39]
    out = np.zeros(12)
    for i in range(pl.shape[1]):
        dm = gm[i] * v[:, i]
        da = gm[i] * np.cross(r[:, i], v[:, i])
        das = gl[:, i] * gm[i]
        out[0:3] += dm
        out[3:6] += da + das
        out[6:9] += dm
        out[9:12] += da + das
        rg = int(pl[103, i])
        if rg >= 0:
            ratio, gl_r2 = md.ring_param[rg][0], md.ring_param[rg][3]
            out[6:9] += dm * (ratio / (1 - ratio))
            out[9:12] += da * (ratio / (1 - ratio))
            out[9:12] += gl[:, i] / np.linalg.norm(gl[:, i]) * (gl_r2 * gm[i] * pl[53, i])
    return out


def test_momentum_conservation(tmp_path):
    """The reference's conservation known-answer test (src/tests/test_conservation.cpp:6-112) on an
    isolated ringed planet (geopotential x3, a ring of 0.2 of its mass, tides, spin) with four tidally
    locked moons: over 6000 steps of 900 s the translational and angular momenta, with the ring's share,
    vary by less than 1e-12 of their size. The ring-correction factor (the same variation over the one
    without the ring's share) is bounded by 2e-8: the reference reaches 1.1e-8 on this system (its own test
    bounds 1e-8 on its Saturn data)."""
    from ephemeris_b200 import synth
    cfg = synth.write_system(synth.make_ringed_subsystem(ring_ratio=0.2), os.path.join(str(tmp_path), "ringed"))
    ms = _load(cfg)
    pl, md = ms.planes(), ms.models()
    c = _ctx(pl, md)
    hi, lo = np.full(12, -np.inf), np.full(12, np.inf)
    t = (0.0, 0.0)
    for _ in range(6000):
        t = c.integrate(900.0, 1, t)
        p = _momenta(c.download(), md)
        hi, lo = np.maximum(hi, p), np.minimum(lo, p)
    d = hi - lo
    err = max(np.linalg.norm(d[6:9]) / np.linalg.norm(hi[6:9]), np.linalg.norm(d[9:12]) / np.linalg.norm(hi[9:12]))
    err_plain = max(np.linalg.norm(d[0:3]) / np.linalg.norm(hi[6:9]), np.linalg.norm(d[3:6]) / np.linalg.norm(hi[9:12]))
    assert err < 1e-12, err
    assert err / err_plain < 2e-8, err / err_plain


def test_full_physics_run_repeats_bit_for_bit(tmp_path):
    """The 504-body full-physics workload, 50 RK12 steps twice from the same upload: identical planes (the
    persistent kernel's reductions and barriers fix every summation order)."""
    from ephemeris_b200 import synth
    cfg = synth.write_system(synth.make_config2(2002), os.path.join(str(tmp_path), "c2"))
    ms = _load(cfg)
    pl, md = ms.planes(), ms.models()
    outs = []
    for _ in range(2):
        c = _ctx(pl, md)
        c.integrate(ms.delta_t, 50)
        outs.append(c.download())
    assert np.isfinite(outs[0][0:12]).all()
    assert np.array_equal(outs[0], outs[1])
