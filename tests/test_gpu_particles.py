"""Massless test particles (eph_particles_*) against the oracle.

The reference has no massless bodies (its loader requires GM > 0, src/mass/mass_loader.cpp:33); its
equivalent is a system of the perturbers plus the particles as bodies of GM = 1e-20 m^3/s^2, whose effect
on anything is below 1e-30 relative. Each test loads such a combined system, integrates it with the
oracle, and integrates the perturbers and the particles separately on the GPU from the same loaded
state. Tolerances are those of tests/test_gpu_parity.py: position 1e-12 of |r - r_0| (body 0 is the
star, or the planet of a planetary subsystem) for perturbers and particles alike.
"""
import os

import numpy as np
import pytest

from tests.parity import position_error

pytestmark = pytest.mark.gpu

POS_TOL = 1e-12


def _combined(tmp_path, sysm, particles, name):
    from ephemeris_b200 import MSystem, synth
    cfg = synth.write_system(synth.with_test_bodies(sysm, particles), os.path.join(str(tmp_path), name))
    ms = MSystem(0)
    assert ms.load(cfg)
    pl, md = ms.planes(), ms.models()
    n_pert = len(sysm.bodies)
    assert (pl[39, n_pert:] == 1e-20).all() and (pl[39, :n_pert] > 1e-10).all()   # perturbers first
    return pl, md, ms.delta_t, n_pert


def _omodels(md):
    from oracle.pyoracle import Models
    return Models(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)


def _gpu(pl, md, n_pert, calls):
    """Perturbers = the first n_pert bodies, particles = the rest; calls: [(dt, n_step), ...]."""
    from ephemeris_b200 import Particles
    p = Particles(0)
    p.upload(np.ascontiguousarray(pl[:, :n_pert]), md, np.ascontiguousarray(pl[0:12, n_pert:]))
    t = (0.0, 0.0)
    for dt, k in calls:
        t = p.integrate(dt, k, t)
    pert, part = p.download()
    p.close()
    out = pl.copy()
    out[:, :n_pert] = pert
    out[0:12, n_pert:] = part
    return out, t


def _check(out, ref, n_pert):
    assert np.isfinite(out[0:12]).all()
    assert position_error(out[:, :n_pert], ref[:, :n_pert]) <= POS_TOL
    # particles: relative to their distance from body 0
    both = np.concatenate([out[:, :1], out[:, n_pert:]], axis=1)
    both_ref = np.concatenate([ref[:, :1], ref[:, n_pert:]], axis=1)
    assert position_error(both, both_ref) <= POS_TOL


def test_particles_against_star_and_planets(tmp_path, oracle):
    """The particle workload's recipe at 300 particles (two CTAs' worth, the second ragged): a star with
    J2 and J3-J4 and 8 planets, Newtonian + 1PN; two calls of 4 and 3 steps."""
    from ephemeris_b200 import synth
    sysm, parts = synth.make_config5(5005, n_particles=300)
    pl, md, dt, n_pert = _combined(tmp_path, sysm, parts, "c5")
    assert n_pert == 9
    ref, t1, _ = oracle.integrate(pl, _omodels(md), dt, 4)
    ref, t2, _ = oracle.integrate(ref, _omodels(md), dt, 3, t1)
    out, t = _gpu(pl, md, n_pert, [(dt, 4), (dt, 3)])
    _check(out, ref, n_pert)
    assert t == t2


def test_particles_around_a_ringed_planet(tmp_path, oracle):
    """Every field a particle can feel: a spinning, tidally deformed planet with J2..J6 and degree-4
    geopotential, a ring annulus (1.2-2.3 radii) and four tidally locked moons; particles at 2.6-12 planet
    radii (some inside the moons' orbits), inclinations up to 30 degrees to the planet's equator plane."""
    from ephemeris_b200 import synth
    sysm = synth.make_ringed_subsystem(ring_ratio=0.05)
    host = sysm.bodies[0]
    rng = np.random.default_rng(6016)
    n = 200
    a = rng.uniform(2.6, 12.0, n) * host.R_km * 1e3
    parts = synth.kepler_cloud(rng, host.GM, a, rng.uniform(0, 0.1, n), rng.uniform(0, 30 * synth.DEG, n),
                               host.r, host.v)
    pl, md, dt, n_pert = _combined(tmp_path, sysm, parts, "ringed")
    ref = oracle.integrate(pl, _omodels(md), dt, 8)[0]
    out, _ = _gpu(pl, md, n_pert, [(dt, 8)])
    _check(out, ref, n_pert)


def test_particles_backwards_and_repeat(tmp_path, oracle):
    """A backward call (negative step count) against the oracle; the same upload and calls repeat bit
    for bit."""
    from ephemeris_b200 import synth
    sysm, parts = synth.make_config5(5006, n_particles=40)
    pl, md, dt, n_pert = _combined(tmp_path, sysm, parts, "back")
    ref = oracle.integrate(pl, _omodels(md), dt, -5)[0]
    out, _ = _gpu(pl, md, n_pert, [(dt, -5)])
    _check(out, ref, n_pert)
    again, _ = _gpu(pl, md, n_pert, [(dt, -5)])
    assert np.array_equal(out[0:12], again[0:12])


def test_mixed_precision_particles(tmp_path, oracle):
    """EPH_PREC_MIXED (EIH 1PN in FP32) on the particle workload's recipe and on the ringed planet (its
    general field path): within the FP64 tolerance of the oracle, and within 1e-14 of the FP64 GPU path
    after 20 steps of 0.5 day."""
    from ephemeris_b200 import Particles, synth
    sysm, parts = synth.make_config5(5007, n_particles=300)
    pl, md, dt, n_pert = _combined(tmp_path, sysm, parts, "mixed")
    ref = oracle.integrate(pl, _omodels(md), dt, 20)[0]
    outs = []
    for mixed in (False, True):
        p = Particles(0)
        p.set_precision(mixed)
        p.upload(np.ascontiguousarray(pl[:, :n_pert]), md, np.ascontiguousarray(pl[0:12, n_pert:]))
        p.integrate(dt, 20)
        pert, part = p.download()
        p.close()
        out = pl.copy()
        out[:, :n_pert] = pert
        out[0:12, n_pert:] = part
        outs.append(out)
        _check(out, ref, n_pert)
    both = [np.concatenate([o[:, :1], o[:, n_pert:]], axis=1) for o in outs]
    assert position_error(both[1], both[0]) <= 1e-14

    sysm = synth.make_ringed_subsystem(ring_ratio=0.05)
    host = sysm.bodies[0]
    rng = np.random.default_rng(6017)
    a = rng.uniform(2.6, 12.0, 64) * host.R_km * 1e3
    parts = synth.kepler_cloud(rng, host.GM, a, rng.uniform(0, 0.1, 64), rng.uniform(0, 30 * synth.DEG, 64),
                               host.r, host.v)
    pl, md, dt, n_pert = _combined(tmp_path, sysm, parts, "ringed_mixed")
    ref = oracle.integrate(pl, _omodels(md), dt, 8)[0]
    p = Particles(0)
    p.set_precision(True)
    p.upload(np.ascontiguousarray(pl[:, :n_pert]), md, np.ascontiguousarray(pl[0:12, n_pert:]))
    p.integrate(dt, 8)
    pert, part = p.download()
    out = pl.copy()
    out[:, :n_pert] = pert
    out[0:12, n_pert:] = part
    _check(out, ref, n_pert)


def test_full_size_workload_properties(tmp_path):
    """The particle workload at its full size (2 000 000 particles, 9 perturbers, dt = 0.5 day): 20 steps
    forward and 20 back return the particles to their start (all but 1e-4 of them within 1e-13 of
    |r - r_star|; a particle passing close to a planet amplifies the round trip's rounding, so the bound on
    every particle is 1e-9), and a sample of 64 particles integrated on their own gives bit-identical results
    (a particle's computation does not depend on the rest of the batch)."""
    from ephemeris_b200 import MSystem, Particles, synth
    sysm, parts = synth.make_config5(5005, n_particles=2_000_000)
    ms = MSystem(0)
    assert ms.load(synth.write_system(sysm, os.path.join(str(tmp_path), "pert")))
    pl, md, dt = ms.planes(), ms.models(), ms.delta_t
    p = Particles(0)
    p.upload(pl, md, parts)
    t = p.integrate(dt, 20)
    _, mid = p.download()
    p.integrate(-dt, 20, t)   # n_step > 0 with a negative dt: backwards
    _, back = p.download()
    assert np.isfinite(mid).all() and np.isfinite(back).all()
    r0 = parts[0:3]
    star = pl[0:3, 0] + pl[3:6, 0]
    err = np.linalg.norm((back[0:3] + back[3:6]) - r0, axis=0) / np.linalg.norm(r0 - star[:, None], axis=0)
    assert err.max() <= 1e-9, err.max()
    assert (err > 1e-13).mean() <= 1e-4, np.sort(err)[-10:]
    rng = np.random.default_rng(11)
    pick = np.sort(rng.choice(parts.shape[1], 64, replace=False))
    q = Particles(0)
    q.upload(pl, md, np.ascontiguousarray(parts[:, pick]))
    q.integrate(dt, 20)
    _, alone = q.download()
    assert np.array_equal(alone, mid[:, pick])


def test_full_size_mixed_precision_error(tmp_path):
    """Mixed precision at the workload's full size (2 000 000 particles, 20 steps of 0.5 day): every particle
    within 1e-14 of |r - r_star| of the FP64 run."""
    from ephemeris_b200 import MSystem, Particles, synth
    sysm, parts = synth.make_config5(5005, n_particles=2_000_000)
    ms = MSystem(0)
    assert ms.load(synth.write_system(sysm, os.path.join(str(tmp_path), "pert")))
    pl, md, dt = ms.planes(), ms.models(), ms.delta_t
    runs = []
    for mixed in (False, True):
        p = Particles(0)
        p.set_precision(mixed)
        p.upload(pl, md, parts)
        p.integrate(dt, 20)
        runs.append(p.download()[1])
        p.close()
    a, b = runs
    star = pl[0:3, 0] + pl[3:6, 0]
    r = b[0:3] + b[3:6]
    err = np.linalg.norm((a[0:3] - b[0:3]) + (a[3:6] - b[3:6]), axis=0) / np.linalg.norm(r - star[:, None], axis=0)
    assert np.isfinite(a).all() and err.max() <= 1e-14, err.max()
