"""Serving (eph_serve_*): massless particles with adaptive RK12 against a device B-spline ephemeris.

The ephemeris is built the way the serving workload builds it: the perturbers (the config4 recipe,
truncated to its first 40 bodies so that the oracle stays quick) are integrated on the GPU with
eph_record_samples (dt = 0.5 day), each body's 10 channels fitted with cubic B-splines at 1-day knots by
eph_bspline_fit. Checks:

* the device evaluation of the ephemeris against the reference's own B-spline sampling
  (src/math/interp.h:263-345, oracle/_ref) at arbitrary times;
* requests of 5 and 300 (32 lanes per particle, 1 and 38 blocks), 4096 (16 lanes) and 40 000 (one lane,
  157 blocks) particles: the first block's particles against the oracle replaying that block's accepted
  step sequence (oracle/serve_oracle.py), position within 1e-12 of |r - r_star|; every particle finite.
  A particle that passes within 0.01 AU of a planet (inside its Hill sphere: the 300-particle draw has one
  at 135 000 km from a Jupiter-mass planet) amplifies rounding differences of the two arithmetics by orders
  of magnitude; such particles are held to 1e-9;
* the tolerance: tol = 1e-13 against a run at tol = 1e-16 over the same span;
* many requests in flight and a memory budget that admits one at a time give the same results bit for bit;
* a backward request, and requests outside the ephemeris or with bad arguments are refused.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-12
DAY = 86400.0


@pytest.fixture(scope="module")
def eph(tmp_path_factory):
    from ephemeris_b200 import Context, MSystem, Server, bspline_fit, synth
    sysm = synth.make_config4_system(4004)
    sysm.bodies = sysm.bodies[:40]
    td = str(tmp_path_factory.mktemp("serve"))
    ms = MSystem(0)
    assert ms.load(synth.write_system(sysm, os.path.join(td, "pert")))
    pl, md = ms.planes(), ms.models()
    c = Context(0)
    c.upload(pl, md)
    days = 60
    samples, _ = c.record_samples(DAY / 2, 2 * days, 1)
    M = pl.shape[1]
    coefs = np.stack([bspline_fit(samples[:, j, :], days, 3) for j in range(M)])
    srv = Server(coefs, pl[39], DAY, 0.0, 3, pl[54])
    return dict(sysm=sysm, pl=pl, md=md, samples=samples, coefs=coefs, srv=srv, M=M, days=days, td=td)


def _particles(seed, n, eph, a=(0.8, 3.0), e=0.3):
    from ephemeris_b200 import synth
    rng = np.random.default_rng(seed)
    s0 = eph["samples"][0, 0]
    return synth.kepler_cloud(rng, synth.GM_SUN, rng.uniform(*a, n) * synth.AU, rng.uniform(0, e, n),
                              rng.uniform(0, 20 * synth.DEG, n), s0[0:3], s0[3:6])


def _rel_pos_err(r, r_ref, star):
    return float((np.linalg.norm(r - r_ref, axis=0) / np.linalg.norm(r_ref - star[:, None], axis=0)).max())


def test_ephemeris_evaluation_matches_reference_sampling(eph):
    from oracle.serve_oracle import RefSpline
    ref = RefSpline(eph["coefs"], 3, DAY)
    rng = np.random.default_rng(1)
    for t in list(rng.uniform(0, eph["days"] * DAY, 12)) + [0.0, 17 * DAY, eph["days"] * DAY]:
        got, want = eph["srv"].eval(t), ref(t)
        for lo, hi in ((0, 3), (3, 6), (6, 9), (9, 10)):
            scale = np.abs(want[:, lo:hi]).max(axis=1, keepdims=True)
            assert (np.abs(got[:, lo:hi] - want[:, lo:hi]) <= 4e-16 * np.maximum(scale, 1e-300) + 1e-300).all(), (t, lo)
    # at the sample times the fit reproduces the integration (cubic, 1-day knots, 0.5-day samples)
    s = eph["samples"]
    for q in (0, 31, 80):
        got = eph["srv"].eval(q * DAY / 2)
        r_err = np.linalg.norm(got[:, 0:3] - s[q, :, 0:3], axis=1) / np.linalg.norm(s[q, :, 0:3] - s[q, 0, 0:3], axis=1).clip(1)
        assert r_err[1:].max() < 1e-6


@pytest.mark.parametrize("n_part,lanes", [(5, 32), (300, 32), (4096, 16), (40000, 1)])
def test_request_matches_oracle_replay(eph, oracle, n_part, lanes):
    from ephemeris_b200 import MSystem, synth
    from oracle.serve_oracle import RefSpline, replay
    parts = _particles(100 + n_part, n_part, eph)
    srv = eph["srv"]
    srv.set_step_log(10000)
    rid = srv.submit(parts, 0.0, 20 * DAY, tol=1e-13, h0=DAY)
    g, per_block, blocks = srv.shape(rid)
    assert g == lanes and blocks == -(-n_part // per_block)
    out, acc, rej, steps = srv.result(rid, log_cap=10000)
    srv.set_step_log(0)
    assert acc >= 3 * n_part and len(steps) >= 3 and abs(sum(steps) - 20 * DAY) < 1e-3
    first = parts[:, :per_block]            # the logged steps are the first block's
    cfg = synth.write_system(synth.with_test_bodies(eph["sysm"], first), os.path.join(eph["td"], f"comb{n_part}"))
    ms = MSystem(0)
    assert ms.load(cfg)
    tmpl = ms.planes()
    z = np.zeros((3, first.shape[1]))
    r, v, mind = replay(oracle, tmpl, oracle_models(ms.models()), eph["M"], RefSpline(eph["coefs"], 3, DAY),
                        np.concatenate([first[0:3], z, first[3:6], z]), 0.0, steps)
    star = RefSpline(eph["coefs"], 3, DAY)(20 * DAY)[0, 0:3]
    got = out[0:3, :first.shape[1]] + out[3:6, :first.shape[1]]
    assert np.isfinite(out).all()
    close = mind < 0.01 * synth.AU
    assert close.sum() <= 2
    assert _rel_pos_err(got[:, ~close], r[:, ~close], star) <= POS_TOL
    if close.any():
        assert _rel_pos_err(got[:, close], r[:, close], star) <= 1e-9


def oracle_models(md):
    from oracle.pyoracle import Models
    return Models(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)


def test_tolerance(eph):
    srv = eph["srv"]
    parts = _particles(7, 64, eph, a=(0.5, 2.0), e=0.6)
    a, acc_a, _ = srv.result(srv.submit(parts, 0.0, 40 * DAY, tol=1e-13, h0=DAY))
    b, acc_b, _ = srv.result(srv.submit(parts, 0.0, 40 * DAY, tol=1e-16, h0=DAY))
    assert acc_b > acc_a
    star = srv.eval(40 * DAY)[0, 0:3]
    assert _rel_pos_err(a[0:3] + a[3:6], b[0:3] + b[3:6], star) <= 1e-12


def test_many_requests_and_budget(eph):
    srv = eph["srv"]
    reqs = [(_particles(200 + k, n, eph), (10 + 3 * k) * DAY) for k, n in enumerate([1, 7, 33, 260, 2, 90])]
    single = []
    for p, t1 in reqs:
        single.append(srv.result(srv.submit(p, 0.0, t1))[0])
    ids = [srv.submit(p, 0.0, t1) for p, t1 in reqs]          # all in flight
    for rid, want in zip(ids, single):
        assert np.array_equal(srv.result(rid)[0], want)
    srv.set_budget(1)                                           # one request at a time
    ids = [srv.submit(p, 0.0, t1) for p, t1 in reqs]
    assert srv.info()[1] == len(reqs) - 1                       # queued behind the first
    assert srv.poll(ids[1]) == 0
    for rid, want in zip(ids, single):
        while srv.poll(rid) == 0:
            pass
        assert np.array_equal(srv.result(rid)[0], want)
    srv.set_budget(0)                                           # back to admission by free memory


def test_backward_request_and_refusals(eph):
    from ephemeris_b200 import EphError
    srv = eph["srv"]
    parts = _particles(9, 12, eph)
    fwd = srv.result(srv.submit(parts, 0.0, 15 * DAY))[0]
    back = srv.result(srv.submit(fwd, 15 * DAY, 0.0))[0]
    start = np.concatenate([parts[0:3], np.zeros((3, 12)), parts[3:6], np.zeros((3, 12))])
    star = srv.eval(0.0)[0, 0:3]
    assert _rel_pos_err(back[0:3] + back[3:6], start[0:3], star) <= 1e-11
    with pytest.raises(EphError):
        srv.submit(parts, 0.0, (eph["days"] + 1) * DAY)
    with pytest.raises(EphError):
        srv.submit(parts, 0.0, DAY, tol=0.0)


@pytest.mark.parametrize("d,n,mn", [(3, 60, 120), (1, 20, 20), (5, 200, 1000), (8, 200, 1000)])
def test_batch_fit_on_device_is_bit_identical(eph, d, n, mn):
    """eph_bspline_fit_batch (one GPU thread per series and channel) against eph_bspline_fit (host)."""
    from ephemeris_b200 import bspline_fit, bspline_fit_batch
    rng = np.random.default_rng(d * 1000 + n)
    i = np.arange(mn + 1)
    series = [np.stack([np.sin(i * 0.1), np.cos(i * 0.1)], 1), rng.normal(0, 1e11, (mn + 1, 2))]
    if (n, mn) == (60, 120):
        series += [eph["samples"][:, j, 0:2] for j in range(3)]
    sm = np.stack(series)
    got = bspline_fit_batch(sm, n, d)
    for k in range(len(series)):
        assert np.array_equal(got[k], bspline_fit(series[k], n, d)), k


def test_full_ephemeris_requests(tmp_path):
    """The serving workload's full perturber set (419 bodies, 2-year ephemeris built and fitted on the GPU):
    30 requests of log-U(1, 4096) particles in flight at once all finish with finite states, and two of them
    rerun alone give the same states bit for bit."""
    from ephemeris_b200 import Context, MSystem, Server, bspline_fit_batch, synth
    sysm = synth.make_config4_system(4004)
    ms = MSystem(0)
    assert ms.load(synth.write_system(sysm, os.path.join(str(tmp_path), "eph419")))
    pl, md = ms.planes(), ms.models()
    c = Context(0)
    c.upload(pl, md)
    days = 730
    samples, _ = c.record_samples(DAY / 2, 2 * days, 1)
    coefs = bspline_fit_batch(np.ascontiguousarray(samples.transpose(1, 0, 2)), days, 3)
    srv = Server(coefs, pl[39], DAY, 0.0, 3, pl[54])
    rng = np.random.default_rng(13)
    reqs = synth.make_requests(rng, 30, days * DAY, years=(0.1, 2.0), star_r=samples[0, 0, 0:3],
                               star_v=samples[0, 0, 3:6])
    ids = [srv.submit(p, 0.0, t) for p, t in reqs]
    outs = [srv.result(i) for i in ids]
    assert all(np.isfinite(o[0]).all() and o[1] > 0 for o in outs)
    for k in (0, 17):
        again = srv.result(srv.submit(reqs[k][0], 0.0, reqs[k][1]))[0]
        assert np.array_equal(again, outs[k][0])
