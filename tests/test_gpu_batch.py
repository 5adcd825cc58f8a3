"""Batched ensembles (eph_batch_*): every system of a batch against the oracle and the single-system path.

Members follow the config1 recipe at sizes from 2 to 300 bodies (Newtonian + 1PN: they share the one
persistent ensemble launch; from 96 bodies on a system is shared by the CTAs of a cluster); a
full-physics system in the same batch goes through the single-system kernel. Tolerances are those of
tests/test_gpu_parity.py: position 1e-12 of |r - r_star|, acceleration 1e-14 of sum_j |GM_j/r_ij^2|,
and the reference's own maxima bound (1e-15 relative, src/tests/test_integrator.cpp:15-20).
"""
import os

import numpy as np
import pytest

from tests.parity import accel_error, position_error, rel_err

pytestmark = pytest.mark.gpu

ACC_TOL = 1e-14
POS_TOL = 1e-12


def _members(tmp_path, sizes, seed=3003):
    from ephemeris_b200 import MSystem, synth
    out = []
    for k, n in enumerate(sizes):
        cfg = synth.write_system(synth.make_ensemble_member(seed * 1000 + k, n), os.path.join(str(tmp_path), f"m{k}"))
        ms = MSystem(0)
        assert ms.load(cfg)
        out.append((ms.planes(), ms.models(), ms.delta_t))
    return out


def _omodels(md):
    from oracle.pyoracle import Models
    return Models(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)


def _check(out, ref):
    assert np.isfinite(out[0:12]).all()
    assert position_error(out, ref) <= POS_TOL
    assert accel_error(out, ref) <= ACC_TOL
    for p in (100, 101):   # min_distance, max_influence
        assert rel_err(out[p], ref[p]) <= 1e-15


def test_ensemble_matches_oracle(tmp_path, oracle):
    from ephemeris_b200 import Batch
    sizes = [2, 8, 17, 33, 64, 120]
    steps = [9, 7, 3, 5, 2, 1]
    mem = _members(tmp_path, sizes)
    b = Batch(0)
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    assert b.info()[0] == len(sizes)          # all in the ensemble launch
    t = b.integrate([m[2] for m in mem], steps)
    outs = b.download()
    for (pl, md, dt), k, out, tt in zip(mem, steps, outs, t):
        ref, tref, _ = oracle.integrate(pl, _omodels(md), dt, k)
        _check(out, ref)
        assert tuple(tt) == tuple(tref)


def test_ensemble_cluster_shared_system(tmp_path, oracle):
    """300 bodies: shared by the CTAs of a thread-block cluster, each owning a slice of the bodies."""
    from ephemeris_b200 import Batch
    mem = _members(tmp_path, [300], seed=3004)
    b = Batch(0)
    b.upload([mem[0][0]], [mem[0][1]])
    b.integrate([mem[0][2]], [1])
    ref = oracle.integrate(mem[0][0], _omodels(mem[0][1]), mem[0][2], 1)[0]
    _check(b.download()[0], ref)


def test_ensemble_matches_single_system_path_and_repeats(tmp_path):
    from ephemeris_b200 import Batch, Context
    mem = _members(tmp_path, [5, 40, 90], seed=3005)
    steps = [4, -3, 6]                          # a backward integration among them
    b = Batch(0)
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    t = b.integrate([m[2] for m in mem], steps)
    outs = b.download()
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    assert all(np.array_equal(x, y) for x, y in zip(outs, (b.integrate([m[2] for m in mem], steps), b.download())[1]))
    for (pl, md, dt), k, out, tt in zip(mem, steps, outs, t):
        c = Context(0)
        c.upload(pl, md)
        tc = c.integrate(dt, k)
        assert position_error(out, c.download()) <= POS_TOL
        assert tuple(tt) == tuple(tc)


def test_full_physics_system_in_a_batch(golden, tmp_path):
    """A full-physics system runs through the single-system kernel: identical to the context path."""
    from ephemeris_b200 import Batch, Context, Models
    g = golden("small_full")
    m = g.models()
    md = Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)
    mem = _members(tmp_path, [12], seed=3006)
    b = Batch(0)
    b.upload([g["load"], mem[0][0]], [md, mem[0][1]])
    assert b.info()[0] == 1
    dt = float(g["dt"])
    b.integrate([dt, mem[0][2]], [3, 0])
    out = b.download()
    c = Context(0)
    c.upload(g["load"], md)
    c.integrate(dt, 3)
    assert np.array_equal(out[0], c.download())
    assert np.array_equal(out[1], mem[0][0])   # zero steps: untouched


def test_full_ensemble_members_match_their_own_runs(tmp_path):
    """The 512-member ensemble at its full size (durations scaled by 0.02 to keep the test short): eight
    members, integrated again on their own, give bit-identical states (a member's computation does not
    depend on the rest of the batch), and every member's state is finite."""
    from ephemeris_b200 import Batch, MSystem, synth
    ens = synth.make_ensemble(512)
    pls, mds, dts, ks = [], [], [], []
    for s_, (m, k) in enumerate(ens):
        ms = MSystem(0)
        assert ms.load(synth.write_system(m, os.path.join(str(tmp_path), f"s{s_}")))
        pls.append(ms.planes())
        mds.append(ms.models())
        dts.append(ms.delta_t)
        ks.append(max(1, int(round(k * 0.02))))
        ms.close()
    b = Batch(0)
    b.upload(pls, mds)
    b.integrate(dts, ks)
    outs = b.download()
    assert all(np.isfinite(o[0:12]).all() for o in outs)
    rng = np.random.default_rng(12)
    for s_ in rng.choice(512, 8, replace=False):
        one = Batch(0)
        one.upload([pls[s_]], [mds[s_]])
        one.integrate([dts[s_]], [ks[s_]])
        assert np.array_equal(one.download()[0], outs[s_]), s_
