"""The 1000-step accuracy criterion on every integration path (GPU).

Criterion: after 1000 RK12 steps the position of every body is within 1e-12 of its distance from the
central body, max_i |dr_i| / |r_i - r_star|, against the FP64 (double-double state) oracle or the
reference's own recorded outputs; angular velocities within 1e-12 of the largest one.

* full physics, single system: the 48-body test system (steps 100 and 1000) and the 504-body workload
  (step 1000) against the reference's outputs recorded by tests/golden/make_golden.py;
* batched ensembles: members of the ensemble recipe through eph_batch against the oracle (a chaotic member
  against its own one-ulp sensitivity);
* massless particles, FP64 and mixed precision, against the oracle (particles = GM 1e-20 bodies).

Each test prints the errors it observed (run pytest with -s to see them).
"""
import os

import numpy as np
import pytest

from tests.parity import position_error, rel_err

pytestmark = pytest.mark.gpu

POS_TOL = 1e-12
W_TOL = 1e-12


def _models(g):
    from ephemeris_b200 import Models
    m = g.models()
    return Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk, m.ring_param, m.ring_disk)


def _omodels(md):
    from oracle.pyoracle import Models
    return Models(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)


def _moon_relative(out, ref):
    """max over bodies of |d(r_i - r_p)| / |r_i - r_p| with p the body nearest to i (a planet for a moon)."""
    r = ref[0:3] + ref[3:6]
    ro = out[0:3] + out[3:6]
    d = np.sqrt(((r[:, :, None] - r[:, None, :]) ** 2).sum(0))
    np.fill_diagonal(d, np.inf)
    p = d.argmin(1)
    num = np.sqrt((((ro - ro[:, p]) - (r - r[:, p])) ** 2).sum(0))
    return float((num / d[np.arange(len(p)), p]).max())


@pytest.mark.parametrize("name", ["small_full", "config2"])
def test_thousand_steps_full_physics(golden, name):
    from ephemeris_b200 import Context
    g = golden(name)
    c = Context(0)
    c.upload(g["load"], _models(g))
    dt = float(g["dt"])
    t, done = (0.0, 0.0), 0
    for k in [s for s in g.meta["steps"] if s >= 100]:
        t = c.integrate(dt, k - done, t)
        done = k
        out, ref = c.download(), g[f"step{k}"]
        pe = position_error(out, ref)
        we = rel_err(out[36:39], ref[36:39], floor=np.abs(ref[36:39]).max())
        print(f"{name} step {k}: position {pe:.2e}, moon-relative {_moon_relative(out, ref):.2e}, w {we:.2e}")
        assert tuple(t) == tuple(g[f"t_eph{k}"])
        assert np.isfinite(out[0:12]).all()
        assert pe <= POS_TOL, (k, pe)
        assert we <= W_TOL, (k, we)
    c.close()


def _ulp_sensitivity(oracle, pl, om, dt, steps, ref):
    """How far the oracle itself moves after `steps` when every starting position is perturbed by about one
    unit in the last place: the accuracy any implementation that is not bit-identical can reach."""
    p2 = pl.copy()
    p2[3:6] += pl[0:3] * 2.2e-16 * np.random.default_rng(1).uniform(-1, 1, size=pl[0:3].shape)
    return position_error(oracle.integrate(p2, om, dt, steps)[0], ref)


@pytest.mark.parametrize("mixed", [False, True])
def test_thousand_steps_ensemble_members(tmp_path, oracle, mixed):
    """Members of the ensemble recipe (Newtonian + 1PN) in one eph_batch launch, 1000 steps against the oracle,
    in FP64 and in the mixed-precision form (FP32 1PN terms).

    The first four are well conditioned (a one-ulp change of the start moves the oracle by < 1e-12 after
    1000 steps): they must meet 1e-12. The last one has a close moon pair whose own one-ulp sensitivity is
    ~5e-8 after 1000 steps, so no arithmetic that is not bit-identical can meet 1e-12 on it; it must stay
    within its own sensitivity."""
    from ephemeris_b200 import Batch, MSystem, synth
    cases = [(3003500, 16), (3003502, 32), (3003504, 48), (3003506, 64), (3003401, 48)]
    mem = []
    for seed, n in cases:
        cfg = synth.write_system(synth.make_ensemble_member(seed, n), os.path.join(str(tmp_path), f"m{seed}"))
        ms = MSystem(0)
        assert ms.load(cfg)
        mem.append((ms.planes(), ms.models(), ms.delta_t))
    b = Batch(0)
    b.set_precision(mixed)
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    assert b.info()[0] == len(cases)
    b.integrate([m[2] for m in mem], [1000] * len(cases))
    outs = b.download()
    for k, ((pl, md, dt), out) in enumerate(zip(mem, outs)):
        om = _omodels(md)
        ref = oracle.integrate(pl, om, dt, 1000)[0]
        pe = position_error(out, ref)
        sens = _ulp_sensitivity(oracle, pl, om, dt, 1000, ref)
        print(f"ensemble member ({'mixed' if mixed else 'fp64'}) seed {cases[k][0]} n={pl.shape[1]} step 1000: "
              f"position {pe:.2e} (oracle one-ulp sensitivity {sens:.2e})")
        assert np.isfinite(out[0:12]).all()
        if k < 4:
            assert sens < POS_TOL
            assert pe <= POS_TOL, pe
        else:
            assert sens > 1e-10
            assert pe <= sens, (pe, sens)
    b.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_thousand_steps_particles(tmp_path, oracle, mixed):
    """64 particles of the particle workload's recipe (star with J2-J4, 8 planets) for 1000 steps of 0.5 day,
    in FP64 and in mixed precision, against the oracle's combined system."""
    from ephemeris_b200 import MSystem, Particles, synth
    sysm, parts = synth.make_config5(5005, n_particles=64)
    cfg = synth.write_system(synth.with_test_bodies(sysm, parts), os.path.join(str(tmp_path), "c5"))
    ms = MSystem(0)
    assert ms.load(cfg)
    pl, md, dt = ms.planes(), ms.models(), ms.delta_t
    n_pert = len(sysm.bodies)
    p = Particles(0)
    if mixed:
        p.set_precision(1)
    p.upload(np.ascontiguousarray(pl[:, :n_pert]), md, np.ascontiguousarray(pl[0:12, n_pert:]))
    p.integrate(dt, 1000)
    pert, part = p.download()
    p.close()
    ref = oracle.integrate(pl, _omodels(md), dt, 1000)[0]
    out = pl.copy()
    out[:, :n_pert] = pert
    out[0:12, n_pert:] = part
    pe_pert = position_error(out[:, :n_pert], ref[:, :n_pert])
    both = np.concatenate([out[:, :1], out[:, n_pert:]], axis=1)
    both_ref = np.concatenate([ref[:, :1], ref[:, n_pert:]], axis=1)
    pe_part = position_error(both, both_ref)
    print(f"particles ({'mixed' if mixed else 'fp64'}) step 1000: perturbers {pe_pert:.2e}, particles {pe_part:.2e}")
    assert np.isfinite(out[0:12]).all()
    assert pe_pert <= POS_TOL
    assert pe_part <= POS_TOL


MIXED_ACC_TOL = 1e-13


def test_mixed_ensemble_stage_acceleration(tmp_path, oracle):
    """The mixed-precision ensemble's accelerations after one step against the oracle's. The 1e-14 per-stage
    bound is the plain FP64 path's; the mixed form's criterion is the 1000-step position error (1e-12, above).
    Its per-stage error is the FP32 rounding of the 1PN terms: each ~6e-8 of a term ~1e-8 of the Newtonian
    acceleration, summed over up to 300 partners, so it is held to MIXED_ACC_TOL of sum_j |GM_j/r_ij^2|. The
    per-pair maxima within 1e-6 (their extremal pair is chosen on FP32 values, then recomputed in FP64)."""
    from ephemeris_b200 import Batch, MSystem, synth
    from tests.parity import accel_error
    mem = []
    for k, n in enumerate((33, 120, 300)):
        cfg = synth.write_system(synth.make_ensemble_member(3003 * 1000 + 600 + k, n), os.path.join(str(tmp_path), f"a{k}"))
        ms = MSystem(0)
        assert ms.load(cfg)
        mem.append((ms.planes(), ms.models(), ms.delta_t))
    b = Batch(0)
    b.set_precision(True)
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    b.integrate([m[2] for m in mem], [1, 1, 1])
    for (pl, md, dt), out in zip(mem, b.download()):
        ref = oracle.integrate(pl, _omodels(md), dt, 1)[0]
        ae = accel_error(out, ref)
        print(f"mixed ensemble n={pl.shape[1]} one step: acceleration {ae:.2e}, position {position_error(out, ref):.2e}")
        assert ae <= MIXED_ACC_TOL
        assert position_error(out, ref) <= POS_TOL
        for p in (100, 101):
            assert rel_err(out[p], ref[p]) <= 1e-6
    b.close()
