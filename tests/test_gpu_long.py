"""The 1000-step accuracy criterion on every integration path (GPU).

Criterion: after 1000 RK12 steps the position of every body is within 1e-12 of its distance from the
central body, max_i |dr_i| / |r_i - r_star|, against the FP64 (double-double state) oracle or the
reference's own recorded outputs; angular velocities within 1e-12 of the largest one.

* full physics, single system: the 48-body test system (steps 100 and 1000) and the 504-body workload
  (step 1000) against the reference's outputs recorded by tests/golden/make_golden.py;
* batched ensembles: two members of the ensemble recipe through eph_batch against the oracle;
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


def test_thousand_steps_ensemble_members(tmp_path, oracle):
    """Two members of the ensemble recipe (24 and 48 bodies, Newtonian + 1PN) in one eph_batch launch."""
    from ephemeris_b200 import Batch, MSystem, synth
    mem = []
    for k, n in enumerate((24, 48)):
        cfg = synth.write_system(synth.make_ensemble_member(3003 * 1000 + 400 + k, n),
                                 os.path.join(str(tmp_path), f"m{k}"))
        ms = MSystem(0)
        assert ms.load(cfg)
        mem.append((ms.planes(), ms.models(), ms.delta_t))
    b = Batch(0)
    b.upload([m[0] for m in mem], [m[1] for m in mem])
    assert b.info()[0] == 2
    b.integrate([m[2] for m in mem], [1000, 1000])
    outs = b.download()
    for (pl, md, dt), out in zip(mem, outs):
        ref = oracle.integrate(pl, _omodels(md), dt, 1000)[0]
        pe = position_error(out, ref)
        print(f"ensemble member n={pl.shape[1]} step 1000: position {pe:.2e}")
        assert np.isfinite(out[0:12]).all()
        assert pe <= POS_TOL, pe
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
