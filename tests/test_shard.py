"""Sharding across ranks (ephemeris_b200.shard), on CPU with gloo ranks.

* The ensemble split: every member on exactly one rank, loads within 0.1 % of the mean for the 512-member
  ensemble on 2, 4 and 8 ranks, the same split on every call.
* Two gloo ranks each integrate their share (the oracle stands in for the GPU here) and one gather brings the
  results to rank 0: ensemble members equal to a one-rank run bit for bit (independent systems); massless
  particles (GM = 1e-20 bodies with the perturbers replicated on both ranks) within 1e-15 of a one-rank run
  of the whole set (the only difference is the particles' mutual pull, ~1e-20 of the star's).
"""
import os
import sys

import numpy as np

from tests.conftest import ROOT


def test_partition_covers_and_balances():
    from ephemeris_b200 import shard, synth
    ens = synth.make_ensemble(512)
    costs = [shard.member_cost(len(m.bodies), k) for m, k in ens]
    for world in (1, 2, 4, 8):
        parts = shard.partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.001 * np.mean(loads), (world, max(loads) / np.mean(loads))
        assert parts == shard.partition(costs, world)
    assert shard.particle_slice(10, 3, 0) == (0, 3) and shard.particle_slice(10, 3, 2) == (6, 10)


def _members():
    """Three small independent systems (the golden fixtures' loaded states)."""
    from tests.conftest import Golden
    out = []
    for name in ("config1", "small_full", "config1"):
        g = Golden(name)
        out.append((np.array(g["load"]), g.models(), float(g["dt"])))
    return out


def _particle_system(n_part):
    """The star and 8 planets of the 33-body fixture with n_part GM = 1e-20 bodies on 1-5 AU orbits, all
    auxiliaries set by one oracle acceleration evaluation."""
    from oracle.pyoracle import Oracle
    from tests.conftest import Golden
    g = Golden("config1")
    pl = np.array(g["load"])[:, :9]
    rng = np.random.default_rng(77)
    tmpl = pl[:, 8:9].copy()
    tmpl[41] = tmpl[39] = 1e-20          # GM0, GM
    tmpl[44] = 1e-3                      # radius (km)
    cols = []
    for _ in range(n_part):
        c = tmpl.copy()
        a = rng.uniform(1.0, 5.0) * 1.495978707e11
        th = rng.uniform(0, 2 * np.pi)
        v = np.sqrt(pl[39, 0] / a)
        c[0:3, 0] = pl[0:3, 0] + a * np.array([np.cos(th), np.sin(th), 0.0])
        c[3:6, 0] = 0.0
        c[6:9, 0] = pl[6:9, 0] + v * np.array([-np.sin(th), np.cos(th), 0.0])
        c[9:12, 0] = 0.0
        cols.append(c)
    full = np.concatenate([pl] + cols, axis=1)
    return Oracle().accel(full, g.models()), g.models(), float(g["dt"])


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from ephemeris_b200 import shard
    from oracle.pyoracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pg = dist.group.WORLD
    orc = Oracle()
    steps = 3
    # ensemble: this rank's share of the members, gathered as objects
    mem = _members()
    parts = shard.partition([shard.member_cost(p.shape[1], steps) for p, _, _ in mem], world)
    mine = {i: orc.integrate(mem[i][0], mem[i][1], mem[i][2], steps)[0] for i in parts[rank]}
    got = [None] * world
    dist.all_gather_object(got, mine, group=pg)
    # particles: this rank's slice of one particle set with the 9 perturbers, one gather of the states
    full, md, dt = _particle_system(40)
    n_part = full.shape[1] - 9
    lo, hi = shard.particle_slice(n_part, world, rank)
    sub = np.concatenate([full[:, :9], full[:, 9 + lo:9 + hi]], axis=1)
    out = orc.integrate(sub, md, dt, steps)[0]
    gathered = shard.gather_rows(np.ascontiguousarray(out[0:12, 9:]), n_part, pg)
    if rank == 0:
        merged = {}
        for d in got:
            merged.update(d)
        ens_ok = all(np.array_equal(merged[i], orc.integrate(p, m, t, steps)[0]) for i, (p, m, t) in enumerate(mem))
        ref = orc.integrate(full, md, dt, steps)[0][0:12, 9:]
        r_ref, r_got = ref[0:3] + ref[3:6], gathered[0:3] + gathered[3:6]
        err = float((np.linalg.norm(r_got - r_ref, axis=0) / np.linalg.norm(r_ref - full[0:3, :1], axis=0)).max())
        q.put((ens_ok, gathered.shape == ref.shape, err))
    dist.barrier(group=pg)
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ens_ok, shape_ok, err = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
    assert ens_ok
    assert shape_ok
    assert err <= 1e-15, err
