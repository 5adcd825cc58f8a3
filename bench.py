"""Benchmark of the B200 RK12 step: body-steps/s on the full-shape synthetic solar system.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload config2]

Workload: the 504-body full-physics synthetic system (ephemeris_b200.synth.make_config2, seed 2002:
geopotentials on 9 bodies, time-lagged tides, a ring, soft masses, radiation pressure), fixed step of
0.05 day. One bench "step" is one call of the integrator over `--rk-steps` RK12 steps (default 100) of
the whole system, i.e. rk_steps * 504 body-steps. The state (double-double position/velocity, full
auxiliaries) is resident in HBM when the timed region starts (`value`); `e2e` repeats the measurement
through the public C-ABI with the system planes uploaded from pinned host memory and downloaded back
every step. The launch shape comes from eph_autotune (cached per system class; --no-autotune keeps the
heuristic plan). The line also carries the reference's own GPU kernel timed on the same system
(`reference_gpu`) and, unless --no-sub-records, one sub-record per other workload.

Multi-GPU: one system does not shard ("replicas only": N ranks integrate N independent copies; value =
all ranks' body-steps / max-over-ranks device time). The ensemble (config3) is partitioned across ranks
longest-member-first and one particle set (config5) is split by index with one final gather
(ephemeris_b200.shard).

--impl reference times the reference's own CPU integrator (oracle/_ref, built from the reference
sources, with its thread pool) on the same workload; without it, the oracle restatement is timed.

Other workloads (--workload; also the sub-records of the default run): config3 (batched ensemble of 512
systems at their full 500-20000-step durations, eph_batch_*: plain FP64 members one by one, the batched
FP64 form and the batched mixed-precision form, with their 1000-step errors against the oracle), config4
(serving small-body requests against a device B-spline ephemeris, eph_serve_*: capacity, then p50/p99
latency under Poisson arrivals at a fixed rate and over a sweep of loads), config5 (2 M massless particles
against 9 perturbers, eph_particles_*; --mixed for FP32 1PN terms). Each prints the same JSON line with
its own unit (body-steps/s or particle-steps/s) and CPU reference arm.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-steps/s vs plain FP64 at <=1e-12 pos err; small-body p50/p99 latency"
UNIT = "body-steps/s"
# DRAM bytes (read + write) of one step_kernel launch, from an ncu capture of that launch
# (dram__bytes_read.sum + dram__bytes_write.sum), keyed by (workload, RK12 steps per launch).
DRAM_BYTES_PER_LAUNCH = {("config2", 100): 1530880 + 461056}
# DRAM bytes (read + write) of one particle_kernel launch per particle, from the ncu capture summarised in
# an ncu capture of one launch (1 M particles x 10 steps: 124.4 + 143.5 MB): the particle state is read
# and written once per launch and the stage store stays in L2, so the traffic scales with the particles and
# not with the steps of the launch.
DRAM_BYTES_PER_PARTICLE_LAUNCH = (124.399360e6 + 143.479040e6) / 1e6

# Algorithmic flop convention per ordered pair and stage evaluation (add, sub, mul, div, sqrt = 1, fma = 2):
FLOP_PASS_A = 20            # potential + Newtonian acceleration
FLOP_PASS_A_TIDE = 120      # time-lagged tidal matrix, extra over the Newtonian part
FLOP_1PN = 80
FLOP_DEFORM = 90            # tidal/rotational deformation force of i and j
FLOP_LT = 80
FLOP_RAD = 10
FLOP_GP = 250               # per (body, geopotential host), Nz=6/Nt=4
FLOP_GP_ZONAL = 80          # per (body, geopotential host), J2-J4 zonal only
FLOP_RING_DISK = 60         # per (body, ring host, disk)
FLOP_RK = 3900              # RK12 combination + update per body-step


def full_class(planes):
    """Bodies for which a term beyond point-mass Newtonian + 1PN can be nonzero, as source or target (the
    kernels' body classes): tides, rotational deformation, J2 rate, luminosity, radiation receptance,
    geopotential, ring, static harmonics or spin. Pair terms between two other bodies are exactly zero and
    the kernels skip them."""
    P = planes
    f = (P[46] != 0) | (P[47] != 0) | (P[43] != 0) | (P[50] != 0) | (P[55] != 0) | (P[102] >= 0) | (P[103] >= 0)
    return f | (P[56:65] != 0).any(0) | (P[36:39] != 0).any(0) | (P[12:18] != 0).any(0)


def algorithmic_flops_per_step(planes, models):
    """FLOPs of one RK12 step (25 stage evaluations) of the whole system by the convention above, counting
    only the terms the kernels evaluate: pass A and 1PN for every ordered pair, the time-lagged tide for pairs
    whose first body has a delayed tide, deformation / Lense-Thirring / radiation for pairs with a full-class
    body, geopotential per (body, host) by model kind, ring per (body, host, disk)."""
    n = planes.shape[1]
    n_point = n - int(full_class(planes).sum())
    pairs = n * (n - 1)
    pairs_full = pairs - n_point * (n_point - 1)
    delayed = int(((planes[46] != 0) & (planes[48] != 0)).sum())
    per_stage = (pairs * (FLOP_PASS_A + FLOP_1PN) + pairs_full * (FLOP_DEFORM + FLOP_LT + FLOP_RAD)
                 + delayed * (n - 1) * FLOP_PASS_A_TIDE)
    for k in range(len(models.gp_nz)):
        hosts = int((planes[102] == k).sum())
        per_stage += hosts * (n - 1) * (FLOP_GP if models.gp_nt[k] > 0 else FLOP_GP_ZONAL)
    for k in range(len(models.ring_ndisk)):
        hosts = int((planes[103] == k).sum())
        per_stage += hosts * (n - 1) * int(models.ring_ndisk[k]) * FLOP_RING_DISK
    return 25 * per_stage + n * FLOP_RK


_CAPTURE = None   # when a list, result lines are collected here (sub-records) instead of printed


def _emit(line):
    if _CAPTURE is not None:
        _CAPTURE.append(line)
    else:
        print(json.dumps(line), flush=True)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_workload(workload: str, tmpdir: str):
    from ephemeris_b200 import synth
    return synth.write_workload(workload, os.path.join(tmpdir, workload))


def dist_setup(n_gpus):
    """Rank / world size from torchrun's environment; NCCL process group when N > 1."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = os.environ.get("EPH_BENCH_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def reduce_max(pg, value: float, device=None) -> float:
    """Maximum of a per-rank float over all ranks (identity without a process group)."""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device=None):
    if pg is None:
        return
    import torch
    t = torch.zeros(1, device=device)
    pg.all_reduce(t)


def cpu_baseline(cfg, n_steps: int):
    """The reference's own CPU integrator (thread pool) on a bounded sample; else the oracle port."""
    from oracle.pyoracle import Oracle, RefSystem, ref_available
    cores = os.cpu_count() or 1
    if ref_available():
        ref = RefSystem(cfg)
        RefSystem.thread_pool(True)
        dt = ref.lib().ref_delta_t(ref.h)
        ref.integrate(dt, 1)                       # warm the pool
        t0 = time.perf_counter()
        ref.integrate(dt, n_steps)
        el = time.perf_counter() - t0
        RefSystem.thread_pool(False)
        return {"value": ref.n * n_steps / el, "unit": UNIT, "cores": min(16, cores), "kind": "reference",
                "sample": f"{n_steps} RK12 steps of the {ref.n}-body system, msystem::integrate(dt,n,0) with "
                          f"ThreadPool (min(16, {cores}) workers), {el:.1f} s"}
    from ephemeris_b200 import MSystem  # noqa: F401  (product loader provides the state)
    raise RuntimeError("oracle/_ref missing")


def reference_gpu_baseline(cfg, rk_steps: int = 10, calls: int = 3):
    """The reference's own GPU integrator (its cooperative kernel compiled unchanged for sm_100a,
    oracle/_ref/libephref_gpu.so) on the same system, in a child process (its CUDA error handler exits the
    process): one step checked against its CPU integrator with its own bounds, then timed by wall clock."""
    path = os.path.join(ROOT, "oracle", "_ref", "libephref_gpu.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libephref_gpu.so not built"}
    try:
        out = subprocess.run([sys.executable, "-m", "oracle.ref_gpu_timing", cfg, str(rk_steps), str(calls)],
                             cwd=ROOT, capture_output=True, text=True, timeout=240)
        lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
        if out.returncode != 0 or not lines:
            return {"unavailable": f"exit {out.returncode}: {(out.stderr or out.stdout)[-200:]}"}
        return json.loads(lines[-1])
    except Exception as exc:
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def run_reference(args):
    """--impl reference: the reference CPU integrator, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pyoracle import Oracle, RefSystem, ref_available
    with tempfile.TemporaryDirectory() as td:
        cfg = load_workload(args.workload, td)
        cores = os.cpu_count() or 1
        per_step = args.ref_rk_steps
        if ref_available():
            ref = RefSystem(cfg)
            RefSystem.thread_pool(True)
            dt = ref.lib().ref_delta_t(ref.h)
            n = ref.n
            for _ in range(args.warmup):
                ref.integrate(dt, per_step)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                ref.integrate(dt, per_step)
            el = time.perf_counter() - t0
            kind, used = "reference", min(16, cores)
            sample = (f"{args.steps} x {per_step} RK12 steps of the {n}-body system, reference "
                      f"msystem::integrate(dt,n,0) with its ThreadPool ({used} workers)")
        else:
            from ephemeris_b200 import MSystem
            ms = MSystem(0)
            assert ms.load(cfg)
            pl, md = ms.planes(), ms.models()
            orc = Oracle()
            from oracle.pyoracle import Models as OM
            om = OM(md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk)
            dt, n = ms.delta_t, pl.shape[1]
            t0 = time.perf_counter()
            for _ in range(args.steps):
                pl, _, _ = orc.integrate(pl, om, dt, per_step)
            el = time.perf_counter() - t0
            kind, used = "port", 1
            sample = f"{args.steps} x {per_step} RK12 steps, C restatement, 1 thread"
        value = n * per_step * args.steps / el
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": f"{args.workload}: {n}-body full-physics synthetic system, dt=0.05 day",
                           "rk_steps_per_step": per_step},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind, "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


def load_ensemble(args, tmpdir, device=0):
    """The batched-ensemble workload: members of the config1 recipe (8-300 bodies), each loaded by the
    product loader; durations scaled by --ens-frac (at least one step)."""
    from ephemeris_b200 import MSystem, synth
    ens = synth.make_ensemble(args.ens_systems)
    pls, mds, dts, ks, cfgs = [], [], [], [], []
    for s, (m, k) in enumerate(ens):
        cfg = synth.write_system(m, os.path.join(tmpdir, f"s{s}"))
        ms = MSystem(device)
        if not ms.load(cfg):
            raise RuntimeError("ensemble member failed to load")
        pls.append(ms.planes())
        mds.append(ms.models())
        dts.append(ms.delta_t)
        ks.append(max(1, int(round(k * args.ens_frac))))
        cfgs.append(cfg)
        ms.close()
    return pls, mds, dts, ks, cfgs


def _ensemble_flops(pls, ks):
    """Algorithmic FLOPs of the ensemble run: Newtonian + 1PN pairs and the RK update, per the convention."""
    return float(sum(k * (25 * n * (n - 1) * (FLOP_PASS_A + FLOP_1PN) + n * FLOP_RK)
                     for n, k in ((p.shape[1], k) for p, k in zip(pls, ks))))


def _ref_member(args):
    """One ensemble member through the reference's serial integrator (a worker process)."""
    cfg, n_step = args
    from oracle.pyoracle import RefSystem
    ref = RefSystem(cfg)
    dt = ref.lib().ref_delta_t(ref.h)
    t0 = time.perf_counter()
    ref.integrate(dt, n_step)
    return ref.n * n_step, time.perf_counter() - t0


# The reference's msystem::load ends with an orbit-structure analysis (msystem::analyse) that does not
# finish within seconds for about a quarter of the synthetic ensemble members (found by loading each with a
# time limit); the integrator is not involved. The CPU sample therefore takes members of at most this many
# bodies whose reference load finishes within ENS_CPU_LOAD_S seconds. Smaller systems cost the CPU less per
# body-step, so the sample favours the CPU.
ENS_CPU_MAX_BODIES = 100
ENS_CPU_LOAD_S = 5.0


def _loadable(cfgs):
    """The configs whose reference load finishes within ENS_CPU_LOAD_S (one child process each)."""
    code = ("import sys; sys.path.insert(0, %r); from oracle.pyoracle import RefSystem; RefSystem(sys.argv[1])"
            % os.path.dirname(os.path.abspath(__file__)))
    procs = [subprocess.Popen([sys.executable, "-c", code, c], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
             for c in cfgs]
    t_end = time.perf_counter() + ENS_CPU_LOAD_S + 10.0   # interpreter start-up on top of the load itself
    ok = []
    for c, p in zip(cfgs, procs):
        try:
            p.wait(timeout=max(0.1, t_end - time.perf_counter()))
            if p.returncode == 0:
                ok.append(c)
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
    return ok


def ensemble_cpu(cfgs, sizes, n_members, n_step):
    """Reference CPU throughput on the ensemble: one member per worker process, all host cores."""
    import concurrent.futures as cf
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    picks = _loadable([c for c, n in zip(cfgs, sizes) if n <= ENS_CPU_MAX_BODIES][:2 * n_members])[:n_members]
    jobs = [(c, n_step) for c in picks]
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_ref_member, [(c, 1) for c in picks[:cores]]))   # start the workers
        t0 = time.perf_counter()
        done = list(ex.map(_ref_member, jobs))
        el = time.perf_counter() - t0
    body_steps = sum(b for b, _ in done)
    return {"value": body_steps / el, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(jobs)} ensemble members of <= {ENS_CPU_MAX_BODIES} bodies (reference load within "
                      f"{ENS_CPU_LOAD_S:.0f} s) x {n_step} RK12 steps, "
                      f"reference msystem::integrate(dt,n,0) serial, one member per process on {cores} processes, "
                      f"{el:.1f} s"}


# Members of the ensemble recipe whose own one-ulp sensitivity after 1000 steps is below 1e-12 (checked by
# tests/test_gpu_long.py): the 1000-step error sample of the config3 comparison.
ENS_ERR_MEMBERS = [(3003500, 16), (3003502, 32), (3003504, 48), (3003506, 64)]


def _oracle_run(job):
    """Worker process: the oracle's integration of one system (planes, model arrays, dt, steps)."""
    pl, mdl, dt, steps = job
    from oracle.pyoracle import Models, Oracle
    return Oracle().integrate(pl, Models(*mdl), dt, steps)[0]


def ensemble_one_by_one(pls, mds, dts, ks, device, stream, n_probe=24, probe_steps=10):
    """The plain FP64 GPU path on the ensemble: members one after another through a Context (the
    single-system kernel, msystem::integrate semantics). Measured on `n_probe` members spread over the
    sizes (CUDA events over `probe_steps` steps each); the whole ensemble's time is the sum over all members
    of their step counts times the per-step time interpolated at their size."""
    import torch
    from ephemeris_b200 import Context
    order = np.argsort([p.shape[1] for p in pls])
    pick = sorted(set(order[np.linspace(0, len(order) - 1, n_probe).round().astype(int)].tolist()))
    sizes, per_step = [], []
    for s in pick:
        c = Context(device)
        c.set_stream(stream.cuda_stream)
        c.upload(pls[s], mds[s])
        c.integrate(dts[s], 2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c.integrate(dts[s], probe_steps)
        e1.record(stream)
        e1.synchronize()
        sizes.append(pls[s].shape[1])
        per_step.append(e0.elapsed_time(e1) / probe_steps)
        c.close()
    n_all = np.array([p.shape[1] for p in pls], float)
    t_ms = float(np.sum(np.asarray(ks, float) * np.interp(n_all, sizes, per_step)))
    body_steps = float(np.sum(n_all * np.asarray(ks, float)))
    return {"value": body_steps / (t_ms / 1e3), "unit": UNIT, "estimated_s": t_ms / 1e3,
            "sample": f"{len(pick)} members of {min(sizes)}-{max(sizes)} bodies, {probe_steps} RK12 steps each through "
                      f"eph_integrate (CUDA events); per-step time interpolated in body count for all members",
            "ms_per_rk_step_by_bodies": dict(zip(map(int, sizes), map(float, per_step)))}


def ensemble_errors(device, td, pool):
    """1000-step position error against the oracle of well-conditioned ensemble members, FP64 and mixed."""
    from ephemeris_b200 import Batch, MSystem, synth
    from tests.parity import position_error
    mem = []
    for seed, n in ENS_ERR_MEMBERS:
        cfg = synth.write_system(synth.make_ensemble_member(seed, n), os.path.join(td, f"err{seed}"))
        ms = MSystem(device)
        if not ms.load(cfg):
            raise RuntimeError("error-sample member failed to load")
        mem.append((ms.planes(), ms.models(), ms.delta_t))
        ms.close()
    futs = [pool.submit(_oracle_run, (pl, (md.gp_nz, md.gp_nt, md.gp_coef, md.ring_ndisk, md.ring_param, md.ring_disk),
                                      dt, 1000)) for pl, md, dt in mem]
    out = {}
    for mixed in (False, True):
        b = Batch(device)
        b.set_precision(mixed)
        b.upload([m[0] for m in mem], [m[1] for m in mem])
        b.integrate([m[2] for m in mem], [1000] * len(mem))
        out[mixed] = b.download()
        b.close()
    refs = [f.result() for f in futs]
    return {"members": [n for _, n in ENS_ERR_MEMBERS],
            "fp64": max(position_error(o, r) for o, r in zip(out[False], refs)),
            "mixed": max(position_error(o, r) for o, r in zip(out[True], refs)),
            "measure": "max_i |dr_i| / |r_i - r_star| after 1000 RK12 steps of dt = 0.05 day, max over the members"}


def run_b200_ensemble(args):
    import torch
    from ephemeris_b200 import Batch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    with tempfile.TemporaryDirectory() as td:
        pls, mds, dts, ks, cfgs = load_ensemble(args, td, local)
        body_steps_all = float(sum(p.shape[1] * k for p, k in zip(pls, ks)))
        if world > 1:   # this rank's share of the members (longest processing time first; no exchange)
            from ephemeris_b200 import shard
            mine = shard.partition([shard.member_cost(p.shape[1], k) for p, k in zip(pls, ks)], world)[rank]
            pls, mds, dts, ks, cfgs = ([x[i] for i in mine] for x in (pls, mds, dts, ks, cfgs))
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        b = Batch(local)
        b.set_stream(stream.cuda_stream)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        for _ in range(args.warmup):   # warm-up: every member, 20 steps at most
            b.upload(pls, mds)
            b.integrate(dts, [min(k, 20) for k in ks])
        tune = None
        if args.ens_compare:   # the cluster-sharing threshold, tuned on 2 % of every member's steps
            b.upload(pls, mds)
            cm, t1, t0 = b.autotune(dts, ks, step_frac=0.02)
            tune = {"coop_min_bodies": cm, "ms_tuned": t1, "ms_default": t0,
                    "by": "eph_batch_autotune on 2 % of each member's steps (outside the timed region)"}
        barrier(pg, dev)
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        l0 = b.info()[1]
        dev_ms = 0.0
        for k in range(args.steps):
            b.upload(pls, mds)                     # inputs in HBM before the timed region
            flush.fill_(float(k))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.integrate(dts, ks)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            dev_ms += e0.elapsed_time(e1)
        clk = clocks.stop()
        launches = b.info()[1] - l0
        dev_ms_max = reduce_max(pg, dev_ms, dev)
        body_steps = float(sum(p.shape[1] * k for p, k in zip(pls, ks)))
        value = body_steps_all * args.steps / (dev_ms_max / 1e3)
        compare = None
        if args.ens_compare and world == 1:
            # the same ensemble in the mixed-precision form, the plain FP64 path one member at a time, and
            # the 1000-step errors of both forms on a sample (oracle in spawned worker processes)
            import concurrent.futures as cf
            import multiprocessing as mp
            pool = cf.ProcessPoolExecutor(max_workers=len(ENS_ERR_MEMBERS), mp_context=mp.get_context("spawn"))
            b.set_precision(True)
            mixed_ms = 0.0
            for k in range(args.steps):
                b.upload(pls, mds)
                flush.fill_(float(k))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.integrate(dts, ks)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                mixed_ms += e0.elapsed_time(e1)
            b.set_precision(False)
            mixed_value = body_steps * args.steps / (mixed_ms / 1e3)
            plain = ensemble_one_by_one(pls, mds, dts, ks, local, stream)
            errs = ensemble_errors(local, td, pool)
            pool.shutdown()
            compare = {"plain_fp64_one_by_one": plain, "batched_fp64": value, "batched_mixed": mixed_value,
                       "ratio_batched_mixed_vs_plain_fp64": mixed_value / plain["value"],
                       "ratio_batched_fp64_vs_plain_fp64": value / plain["value"],
                       "error_1000_steps": errs}
        # end to end: host planes up, integrate, host planes down
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            b.upload(pls, mds)
            b.integrate(dts, ks)
            b.download()
        e2e_s = reduce_max(pg, time.perf_counter() - t0, dev)
        e2e = body_steps_all * args.steps / e2e_s
        bytes_io = int(sum(p.nbytes for p in pls))
        flops = _ensemble_flops(pls, ks)
        achieved = flops / (dev_ms / args.steps / 1e3) / 1e12
        peak, peak_src = fp64_peak(dev)
        pipe = fp64_pipe_peak(local)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                cpu = ensemble_cpu(cfgs, [p.shape[1] for p in pls], args.ens_cpu_members, args.ens_cpu_steps)
            except Exception as exc:
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(exc)}
        if rank == 0:
            sizes = [p.shape[1] for p in pls]
            line = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic",
                "config": {"workload": f"config3: {len(pls)}-system ensemble, {min(sizes)}-{max(sizes)} bodies "
                                       f"(Newtonian + 1PN), durations {min(ks)}-{max(ks)} RK12 steps "
                                       f"(the 500-20000 draw scaled by {args.ens_frac}), dt=0.05 day",
                           "systems": len(pls), "bodies": int(sum(sizes)), "body_steps_per_step": body_steps,
                           "parallelism": (f"members sharded over {world} GPUs (longest processing time first, no "
                                           f"exchange)") if world > 1 else "one persistent launch, 1 GPU",
                           "autotune": tune,
                           "l2": "flushed between timed steps (256 MB write)"},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
                "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak if peak else None, "traffic": None, "peak_source": peak_src,
                             "flops_per_launch": flops},
                "gpu_launches": launches,
                "clocks": clk,
            }
            if compare is not None:
                line["comparison"] = compare
            if cpu is not None:
                line["cpu_baseline"] = cpu
            _emit(line)
    if pg is not None:
        pg.destroy_process_group()


def run_reference_ensemble(args):
    """--impl reference --workload config3: the reference CPU integrator on a sample of the ensemble."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as td:
        from ephemeris_b200 import synth
        ens = [(m, k) for m, k in synth.make_ensemble(args.ens_systems) if len(m.bodies) <= ENS_CPU_MAX_BODIES]
        ens = ens[:2 * args.ens_cpu_members]
        cfgs = [synth.write_system(m, os.path.join(td, f"s{s}")) for s, (m, _) in enumerate(ens)]
        sizes = [len(m.bodies) for m, _ in ens]
        vals, cpu = [], None
        for _ in range(max(1, args.steps)):
            cpu = ensemble_cpu(cfgs, sizes, args.ens_cpu_members, args.ens_cpu_steps)
            vals.append(cpu["value"])
        value = statistics.median(vals)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic", "impl": "reference",
                "config": {"workload": "config3 ensemble, reference CPU sample (see cpu_baseline.sample)"},
                "cpu_baseline": dict(cpu, value=value),
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- config5: massless test particles
P_CPU_CHUNK = 64   # particles per reference system (with the perturbers as its first bodies)


def particle_flops_per_step(pl, models):
    """Algorithmic FLOPs of one RK12 step of one particle against the perturbers, by the convention of
    algorithmic_flops_per_step: M perturbers x (pass A + 1PN) per stage; a zonal-only geopotential host
    (J2-J4: its static J2 included) FLOP_GP_ZONAL, a tesseral one FLOP_GP, each ring disk FLOP_RING_DISK;
    a tidally deformable or spinning perturber adds its side (half) of the deformation and
    Lense-Thirring terms; FLOP_RK per step."""
    from ephemeris_b200.msystem import P
    m = pl.shape[1]
    per_stage = m * (FLOP_PASS_A + FLOP_1PN)
    for j in range(m):
        tidal_or_spin = pl[P["K2"], j] != 0 or pl[P["K2R"], j] != 0 or (pl[P["W"]:P["W"] + 3, j] != 0).any() or \
            (pl[P["GL_HI"]:P["GL_HI"] + 6, j] != 0).any()
        per_stage += (FLOP_DEFORM + FLOP_LT) // 2 if tidal_or_spin else 0
        g = int(pl[P["GP_INDEX"], j])
        if g >= 0:
            per_stage += FLOP_GP_ZONAL if models.gp_nt[g] == 0 else FLOP_GP
    per_stage += int(np.sum(models.ring_ndisk)) * FLOP_RING_DISK
    return 25 * per_stage + FLOP_RK


def load_particles(args, tmpdir, rank, device=0, world=1):
    """Perturbers (loaded by the product loader) and this rank's particles [6][n]: one particle set of
    --particles x world particles, cut into contiguous slices, one per rank (the perturbers replicated)."""
    from ephemeris_b200 import MSystem, shard, synth
    sysm, parts = synth.make_config5(5005, n_particles=args.particles * world)
    lo, hi = shard.particle_slice(parts.shape[1], world, rank)
    parts = np.ascontiguousarray(parts[:, lo:hi])
    cfg = synth.write_system(sysm, os.path.join(tmpdir, "perturbers"))
    ms = MSystem(device)
    if not ms.load(cfg):
        raise RuntimeError("perturbers failed to load")
    out = ms.planes(), ms.models(), ms.delta_t, parts, sysm
    ms.close()
    return out


def _ref_chunk(args):
    """One chunk of particles (as GM = 1e-20 bodies) with the perturbers through the reference's serial
    integrator (a worker process)."""
    cfg, n_step, n_part = args
    from oracle.pyoracle import RefSystem
    ref = RefSystem(cfg)
    dt = ref.lib().ref_delta_t(ref.h)
    t0 = time.perf_counter()
    ref.integrate(dt, n_step)
    return n_part * n_step, time.perf_counter() - t0


def particles_cpu(sysm, parts, n_step, tmpdir):
    """Reference CPU throughput on massless particles: chunks of P_CPU_CHUNK particles plus the 9
    perturbers per reference system, one chunk per worker process, all host cores."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from ephemeris_b200 import synth
    cores = os.cpu_count() or 1
    cfgs = []
    for c in range(cores):
        chunk = parts[:, c * P_CPU_CHUNK:(c + 1) * P_CPU_CHUNK]
        cfgs.append(synth.write_system(synth.with_test_bodies(sysm, chunk), os.path.join(tmpdir, f"chunk{c}")))
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_ref_chunk, [(c, 1, P_CPU_CHUNK) for c in cfgs]))   # start the workers
        t0 = time.perf_counter()
        done = list(ex.map(_ref_chunk, [(c, n_step, P_CPU_CHUNK) for c in cfgs]))
        el = time.perf_counter() - t0
    steps = sum(b for b, _ in done)
    return {"value": steps / el, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{cores} chunks of {P_CPU_CHUNK} particles (GM=1e-20 bodies) + {len(sysm.bodies)} perturbers, "
                      f"{n_step} RK12 steps each, reference msystem::integrate(dt,n,0) serial, one chunk per process "
                      f"on {cores} processes, {el:.1f} s"}


def run_b200_particles(args):
    import torch
    from ephemeris_b200 import Particles
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    with tempfile.TemporaryDirectory() as td:
        pl, md, dt, parts, sysm = load_particles(args, td, rank, local, world)
        n_part, ks = parts.shape[1], args.p_steps
        n_total = args.particles * world
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        p = Particles(local)
        p.set_stream(stream.cuda_stream)
        p.set_precision(args.mixed)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        for _ in range(args.warmup):
            p.upload(pl, md, parts)
            p.integrate(dt, min(ks, 20))
        barrier(pg, dev)
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        l0, k0 = p.info()
        dev_ms = 0.0
        for k in range(args.steps):
            p.upload(pl, md, parts)                  # inputs in HBM before the timed region
            flush.fill_(float(k))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            p.integrate(dt, ks)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            dev_ms += e0.elapsed_time(e1)
        clk = clocks.stop()
        l1, k1 = p.info()
        part_launches = args.steps                   # one particle-kernel launch per call (all steps fit one round)
        kern_ms = (k1 - k0) / part_launches
        dev_ms_max = reduce_max(pg, dev_ms, dev)
        value = n_total * ks * args.steps / (dev_ms_max / 1e3)
        # end to end through the public API: host particles up, integrate, host particles down (pinned
        # host buffers: the state as double-double rows, as the API takes and returns it)
        z = np.zeros((3, n_part))
        pin = torch.from_numpy(np.concatenate([parts[0:3], z, parts[3:6], z])).pin_memory().numpy()
        pin_out = torch.empty((12, n_part), dtype=torch.float64).pin_memory().numpy()
        pl_out = np.empty_like(pl)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            p.upload(pl, md, pin)
            p.integrate(dt, ks)
            p.download(pl_out, pin_out)
            if pg is not None:   # the one collective: the final states of every slice gathered to rank 0
                from ephemeris_b200 import shard
                shard.gather_rows(pin_out, n_total, pg, device=dev)
        e2e_s = reduce_max(pg, time.perf_counter() - t0, dev)
        e2e = n_total * ks * args.steps / e2e_s
        mixed_err = None
        if args.mixed:   # position error of the mixed run against the FP64 run of the same particles
            part_mixed = pin_out.copy()
            p.set_precision(False)
            p.upload(pl, md, parts)
            p.integrate(dt, ks)
            _, part_fp64 = p.download()
            r_m, r_d = part_mixed[0:3] + part_mixed[3:6], part_fp64[0:3] + part_fp64[3:6]
            star = pl[0:3, 0] + pl[3:6, 0]
            mixed_err = float((np.linalg.norm((part_mixed[0:3] - part_fp64[0:3]) + (part_mixed[3:6] - part_fp64[3:6]),
                                              axis=0) / np.linalg.norm(r_d - star[:, None], axis=0)).max())
        h2d = int(12 * n_part * 8 + pl.nbytes)
        d2h = int(12 * n_part * 8 + pl.nbytes)
        fps = particle_flops_per_step(pl, md)
        achieved = fps * n_part * ks / (kern_ms / 1e3) / 1e12
        peak, peak_src = fp64_peak(dev)
        pipe = fp64_pipe_peak(local)
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                cpu = particles_cpu(sysm, parts, args.p_cpu_steps, td)
            except Exception as exc:
                cpu = {"value": None, "unit": "particle-steps/s", "cores": 0, "kind": "unavailable", "sample": str(exc)}
        if rank == 0:
            line = {
                "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 state, f32 1PN terms" if args.mixed else "f64 (double-double state)", "data": "synthetic",
                "config": {"workload": f"config5: {n_part} massless particles per GPU (a 1.5-50 AU, e < 0.3, "
                                       f"i < 20 deg) against {pl.shape[1]} perturbers (star with J2-J4, 8 planets; "
                                       f"Newtonian + 1PN), dt=0.5 day, {ks} RK12 steps per bench step",
                           "particles": n_part, "perturbers": int(pl.shape[1]), "rk_steps_per_step": ks,
                           "parallelism": (f"one set of {n_total} particles cut into {world} slices, perturbers "
                                           f"replicated, one gather of the final states (e2e)") if world > 1
                           else "1 GPU",
                           "l2": "flushed between timed steps (256 MB write); particle state 240 MB > L2",
                           "precision": "mixed (EIH 1PN in FP32)" if args.mixed else "fp64"},
                "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "roofline": {"bound": "fp64", "kernel": "particle_kernel", "achieved": achieved, "peak": peak,
                             "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                             "traffic": DRAM_BYTES_PER_PARTICLE_LAUNCH * n_part,
                             "traffic_unit": "bytes per launch (ncu, scaled by particles)",
                             "peak_source": peak_src, "flops_per_launch": fps * n_part * ks,
                             "kernel_ms": kern_ms},
                "gpu_launches": l1 - l0,
                "clocks": clk,
            }
            if mixed_err is not None:
                line["mixed_vs_fp64_position_error"] = mixed_err
            if cpu is not None:
                line["cpu_baseline"] = cpu
            _emit(line)
        p.close()
    if pg is not None:
        pg.destroy_process_group()


def run_reference_particles(args):
    """--impl reference --workload config5: the reference CPU integrator on chunks of the particles."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ephemeris_b200 import synth
    with tempfile.TemporaryDirectory() as td:
        sysm, parts = synth.make_config5(5005, n_particles=P_CPU_CHUNK * (os.cpu_count() or 1))
        vals, cpu = [], None
        for _ in range(max(1, args.steps)):
            cpu = particles_cpu(sysm, parts, args.p_cpu_steps, td)
            vals.append(cpu["value"])
        value = statistics.median(vals)
        line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic", "impl": "reference",
                "config": {"workload": "config5 particles, reference CPU sample (see cpu_baseline.sample)"},
                "cpu_baseline": dict(cpu, value=value),
                "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- config4: serving against a B-spline ephemeris
DAY = 86400.0


def build_serving_ephemeris(args, tmpdir, device=0):
    """The perturber ephemeris of the serving workload: synth.make_config4_system (419 point masses)
    integrated on the GPU for --serve-years at dt = 0.5 day (eph_record_samples), each body's 10 channels
    fitted with cubic B-splines at 1-day knots on the GPU (eph_bspline_fit_batch). Returns (coefs, gm, sr2, samples0, setup_s)."""
    from ephemeris_b200 import Context, MSystem, bspline_fit_batch, synth
    t0 = time.perf_counter()
    sysm = synth.make_config4_system(4004)
    ms = MSystem(device)
    if not ms.load(synth.write_system(sysm, os.path.join(tmpdir, "ephemeris"))):
        raise RuntimeError("serving perturbers failed to load")
    pl, md = ms.planes(), ms.models()
    ms.close()
    days = int(round(args.serve_years * 365.25))
    c = Context(device)
    c.upload(pl, md)
    samples, _ = c.record_samples(DAY / 2, 2 * days, 1)
    c.close()
    coefs = bspline_fit_batch(np.ascontiguousarray(samples.transpose(1, 0, 2)), days, 3, device)
    return coefs, pl[39].copy(), pl[54].copy(), samples[0], time.perf_counter() - t0, sysm


def serve_flops_per_particle_step(m):
    """Useful work of one accepted particle-step: 25 stages x M perturbers x (pass A + 1PN) + the RK
    update (the step-doubling evaluations and rejected steps are not counted)."""
    return 25 * m * (FLOP_PASS_A + FLOP_1PN) + FLOP_RK


def run_serving_window(srv, reqs, rate, rng):
    """Open-loop Poisson arrivals at `rate` per second: each request is submitted at its arrival time and
    collected as soon as it is done. Returns (latencies [s], particle_steps, wall_s, h2d, d2h)."""
    if np.isinf(rate):
        arrivals = np.zeros(len(reqs))
    else:
        gaps = rng.exponential(1.0 / rate, len(reqs))
        arrivals = np.cumsum(gaps) - gaps[0]
    pending = {}
    lat, steps, h2d, d2h = [], 0, 0, 0
    run_serving_window.rejected = 0
    t0 = time.perf_counter()
    nxt = 0
    while nxt < len(reqs) or pending:
        now = time.perf_counter() - t0
        while nxt < len(reqs) and arrivals[nxt] <= now:
            parts, t_end = reqs[nxt]
            rid = srv.submit(parts, 0.0, t_end, tol=1e-13, h0=DAY)
            pending[rid] = arrivals[nxt]
            h2d += 12 * parts.shape[1] * 8
            nxt += 1
        done = [rid for rid in list(pending) if srv.poll(rid) == 2]
        for rid in done:
            out, acc, rej = srv.result(rid)
            lat.append(time.perf_counter() - t0 - pending.pop(rid))
            steps += acc
            run_serving_window.rejected += rej
            d2h += out.nbytes
        if not done:
            time.sleep(0.0005)
    return np.array(lat), steps, time.perf_counter() - t0, h2d, d2h


def run_b200_serving(args):
    import torch
    from ephemeris_b200 import Server, synth
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    with tempfile.TemporaryDirectory() as td:
        coefs, gm, sr2, s0, setup_s, sysm = build_serving_ephemeris(args, td, local)
        m = coefs.shape[0]
        srv = Server(coefs, gm, DAY, 0.0, 3, sr2, device=local)
        span = srv.span[1]
        rng = np.random.default_rng(4004 + rank)
        mk = lambda count: synth.make_requests(rng, count, span, p_max=args.serve_pmax, years=(1.0, args.serve_years),
                                               star_r=s0[0, 0:3], star_v=s0[0, 3:6])
        run_serving_window(srv, mk(max(1, args.warmup)), args.serve_rate, rng)    # warm-up
        # capacity: the whole request set at once, drained as fast as the GPU can (value, e2e)
        reqs = mk(args.serve_requests)
        launches0 = srv.info()[0]
        barrier(pg, dev)
        clocks = ClockSampler(local)
        clocks.start()
        _, psteps, wall, h2d, d2h = run_serving_window(srv, reqs, float("inf"), rng)
        rejected = run_serving_window.rejected
        clk = clocks.stop()
        launches = srv.info()[0] - launches0
        wall_max = reduce_max(pg, wall, dev)
        value = world * psteps / wall_max
        # latency: a fresh request set arriving as a Poisson process at --serve-rate
        lat, lsteps, lwall, _, _ = run_serving_window(srv, mk(args.serve_requests), args.serve_rate, rng)
        # load sweep: Poisson arrivals at fractions of the capacity's request rate; a rate is "bounded" while its
        # p99 stays within twice the p99 at --serve-rate (no backlog builds up over the window)
        cap_rate = len(reqs) / wall
        sweep = []
        for frac in args.serve_sweep:
            lat_f, _, wall_f, _, _ = run_serving_window(srv, mk(args.serve_sweep_requests), frac * cap_rate, rng)
            sweep.append({"load": frac, "rate_per_s": frac * cap_rate, "p50": float(np.percentile(lat_f, 50)),
                          "p99": float(np.percentile(lat_f, 99)), "max": float(lat_f.max()),
                          "requests": int(len(lat_f)), "window_s": wall_f})
        p99_ref = float(np.percentile(lat, 99))
        bounded = [w for w in sweep if w["p99"] <= 2 * p99_ref]
        fps = serve_flops_per_particle_step(m)
        peak, peak_src = fp64_peak(dev)
        achieved = fps * psteps / wall / 1e12
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                cpu = serving_cpu(sysm, s0, args.p_cpu_steps // 10, td)
            except Exception as exc:
                cpu = {"value": None, "unit": "particle-steps/s", "cores": 0, "kind": "unavailable", "sample": str(exc)}
        if rank == 0:
            sizes = [p.shape[1] for p, _ in reqs]
            line = {
                "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": 1,
                "warmup": args.warmup, "ms_per_step": wall_max * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic",
                "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": p99_ref,
                              "max": float(lat.max()), "requests": int(len(lat)), "rate_per_s": args.serve_rate,
                              "window_s": lwall, "particle_steps_per_s": lsteps / lwall,
                              "capacity_rate_per_s": cap_rate, "sweep": sweep,
                              "highest_bounded": (max(bounded, key=lambda w: w["rate_per_s"]) if bounded else None),
                              "bounded_rule": "p99 <= 2 x the p99 at rate_per_s"},
                "config": {"workload": f"config4: serving against a {m}-body B-spline ephemeris (config2 recipe, moons "
                                       f"merged into their hosts; cubic, 1-day knots, {args.serve_years:g} yr), "
                                       f"Poisson {args.serve_rate:g} requests/s, P = log-U(1, {args.serve_pmax}) "
                                       f"particles (a 0.5-50 AU, e < 0.6), durations log-U(1, {args.serve_years:g}) yr, "
                                       f"adaptive RK12 (step doubling) tol 1e-13",
                           "requests": len(reqs), "particles": int(sum(sizes)), "perturbers": m,
                           "rejected_step_fraction": rejected / max(1, rejected + psteps),
                           "ephemeris_setup_s": setup_s, "parallelism": f"independent servers x{world}" if world > 1
                           else "1 GPU, 128 streams",
                           "note": "value = accepted particle-steps / wall clock with all requests submitted at once "
                                   "(capacity; H2D/D2H included); latency_s from a second request set arriving as a "
                                   "Poisson process at rate_per_s"},
                "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                "roofline": {"bound": "fp64", "kernel": "serve_kernel", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak if peak else None, "traffic": None, "peak_source": peak_src,
                             "flops_per_particle_step": fps, "basis": "useful flops of accepted steps over the window"},
                "gpu_launches": launches,
                "clocks": clk,
            }
            if cpu is not None:
                line["cpu_baseline"] = cpu
            _emit(line)
        srv.close()
    if pg is not None:
        pg.destroy_process_group()


def serving_cpu(sysm, s0, n_step, tmpdir):
    """The reference CPU integrator on the serving perturbers: chunks of P_CPU_CHUNK particles (GM = 1e-20
    bodies, a 0.5-50 AU) with all perturbers in one msystem, fixed steps of 0.5 day, one chunk per process on
    every host core (the reference has neither B-spline perturbers nor adaptive stepping)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from ephemeris_b200 import synth
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(4005)
    cfgs = []
    for c in range(cores):
        parts = synth.kepler_cloud(rng, synth.GM_SUN, rng.uniform(0.5, 50, P_CPU_CHUNK) * synth.AU,
                                   rng.uniform(0, 0.6, P_CPU_CHUNK), rng.uniform(0, 20 * synth.DEG, P_CPU_CHUNK),
                                   s0[0, 0:3], s0[0, 3:6])
        cfgs.append(synth.write_system(synth.with_test_bodies(sysm, parts), os.path.join(tmpdir, f"serve_chunk{c}")))
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_ref_chunk, [(c, 1, P_CPU_CHUNK) for c in cfgs]))
        t0 = time.perf_counter()
        done = list(ex.map(_ref_chunk, [(c, n_step, P_CPU_CHUNK) for c in cfgs]))
        el = time.perf_counter() - t0
    steps = sum(b for b, _ in done)
    return {"value": steps / el, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{cores} chunks of {P_CPU_CHUNK} particles (GM=1e-20 bodies) + {len(sysm.bodies)} perturbers, "
                      f"{n_step} fixed RK12 steps of 0.5 day each, reference msystem::integrate(dt,n,0) serial, one chunk "
                      f"per process on {cores} processes, {el:.1f} s"}


def run_reference_serving(args):
    """--impl reference --workload config4: the reference CPU integrator on chunks of serving particles."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ephemeris_b200 import synth
    with tempfile.TemporaryDirectory() as td:
        sysm = synth.make_config4_system(4004)
        s0 = np.zeros((len(sysm.bodies), 10))
        s0[0, 0:3], s0[0, 3:6] = sysm.bodies[0].r, sysm.bodies[0].v
        vals, cpu = [], None
        for _ in range(max(1, args.steps)):
            cpu = serving_cpu(sysm, s0, args.p_cpu_steps // 10, td)
            vals.append(cpu["value"])
        value = statistics.median(vals)
        line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic", "impl": "reference",
                "config": {"workload": "config4 serving particles, reference CPU sample (see cpu_baseline.sample)"},
                "cpu_baseline": dict(cpu, value=value),
                "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    from ephemeris_b200 import Context, MSystem
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    with tempfile.TemporaryDirectory() as td:
        cfg = load_workload(args.workload, td)
        ms = MSystem(local)
        if not ms.load(cfg):
            raise RuntimeError("workload failed to load")
        planes0 = ms.planes()
        models = ms.models()
        n = planes0.shape[1]
        dt = ms.delta_t
        rk = args.rk_steps
        ctx = Context(local)
        ctx.upload(planes0, models)
        tune = None
        if args.grid or args.per_cta:
            ctx.set_launch(args.grid, args.per_cta)
        elif not args.no_autotune:
            g_, b_, t_tuned, t_default = ctx.autotune(dt, n_step=3, reps=2, use_cache=False)
            tune = {"grid": g_, "bodies_per_cta": b_, "ms_per_rk_step_tuned": t_tuned,
                    "ms_per_rk_step_heuristic": t_default, "by": "eph_autotune (outside the timed region)"}
        # a dedicated (non-default) stream: the context's kernels, the L2 flush and the events all go on it
        stream = torch.cuda.Stream(dev)
        ctx.set_stream(stream.cuda_stream)
        torch.cuda.set_stream(stream)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

        # ---- device-resident throughput: CUDA events on the launching stream, L2 flushed between steps.
        # Every step integrates the same initial state (restored from an HBM snapshot outside the events),
        # so each timed step is the same workload.
        snap = torch.from_numpy(planes0.copy()).to(dev)
        for _ in range(args.warmup):
            ctx.upload_device(snap.data_ptr())
            ctx.integrate(dt, rk)
        barrier(pg, dev)
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        launches0 = ctx.launches()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        wall0 = time.perf_counter()
        for k in range(args.steps):
            ctx.upload_device(snap.data_ptr())
            flush.fill_(float(k))
            starts[k].record(stream)
            ctx.integrate(dt, rk)
            ends[k].record(stream)
        torch.cuda.synchronize(dev)
        clk = clocks.stop()
        launches = ctx.launches() - launches0
        dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        wall_ms = (time.perf_counter() - wall0) * 1e3
        if dev_ms < 0.8 * wall_ms:   # the events must bracket the kernels (same stream)
            print(f"warning: device-timed {dev_ms:.3f} ms < 0.8 x host-timed {wall_ms:.3f} ms", file=sys.stderr)
        barrier(pg, dev)
        dev_ms_max = reduce_max(pg, dev_ms, dev)
        value = world * n * rk * args.steps / (dev_ms_max / 1e3)
        kern_ms = dev_ms / args.steps

        # ---- end to end through the public C ABI with host buffers (pinned)
        host_in = torch.from_numpy(planes0.copy()).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        pin_in, pin_out = host_in.numpy(), host_out.numpy()
        for _ in range(max(1, args.warmup // 2)):
            ctx.upload(pin_in, models)
            ctx.integrate(dt, rk)
            ctx.download(pin_out)
        barrier(pg, dev)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ctx.upload(pin_in, models)
            ctx.integrate(dt, rk)
            ctx.download(pin_out)
        torch.cuda.synchronize(dev)
        e2e_s = reduce_max(pg, time.perf_counter() - t0, dev)
        e2e = world * n * rk * args.steps / e2e_s

        flops_step = algorithmic_flops_per_step(planes0, models)
        achieved = flops_step * rk / (kern_ms / 1e3) / 1e12
        peak, peak_src = fp64_peak(dev)
        pipe = fp64_pipe_peak(local)
        cpu = None
        ref_gpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(cfg, args.cpu_rk_steps)
            except Exception as exc:   # the baseline is reported, not required
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(exc)}
            ref_gpu = reference_gpu_baseline(cfg)
        if rank == 0:
            grid, per = ctx.launch_shape()
            line = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (double-double state)", "data": "synthetic",
                "config": {"workload": f"{args.workload}: {n}-body full-physics synthetic system (seeded), "
                                       f"dt=0.05 day", "rk_steps_per_step": rk, "bodies": n,
                           "parallelism": f"replicas x{world}" if world > 1 else "single system, 1 GPU",
                           "l2": "flushed between timed steps (256 MB write)", "grid": grid, "bodies_per_cta": per,
                           "autotune": tune},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(planes0.nbytes),
                        "d2h_bytes_per_step": int(planes0.nbytes)},
                "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak if peak else None,
                             "traffic": DRAM_BYTES_PER_LAUNCH.get((args.workload, rk)),
                             "traffic_unit": "DRAM bytes read + written per step_kernel launch (ncu)",
                             "peak_source": peak_src, "flops_per_launch": flops_step * rk,
                             "fp64_pipe_peak": pipe, "frac_of_fp64_pipe": achieved / pipe if pipe else None,
                             "fp64_pipe_peak_source": "eph_fp64_fma_rate: independent FMA chains on every SM"},
                "gpu_launches": launches,
                "clocks": clk,
            }
            if cpu is not None:
                line["cpu_baseline"] = cpu
            if ref_gpu is not None:
                if "value" in ref_gpu:
                    ref_gpu["speedup_of_value"] = value / ref_gpu["value"]
                line["reference_gpu"] = ref_gpu
            if world == 1 and args.workload == "config2" and not args.no_sub_records:
                ctx.close()
                line["sub_records"] = collect_sub_records(args)
            _emit(line)
    if pg is not None:
        pg.destroy_process_group()


def collect_sub_records(args):
    """The other workloads of the path on the same GPU, each with its own metric, value, roofline, e2e,
    clocks and CPU reference sample: config3 (the 512-system ensemble at its full 500-20000-step durations,
    with the mixed-precision form, the plain FP64 path one member at a time and 1000-step errors), config5
    (2 M massless particles x 100 steps per bench step) and config4 (serving: capacity and p50/p99 latency)."""
    import copy
    global _CAPTURE
    plans = [("config3", run_b200_ensemble, dict(ens_frac=1.0, steps=1, warmup=1, ens_compare=True,
                                                 ens_cpu_members=32, ens_cpu_steps=100)),
             ("config5", run_b200_particles, dict(steps=3, warmup=2, p_cpu_steps=100, mixed=False)),
             ("config4", run_b200_serving, dict(warmup=3, serve_requests=100, serve_rate=10.0, p_cpu_steps=100))]
    subs = {}
    for name, fn, over in plans:
        a = copy.copy(args)
        a.workload = name
        for k, v in over.items():
            setattr(a, k, v)
        _CAPTURE = []
        try:
            fn(a)
            subs[name] = _CAPTURE[0] if _CAPTURE else {"unavailable": "the run produced no result"}
        except Exception as exc:   # a sub-record is reported, never fatal to the main line
            subs[name] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        finally:
            _CAPTURE = None
    return subs


_PEAKS = {}


def fp64_pipe_peak(device: int):
    """Measured throughput of the FP64 CUDA-core pipe (TFLOP/s), the pipe the RK12 kernels run on."""
    import ctypes
    from ephemeris_b200 import load_library
    if ("pipe", device) in _PEAKS:
        return _PEAKS[("pipe", device)]
    v = ctypes.c_double(0)
    out = v.value if load_library().eph_fp64_fma_rate(device, ctypes.byref(v)) == 0 else None
    _PEAKS[("pipe", device)] = out
    return out


def fp64_peak(dev):
    """Measured FP64 peak: cuBLAS DGEMM 8192^3 (best of 5, CUDA events), once per process."""
    if ("dgemm", str(dev)) not in _PEAKS:
        _PEAKS[("dgemm", str(dev))] = _fp64_peak(dev)
    return _PEAKS[("dgemm", str(dev))]


def _fp64_peak(dev):
    import torch
    try:
        a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
        b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
        torch.matmul(a, b)
        torch.cuda.synchronize(dev)
        best = None
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            ms = s.elapsed_time(e)
            best = ms if best is None else min(best, ms)
        del a, b
        return 2 * 8192 ** 3 / (best / 1e3) / 1e12, "cuBLAS DGEMM 8192^3, measured in bench.py (best of 5)"
    except Exception as exc:
        return None, f"unavailable: {exc}"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="config2")
    ap.add_argument("--rk-steps", type=int, default=100, help="RK12 steps per bench step")
    ap.add_argument("--ref-rk-steps", type=int, default=2, help="RK12 steps per reference bench step")
    ap.add_argument("--cpu-rk-steps", type=int, default=20, help="RK12 steps of the CPU baseline sample")
    ap.add_argument("--grid", type=int, default=0)
    ap.add_argument("--per-cta", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="config2: keep the built-in launch shape")
    ap.add_argument("--ens-systems", type=int, default=512, help="config3: ensemble members")
    ap.add_argument("--ens-frac", type=float, default=0.1, help="config3: fraction of each member's drawn duration")
    ap.add_argument("--ens-cpu-members", type=int, default=64, help="config3: members in the CPU sample")
    ap.add_argument("--ens-compare", action="store_true",
                    help="config3: also the mixed-precision form, the plain FP64 path one member at a time, and "
                         "1000-step errors against the oracle")
    ap.add_argument("--no-sub-records", action="store_true",
                    help="config2 on 1 GPU: skip the config3/config5/config4 sub-records of the default run")
    ap.add_argument("--ens-cpu-steps", type=int, default=200, help="config3: RK12 steps per member in the CPU sample")
    ap.add_argument("--particles", type=int, default=2_000_000, help="config5: massless particles per GPU")
    ap.add_argument("--p-steps", type=int, default=100, help="config5: RK12 steps per bench step")
    ap.add_argument("--p-cpu-steps", type=int, default=300, help="config5: RK12 steps per chunk in the CPU sample")
    ap.add_argument("--mixed", action="store_true", help="config5: mixed precision (EIH 1PN in FP32)")
    ap.add_argument("--serve-years", type=float, default=10.0, help="config4: ephemeris span and longest request")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="config4: Poisson request rate per second")
    ap.add_argument("--serve-requests", type=int, default=200, help="config4: requests in the timed window")
    ap.add_argument("--serve-pmax", type=int, default=4096, help="config4: most particles in a request")
    ap.add_argument("--serve-sweep", type=float, nargs="*", default=[0.25, 0.5, 0.75, 0.9],
                    help="config4: loads (fractions of the capacity's request rate) of the latency sweep")
    ap.add_argument("--serve-sweep-requests", type=int, default=60, help="config4: requests per sweep window")
    args = ap.parse_args()
    if args.workload == "config4":
        if args.impl == "reference":
            run_reference_serving(args)
        else:
            run_b200_serving(args)
    elif args.workload == "config5":
        if args.impl == "reference":
            run_reference_particles(args)
        else:
            run_b200_particles(args)
    elif args.workload == "config3":
        if args.impl == "reference":
            run_reference_ensemble(args)
        else:
            run_b200_ensemble(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
