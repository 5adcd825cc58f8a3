"""Host-side checks that need no GPU: the C ABI library, the loader's error paths, the synthetic
generator and the multi-rank reduction used by bench.py."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from tests.conftest import GOLDEN, ROOT, gpu_available

HEADERS = ["eph_b200.h", "eph_msystem.h"]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(eph_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from ephemeris_b200 import load_library, LIB_PATH
    lib = load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (eph_\w+)", out))
    assert set(declared_functions()) <= exported


def test_build_targets_sm100a_only():
    from ephemeris_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_context_without_device_reports_error():
    from ephemeris_b200 import load_library
    lib = load_library()
    h = ctypes.c_void_p()
    assert lib.eph_ctx_create(0, ctypes.byref(h)) == 1     # EPH_ERR_ARG, nothing allocated
    assert not h.value


def test_loader_rejects_missing_and_malformed_files(tmp_path):
    from ephemeris_b200 import load_library
    lib = load_library()
    h = ctypes.c_void_p()
    assert lib.eph_msystem_load(str(tmp_path / "nope" / "Config.txt").encode(), 0, ctypes.byref(h)) == 6
    cfg = tmp_path / "Config.txt"
    cfg.write_text("Initial\tInitial.txt\nBogusKey\t1\n")
    assert lib.eph_msystem_load(str(cfg).encode(), 0, ctypes.byref(h)) == 6
    cfg.write_text("Initial\tInitial.txt\n")
    (tmp_path / "Initial.txt").write_text("Star\tS0\t1.0\t2.0\n")      # too few columns
    assert lib.eph_msystem_load(str(cfg).encode(), 0, ctypes.byref(h)) == 6
    (tmp_path / "Initial.txt").write_text("")                            # no bodies
    assert lib.eph_msystem_load(str(cfg).encode(), 0, ctypes.byref(h)) == 6


def test_msystem_without_gpu_flag_is_unsupported():
    """USE_GPU=0 / parallel_option<=0 ask for the CPU path, which this library does not provide."""
    from ephemeris_b200 import load_library
    lib = load_library()
    assert lib.eph_msystem_integrate(None, 1.0, 1, 0) == 1      # null system: EPH_ERR_ARG first


def test_synthetic_systems_are_reproducible(tmp_path):
    from ephemeris_b200 import synth
    from tests.golden.make_golden import system_hash
    import json
    meta = json.load(open(os.path.join(GOLDEN, "manifest.json")))
    for name in ["config1", "small_full", "config2"]:
        d = tmp_path / name
        synth.write_workload(meta[name]["generator"], str(d), **meta[name]["kwargs"])
        assert system_hash(str(d)) == meta[name]["sha256"], name
    for name in ["config1", "small_full"]:
        assert system_hash(str(tmp_path / name)) == system_hash(os.path.join(GOLDEN, "systems", name))


def test_config2_shape():
    from ephemeris_b200 import synth
    s = synth.make_config2()
    assert len(s.bodies) == 504
    assert len(s.geopotentials) == 9 and len(s.rings) == 1
    soft = [b for b in s.bodies if b.R_km < 0]
    assert len(soft) == 36


def test_algorithmic_flop_count(golden):
    import bench
    from ephemeris_b200 import Models
    g = golden("config1")
    m = g.models()
    f = bench.algorithmic_flops_per_step(g["load"], Models(m.gp_nz, m.gp_nt, m.gp_coef, m.ring_ndisk,
                                                          m.ring_param, m.ring_disk))
    n = 33
    # point-like bodies only: pass A (20) and 1PN (80) per ordered pair; the deformation, Lense-Thirring and
    # radiation terms are exactly zero and not evaluated
    assert f == 25 * n * (n - 1) * 100 + n * 3900
    g2 = golden("config2")
    m2 = g2.models()
    pl = g2["load"]
    f2 = bench.algorithmic_flops_per_step(pl, Models(m2.gp_nz, m2.gp_nt, m2.gp_coef, m2.ring_ndisk, m2.ring_param,
                                                     m2.ring_disk))
    n, nf = pl.shape[1], int(bench.full_class(pl).sum())
    delayed = int(((pl[46] != 0) & (pl[48] != 0)).sum())
    pairs_full = n * (n - 1) - (n - nf) * (n - nf - 1)
    want = 25 * (n * (n - 1) * 100 + pairs_full * 180 + delayed * (n - 1) * 120 + 9 * (n - 1) * 250
                 + 2 * (n - 1) * 60) + n * 3900
    assert (nf, delayed) == (107, 86)
    assert f2 == want


def _gloo_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), EPH_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    r, w, local, pg = bench.dist_setup(world)
    got = bench.reduce_max(pg, float(10 + rank), device="cpu")
    bench.barrier(pg, device="cpu")
    q.put((r, w, got))
    pg.destroy_process_group()


def test_bench_rank_reduction_gloo():
    """bench.py's max-over-ranks timing with two gloo ranks on CPU."""
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == [(0, 2, 11.0), (1, 2, 11.0)]


def test_serving_and_particle_workloads_are_seeded():
    """The config4/config5 generators: same seed, same bodies and particles; the stated shapes."""
    from ephemeris_b200 import synth
    a, b = synth.make_config4_system(4004), synth.make_config4_system(4004)
    assert len(a.bodies) == 419 and [x.r for x in a.bodies] == [x.r for x in b.bodies]
    assert all(x.k2 == 0 and x.j2 == 0 and x.gp_factor == 0 for x in a.bodies)   # point masses
    s1, p1 = synth.make_config5(5005, n_particles=1000)
    s2, p2 = synth.make_config5(5005, n_particles=1000)
    assert np.array_equal(p1, p2) and len(s1.bodies) == 9
    c1 = synth.make_config1(1001)
    assert [x.r for x in s1.bodies[1:]] != [] and s1.bodies[0].j2 == 2e-4
    assert [x.GM for x in s1.bodies] == [x.GM for x in c1.bodies[:9]]      # config1's star and planets
    r = np.linalg.norm(p1[0:3] - np.asarray(s1.bodies[0].r)[:, None], axis=0) / synth.AU
    assert r.min() > 1.5 * 0.7 - 1e-9 and r.max() < 50 * 1.3 + 1e-9        # a in [1.5, 50] AU, e < 0.3
    rng = np.random.default_rng(1)
    reqs = synth.make_requests(rng, 50, 10 * 365.25 * 86400, years=(1, 10))
    assert all(1 <= q.shape[1] <= 4096 and 365.25 * 86400 * 0.999 <= t <= 10 * 365.25 * 86400 for q, t in reqs)
