"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run from the repository root, in a container where the reference tree is available and
oracle/_ref/libephref.so has been built (`make -C oracle`):

    python tests/golden/make_golden.py

For each synthetic system it writes <name>.npz with the reference's outputs, all in the plane layout
of include/eph_planes.h:
  load      planes after msystem::load(config)          (src/modules/mass_loader.cpp:67-294)
  accel     planes after msystem::accel(-1) on `load`   (src/physics/mass.cpp:216-397, serial branch)
  step<k>   planes after msystem::integrate(dt, k, 0)   (src/physics/mass.cpp:399-442), serial branch
  stage_acc gaccel+daccel+naccel after each of the 25 accel() calls of the first step
  models    geopotential / ring tables; t_eph after each integrate; dt
The systems' text files (reference initials formats, written by ephemeris_b200.synth) are stored in
tests/golden/systems/<name>/ for the small systems; config2 (504 bodies) is regenerated from its seed
and checked against the recorded SHA-256 of its files.
"""
import hashlib
import json
import os
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ephemeris_b200 import synth  # noqa: E402
from oracle.pyoracle import RefSystem  # noqa: E402

HERE = os.path.join(ROOT, "tests", "golden")
SYSTEMS = {
    # name: (generator, kwargs, stored text files?, steps to record)
    "config1": ("config1", {}, True, [1, 10, 1000]),
    "small_full": ("small_full", {}, True, [1, 10, 100, 1000]),
    "config2": ("config2", {}, False, [1, 1000]),
}


def system_hash(directory):
    h = hashlib.sha256()
    for root, _, files in sorted(os.walk(directory)):
        for f in sorted(files):
            p = os.path.join(root, f)
            h.update(os.path.relpath(p, directory).encode())
            with open(p, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()


def main():
    manifest = {}
    for name, (gen, kw, store, steps) in SYSTEMS.items():
        sysdir = os.path.join(HERE, "systems", name) if store else os.path.join(HERE, "_tmp", name)
        if os.path.exists(sysdir):
            shutil.rmtree(sysdir)
        cfg = synth.write_workload(gen, sysdir, **kw)
        digest = system_hash(sysdir)
        ref = RefSystem(cfg)
        RefSystem.thread_pool(False)
        out = {"load": ref.planes()}
        m = ref.models()
        out.update(gp_nz=m.gp_nz, gp_nt=m.gp_nt, gp_coef=m.gp_coef, ring_ndisk=m.ring_ndisk,
                   ring_param=m.ring_param, ring_disk=m.ring_disk)
        dt = ref.lib().ref_delta_t(ref.h)
        out["dt"] = np.array(dt)
        a = ref.clone()
        a.accel(-1)
        out["accel"] = a.planes()
        cap = ref.clone()
        stages = cap.integrate_capture(dt, 1)
        out["stage_acc"] = stages[:, 76:79] + stages[:, 70:73] + stages[:, 67:70]
        done = 0
        cur = ref.clone()
        for k in steps:
            cur.integrate(dt, k - done)
            done = k
            out[f"step{k}"] = cur.planes()
            out[f"t_eph{k}"] = np.array(cur.t_eph)
        out["sids"] = np.array(ref.sids())
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        manifest[name] = {"generator": gen, "kwargs": kw, "sha256": digest, "stored": store, "steps": steps,
                          "n": int(out["load"].shape[1]), "dt": dt}
        print(name, out["load"].shape, "steps", steps)
    tmp = os.path.join(HERE, "_tmp")
    if os.path.exists(tmp):
        shutil.rmtree(tmp)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
