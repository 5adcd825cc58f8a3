"""Timing of the reference's own GPU integrator (test infrastructure; baseline only).

    python -m oracle.ref_gpu_timing <Config.txt> <rk_steps> [calls]

Loads the system with the reference's loader and integrates it with msystem::integrate(dt, n, USE_GPU=1),
i.e. the reference's unchanged cooperative kernel (src/integrators/RungeKutta.cu:391-412) compiled for
sm_100a (oracle/_ref/libephref_gpu.so, built by oracle/Makefile). First one step is checked against the
reference's CPU integrator with the reference's own CPU-vs-GPU bounds (src/tests/test_integrator.cpp:15-45);
then `calls` calls of `rk_steps` steps each are timed by wall clock (each call copies the body list to the
device and back, as the reference does). Prints one JSON object. Runs in a process of its own: the
reference's CUDA error handler exits the process.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

GPU_LIB = os.path.join(HERE, "_ref", "libephref_gpu.so")


def _bounds(gpu, cpu, t):
    """Largest ratio of a test_integrator.cpp:22-45 error to its bound (ref_cgpu_err, :16), scaled 86400/t."""
    f = 86400.0 / t
    norm = lambda d: np.sqrt((d ** 2).sum(0)).max()
    dr = (gpu[0:3] - cpu[0:3]) + (gpu[3:6] - cpu[3:6])
    dv = (gpu[6:9] - cpu[6:9]) + (gpu[9:12] - cpu[9:12])
    return max(norm(dr) * f / 1e-6, norm(dv) * f / 1e-8, norm(gpu[36:39] - cpu[36:39]) * f / 1e-16,
               norm(gpu[18:21] - cpu[18:21]) * f / 1e-13, norm(gpu[24:27] - cpu[24:27]) * f / 1e-13)


def main():
    from oracle.pyoracle import RefSystem
    cfg, steps = sys.argv[1], int(sys.argv[2])
    calls = int(sys.argv[3]) if len(sys.argv) > 3 else 3
    base = RefSystem(cfg, lib_path=GPU_LIB)
    dt = base.lib().ref_delta_t(base.h)
    g, c = base.clone(), base.clone()
    RefSystem.thread_pool(True)
    g.integrate(dt, 1, use_gpu=1)
    c.integrate(dt, 1, use_gpu=0)
    check = _bounds(g.planes(), c.planes(), abs(dt))
    run = base.clone()
    run.integrate(dt, steps, use_gpu=1)    # warm-up (context creation, module load)
    t0 = time.perf_counter()
    for _ in range(calls):
        run.integrate(dt, steps, use_gpu=1)
    el = time.perf_counter() - t0
    n = base.n
    print(json.dumps({"value": n * steps * calls / el, "unit": "body-steps/s", "ms_per_rk_step": 1e3 * el / (steps * calls),
                      "bodies": n, "rk_steps_per_call": steps, "calls": calls,
                      "one_step_vs_reference_cpu": {"max_ratio_to_test_integrator_bound": check,
                                                    "within_bounds": bool(check < 1.0)},
                      "what": "reference msystem::integrate(dt,n,1): its cooperative kernel (RungeKutta.cu) compiled "
                              "unchanged for sm_100a, wall clock per call including its host<->device copies"}))


if __name__ == "__main__":
    main()
