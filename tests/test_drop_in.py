"""The drop-in itself: the unmodified reference host code with its GPU members served by the B200
bridge (ephemeris_b200/bridge/cuda_rk12_bridge.cpp linked in place of src/integrators/RungeKutta.cu).

Mirrors the first check of the reference's test_integrator (src/tests/test_integrator.cpp:53-82): the
same system is integrated one step with USE_GPU=0 (the reference CPU integrator) and USE_GPU=1 (the
B200 kernels through msystem::integrate), and the results must agree within ref_cgpu_err (:16,41-43)
and 1e-15 relative on min_distance / max_influence (:20,36-40).
"""
import numpy as np
import pytest

from oracle.pyoracle import BRIDGE_LIB, RefSystem, ref_available
from tests.parity import accel_error, position_error
from tests.test_gpu_parity import _test_integrator_bounds

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(BRIDGE_LIB), reason="bridge build oracle/_ref/libephref_b200.so absent")]


@pytest.mark.parametrize("name", ["config1", "small_full", "config2"])
def test_reference_host_cpu_vs_b200_gpu_one_step(golden, tmp_path, name):
    g = golden(name)
    cfg = g.config_path(tmp_path)
    cpu = RefSystem(cfg, lib_path=BRIDGE_LIB)
    gpu = cpu.clone()
    dt = float(g["dt"])
    cpu.integrate(dt, 1, use_gpu=0)
    gpu.integrate(dt, 1, use_gpu=1)
    a, b = gpu.planes(), cpu.planes()
    t = cpu.t_eph
    assert gpu.t_eph == t
    assert position_error(a, b) <= 1e-12
    assert _test_integrator_bounds(a, b, t[0] + t[1]) < 1.0


def test_reference_accel_gpu_option(golden, tmp_path):
    g = golden("small_full")
    cpu = RefSystem(g.config_path(tmp_path), lib_path=BRIDGE_LIB)
    gpu = cpu.clone()
    cpu.accel(-1)
    gpu.accel(1)
    assert accel_error(gpu.planes(), cpu.planes()) <= 1e-14


def test_reference_host_many_calls(golden, tmp_path):
    """Repeated integrate() calls through the bridge keep matching the CPU path (state round trips)."""
    g = golden("config1")
    cpu = RefSystem(g.config_path(tmp_path), lib_path=BRIDGE_LIB)
    gpu = cpu.clone()
    dt = float(g["dt"])
    for k in range(5):
        cpu.integrate(dt, 7, use_gpu=0)
        gpu.integrate(dt, 7, use_gpu=1)
    assert position_error(gpu.planes(), cpu.planes()) <= 1e-12
