"""B200-native RK12 step of Ephemeris: CUDA kernels for sm_100a behind a C ABI.

Public entry points (mirroring the reference's msystem for the RK12 path):
    MSystem   - load(config) / integrate(dt, n_step, 1) / accel(1) / planes()
    Context   - the lower-level C ABI: upload a plane array, rk12 / integrate / accel, download
    Batch     - many independent systems integrated together (ensembles)
    Particles - massless test particles against perturbers
    Server    - small-body requests (adaptive RK12) against a device B-spline ephemeris
    EphemerisInterpolator - one compressed orbital record of the reference's ephemeris files, decoded
    synth     - seeded synthetic systems written in the reference's initials formats
"""
from .msystem import MSystem, Context, Batch, Particles, Server, bspline_fit, bspline_fit_batch, Models, P as PLANES, set_log_level, CPU_RK12, GPU_RK12, COMBINED_RK12
from ._lib import load_library, EphError, NPLANES, LIB_PATH
from .ephemeris_record import EphemerisInterpolator

__all__ = ["MSystem", "Context", "Batch", "Particles", "Server", "bspline_fit", "bspline_fit_batch", "Models", "PLANES", "set_log_level", "load_library", "EphError", "NPLANES",
           "LIB_PATH", "CPU_RK12", "GPU_RK12", "COMBINED_RK12", "EphemerisInterpolator"]
