"""Build recipe of libeph_b200.so (CUDA kernels for sm_100a + the C ABI + the host loader).

    python -m ephemeris_b200.build          # or ephemeris_b200.build.build()

nvcc compiles every translation unit for sm_100a only (-gencode arch=compute_100a,code=sm_100a) and
links them into ephemeris_b200/libeph_b200.so, in the source tree, so the library travels with the
repository checkout. Rebuilds only when a source is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libeph_b200.so")
BUILD = os.path.join(HERE, "_build")

CUDA_UNITS = ["eph_step.cu", "eph_capi.cu", "eph_noalloc.cu", "eph_batch.cu", "eph_particles.cu", "eph_serve.cu",
              "eph_fields.cu"]
CXX_UNITS = ["eph_msystem.cpp", "eph_bspline.cpp", "eph_ephemeris.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *ARCH]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    srcs = [os.path.join(CSRC, f) for f in CUDA_UNITS + CXX_UNITS]
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return srcs, deps


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    mtime = os.path.getmtime(LIB)
    _, deps = _sources()
    return any(os.path.getmtime(d) > mtime for d in deps + [__file__])


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for unit in CUDA_UNITS + CXX_UNITS:
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj]
        if unit.endswith(".cpp"):
            cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-fPIC", "-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", *ARCH, "-o", tmp, *objs, "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
