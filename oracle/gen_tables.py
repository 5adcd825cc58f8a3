"""Regenerate the two constant data tables that the reference ships as hex source data.

Run from the repository root with the reference tree available:
    python oracle/gen_tables.py [REFERENCE_ROOT]
(default: the REF_ROOT environment variable, as for oracle/Makefile)

Outputs (committed, plain C headers usable from C, C++ and CUDA):
  include/eph_rk12_table.h  Feagin's 12th-order, 25-stage Runge-Kutta coefficients as 325
                            double-double values, row k at k*(k-1)/2 (src/integrators/RungeKutta.impl:37-104).
  include/eph_ring_table.h  the fp32 bicubic correction table of the disk-field approximation,
                            2048 cells x 16 coefficients (src/physics/ring.impl:19-2068).

Both are numeric tables, not code: parity with the reference's integrator needs the identical
coefficients, so they are carried over as data, bit for bit.
"""
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT", "")
if not REF:
    sys.exit("usage: python oracle/gen_tables.py REFERENCE_ROOT (or set REF_ROOT)")
HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(HERE, "..", "include")


def _hex_block(path, start_marker):
    text = open(path, "r", encoding="latin-1").read().replace("\r", "")
    i = text.index(start_marker)
    j = text.index("};", i)
    return re.findall(r"0x[0-9a-fA-F]+", text[i:j])


def main():
    rk = _hex_block(os.path.join(REF, "src/integrators/RungeKutta.impl"), "rk12_coefs[]")
    assert len(rk) == 650, len(rk)
    with open(os.path.join(INC, "eph_rk12_table.h"), "w") as f:
        f.write("/* Generated by oracle/gen_tables.py - do not edit.\n"
                " * Feagin RK12 (25 stages) coefficients a[k][j], k=1..25, j<k, as double-double (hi, lo)\n"
                " * IEEE-754 bit patterns; entry k*(k-1)/2+j; row 25 is the weight vector b.\n"
                " * Data as in src/integrators/RungeKutta.impl:37-104 of the reference. */\n")
        f.write("#ifndef EPH_RK12_TABLE_H\n#define EPH_RK12_TABLE_H\n#include <stdint.h>\n")
        f.write("#define EPH_RK12_STAGES 25\n#define EPH_RK12_NCOEF 325\n")
        f.write("static const uint64_t EPH_RK12_COEF_BITS[2 * EPH_RK12_NCOEF] = {\n")
        for r in range(0, len(rk), 6):
            f.write("    " + ", ".join(x.lower() + "ull" for x in rk[r:r + 6]) + ",\n")
        f.write("};\n#endif\n")
    ring = _hex_block(os.path.join(REF, "src/physics/ring.impl"), "disk_approx_table[]")
    assert len(ring) == 2048 * 16, len(ring)
    with open(os.path.join(INC, "eph_ring_table.h"), "w") as f:
        f.write("/* Generated by oracle/gen_tables.py - do not edit.\n"
                " * fp32 bicubic correction of the ring disk-field angle term: 2*32 x 32 cells of 16\n"
                " * coefficients (IEEE-754 binary32 bit patterns), indexed [(2*32*i + j)*16 + c].\n"
                " * Data as in src/physics/ring.impl:19-2068 of the reference. */\n")
        f.write("#ifndef EPH_RING_TABLE_H\n#define EPH_RING_TABLE_H\n#include <stdint.h>\n")
        f.write("#define EPH_RING_TABLE_WORDS 32768\n")
        f.write("#ifdef __CUDACC__\n#define EPH_RING_TABLE_QUAL static __device__ const\n#else\n"
                "#define EPH_RING_TABLE_QUAL static const\n#endif\n")
        f.write("EPH_RING_TABLE_QUAL uint32_t EPH_RING_TABLE_BITS[EPH_RING_TABLE_WORDS] = {\n")
        for r in range(0, len(ring), 16):
            f.write("    " + ",".join(x.lower() for x in ring[r:r + 16]) + ",\n")
        f.write("};\n")
        f.write("#endif\n")


if __name__ == "__main__":
    main()
