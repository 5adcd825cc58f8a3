// eph_rk12_host.h - host-side expansion of the Feagin RK12 table (include/eph_rk12_table.h) into the
// arrays the kernels keep in constant memory: a_kj as double-double (hi, lo) and the stage nodes c_k.
#pragma once
#include <cstring>

#include "../../include/eph_rk12_table.h"

namespace eph {

// c_k is accumulated exactly as RungeKutta.impl:118-152: zero coefficients skipped, hi + lo added in j order.
inline void rk12_expand(double *hi, double *lo, double *dtk) {
    for (int q = 0; q < EPH_RK12_NCOEF; ++q) {
        memcpy(&hi[q], &EPH_RK12_COEF_BITS[2 * q], 8);
        memcpy(&lo[q], &EPH_RK12_COEF_BITS[2 * q + 1], 8);
    }
    dtk[0] = 0;
    for (int k = 1; k <= EPH_RK12_STAGES; ++k) {
        double acc = 0;
        for (int j = 0; j < k; ++j) {
            const int ci = k * (k - 1) / 2 + j;
            if (hi[ci] != 0) acc += hi[ci] + lo[ci];
        }
        dtk[k] = acc;
    }
}

}  // namespace eph
