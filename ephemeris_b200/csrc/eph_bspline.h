// eph_bspline.h - the grid part of the B-spline fit (eph_bspline.cpp), shared by the host fit and the
// device batch fit (eph_serve.cu).
//
// The normal-equation matrix of the least-squares fit depends only on the degree and the sample grid,
// not on the data, so it is assembled, row-scaled and LU-factored once; a data series then needs only its
// right-hand side and the two substitutions. Double-double values are kept as (hi, lo) pairs.
#pragma once
#include <cstdint>
#include <vector>

namespace eph {

struct BsplineFactor {
    int d = 0, J = 0;                  // degree; most samples in one row's support
    int64_t n = 0, mn = 0, m = 0;      // knot intervals, sample intervals, coefficients (n + d)
    std::vector<int64_t> jmin;         // [m] first sample of row i's support
    std::vector<int> cnt;              // [m] samples in it
    std::vector<double> bval;          // [m][J] B[d, x_j - i] on them
    std::vector<double> rw_hi, rw_lo;  // [m] 1 / sum_j B[d, x_j - i]
    std::vector<double> lu_hi, lu_lo;  // [m][2d + 1] L (below the diagonal) and U, band[i][j - i + d]
    std::vector<double> rd_hi, rd_lo;  // [m] 1 / U(i, i)
};

// 0 on success; nonzero for sizes the fit does not take (see eph_bspline_fit).
int bspline_factor(int d, int64_t n, int64_t mn, BsplineFactor &f);

}  // namespace eph
