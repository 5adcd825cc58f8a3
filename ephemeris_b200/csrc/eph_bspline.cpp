// eph_bspline.cpp - host side of the B-spline ephemeris: the least-squares fit of uniformly sampled
// channels with degree-d B-splines, and the Chebyshev form of the B-spline basis that the device
// evaluator uses.
//
// Basis (src/math/interp.h:10-22): B[0,x] = 1 on [0,1); B[d,x] = ((x+d) B[d-1,x+1] + (1-x) B[d-1,x]) / d,
// positive on (-d,1). On x in [0,1) the piece B[d, x-k] (k = 0..d) is a polynomial of degree d, written
// here as sum_j c(d,k,j) T_j(2x-1) (src/math/interp.h:24-30); c is derived below from the recursion.
//
// Fit (src/math/interp.h:68-150): n + d basis functions B[d, x - i], i = 0..n+d-1, on the sample grid
// x_j = j n / mn, j = 0..mn; normal equations sum_j B_i(x_j) B_k(x_j) a_k = sum_j B_i(x_j) y_j, each row
// scaled by 1 / sum_j B_i(x_j), solved by banded LU without pivoting (bandwidth d), all in double-double.
// The matrix part depends only on the grid (bspline_factor); each data series then takes its right-hand
// side and the two substitutions, in the reference's operation order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/eph_b200.h"
#include "eph_bspline.h"

namespace {

constexpr int kMaxDeg = EPH_BSPLINE_MAX_DEGREE;

// ------------------------------------------------------------------ Chebyshev coefficients of the pieces
struct ChebTable {
    double c[kMaxDeg + 1][kMaxDeg + 1][kMaxDeg + 1];   // [d][k][j]
    ChebTable() {
        std::memset(c, 0, sizeof(c));
        // pieces as polynomials in x on [0,1): P[d][k][m] = coefficient of x^m of B[d, x - k]
        long double P[kMaxDeg + 1][kMaxDeg + 1][kMaxDeg + 1] = {};
        P[0][0][0] = 1;
        for (int d = 1; d <= kMaxDeg; ++d)
            for (int k = 0; k <= d; ++k) {
                // B[d, x-k] = ((x-k+d) B[d-1, x-k+1] + (1-x+k) B[d-1, x-k]) / d; B[d-1, x-(k-1)] is piece k-1
                long double out[kMaxDeg + 2] = {};
                if (k - 1 >= 0)
                    for (int m = 0; m < d; ++m) {
                        out[m + 1] += P[d - 1][k - 1][m];
                        out[m] += (long double)(d - k) * P[d - 1][k - 1][m];
                    }
                if (k <= d - 1)
                    for (int m = 0; m < d; ++m) {
                        out[m + 1] -= P[d - 1][k][m];
                        out[m] += (long double)(1 + k) * P[d - 1][k][m];
                    }
                for (int m = 0; m <= d; ++m) P[d][k][m] = out[m] / d;
            }
        // x = (u + 1) / 2, then powers of u to Chebyshev: u^l = 2^(1-l) sum_{i} binom(l, i) T_{l-2i} (halved at 0)
        for (int d = 0; d <= kMaxDeg; ++d)
            for (int k = 0; k <= d; ++k) {
                long double q[kMaxDeg + 1] = {};   // coefficients in u
                for (int m = 0; m <= d; ++m) {
                    long double scale = P[d][k][m] / std::pow(2.0L, m);
                    long double binom = 1;          // binom(m, l)
                    for (int l = 0; l <= m; ++l) {
                        q[l] += scale * binom;
                        binom = binom * (m - l) / (l + 1);
                    }
                }
                long double t[kMaxDeg + 1] = {};
                for (int l = 0; l <= d; ++l) {
                    long double binom = 1;          // binom(l, i)
                    for (int i = 0; 2 * i <= l; ++i) {
                        const int j = l - 2 * i;
                        long double w = q[l] * binom / std::pow(2.0L, l - 1);
                        if (j == 0) w /= 2;
                        t[j] += w;
                        binom = binom * (l - i) / (i + 1);
                    }
                }
                for (int j = 0; j <= d; ++j) c[d][k][j] = (double)t[j];
            }
    }
};
const ChebTable &cheb() {
    static const ChebTable t;
    return t;
}

// B[d, x] from the Chebyshev pieces (src/math/interp.cpp:116-137 evaluates the same expansion)
double basis(int d, double x) {
    if (!(x < 1 && x >= -d)) return 0;
    const int k = -(int)std::floor(x);
    const double *c = cheb().c[d][k];
    x += k;
    const double u = 2 * x - 1, u2 = 2 * u;
    double s = c[0];
    if (d > 0) {
        s += c[1] * u;
        double tm, t = 1, tp = u;
        for (int j = 2; j <= d; ++j) {
            tm = t;
            t = tp;
            tp = u2 * t - tm;
            s += c[j] * tp;
        }
    }
    return s;
}

// ------------------------------------------------------------------ double-double
struct dd {
    double hi, lo;
};
inline dd two_sum(double a, double b) {
    const double s = a + b, bb = s - a;
    return dd{s, (a - (s - bb)) + (b - bb)};
}
inline dd quick(double a, double b) {
    const double s = a + b;
    return dd{s, b - (s - a)};
}
inline dd add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return quick(s.hi, s.lo);
}
inline dd neg(dd a) { return dd{-a.hi, -a.lo}; }
inline dd sub(dd a, dd b) { return add(a, neg(b)); }
inline dd mul(dd a, dd b) {
    const double p = a.hi * b.hi;
    const double e = std::fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
    return quick(p, e);
}
inline dd div(dd a, dd b) {
    const double q1 = a.hi / b.hi;
    const dd r = sub(a, mul(dd{q1, 0}, b));
    const double q2 = r.hi / b.hi;
    const dd r2 = sub(r, mul(dd{q2, 0}, b));
    const double q3 = r2.hi / b.hi;
    return add(quick(q1, q2), dd{q3, 0});
}
inline dd mk(double a) { return dd{a, 0}; }

}  // namespace

namespace eph {

int bspline_factor(int d, int64_t n, int64_t mn, BsplineFactor &f) {
    if (d < 1 || d > kMaxDeg || n < 1 || mn < 1 || mn + 1 < n + d) return 1;
    const int64_t m = n + d, w = 2 * d + 1;
    f.d = d; f.n = n; f.mn = mn; f.m = m;
    f.jmin.assign(m, 0);
    f.cnt.assign(m, 0);
    f.J = 0;
    for (int64_t i = 0; i < m; ++i) {
        f.jmin[i] = std::max<int64_t>(0, mn * (i - d) + n) / n;
        const int64_t jmax = std::min<int64_t>(mn, (mn * (i + 1) - 1) / n);
        f.cnt[i] = (int)std::max<int64_t>(0, jmax - f.jmin[i] + 1);
        f.J = std::max(f.J, f.cnt[i]);
    }
    f.bval.assign((size_t)m * f.J, 0.0);
    std::vector<dd> band((size_t)m * w, mk(0));          // band[i][j - i + d]
    auto A = [&](int64_t i, int64_t j) -> dd & { return band[(size_t)i * w + (j - i + d)]; };
    std::vector<dd> rw(m);
    const double rmn = 1.0 / (double)mn;
    for (int64_t i = 0; i < m; ++i) {
        dd wsum = mk(0);
        for (int q = 0; q < f.cnt[i]; ++q) {
            const int64_t j = f.jmin[i] + q;
            const double xj = (double)(j * n) * rmn;
            const double bij = basis(d, xj - (double)i);
            f.bval[(size_t)i * f.J + q] = bij;
            const dd b = mk(bij);
            const int64_t kmin = j * n / mn, kmax = (j * n + mn - 1) / mn + d - 1;
            for (int64_t k = kmin; k <= kmax; ++k)
                if (k >= 0 && k < m && std::llabs(k - i) <= d) A(i, k) = add(A(i, k), mul(mk(basis(d, xj - (double)k)), b));
            wsum = add(wsum, b);
        }
        rw[i] = div(mk(1), wsum);
        for (int64_t k = std::max<int64_t>(0, i - d); k <= std::min<int64_t>(m - 1, i + d); ++k) A(i, k) = mul(A(i, k), rw[i]);
    }
    // banded LU without pivoting (Doolittle)
    for (int64_t i = 0; i < m; ++i) {
        const int64_t lo = std::max<int64_t>(0, i - d), hi = std::min<int64_t>(m - 1, i + d);
        for (int64_t j = lo; j < i; ++j) {
            dd s = mk(0);
            for (int64_t k = lo; k < j; ++k) s = add(s, mul(A(i, k), A(k, j)));
            A(i, j) = div(sub(A(i, j), s), A(j, j));
        }
        for (int64_t j = i; j <= hi; ++j) {
            dd s = mk(0);
            for (int64_t k = std::max<int64_t>(0, j - d); k < i; ++k) s = add(s, mul(A(i, k), A(k, j)));
            A(i, j) = sub(A(i, j), s);
        }
    }
    f.rw_hi.resize(m); f.rw_lo.resize(m); f.rd_hi.resize(m); f.rd_lo.resize(m);
    f.lu_hi.resize((size_t)m * w); f.lu_lo.resize((size_t)m * w);
    for (int64_t i = 0; i < m; ++i) {
        f.rw_hi[i] = rw[i].hi; f.rw_lo[i] = rw[i].lo;
        const dd r = div(mk(1), A(i, i));
        f.rd_hi[i] = r.hi; f.rd_lo[i] = r.lo;
    }
    for (size_t q = 0; q < band.size(); ++q) { f.lu_hi[q] = band[q].hi; f.lu_lo[q] = band[q].lo; }
    return 0;
}

}  // namespace eph

extern "C" {

double eph_bspline_cheb_coef(int d, int k, int j) {
    if (d < 0 || d > kMaxDeg || k < 0 || k > d || j < 0 || j > d) return 0;
    return cheb().c[d][k][j];
}

int eph_bspline_fit(int d, int64_t n, int64_t mn, int channels, const double *samples, double *coefs) {
    if (channels < 1 || !samples || !coefs) return EPH_ERR_ARG;
    eph::BsplineFactor f;
    if (eph::bspline_factor(d, n, mn, f)) return EPH_ERR_ARG;
    const int64_t m = f.m, w = 2 * d + 1;
    std::vector<dd> y((size_t)m * channels);
    for (int c = 0; c < channels; ++c) {
        // right-hand side (rows scaled) and forward substitution with L
        for (int64_t i = 0; i < m; ++i) {
            dd yi = mk(0);
            for (int q = 0; q < f.cnt[i]; ++q)
                yi = add(yi, mul(mk(samples[(size_t)(f.jmin[i] + q) * channels + c]), mk(f.bval[(size_t)i * f.J + q])));
            yi = mul(yi, dd{f.rw_hi[i], f.rw_lo[i]});
            for (int64_t k = std::max<int64_t>(0, i - d); k < i; ++k) {
                const size_t q = (size_t)i * w + (k - i + d);
                yi = sub(yi, mul(dd{f.lu_hi[q], f.lu_lo[q]}, y[(size_t)k * channels + c]));
            }
            y[(size_t)i * channels + c] = yi;
        }
        // back substitution with U
        for (int64_t i = m - 1; i >= 0; --i) {
            dd yi = y[(size_t)i * channels + c];
            for (int64_t j = i + 1; j <= std::min<int64_t>(m - 1, i + d); ++j) {
                const size_t q = (size_t)i * w + (j - i + d);
                yi = sub(yi, mul(dd{f.lu_hi[q], f.lu_lo[q]}, y[(size_t)j * channels + c]));
            }
            y[(size_t)i * channels + c] = mul(yi, dd{f.rd_hi[i], f.rd_lo[i]});
        }
    }
    for (int64_t i = 0; i < m; ++i)
        for (int c = 0; c < channels; ++c) coefs[(size_t)i * channels + c] = y[(size_t)i * channels + c].hi + y[(size_t)i * channels + c].lo;
    return EPH_OK;
}

}  // extern "C"
