/*
 * ref_bspline.cpp - flat C entry points over the reference's own B-spline fitter.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY. Compiled with the unmodified reference sources
 * (src/math/interp.cpp, src/math/interp.h) into oracle/_ref/libephref.so by oracle/Makefile, so the
 * tests can pin the product's fitter (eph_bspline_fit) and spline evaluation against
 *   bspline_fitter<double,N>(d, n, samples, mn)      src/math/interp.h:68-150
 *   bspline_fitter<double,N>::expand / operator()    src/math/interp.h:252-345
 *   bspline_basis_chebyshev_coef(d, k, j)            src/math/interp.cpp:110-114
 * for the channel counts the tests use (2 and 10).
 */
#include "math/interp.h"

#include <cstdint>
#include <cstring>

namespace {
template <size_t C>
int fit(int d, int64_t n, int64_t mn, const double *samples, double *coefs) {
    bspline_fitter<double, C> f(d, n, samples, mn);
    if (!f) return 1;
    std::memcpy(coefs, f.get_fitted_data(), sizeof(double) * C * (n + d));
    return 0;
}
template <size_t C>
int eval(const double *coefs, int d, int64_t n, double range, int expanded, int64_t m, const double *pos,
         double *value, double *deriv) {
    bspline_fitter<double, C> f(coefs, d, n, range);
    if (!f) return 1;
    if (expanded) f.expand();
    for (int64_t i = 0; i < m; ++i) f(pos[i], value + C * i, deriv + C * i);
    return 0;
}
}  // namespace

extern "C" {
double ref_bspline_cheb_coef(int d, int k, int j) { return bspline_basis_chebyshev_coef(d, k, j); }

int ref_bspline_fit(int channels, int d, int64_t n, int64_t mn, const double *samples, double *coefs) {
    switch (channels) {
        case 2: return fit<2>(d, n, mn, samples, coefs);
        case 10: return fit<10>(d, n, mn, samples, coefs);
        default: return 2;
    }
}

int ref_bspline_eval(int channels, const double *coefs, int d, int64_t n, double range, int expanded, int64_t m,
                     const double *pos, double *value, double *deriv) {
    switch (channels) {
        case 2: return eval<2>(coefs, d, n, range, expanded, m, pos, value, deriv);
        case 10: return eval<10>(coefs, d, n, range, expanded, m, pos, value, deriv);
        default: return 2;
    }
}
}  // extern "C"
