// eph_math.cuh - device arithmetic for the RK12 kernels: double-double numbers, 3-vectors and
// 3x3 matrices with the reference's semantics.
//
// Semantics follow the reference's math headers: double-double operations of
// src/math/dfloat_t.h:49-141 (TwoSum / quick TwoSum / TwoDiff / fma-based TwoProd), the vector and
// matrix conventions of src/math/vec_t.h (a matrix is its three axis columns x, y, z; `dot` is the
// reference's `%`, `cross` its vector `*`), the scaled normalisation of hypot_t (vec_t.h:30-92) and
// rotation_matrix (vec_t.h:540-559). Error-free transforms use explicit round-to-nearest intrinsics so
// the compiler cannot contract them; the physics terms around them may use FMA.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace eph {

struct dd { double hi, lo; };
struct v3 { double x, y, z; };
struct v3d { dd x, y, z; };
struct m3 { v3 x, y, z; };

// ----------------------------------------------------------------- double-double
__device__ __forceinline__ dd dd_make(double h) { return dd{h, 0.0}; }
__device__ __forceinline__ double dd_val(dd a) { return __dadd_rn(a.hi, a.lo); }

__device__ __forceinline__ void two_sum(double x, double y, double &r, double &e) {
    r = __dadd_rn(x, y);
    double t = __dsub_rn(r, x);
    e = __dadd_rn(__dsub_rn(x, __dsub_rn(r, t)), __dsub_rn(y, t));
}
__device__ __forceinline__ void two_sum_quick(double x, double y, double &r, double &e) {
    double s = __dadd_rn(x, y);
    e = __dsub_rn(y, __dsub_rn(s, x));
    r = s;
}
__device__ __forceinline__ dd dd_add(dd x, dd y) {
    dd r;
    two_sum(x.hi, y.hi, r.hi, r.lo);
    r.lo = __dadd_rn(r.lo, __dadd_rn(x.lo, y.lo));
    two_sum_quick(r.hi, r.lo, r.hi, r.lo);
    return r;
}
__device__ __forceinline__ dd dd_sub(dd x, dd y) {
    dd r;
    r.hi = __dsub_rn(x.hi, y.hi);
    double t = __dsub_rn(r.hi, x.hi);
    r.lo = __dsub_rn(__dsub_rn(x.hi, __dsub_rn(r.hi, t)), __dadd_rn(y.hi, t));
    r.lo = __dadd_rn(r.lo, __dsub_rn(x.lo, y.lo));
    two_sum_quick(r.hi, r.lo, r.hi, r.lo);
    return r;
}
__device__ __forceinline__ dd dd_mul(dd x, dd y) {
    dd r;
    r.hi = __dmul_rn(x.hi, y.hi);
    r.lo = __fma_rn(x.hi, y.hi, -r.hi);
    r.lo = __dadd_rn(r.lo, __dadd_rn(__dmul_rn(x.hi, y.lo), __dmul_rn(y.hi, x.lo)));
    two_sum_quick(r.hi, r.lo, r.hi, r.lo);
    return r;
}
__device__ __forceinline__ bool dd_finite(dd a) { return isfinite(a.hi) && isfinite(a.lo); }

// ----------------------------------------------------------------- vectors
__device__ __forceinline__ v3 mk(double x, double y, double z) { return v3{x, y, z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return v3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return v3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator-(v3 a) { return v3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ v3 operator*(double s, v3 a) { return v3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 &operator+=(v3 &a, v3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ v3 &operator-=(v3 &a, v3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return v3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ v3 vdiv(v3 a, double s) { double r = 1.0 / s; return v3{a.x * r, a.y * r, a.z * r}; }
__device__ __forceinline__ bool v3_finite(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

__device__ __forceinline__ v3 v3_of(v3d a) { return v3{dd_val(a.x), dd_val(a.y), dd_val(a.z)}; }
__device__ __forceinline__ v3d v3d_of(v3 a) { return v3d{dd_make(a.x), dd_make(a.y), dd_make(a.z)}; }
__device__ __forceinline__ v3d add(v3d a, v3d b) { return v3d{dd_add(a.x, b.x), dd_add(a.y, b.y), dd_add(a.z, b.z)}; }
__device__ __forceinline__ v3d scale(dd s, v3d a) { return v3d{dd_mul(s, a.x), dd_mul(s, a.y), dd_mul(s, a.z)}; }
// double-double difference of two positions rounded to double (`fast_mpvec r = mj.r - mi.r`)
__device__ __forceinline__ double dd_diff(double ahi, double alo, double bhi, double blo) {
    return dd_val(dd_sub(dd{ahi, alo}, dd{bhi, blo}));
}
// The same separation in three operations, for the O(N^2) pair sweeps. When ahi - bhi is exact (any two
// coordinates within a factor of two of each other, e.g. every close pair), the result equals dd_diff;
// otherwise it differs by at most about one unit in the last place of the separation.
__device__ __forceinline__ double sep_diff(double ahi, double alo, double bhi, double blo) {
    return __dadd_rn(__dsub_rn(ahi, bhi), __dsub_rn(alo, blo));
}

// ----------------------------------------------------------------- matrices (columns x, y, z)
__device__ __forceinline__ m3 mident(double a) { return m3{{a, 0, 0}, {0, a, 0}, {0, 0, a}}; }
__device__ __forceinline__ m3 outer(v3 a, v3 b) { return m3{b.x * a, b.y * a, b.z * a}; }
__device__ __forceinline__ m3 operator+(m3 a, m3 b) { return m3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ m3 operator-(m3 a, m3 b) { return m3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ m3 operator*(double s, m3 a) { return m3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ m3 add_diag(m3 a, double s) { a.x.x += s; a.y.y += s; a.z.z += s; return a; }
__device__ __forceinline__ v3 mul(m3 a, v3 b) { return (b.x * a.x + b.y * a.y) + b.z * a.z; }      // a % b
__device__ __forceinline__ v3 tmul(v3 a, m3 b) { return v3{dot(a, b.x), dot(a, b.y), dot(a, b.z)}; } // a % b
__device__ __forceinline__ m3 mul(m3 a, m3 b) { return m3{mul(a, b.x), mul(a, b.y), mul(a, b.z)}; }
__device__ __forceinline__ m3 transpose(m3 m) {
    return m3{{m.x.x, m.y.x, m.z.x}, {m.x.y, m.y.y, m.z.y}, {m.x.z, m.y.z, m.z.z}};
}
__device__ __forceinline__ v3 tolocal(m3 s, v3 a) { return tmul(a, s); }
__device__ __forceinline__ v3 toworld(m3 s, v3 a) { return mul(s, a); }
__device__ __forceinline__ m3 toworld(m3 s, m3 a) {   // s a s^T
    m3 sa = mul(s, a);
    return m3{(s.x.x * sa.x + s.y.x * sa.y) + s.z.x * sa.z,
              (s.x.y * sa.x + s.y.y * sa.y) + s.z.y * sa.z,
              (s.x.z * sa.x + s.y.z * sa.y) + s.z.z * sa.z};
}
__device__ __forceinline__ m3 tolocal(m3 s, m3 a) {   // s^T a s
    m3 sTa{tmul(a.x, s), tmul(a.y, s), tmul(a.z, s)};
    return mul(sTa, s);
}
__device__ __forceinline__ double det(m3 a) { return dot(cross(a.x, a.y), a.z); }
__device__ __forceinline__ m3 inverse(m3 m) {
    m3 a{{m.y.y * m.z.z - m.y.z * m.z.y, m.z.y * m.x.z - m.x.y * m.z.z, m.x.y * m.y.z - m.x.z * m.y.y},
         {m.y.z * m.z.x - m.y.x * m.z.z, m.z.z * m.x.x - m.x.z * m.z.x, m.x.z * m.y.x - m.x.x * m.y.z},
         {m.y.x * m.z.y - m.y.y * m.z.x, m.z.x * m.x.y - m.x.x * m.z.y, m.x.x * m.y.y - m.x.y * m.y.x}};
    double rdet = 1.0 / (a.x.z * m.z.x + a.y.z * m.z.y + a.z.z * m.z.z);
    return rdet * a;
}

// Scaled normalisation (hypot_t::normalize): returns the norm, leaves the unit vector in place,
// and maps the zero vector to the last argument's axis.
__device__ __forceinline__ double normalize3(double &a, double &b, double &c) {
    const double high = 0x1p960, mul_ = 0x1p768, div_ = 0x1p-768, low = 0x1p-960;
    double x = a, y = b, z = c;
    double r = x * x + y * y + z * z;
    double scale_back = 1.0;
    if (r < low) {
        x *= mul_; y *= mul_; z *= mul_;
        r = x * x + y * y + z * z;
        if (r == 0) { a = 0; b = 0; c = 1; return 0; }
        scale_back = div_;
    } else if (!(r < high)) {
        x *= div_; y *= div_; z *= div_;
        r = x * x + y * y + z * z;
        scale_back = mul_;
    }
    double s = sqrt(r), rs = 1.0 / s;
    a = x * rs; b = y * rs; c = z * rs;
    return scale_back * s;
}
__device__ __forceinline__ double normalize2(double &a, double &b) {
    const double high = 0x1p960, mul_ = 0x1p768, div_ = 0x1p-768, low = 0x1p-960;
    double x = a, y = b;
    double r = x * x + y * y;
    double scale_back = 1.0;
    if (r < low) {
        x *= mul_; y *= mul_;
        r = x * x + y * y;
        if (r == 0) { a = 0; b = 1; return 0; }
        scale_back = div_;
    } else if (!(r < high)) {
        x *= div_; y *= div_;
        r = x * x + y * y;
        scale_back = mul_;
    }
    double s = sqrt(r), rs = 1.0 / s;
    a = x * rs; b = y * rs;
    return scale_back * s;
}
__device__ __forceinline__ double normalize(v3 &v) { return normalize3(v.x, v.y, v.z); }

// (I + R) rotates a vector about w by |w| t (vec_t.h:540-559). sin(wt) and 2 sin^2(wt/2) come from one
// sincos of the half angle (sin wt = 2 sin(wt/2) cos(wt/2)), one range reduction instead of two.
__device__ __forceinline__ m3 rotation_matrix(v3 w, double t) {
    double x = w.x, y = w.y, z = w.z;
    double wt = normalize3(x, y, z) * t;
    double sh, ch;
    sincos(wt / 2, &sh, &ch);
    const double st = 2 * sh * ch, st222 = 2 * sh * sh;
    m3 dr{{x * x - 1, x * y, x * z}, {x * y, y * y - 1, y * z}, {x * z, y * z, z * z - 1}};
    dr = st222 * dr;
    dr.x.y += z * st;
    dr.y.x -= z * st;
    dr.x.z -= y * st;
    dr.z.x += y * st;
    dr.y.z += x * st;
    dr.z.y -= x * st;
    return dr;
}

// NaN-propagating running maximum (checked_maximize, src/math/basic_math.h:34-45)
__device__ __forceinline__ void checked_maximize(double &a, double b) { a = (a != a || b < a) ? a : b; }

}  // namespace eph
