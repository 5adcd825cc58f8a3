// eph_ephemeris.cpp - reading the reference's compressed ephemeris records on the host, and
// resampling them into the B-spline tables of the device ephemeris (eph_bspline_fit, eph_serve_*).
//
// Record format (src/modules/ephemeris_compressor.h:50-72 and ephemeris_compressor.cpp:9-66): a 24-byte
// common header {float relative_error; int16 degree; uint16 ~format; int64 n; float smooth_range[2]},
// the format's end corrections fix[4][channels] (left value, left derivative, right value, right
// derivative), the format's extra constants, then (n + degree) B-spline coefficients of `channels` values
// over n uniform segments spanning the record's time range. The orbital formats:
//
//   1 STATE_VECTORS       channel: position vector                        (fix: 4 vectors)
//   2 KEPLERIAN_VECTORS   channel: position vector, then GM               (fix: 4 vectors)
//   3 KEPLERIAN_CIRCULAR  6 channels j[3], ex, ey, mean longitude; GM      (fix: 4 x 6)
//   4 KEPLERIAN_RAW       6 channels j[3], q, el, modified mean anomaly; GM (fix: 4 x 6)
//
// Evaluation at time t in [0, range] (ephemeris_compressor.cpp:1017-1053): the spline's value and time
// derivative at x = t n / range, a cubic blend of the end corrections inside the first / last
// smooth_range segments (ephemeris_compressor.cpp:719-735), then the format's conversion to position and
// velocity: the vector formats take value and derivative as they are; the element formats turn the
// interpolated elements into a state (state_parameters.cpp:69-86,137-168 for the element sets,
// keplerian.cpp:138-224 for the state), with velocities scaled by sqrt(GM).
//
// The rotational formats give a body's angular velocity and surface-frame axes x, z:
//
//   5 AXIAL_OFFSET        6 channels w[3], spin-axis offsets py, pz, rotation angle; local-axis angles
//   6 QUATERNION          4 channels (x, y, z, w) of the frame's quaternion
//   7 TIDAL_LOCK          the same, relative to the orbit frame; needs the orbital state at the same time
//
// (ephemeris_compressor.cpp:761-790, state_parameters.cpp:29-57).
//
// Own implementation: the B-spline pieces come from the degree recursion evaluated at the point (not the
// reference's Chebyshev tables), the element-to-state conversion is the textbook perifocal form with
// Kepler's equation solved by Newton steps (in a form that keeps near-parabolic orbits accurate), and the
// frames are built as rotations of explicit axis triples; agreement with the reference interpolator is to
// rounding, not bit for bit.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/eph_b200.h"

namespace {

constexpr int kMaxRecordDegree = 11;   // the compressor's largest (odd) degree
constexpr size_t kCommonHeader = 24;

struct Header {
    float relative_error;
    int16_t degree;
    uint16_t uformat;
    int64_t n;
    float smooth[2];
};
static_assert(sizeof(Header) == kCommonHeader, "the record's common header is 24 bytes");

// per-format layout: channels (doubles per coefficient), bytes of the header before the coefficients, the
// doubles that follow the end corrections (GM; or the local axis's polar and azimuthal angles)
struct Layout {
    int channels;
    size_t header_bytes;
    int extras;
};
bool layout_of(int format, Layout &L) {
    switch (format) {
        case 1: L = {3, kCommonHeader + 4 * 3 * 8, 0}; return true;
        case 2: L = {3, kCommonHeader + 4 * 3 * 8 + 8, 1}; return true;
        case 3:
        case 4: L = {6, kCommonHeader + 4 * 6 * 8 + 8, 1}; return true;
        case 5: L = {6, kCommonHeader + 4 * 6 * 8 + 16, 2}; return true;   // AXIAL_OFFSET
        case 6:
        case 7: L = {4, kCommonHeader + 4 * 4 * 8, 0}; return true;        // QUATERNION, TIDAL_LOCK
        default: return false;
    }
}

}  // namespace

struct eph_ephem {
    int format = 0, degree = 0, channels = 0;
    int64_t n = 0;
    double range = 0, relative_error = 0, gm = 0;
    double smooth[2] = {0, 0};
    double fix[4][6] = {};
    double axis_theta = 0, axis_phi = 0;   // AXIAL_OFFSET: the local spin axis's polar / azimuthal angle
    double orb_r[3] = {0, 0, 0}, orb_v[3] = {0, 0, 0};   // TIDAL_LOCK: the orbital state at the same time
    bool orb_set = false;
    std::vector<double> coef;   // [n + degree][channels]
};

namespace {

// Values and x-derivatives of the degree-d pieces at u in [0, 1]: piece k is the basis function of
// coefficient (segment + k), B[d, u - k] with B[0, x] = 1 on [0, 1) and
// B[d, x] = ((x + d) B[d-1, x+1] + (1 - x) B[d-1, x]) / d (src/math/interp.h:10-22); the derivative is
// B[d-1, x+1] - B[d-1, x].
void pieces(int d, double u, double *b, double *db) {
    double prev[kMaxRecordDegree + 1] = {1.0};
    for (int e = 1; e <= d; ++e) {
        double cur[kMaxRecordDegree + 1];
        for (int k = 0; k <= e; ++k) {
            const double left = k >= 1 ? prev[k - 1] : 0.0;   // B[e-1, u-k+1]: piece k-1 of degree e-1
            const double right = k <= e - 1 ? prev[k] : 0.0;  // B[e-1, u-k]: piece k of degree e-1
            if (e == d) db[k] = left - right;
            cur[k] = ((u - k + e) * left + (1 - u + k) * right) / e;
        }
        for (int k = 0; k <= e; ++k) prev[k] = cur[k];
    }
    if (d == 0) db[0] = 0;
    for (int k = 0; k <= d; ++k) b[k] = prev[k];
}

// Spline value and time derivative of every channel at t; false outside [0, range].
bool spline_at(const eph_ephem &E, double t, double *val, double *der) {
    const double x = t / E.range * (double)E.n;
    if (!(x >= 0 && x <= (double)E.n)) return false;
    int64_t seg = (int64_t)std::floor(x);
    if (seg == E.n) seg -= 1;
    const double u = x - (double)seg;
    double b[kMaxRecordDegree + 1], db[kMaxRecordDegree + 1];
    pieces(E.degree, u, b, db);
    const double dxdt = (double)E.n / E.range;
    const int C = E.channels;
    for (int c = 0; c < C; ++c) { val[c] = 0; der[c] = 0; }
    for (int k = 0; k <= E.degree; ++k) {
        const double *a = E.coef.data() + (size_t)(seg + k) * C;
        for (int c = 0; c < C; ++c) {
            val[c] += b[k] * a[c];
            der[c] += db[k] * a[c];
        }
    }
    for (int c = 0; c < C; ++c) der[c] *= dxdt;
    return true;
}

// The end corrections: inside the first (last) smooth[0] (smooth[1]) segments the spline is pulled toward
// the recorded end state by value + derivative * distance, weighted by the cubic (1 - s)^2 (1 + 2 s) of the
// fraction s of the blending range (ephemeris_compressor.cpp:719-735, 1017-1030).
void blend_ends(const eph_ephem &E, double t, double *val, double *der) {
    const double x = t / E.range * (double)E.n, nn = (double)E.n;
    const double vscale = nn / E.range;
    auto pull = [&](const double *fv, const double *fd, double dist, double width) {
        const double s = dist / width, w1 = 1 - s;
        const double w = w1 * w1 * (1 + 2 * s), dw = -6 * s * w1 / width;
        for (int c = 0; c < E.channels; ++c) {
            const double dr = fv[c] + fd[c] * dist;
            val[c] += w * dr;
            der[c] += (dw * dr + w * fd[c]) * vscale;
        }
    };
    if (std::floor(x) == 0 && x < E.smooth[0]) pull(E.fix[0], E.fix[1], x, E.smooth[0]);
    if (std::ceil(x) == nn && nn - x < E.smooth[1]) pull(E.fix[2], E.fix[3], nn - x, E.smooth[1]);
}

// ------------------------------------------------------------------ orbital elements to state
struct V3 {
    double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// Unit vector toward the ascending node of the plane normal to j: (-j.y, j.x, 0) normalised, or the x axis
// when j is along z (src/math/vec_t.h:226-230).
V3 ascending_node(V3 j) {
    const double h = std::hypot(j.x, j.y);
    if (h == 0) return {1, 0, 0};
    return {-j.y / h, j.x / h, 0};
}

// The reference's element set (src/math/keplerian.h:6-22), with time scaled by sqrt(GM):
//   j  angular momentum per mass / sqrt(GM)      q  e - 1
//   w  argument of the eccentricity vector from the ascending node, in the orbit plane
//   m  mean anomaly / |1 - e^2|^(3/2)            (dm/dt = 1 / |j|^3)
struct Elements {
    V3 j;
    double q, w, m;
};

// The interpolated channels of a record as elements (state_parameters.cpp:69-86 with 137-168): circular
// sets hold j, e (cos, sin) of the longitude of periapsis and the mean longitude; raw sets hold j, q, the
// longitude of periapsis and m. Longitudes count from the x axis: w = longitude - phi(ascending node).
Elements elements_from(const double *p, bool circular) {
    Elements k;
    k.j = {p[0], p[1], p[2]};
    const V3 an = ascending_node(k.j);
    const double node = std::atan2(an.y, an.x);
    if (circular) {
        const double e = std::sqrt(p[3] * p[3] + p[4] * p[4]);
        const double lp = std::atan2(p[4], p[3]);
        k.q = e - 1;
        const double s = -k.q * (k.q + 2);   // 1 - e^2
        k.m = (p[5] - lp) / (s * std::sqrt(s));
        k.w = lp - node;
    } else {
        k.q = p[3];
        k.m = p[5];
        k.w = p[4] - node;
    }
    return k;
}

// x - sin x and sinh x - x, by their series below |x| = 1 (where the difference cancels), else directly.
double x_minus_sin(double x) {
    if (std::fabs(x) >= 1) return x - std::sin(x);
    const double x2 = x * x;
    double term = x * x2 / 6, sum = 0;
    for (int k = 2; k < 40 && term != 0; ++k) {   // x^3/3! - x^5/5! + ...
        sum += term;
        term *= -x2 / ((2 * k) * (2 * k + 1));
        if (std::fabs(term) < 1e-18 * std::fabs(sum)) break;
    }
    return sum;
}
double sinh_minus_x(double x) {
    if (std::fabs(x) >= 1) return std::sinh(x) - x;
    const double x2 = x * x;
    double term = x * x2 / 6, sum = 0;
    for (int k = 2; k < 40 && term != 0; ++k) {   // x^3/3! + x^5/5! + ...
        sum += term;
        term *= x2 / ((2 * k) * (2 * k + 1));
        if (std::fabs(term) < 1e-18 * std::fabs(sum)) break;
    }
    return sum;
}

// Mean anomaly reduced into [-pi, pi].
double wrap_pi(double a) {
    constexpr double two_pi = 6.283185307179586476925286766559;
    if (a > -M_PI && a <= M_PI) return a;
    return a - two_pi * std::nearbyint(a / two_pi);
}

// Position and velocity / sqrt(GM) of elements k at their epoch (keplerian.cpp:138-224 for the quantity;
// the conics in perifocal coordinates scaled by the semi-latus rectum p = |j|^2: x = X / p, y = Y / p,
// velocity (-y, e - Q x) |j| / r with Q = e^2 - 1).
void elements_to_state(const Elements &k, V3 &r, V3 &v) {
    const double jj = dot(k.j, k.j), jn = std::sqrt(jj);
    const double e = k.q + 1;
    const double Q = k.q * (k.q + 2);   // e^2 - 1 without cancellation
    const double aQ = std::fabs(Q), sQ = std::sqrt(aQ);
    double x, y, vyn;   // perifocal position / p; vyn = e - Q x (cos E, cosh H or 1) without cancellation
    if (Q < 0) {
        // ellipse: E - e sin E = M; x = (cos E - e) / (1 - e^2), y = sin E / sqrt(1 - e^2), with
        // cos E - e = -2 sin^2(E/2) - q kept free of cancellation near periapsis of a near-parabolic orbit
        // written as (1 - e) E + e (E - sin E) = M, with 1 - e = -q and E - sin E from its series at small E,
        // so that near-parabolic orbits (M and 1 - e both small) keep full relative precision
        const double M = wrap_pi(k.m * aQ * sQ);
        double E = M + 0.85 * e * (M >= 0 ? 1 : -1);   // Danby's start: Newton converges for every e < 1
        for (int it = 0; it < 100; ++it) {
            const double sh = std::sin(0.5 * E);
            const double f = -k.q * E + e * x_minus_sin(E) - M, fp = -k.q + 2 * e * sh * sh;
            const double dE = f / fp;
            E -= dE;
            if (std::fabs(dE) <= 1e-16 * std::fabs(E) || f == 0) break;
        }
        const double sh = std::sin(0.5 * E);
        x = (-2 * sh * sh - k.q) / aQ;
        y = std::sin(E) / sQ;
        vyn = std::cos(E);
    } else if (Q > 0) {
        // hyperbola: e sinh H - H = M; x = (e - cosh H) / (e^2 - 1), y = sinh H / sqrt(e^2 - 1)
        // written as (e - 1) H + e (sinh H - H) = M, the same way as the ellipse
        const double M = k.m * aQ * sQ;
        // start: the cubic root cbrt(6 |M| / e) lies beyond the solution (sinh H - H >= H^3 / 6); for large |M|
        // asinh(|M| / e) + 1 is closer. f is odd and convex for H > 0, so Newton converges from either side.
        const double aM = std::fabs(M);
        double H = std::fmin(std::cbrt(6 * aM / e), std::asinh(aM / e) + 1) * (M >= 0 ? 1 : -1);
        for (int it = 0; it < 200; ++it) {
            const double sh = std::sinh(0.5 * H);
            const double f = k.q * H + e * sinh_minus_x(H) - M, fp = k.q + 2 * e * sh * sh;
            const double dH = f / fp;
            H -= dH;
            if (std::fabs(dH) <= 1e-16 * std::fabs(H) || f == 0) break;
        }
        const double sh = std::sinh(0.5 * H);
        x = (k.q - 2 * sh * sh) / aQ;   // e - cosh H = q - 2 sinh^2(H/2)
        y = std::sinh(H) / sQ;
        vyn = std::cosh(H);
    } else {
        // parabola: Barker's equation for D = tan(nu/2): D / 2 + D^3 / 6 = m (the limit of the modified
        // mean anomaly); x = (1 - D^2) / 2, y = D
        const double m3 = 3 * k.m, s = std::cbrt(m3 + std::sqrt(1 + m3 * m3));
        const double D = s - 1 / s;
        x = (1 - D * D) / 2;
        y = D;
        vyn = 1;
    }
    const double rn = jj * std::sqrt(x * x + y * y);   // |r|
    const double vv = jn / rn;
    const double vx = -y * vv, vy = vyn * vv;
    const V3 jx = ascending_node(k.j), jy = (1 / jn) * cross(k.j, jx);
    const double cw = std::cos(k.w), sw = std::sin(k.w);
    const double X = jj * x, Y = jj * y;
    r = (X * cw - Y * sw) * jx + (X * sw + Y * cw) * jy;
    v = (vx * cw - vy * sw) * jx + (vx * sw + vy * cw) * jy;
}

// ------------------------------------------------------------------ rotational records to frame and spin
// A body's rotation state is its angular velocity w and two axes of its surface frame, x and z (y = z x x).
V3 unit_or_z(V3 a) {   // a / |a|, or the z axis for a zero vector (src/math/vec_t.h:166-175)
    const double n = std::sqrt(dot(a, a));
    if (n == 0) return {0, 0, 1};
    return (1 / n) * a;
}
// the world image of local coordinates a in the frame (ex, ey, ez)
V3 to_world(V3 ex, V3 ey, V3 ez, V3 a) { return a.x * ex + a.y * ey + a.z * ez; }

// AXIAL_OFFSET channels {w[3], py, pz, angle} (ephemeris_compressor.cpp:420-466, state_parameters.cpp:29-57):
// the spin axis's polar angle theta (cos theta = pz) and azimuth phi (sin theta sin phi = py) in the frame
// built on w (x toward w's ascending node, z along w), the rotation angle about w; the surface frame is
// that frame turned by -theta about its y axis and -phi about its z axis, then by the angle about w, then
// taken to the record's local axis (polar angle, azimuth stored in the header).
void axial_to_rotation(const eph_ephem &E, const double *a, V3 &w, V3 &x, V3 &z) {
    w = {a[0], a[1], a[2]};
    const V3 wz = unit_or_z(w);
    const double th = std::acos(a[4]), ph = std::asin(a[3] / std::sqrt(1 - a[4] * a[4]));
    V3 X = ascending_node(w), Z = wz, Y = cross(Z, X);
    {   // -theta about the frame's y axis
        const double c = std::cos(th), s = std::sin(th);
        const V3 nz = c * Z + (-s) * X;
        X = c * X + s * Z;
        Z = nz;
    }
    {   // -phi about the frame's z axis
        const double c = std::cos(ph), s = std::sin(ph);
        const V3 nx = c * X + (-s) * Y;
        Y = c * Y + s * X;
        X = nx;
    }
    const double c = std::cos(a[5]), s = std::sin(a[5]);
    auto spin = [&](V3 v) {   // v turned by the angle about wz: v + (c - 1) v_perp + s wz x v
        const V3 perp = v + (-dot(wz, v)) * wz;
        return v + (c - 1) * perp + s * cross(wz, v);
    };
    X = spin(X);
    Y = spin(Y);
    Z = spin(Z);
    // local axis frame (u, v, u x v) from the header's angles; the surface axes are the rows of its
    // transpose taken through (X, Y, Z)
    const double t0 = E.axis_theta, p0 = E.axis_phi, t1 = t0 + M_PI / 2;
    const V3 u = {std::sin(t0) * std::cos(p0), std::sin(t0) * std::sin(p0), std::cos(t0)};
    const V3 v = {std::sin(t1) * std::cos(p0), std::sin(t1) * std::sin(p0), std::cos(t1)};
    const V3 n = cross(u, v);
    x = to_world(X, Y, Z, {u.x, v.x, n.x});
    z = to_world(X, Y, Z, {u.z, v.z, n.z});
}

// Unit quaternion (x, y, z, w) to the frame's x and z axes (src/math/vec_t.h:612-623).
void quat_axes(const double *q, V3 &x, V3 &z) {
    double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    double a = q[0], b = q[1], c = q[2], d = q[3];
    if (n == 0) { a = b = c = 0; d = 1; n = 1; }
    a /= n; b /= n; c /= n; d /= n;
    x = {d * d + a * a - (b * b + c * c), 2 * (a * b + d * c), 2 * (c * a - d * b)};
    z = {2 * (c * a + d * b), 2 * (b * c - d * a), d * d + c * c - (a * a + b * b)};
}

// Angular velocity of a rotating quaternion q with derivative qd: the vector part of 2 qd q^-1.
V3 quat_spin(const double *q, const double *qd) {
    const double nn = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    // qd (x) conj(q), Hamilton product, vector part
    const double px = -qd[3] * q[0] + qd[0] * q[3] - qd[1] * q[2] + qd[2] * q[1];
    const double py = -qd[3] * q[1] + qd[1] * q[3] - qd[2] * q[0] + qd[0] * q[2];
    const double pz = -qd[3] * q[2] + qd[2] * q[3] - qd[0] * q[1] + qd[1] * q[0];
    return (2 / nn) * V3{px, py, pz};
}

// QUATERNION / TIDAL_LOCK channels (ephemeris_compressor.cpp:769-790): the frame of the quaternion and the
// spin 2 q' q^-1; a tidally locked record holds them relative to the orbit frame (x toward the orbital
// centre, z along r x v), which the orbital state at the same time takes back to the world, adding the
// orbit's own angular velocity r x v / r^2.
void quat_to_rotation(const eph_ephem &E, const double *q, const double *qd, V3 &w, V3 &x, V3 &z) {
    quat_axes(q, x, z);
    w = quat_spin(q, qd);
    if (E.format != 7) return;
    const V3 r = {E.orb_r[0], E.orb_r[1], E.orb_r[2]}, v = {E.orb_v[0], E.orb_v[1], E.orb_v[2]};
    const double r2 = dot(r, r);
    const V3 wo = (1 / r2) * cross(r, v);
    const V3 jx = (-1 / std::sqrt(r2)) * r, jz = unit_or_z(wo), jy = cross(jz, jx);
    x = to_world(jx, jy, jz, x);
    z = to_world(jx, jy, jz, z);
    w = to_world(jx, jy, jz, w) + wo;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int eph_ephem_open(const void *record, int64_t size, double range, eph_ephem **out) {
    if (!out) return EPH_ERR_ARG;
    *out = nullptr;
    if (!record || size < (int64_t)kCommonHeader || !(range != 0 && range * 0 == 0)) return EPH_ERR_ARG;
    const uint8_t *p = static_cast<const uint8_t *>(record);
    Header h;
    std::memcpy(&h, p, sizeof(h));
    const double rel = h.relative_error;
    if (!(rel >= 0 && rel < 1)) return EPH_ERR_LOAD;   // an uncompressed or failed record
    const int format = (uint16_t)~h.uformat;
    Layout L;
    if (!layout_of(format, L)) return EPH_ERR_LOAD;
    // (n above the record's size cannot fit its coefficients; checked first so that n + degree cannot overflow)
    if (h.degree < 1 || h.degree > kMaxRecordDegree || h.n < 1 || h.n > size) return EPH_ERR_LOAD;
    const int64_t per = (int64_t)L.channels * 8;
    if (size < (int64_t)L.header_bytes || (size - (int64_t)L.header_bytes) % per != 0 ||
        (size - (int64_t)L.header_bytes) / per != h.n + h.degree)
        return EPH_ERR_LOAD;
    eph_ephem *E = new (std::nothrow) eph_ephem;
    if (!E) return EPH_ERR_LIMIT;
    E->format = format;
    E->degree = h.degree;
    E->channels = L.channels;
    E->n = h.n;
    E->range = range;
    E->relative_error = rel;
    E->smooth[0] = h.smooth[0];
    E->smooth[1] = h.smooth[1];
    const uint8_t *q = p + kCommonHeader;
    for (int a = 0; a < 4; ++a, q += per) std::memcpy(E->fix[a], q, (size_t)per);
    if (format == 5) {
        std::memcpy(&E->axis_theta, q, 8);
        std::memcpy(&E->axis_phi, q + 8, 8);
    } else if (L.extras == 1) {
        std::memcpy(&E->gm, q, 8);
    }
    try {
        E->coef.resize((size_t)(h.n + h.degree) * L.channels);
    } catch (...) {
        delete E;
        return EPH_ERR_LIMIT;
    }
    std::memcpy(E->coef.data(), p + L.header_bytes, E->coef.size() * 8);
    *out = E;
    return EPH_OK;
}

int eph_ephem_close(eph_ephem *E) {
    delete E;
    return EPH_OK;
}

int eph_ephem_info(const eph_ephem *E, int *format, int *degree, int64_t *segments, double *relative_error,
                   double *gm) {
    if (!E) return EPH_ERR_ARG;
    if (format) *format = E->format;
    if (degree) *degree = E->degree;
    if (segments) *segments = E->n;
    if (relative_error) *relative_error = E->relative_error;
    if (gm) *gm = E->format == 1 ? 0.0 : E->gm;
    return EPH_OK;
}

int eph_ephem_set_orbital_state(eph_ephem *E, const double *r, const double *v) {
    if (!E || !r || !v) return EPH_ERR_ARG;
    for (int c = 0; c < 3; ++c) { E->orb_r[c] = r[c]; E->orb_v[c] = v[c]; }
    E->orb_set = true;
    return EPH_OK;
}

int eph_ephem_rotation(const eph_ephem *E, double t, double *w, double *x, double *z) {
    if (!E || !w || !x || !z) return EPH_ERR_ARG;
    if (E->format < 5) return EPH_ERR_UNSUPPORTED;
    if (E->format == 7 && !E->orb_set) return EPH_ERR_STATE;   // no orbital state to take the frame back
    double val[6], der[6];
    if (!spline_at(*E, t, val, der)) {
        for (int c = 0; c < 3; ++c) w[c] = x[c] = z[c] = NAN;
        return EPH_ERR_ARG;
    }
    blend_ends(*E, t, val, der);
    V3 ww, xx, zz;
    if (E->format == 5) axial_to_rotation(*E, val, ww, xx, zz);
    else quat_to_rotation(*E, val, der, ww, xx, zz);
    w[0] = ww.x; w[1] = ww.y; w[2] = ww.z;
    x[0] = xx.x; x[1] = xx.y; x[2] = xx.z;
    z[0] = zz.x; z[1] = zz.y; z[2] = zz.z;
    return EPH_OK;
}

int eph_ephem_state(const eph_ephem *E, double t, double *r, double *v, double *gm) {
    if (!E || !r || !v) return EPH_ERR_ARG;
    if (E->format > 4) return EPH_ERR_UNSUPPORTED;   // a rotational record: eph_ephem_rotation
    double val[6], der[6];
    if (!spline_at(*E, t, val, der)) {
        for (int c = 0; c < 3; ++c) r[c] = v[c] = NAN;
        return EPH_ERR_ARG;
    }
    blend_ends(*E, t, val, der);
    if (E->format <= 2) {
        for (int c = 0; c < 3; ++c) { r[c] = val[c]; v[c] = der[c]; }
    } else {
        V3 rr, vv;
        elements_to_state(elements_from(val, E->format == 3), rr, vv);
        const double sg = std::sqrt(E->gm);
        r[0] = rr.x; r[1] = rr.y; r[2] = rr.z;
        v[0] = sg * vv.x; v[1] = sg * vv.y; v[2] = sg * vv.z;
    }
    if (gm) *gm = E->format == 1 ? 0.0 : E->gm;
    return EPH_OK;
}

int eph_ephem_states(const eph_ephem *E, int64_t count, const double *t, double *out) {
    if (!E || count < 0 || (count > 0 && (!t || !out))) return EPH_ERR_ARG;
    if (E->format > 4) return EPH_ERR_UNSUPPORTED;
    int status = EPH_OK;
    for (int64_t k = 0; k < count; ++k) {
        double *o = out + 6 * k;
        const int rc = eph_ephem_state(E, t[k], o, o + 3, nullptr);
        if (rc && !status) status = rc;   // the state is NaN there; the rest are still evaluated
    }
    return status;
}

int eph_ephem_to_bspline(const eph_ephem *E, int d, int64_t n, int64_t mn, double *coefs) {
    if (!E || !coefs || mn < 1 || n < 1 || mn + 1 < n + d) return EPH_ERR_ARG;
    if (E->format > 4) return EPH_ERR_UNSUPPORTED;
    std::vector<double> samples;
    try {
        samples.resize((size_t)(mn + 1) * 3);
    } catch (...) {
        return EPH_ERR_LIMIT;
    }
    for (int64_t k = 0; k <= mn; ++k) {
        const double t = k == mn ? E->range : E->range * ((double)k / (double)mn);
        double v[3];
        const int rc = eph_ephem_state(E, t, samples.data() + 3 * k, v, nullptr);
        if (rc) return rc;
    }
    return eph_bspline_fit(d, n, mn, 3, samples.data(), coefs);
}

}  // extern "C"
