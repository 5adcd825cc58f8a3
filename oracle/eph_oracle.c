/*
 * eph_oracle.c - CPU restatement of the reference's RK12 step. TEST INFRASTRUCTURE ONLY:
 * the parity tests, smoke() and bench.py's cpu_baseline leg call it as the checker; the product
 * library never links or loads it.
 *
 * Every function follows the cited reference code operation by operation (same association order,
 * compiled with -ffp-contract=off to honour `#pragma fp_contract (off)` in src/definitions.h:2), so
 * its output is bit-identical to the reference's serial CPU path. Operator spellings of the
 * reference: `%` is the dot product / matrix product, `*` between vectors is the cross product
 * (src/math/vec_t.h:248-253,476-484).
 */
#include "eph_oracle.h"
#include "eph_planes.h"
#include "eph_rk12_table.h"
#include "eph_ring_table.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- constants (basic_math.h:9-31) */
static const double C_LIGHT = 299792458.0;
#define C2 (C_LIGHT * C_LIGHT)
static const double PI = 3.1415926535897932;

/* ---------------------------------------------------------------- double-double (dfloat_t.h:49-141) */
typedef struct { double hi, lo; } dd;

static void two_sum(double x, double y, double *r, double *e) {      /* dfloat_t.h:124-128 */
    *r = x + y;
    double t = *r - x;
    *e = (x - (*r - t)) + (y - t);
}
static void two_sum_quick(double x, double y, double *r, double *e) { /* dfloat_t.h:129-132 */
    double s = x + y;
    *e = y - (s - x);
    *r = s;
}
static void two_diff(double x, double y, double *r, double *e) {     /* dfloat_t.h:133-137 */
    *r = x - y;
    double t = *r - x;
    *e = (x - (*r - t)) - (y + t);
}
static dd dd_make(double h) { dd r = {h, 0.0}; return r; }
static double dd_val(dd a) { return a.hi + a.lo; }                   /* dfloat_t.h:19 */
static dd dd_add(dd x, dd y) {                                         /* dfloat_t.h:49-55 */
    dd r;
    two_sum(x.hi, y.hi, &r.hi, &r.lo);
    r.lo = r.lo + (x.lo + y.lo);
    two_sum_quick(r.hi, r.lo, &r.hi, &r.lo);
    return r;
}
static dd dd_sub(dd x, dd y) {                                         /* dfloat_t.h:57-63 */
    dd r;
    two_diff(x.hi, y.hi, &r.hi, &r.lo);
    r.lo = r.lo + (x.lo - y.lo);
    two_sum_quick(r.hi, r.lo, &r.hi, &r.lo);
    return r;
}
static dd dd_mul(dd x, dd y) {                                         /* dfloat_t.h:65-71 */
    dd r;
    r.hi = x.hi * y.hi;
    r.lo = fma(x.hi, y.hi, -r.hi);
    r.lo = r.lo + (x.hi * y.lo + y.hi * x.lo);
    two_sum_quick(r.hi, r.lo, &r.hi, &r.lo);
    return r;
}
static int dd_is_finite(dd a) { return !(0 * a.hi != 0 || 0 * a.lo != 0); } /* dfloat_t.h:35 */

/* ---------------------------------------------------------------- vectors / matrices (vec_t.h) */
typedef struct { double x, y, z; } v3;
typedef struct { dd x, y, z; } v3d;
typedef struct { v3 x, y, z; } m3;     /* columns (axes) x, y, z: vec_t.h:270-272 */
typedef struct { v3d x, y, z; } m3d;

static v3 v3_make(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 v3_add(v3 a, v3 b) { return v3_make(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 v3_sub(v3 a, v3 b) { return v3_make(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 v3_neg(v3 a) { return v3_make(-a.x, -a.y, -a.z); }
static v3 v3_cross(v3 a, v3 b) {                                        /* vec_t.h:248-250 */
    return v3_make(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double v3_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; } /* vec_t.h:251-253 */
static v3 v3_scale(double a, v3 b) { return v3_make(a * b.x, a * b.y, a * b.z); } /* vec_t.h:255-260 */
static v3 v3_div(v3 b, double a) { double reca = 1 / a; return v3_make(b.x * reca, b.y * reca, b.z * reca); }
static double v3_normsqr(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }

static v3 v3_from_dd(v3d a) { return v3_make(dd_val(a.x), dd_val(a.y), dd_val(a.z)); }
static v3d v3d_from(v3 a) { v3d r = {dd_make(a.x), dd_make(a.y), dd_make(a.z)}; return r; }
static v3d v3d_add(v3d a, v3d b) { v3d r = {dd_add(a.x, b.x), dd_add(a.y, b.y), dd_add(a.z, b.z)}; return r; }
static v3d v3d_sub(v3d a, v3d b) { v3d r = {dd_sub(a.x, b.x), dd_sub(a.y, b.y), dd_sub(a.z, b.z)}; return r; }
static v3d v3d_scale(dd a, v3d b) { v3d r = {dd_mul(a, b.x), dd_mul(a, b.y), dd_mul(a, b.z)}; return r; }
static int v3d_is_finite(v3d a) { return dd_is_finite(a.z) && dd_is_finite(a.y) && dd_is_finite(a.x); }
/* `fast_mpvec r = mj.r - mi.r`: double-double difference rounded to double */
static v3 v3d_diff(v3d a, v3d b) { return v3_from_dd(v3d_sub(a, b)); }

static m3 m3_make(v3 x, v3 y, v3 z) { m3 r = {x, y, z}; return r; }
static m3 m3_ident(double a) {                                            /* vec_t.h:275 */
    return m3_make(v3_make(a, 0, 0), v3_make(0, a, 0), v3_make(0, 0, a));
}
static m3 m3_outer(v3 a, v3 b) {                                          /* vec_t.h:277 */
    return m3_make(v3_scale(b.x, a), v3_scale(b.y, a), v3_scale(b.z, a));
}
static m3 m3_add(m3 a, m3 b) { return m3_make(v3_add(a.x, b.x), v3_add(a.y, b.y), v3_add(a.z, b.z)); }
static m3 m3_sub(m3 a, m3 b) { return m3_make(v3_sub(a.x, b.x), v3_sub(a.y, b.y), v3_sub(a.z, b.z)); }
static m3 m3_scale(double a, m3 b) { return m3_make(v3_scale(a, b.x), v3_scale(a, b.y), v3_scale(a, b.z)); }
static m3 m3_add_diag(m3 b, double a) { b.x.x += a; b.y.y += a; b.z.z += a; return b; }  /* vec_t.h:388-393 */
static m3 m3_sub_diag(m3 b, double a) { b.x.x -= a; b.y.y -= a; b.z.z -= a; return b; }  /* vec_t.h:394-399 */
static m3 m3_neg(m3 a) { return m3_make(v3_neg(a.x), v3_neg(a.y), v3_neg(a.z)); }
static v3 m3_mulv(m3 a, v3 b) {                                           /* vec_t.h:476-478 */
    return v3_add(v3_add(v3_scale(b.x, a.x), v3_scale(b.y, a.y)), v3_scale(b.z, a.z));
}
static v3 v3_mulm(v3 a, m3 b) { return v3_make(v3_dot(a, b.x), v3_dot(a, b.y), v3_dot(a, b.z)); } /* :479-481 */
static m3 m3_mul(m3 a, m3 b) { return m3_make(m3_mulv(a, b.x), m3_mulv(a, b.y), m3_mulv(a, b.z)); } /* :482-484 */
static v3 m3_tolocal(m3 s, v3 a) { return v3_mulm(a, s); }                 /* vec_t.h:326 */
static v3 m3_toworld(m3 s, v3 a) { return m3_mulv(s, a); }                 /* vec_t.h:328 */
static m3 m3_toworld_m(m3 s, m3 a) {                                       /* vec_t.h:335-338 */
    m3 sa = m3_mul(s, a);
    return m3_make(
        v3_add(v3_add(v3_scale(s.x.x, sa.x), v3_scale(s.y.x, sa.y)), v3_scale(s.z.x, sa.z)),
        v3_add(v3_add(v3_scale(s.x.y, sa.x), v3_scale(s.y.y, sa.y)), v3_scale(s.z.y, sa.z)),
        v3_add(v3_add(v3_scale(s.x.z, sa.x), v3_scale(s.y.z, sa.y)), v3_scale(s.z.z, sa.z)));
}
static double m3_det(m3 a) { return v3_dot(v3_cross(a.x, a.y), a.z); }  /* vec_t.h:432-434 */
static m3 m3_adjoint(m3 m) {                                                /* vec_t.h:443-449 */
    return m3_make(
        v3_make(m.y.y * m.z.z - m.y.z * m.z.y, m.z.y * m.x.z - m.x.y * m.z.z, m.x.y * m.y.z - m.x.z * m.y.y),
        v3_make(m.y.z * m.z.x - m.y.x * m.z.z, m.z.z * m.x.x - m.x.z * m.z.x, m.x.z * m.y.x - m.x.x * m.y.z),
        v3_make(m.y.x * m.z.y - m.y.y * m.z.x, m.z.x * m.x.y - m.x.x * m.z.y, m.x.x * m.y.y - m.x.y * m.y.x));
}
static m3 m3_inverse(m3 m) {                                                /* vec_t.h:450-454 */
    m3 madj = m3_adjoint(m);
    double rdet = 1 / (madj.x.z * m.z.x + madj.y.z * m.z.y + madj.z.z * m.z.z);
    return m3_scale(rdet, madj);
}
static m3 m3_transpose(m3 m) {
    return m3_make(v3_make(m.x.x, m.y.x, m.z.x), v3_make(m.x.y, m.y.y, m.z.y), v3_make(m.x.z, m.y.z, m.z.z));
}
static m3 m3_from_dd(m3d a) { return m3_make(v3_from_dd(a.x), v3_from_dd(a.y), v3_from_dd(a.z)); }
static m3d m3d_add_fast(m3d a, m3 b) {  /* mpmat += fast_mpmat (widened to double-double) */
    m3d r = {v3d_add(a.x, v3d_from(b.x)), v3d_add(a.y, v3d_from(b.y)), v3d_add(a.z, v3d_from(b.z))};
    return r;
}

/* hypot_t<double>::normalize for 3 and 2 arguments (vec_t.h:30-92): scaled to avoid
 * over/underflow; a zero vector becomes the last axis. */
static const double HYP_HIGH = 0x1p960, HYP_MUL = 0x1p768;
static double hyp_normalize3(double *a, double *b, double *c) {
    const double high = HYP_HIGH, mul = HYP_MUL, div = 1 / HYP_MUL, low = 1 / HYP_HIGH;
    double x = *a, y = *b, z = *c;
    double r = x * x + y * y + z * z;
    if (r < low) {
        x *= mul; y *= mul; z *= mul;
        r = x * x + y * y + z * z;
        if (r == 0) {
            *a = 0; *b = 0; *c = 1;
            return r;
        }
        double s = sqrt(r), rs = 1 / s;
        *a = x * rs; *b = y * rs; *c = z * rs;
        return div * s;
    }
    if (!(r < high)) {
        x *= div; y *= div; z *= div;
        r = x * x + y * y + z * z;
        double s = sqrt(r), rs = 1 / s;
        *a = x * rs; *b = y * rs; *c = z * rs;
        return mul * s;
    }
    double s = sqrt(r), rs = 1 / s;
    *a = x * rs; *b = y * rs; *c = z * rs;
    return s;
}
static double hyp_normalize2(double *a, double *b) {
    const double high = HYP_HIGH, mul = HYP_MUL, div = 1 / HYP_MUL, low = 1 / HYP_HIGH;
    double x = *a, y = *b;
    double r = x * x + y * y;
    if (r < low) {
        x *= mul; y *= mul;
        r = x * x + y * y;
        if (r == 0) {
            *a = 0; *b = 1;
            return r;
        }
        double s = sqrt(r), rs = 1 / s;
        *a = x * rs; *b = y * rs;
        return div * s;
    }
    if (!(r < high)) {
        x *= div; y *= div;
        r = x * x + y * y;
        double s = sqrt(r), rs = 1 / s;
        *a = x * rs; *b = y * rs;
        return mul * s;
    }
    double s = sqrt(r), rs = 1 / s;
    *a = x * rs; *b = y * rs;
    return s;
}
static double v3_normalize(v3 *v) { return hyp_normalize3(&v->x, &v->y, &v->z); }  /* vec_t.h:168-170 */
static v3 v3_unit(v3 v) { v3_normalize(&v); return v; }
static v3 v3_asc_node(v3 v) {                                             /* vec_t.h:226-230 */
    v3 p = v3_make(-v.y, v.x, 0);
    hyp_normalize2(&p.y, &p.x);
    return p;
}
static m3 v3_rotation_matrix(v3 w, double t) {                           /* vec_t.h:540-559 */
    double x = w.x, y = w.y, z = w.z;
    double wt = hyp_normalize3(&x, &y, &z) * t;
    double st = sin(wt), st222 = sin(wt / 2);
    st222 *= 2 * st222;
    m3 dr = m3_make(v3_make(x * x - 1, x * y, x * z), v3_make(x * y, y * y - 1, y * z), v3_make(x * z, y * z, z * z - 1));
    dr = m3_scale(st222, dr);
    dr.x.y += z * st;
    dr.y.x -= z * st;
    dr.x.z -= y * st;
    dr.z.x += y * st;
    dr.y.z += x * st;
    dr.z.y -= x * st;
    return dr;
}

/* checked_maximize (basic_math.h:34-45): NaN-propagating running maximum */
static void checked_maximize(double *a, double b) { *a = (*a != *a || b < *a) ? *a : b; }
static double dmax(double a, double b) { return (a < b) ? b : a; }  /* std::max */

/* ---------------------------------------------------------------- body record (mass.h:67-143) */
typedef struct body {
    v3d r, v, GL;
    m3d s;
    v3 w;
    double GM, exJ2;
    double GM0, dGM, dJ2, R, inertia, k2, k2r, tide_delay, tide_delay_factor, lum, recpt, A, R2, sR2, rR2G_4c;
    m3 C_static;
    int gp, ring;
    double phi, beta2;
    v3 naccel, daccel, dtorque, gaccel, beta;
    m3 GI, C_potential;
    v3 Egrad;
    double min_distance, max_influence;
} body;

typedef struct stage_state {   /* mass_state (mass.h:168-195) */
    v3d r, v, GL;
    m3d s;
    v3 w, naccel, dtorque;
} stage_state;

#define PL(p, i) planes[(int64_t)(p) * n + (i)]
static v3 get3(const double *planes, int64_t n, int p, int64_t i) { return v3_make(PL(p, i), PL(p + 1, i), PL(p + 2, i)); }
static v3d get3d(const double *planes, int64_t n, int ph, int pl, int64_t i) {
    v3d r = {{PL(ph, i), PL(pl, i)}, {PL(ph + 1, i), PL(pl + 1, i)}, {PL(ph + 2, i), PL(pl + 2, i)}};
    return r;
}
static m3 get9(const double *planes, int64_t n, int p, int64_t i) {
    return m3_make(get3(planes, n, p, i), get3(planes, n, p + 3, i), get3(planes, n, p + 6, i));
}
static m3d get9d(const double *planes, int64_t n, int ph, int pl, int64_t i) {
    m3d r = {get3d(planes, n, ph, pl, i), get3d(planes, n, ph + 3, pl + 3, i), get3d(planes, n, ph + 6, pl + 6, i)};
    return r;
}
static void put3(double *planes, int64_t n, int p, int64_t i, v3 v) { PL(p, i) = v.x; PL(p + 1, i) = v.y; PL(p + 2, i) = v.z; }
static void put3d(double *planes, int64_t n, int ph, int pl, int64_t i, v3d v) {
    PL(ph, i) = v.x.hi; PL(ph + 1, i) = v.y.hi; PL(ph + 2, i) = v.z.hi;
    PL(pl, i) = v.x.lo; PL(pl + 1, i) = v.y.lo; PL(pl + 2, i) = v.z.lo;
}
static void put9(double *planes, int64_t n, int p, int64_t i, m3 m) {
    put3(planes, n, p, i, m.x); put3(planes, n, p + 3, i, m.y); put3(planes, n, p + 6, i, m.z);
}
static void put9d(double *planes, int64_t n, int ph, int pl, int64_t i, m3d m) {
    put3d(planes, n, ph, pl, i, m.x); put3d(planes, n, ph + 3, pl + 3, i, m.y); put3d(planes, n, ph + 6, pl + 6, i, m.z);
}

static void load_bodies(int64_t n, const double *planes, body *b) {
    for (int64_t i = 0; i < n; ++i) {
        body *m = &b[i];
        m->r = get3d(planes, n, EPH_P_R_HI, EPH_P_R_LO, i);
        m->v = get3d(planes, n, EPH_P_V_HI, EPH_P_V_LO, i);
        m->GL = get3d(planes, n, EPH_P_GL_HI, EPH_P_GL_LO, i);
        m->s = get9d(planes, n, EPH_P_S_HI, EPH_P_S_LO, i);
        m->w = get3(planes, n, EPH_P_W, i);
        m->GM = PL(EPH_P_GM, i); m->exJ2 = PL(EPH_P_EXJ2, i);
        m->GM0 = PL(EPH_P_GM0, i); m->dGM = PL(EPH_P_DGM, i); m->dJ2 = PL(EPH_P_DJ2, i);
        m->R = PL(EPH_P_RADIUS, i); m->inertia = PL(EPH_P_INERTIA, i); m->k2 = PL(EPH_P_K2, i);
        m->k2r = PL(EPH_P_K2R, i); m->tide_delay = PL(EPH_P_TIDE_DELAY, i);
        m->tide_delay_factor = PL(EPH_P_TIDE_DELAY_FACTOR, i); m->lum = PL(EPH_P_LUM, i);
        m->recpt = PL(EPH_P_RECPT, i); m->A = PL(EPH_P_A, i); m->R2 = PL(EPH_P_R2, i);
        m->sR2 = PL(EPH_P_SR2, i); m->rR2G_4c = PL(EPH_P_RR2G_4C, i);
        m->C_static = get9(planes, n, EPH_P_C_STATIC, i);
        m->gp = (int)PL(EPH_P_GP_INDEX, i); m->ring = (int)PL(EPH_P_RING_INDEX, i);
        m->phi = PL(EPH_P_PHI, i); m->beta2 = PL(EPH_P_BETA2, i);
        m->naccel = get3(planes, n, EPH_P_NACCEL, i); m->daccel = get3(planes, n, EPH_P_DACCEL, i);
        m->dtorque = get3(planes, n, EPH_P_DTORQUE, i); m->gaccel = get3(planes, n, EPH_P_GACCEL, i);
        m->beta = get3(planes, n, EPH_P_BETA, i);
        m->GI = get9(planes, n, EPH_P_GI, i); m->C_potential = get9(planes, n, EPH_P_C_POTENTIAL, i);
        m->min_distance = PL(EPH_P_MIN_DISTANCE, i); m->max_influence = PL(EPH_P_MAX_INFLUENCE, i);
        m->Egrad = v3_make(0, 0, 0);
    }
}
static void store_bodies(int64_t n, double *planes, const body *b) {
    for (int64_t i = 0; i < n; ++i) {
        const body *m = &b[i];
        put3d(planes, n, EPH_P_R_HI, EPH_P_R_LO, i, m->r);
        put3d(planes, n, EPH_P_V_HI, EPH_P_V_LO, i, m->v);
        put3d(planes, n, EPH_P_GL_HI, EPH_P_GL_LO, i, m->GL);
        put9d(planes, n, EPH_P_S_HI, EPH_P_S_LO, i, m->s);
        put3(planes, n, EPH_P_W, i, m->w);
        PL(EPH_P_GM, i) = m->GM; PL(EPH_P_EXJ2, i) = m->exJ2;
        PL(EPH_P_PHI, i) = m->phi; PL(EPH_P_BETA2, i) = m->beta2;
        put3(planes, n, EPH_P_NACCEL, i, m->naccel); put3(planes, n, EPH_P_DACCEL, i, m->daccel);
        put3(planes, n, EPH_P_DTORQUE, i, m->dtorque); put3(planes, n, EPH_P_GACCEL, i, m->gaccel);
        put3(planes, n, EPH_P_BETA, i, m->beta);
        put9(planes, n, EPH_P_GI, i, m->GI); put9(planes, n, EPH_P_C_POTENTIAL, i, m->C_potential);
        PL(EPH_P_MIN_DISTANCE, i) = m->min_distance; PL(EPH_P_MAX_INFLUENCE, i) = m->max_influence;
    }
}

/* ---------------------------------------------------------------- extended-body models */
#define GPJ(n) ((n) * (n) - 4)  /* geopotential.impl:22-24 */

/* geopotential::sum (src/physics/geopotential.impl:26-106) */
static v3 gp_sum(const orc_models *md, int k, double R, v3 r) {
    const int64_t Nz = md->gp_nz[k], Nt = md->gp_nt[k];
    const double *c_table = md->gp_coef + (int64_t)k * EPH_GP_TABLE_SIZE;
    double rho2 = r.x * r.x + r.y * r.y;
    double rr2 = 1 / (rho2 + r.z * r.z);
    double rho1 = sqrt(rho2);
    double rr1 = sqrt(rr2);
    double rb1 = R * rr1;
    double rbn = rb1;
    double cphi = rho1 * rr1;
    double sphi = r.z * rr1;
    double cm, sm;
    if (rho2 < DBL_MIN) { cm = 1; sm = 0; }
    else { cm = r.x / rho1; sm = r.y / rho1; }
    double pnm[EPH_GP_MAX_DEGREE], pn1m[EPH_GP_MAX_DEGREE];
    pnm[0] = 0;
    pn1m[0] = 1;
    double ppn = 1, pn = 1, pn1 = sphi;
    double zx = 0, zz = 0;
    v3 t = v3_make(0, 0, 0);
    for (int64_t n = 2; n <= Nz; ++n) {
        rbn *= rb1;
        const double *JCSn = c_table + GPJ(n);
        pn = ((double)(2 * n - 1) * sphi * pn1 - (double)(n - 1) * pn) / (double)n;
        ppn = sphi * ppn + (double)n * pn1;
        double z1 = JCSn[0] * rbn;
        zx += (double)(n + 1) * z1 * pn;
        zz -= z1 * ppn;
        { double sw = pn; pn = pn1; pn1 = sw; }
        if (n > Nt) continue;
        v3 f = v3_make(0, 0, 0);
        double m1 = (double)(2 * n - 1) * sphi;
        double m2 = (double)(-n) * sphi;
        double smm = 0, cmm = 0, smm1 = 0, cmm1 = 0;
        for (int64_t m = 1; m <= n; ++m) {
            if (m == n) {
                pn1m[m - 1] = 0;
                pnm[m - 1] = (double)(2 * n - 1) * cphi * pnm[m - 2];
            } else pnm[m - 1] = (m1 * pn1m[m - 1] - (double)(n + m - 1) * pnm[m - 1]) / (double)(n - m);
            if (m == 1) { smm = sm; cmm = cm; smm1 = 0; cmm1 = 1; }
            else {
                smm = 2 * cm * smm1 - smm;
                cmm = 2 * cm * cmm1 - cmm;
            }
            double t1 = JCSn[2 * m] * smm + JCSn[2 * m - 1] * cmm;
            double t2 = JCSn[2 * m] * cmm - JCSn[2 * m - 1] * smm;
            double ppnm = m2 * pnm[m - 1] + (double)(n + m) * pn1m[m - 1];
            f.x += t1 * pnm[m - 1];
            f.y += (double)m * t2 * pnm[m - 1];
            f.z += t1 * ppnm;
            { double sw = cmm; cmm = cmm1; cmm1 = sw; }
            { double sw = smm; smm = smm1; smm1 = sw; }
            { double sw = pnm[m - 1]; pnm[m - 1] = pn1m[m - 1]; pn1m[m - 1] = sw; }
        }
        f.x *= (double)(n + 1);
        t = v3_add(t, v3_scale(rbn, f));
    }
    t.x = zx - cphi * t.x;
    t.z += zz * cphi;
    t = v3_scale(rr2, t);   /* t *= rr2 */
    double g1 = t.x * cphi - t.z * sphi;
    return v3_make(g1 * cm - t.y * sm, g1 * sm + t.y * cm, cphi * t.z + sphi * t.x);
}

/* fzcorr / padesum / ring::sum (src/physics/ring.impl:2070-2195) */
static float ring_fzcorr(float x, float y, int kh) {
    const unsigned long N = 32;
    const float *table = (const float *)EPH_RING_TABLE_BITS;
    x *= (float)N;
    y *= (float)N;
    int i = (int)floorf(x), j = (int)floorf(y);
    j -= kh * (int)N;
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i >= (int)N) i = N - 1;
    if (j >= (int)N) j = N - 1;
    j += kh * (int)N;
    x -= (float)i;
    y -= (float)j;
    const float *p = table + 16 * (2 * N * i + j);
    return p[0] + x * (p[4] + x * (p[8] + x * p[12]))
         + y * (p[1] + x * (p[5] + x * (p[9] + x * p[13]))
         + y * (p[2] + x * (p[6] + x * (p[10] + x * p[14]))
         + y * (p[3] + x * (p[7] + x * (p[11] + x * p[15])))));
}
static double padesum(double x, const double coef[][2], int n) {
    double resn = 0, resd = 0;
    while (n > 0) {
        --n;
        resn = x * resn + coef[n][0];
        resd = x * resd + coef[n][1];
    }
    return resn / resd;
}
/* Pade coefficients of the disk field (src/physics/ring.impl:2101-2107) */
static const double XSERKK[][2] = {{-4228.1846570321674587, 6387.9414439779279738}, {-13276.372802884782407, 16984.953742612298093}, {-11316.549465243054011, 8997.7319379726254196}, {-3242.2867356286923985, 403.15182320396046619}, {-704.60633921130372399, -5.7789477668119521439}};
static const double XSERKM[][2] = {{-2530.8255093002657219, 7950.8733392382639504}, {-5471.7803365810451727, 17189.101860053144376}, {-1624.0389725420726306, 7100.5562444641275465}, {1164.6058458813108946, 532.54915854738706820}, {270.03897254207263065, -5.0806023029229406554}};
static const double XSER0[][2] = {{3216.9908772759482762, 32768.000000000000000}, {-6727.1375380948220662, -93098.060290997395032}, {4534.8257724052420971, 96814.901233532309690}, {-1004.5251977686921953, -43973.540867249017404}, {17.915064837735955511, 7754.0323173314244943}, {-0.039157108395559676838, -224.00490789882410101}};
static const double KSERKK[][2] = {{-2373.3522804139070577, 1124.9866194216978637}, {-8300.7524798211745830, 17215.217000406477760}, {15279.068333441193395, 26590.060415743810476}, {-4354.4701057632348105, -9776.5071563707548874}, {-250.49346744287694398, -2385.7568792012312128}};
static const double KSERKM[][2] = {{-523.02599873176918199, 290.10526315789473684}, {-5485.2200380469245403, 5336.9790741915028535}, {-8338.1052631578947368, 15206.361445783132530}, {-2017.9378566899175650, 10515.743817374762207}, {-19.710843373493975904, 1418.8103994927076728}};
static const double KSER0[][2] = {{51471.854036415172419, 32768.000000000000000}, {-119621.18573838632696, -84345.212035111671234}, {96754.491735189724987, 78074.125512775430927}, {-31810.735585315211544, -31108.829182924968396}, {3678.1383813624327949, 4926.4461273804873303}, {-74.040670509817904983, -206.66608791871105442}};
#define PADE(x, c) padesum(x, c, (int)(sizeof(c) / sizeof(c[0])))

static v3 ring_sum(const orc_models *md, int k, double host_R, v3 r) {
    const int64_t N = md->ring_ndisk[k];
    const double *disks = md->ring_disk + (int64_t)k * EPH_RING_MAX_DISKS * 3;
    int psign = r.z < 0;
    if (psign) r.z = -r.z;
    const double re2 = r.x * r.x + r.y * r.y;
    const double re = sqrt(re2);
    const double rz2 = r.z * r.z;
    const double r2 = re2 + rz2;
    const double rz = r.z;
    v3 ret = v3_make(0, 0, 0);
    for (int64_t i = 0; i < N; ++i) {
        const double GsR2 = disks[i * 3 + 0], R_R = disks[i * 3 + 1], H_R = disks[i * 3 + 2];
        double R = R_R * host_R;
        double H = H_R * host_R;
        double reR = re * R;
        double R2 = R * R, H2, fzh = 1;
        double k2dre = 4 / (r2 + R2 + 2 * reR);
        if (H > 0) {
            H2 = H * H;
            k2dre -= H2 * (k2dre * k2dre) * (1 - k2dre * rz2) / 48;
            fzh = (re > R ? re - R : 0);
            fzh = 4 * (rz2 + fzh * fzh);
            fzh = sqrt(fzh / (fzh + H2));
        }
        double k2 = reR * k2dre;
        k2dre *= R2 * sqrt(k2dre);
        double phi = atan2(rz, re - R);
        double kk = 0, lk = 0, fx;
        int lkh = k2 >= 0.45;
        if (lkh) {
            kk = sqrt(k2);
            lk = log((1 - k2) / (8 * (1 + kk)));
            fx = (PADE(kk, XSERKK) + lk * PADE(kk, XSERKM)) / (k2 * k2);
        } else {
            fx = PADE(k2, XSER0);
        }
        fx *= k2dre;
        double fz;
        double s = sin(phi), c = cos(phi);
        int kh = k2 >= .5;
        int exphi;
        if (kh) {
            const double phimax = (PI / 2);
            exphi = c > 0;
            double ck = 1 - k2, lk2 = log(ck / 16), sk = sqrt(ck);
            double cc = exphi ? -c : c;
            double cphi = exphi ? PI - phi : phi;
            fz = cphi - (s / 8) * ((lk2 * (k2 - 5) - 2 * ck) * sk + 2 * cc * (1 + lk2) * ck);
            fz *= ring_fzcorr((float)((exphi ? phi : PI - phi) * (1 / phimax)), (float)(k2 * 2), kh);
        } else {
            const double phimax = (809. / 512);
            exphi = phi > phimax;
            double cr2 = exphi ? R2 + rz2 : r2;
            double cRdr2 = (exphi ? re2 : R2) / cr2;
            fz = (PI / 8) * (4 - 3 * cRdr2) * (rz / sqrt(cr2) * cRdr2);
            fz *= ring_fzcorr((float)((exphi ? PI - phi : phi) * (1 / phimax)), (float)(k2 * 2), kh);
        }
        if (exphi) {
            double ek;
            if (lkh) ek = PADE(kk, KSERKK) + lk * PADE(kk, KSERKM);
            else ek = PADE(k2, KSER0);
            fz = PI - 2 * sqrt(1 - k2) * ek * s - fz;
        }
        double Gs = GsR2 / (host_R * host_R);
        fx *= Gs;
        fz *= Gs;
        ret = v3_add(ret, v3_make(-4 * fx * r.x, -4 * fx * r.y, -2 * fz * fzh));
    }
    if (psign) ret.z = -ret.z;
    return ret;
}

void orc_geopotential_sum(const orc_models *models, int32_t k, double R, const double r[3], double out[3]) {
    v3 g = gp_sum(models, k, R, v3_make(r[0], r[1], r[2]));
    out[0] = g.x; out[1] = g.y; out[2] = g.z;
}
void orc_ring_sum(const orc_models *models, int32_t k, double R, const double r[3], double out[3]) {
    v3 g = ring_sum(models, k, R, v3_make(r[0], r[1], r[2]));
    out[0] = g.x; out[1] = g.y; out[2] = g.z;
}

/* ---------------------------------------------------------------- pass A: deform_by (mass.cpp:78-103) */
typedef struct pass_a_acc { double phi; v3 naccel; m3 C; } pass_a_acc;

static void deform_by(int64_t n, body *b, int64_t i) {
    body *mi = &b[i];
    pass_a_acc M;
    M.phi = 0;
    M.naccel = v3_make(0, 0, 0);
    M.C = m3_ident(0);
    for (int64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        const body *mj = &b[j];
        v3 r = v3d_diff(mj->r, mi->r);
        v3 v = v3d_diff(mj->v, mi->v);
        double rr2 = 1 / dmax(v3_dot(r, r), mi->sR2 + mj->sR2);
        double rr = sqrt(rr2);
        double tp_dphi = rr * mj->GM;
        if (mi->k2 != 0 && mi->tide_delay != 0) {
            /* DAMPED_TIDAL_DEFORMATION_MATRIX (mass.impl:1-23) */
            M.phi -= tp_dphi;
            double tp_dg = rr2 * tp_dphi;
            M.naccel = v3_add(M.naccel, v3_scale(tp_dg, r));
            double fmj = -3 * tp_dg;
            v3 dw = v3_scale(rr2, v3_cross(r, v3_sub(v3_cross(mi->w, r), v)));
            double dwt = v3_normalize(&dw);
            dwt *= mi->tide_delay * mj->tide_delay_factor;
            double ecwt2 = 1 + 4 * dwt * dwt,
                   secwt2 = sqrt(ecwt2),
                   x0 = sqrt((1 + secwt2) / (2 * ecwt2)),
                   y0 = dwt * sqrt(2 / (ecwt2 * (1 + secwt2))),
                   z02 = dwt * dwt * (2 / (ecwt2 + secwt2));
            v3 dr = v3_add(v3_scale(x0, r), v3_scale(y0, v3_cross(dw, r)));
            m3 t = m3_add_diag(m3_sub(m3_outer(v3_scale(rr2, dr), dr), m3_outer(v3_scale(z02, dw), dw)), z02 - 1.0 / 3);
            M.C = m3_sub(M.C, m3_scale(fmj * mi->k2, t));
        } else if (mi->k2 != 0) {
            /* DAMPED_TIDAL_DEFORMATION_MATRIX_NDELAY (mass.impl:25-36) */
            M.phi -= tp_dphi;
            double tp_dg = rr2 * tp_dphi;
            M.naccel = v3_add(M.naccel, v3_scale(tp_dg, r));
            double fmj = -3 * tp_dg;
            m3 t = m3_sub_diag(m3_outer(v3_scale(rr2, r), r), 1.0 / 3);
            M.C = m3_sub(M.C, m3_scale(fmj * mi->k2, t));
        } else {
            /* DAMPED_TIDAL_DEFORMATION_MATRIX_NK2 (mass.impl:38-46) */
            double tp_dg = rr2 * tp_dphi;
            M.phi -= tp_dphi;
            M.naccel = v3_add(M.naccel, v3_scale(tp_dg, r));
        }
    }
    mi->phi = M.phi;
    mi->naccel = M.naccel;
    mi->C_potential = M.C;
    /* UPDATE_HARMONICS (mass.impl:48-61) */
    double w2 = v3_dot(mi->w, mi->w);
    mi->C_potential = m3_add_diag(mi->C_potential, w2 * mi->k2r / 3);
    mi->C_potential = m3_sub(mi->C_potential, m3_outer(v3_scale(mi->k2r, mi->w), mi->w));
    mi->C_potential = m3_scale(mi->R * mi->R2 / (2 * mi->GM), mi->C_potential);
    m3 fmis = m3_from_dd(mi->s);
    m3 mc = mi->C_static;
    mc.x.x += mi->exJ2 / 2;
    mc.y.y += mi->exJ2 / 2;
    mc.z.z -= mi->exJ2;
    mc = m3_toworld_m(fmis, mc);
    mi->C_potential = m3_add(mi->C_potential, mc);
    mi->GI = m3_scale((-2.0) / 3 * mi->R2, m3_sub_diag(mi->C_potential, mi->A));
}

/* UPDATE_ANGULAR_VELOCITY (mass.impl:63-72); returns should_break */
static int update_angular_velocity(body *mi) {
    if (v3d_is_finite(mi->GL)) {
        v3 oldw = mi->w;
        mi->w = m3_mulv(m3_inverse(mi->GI), v3_from_dd(mi->GL));
        return v3_normsqr(v3_sub(mi->w, oldw)) < 1e-18 * v3_normsqr(oldw);
    }
    mi->GL = v3d_from(m3_mulv(mi->GI, mi->w));
    return 1;
}

void orc_deform(int64_t n, double *planes, const orc_models *models) {
    (void)models;
    body *b = (body *)malloc(sizeof(body) * (size_t)(n ? n : 1));
    load_bodies(n, planes, b);
    for (int64_t i = 0; i < n; ++i) deform_by(n, b, i);
    store_bodies(n, planes, b);
    free(b);
}

/* ---------------------------------------------------------------- accel, serial branch (mass.cpp:216-397) */
static void accel_serial(int64_t n, body *b, const orc_models *md) {
    const double c = C_LIGHT;
    for (int64_t i = 0; i < n; ++i) {   /* mass.cpp:311-326 */
        body *mi = &b[i];
        int max_iter = 4;   /* MAX_ANGULAR_VELOCITY_ITER, mass.impl:74 */
        do {
            deform_by(n, b, i);
            if (update_angular_velocity(mi)) break;
        } while (--max_iter);
        /* PREPARE_RELATIVITY (mass.impl:76-80) */
        mi->beta = v3_div(v3_from_dd(mi->v), c);
        mi->beta2 = v3_dot(mi->beta, mi->beta);
        mi->phi /= C2;
        mi->naccel = v3_div(mi->naccel, C2);
        mi->daccel = mi->dtorque = mi->gaccel = v3_make(0, 0, 0);
    }
    for (int64_t i = 0; i < n; ++i) {   /* mass.cpp:329-373 */
        body *mi = &b[i];
        for (int64_t j = 0; j < n; ++j) {
            if (i == j) continue;
            body *mj = &b[j];
            /* RELATIVITY (mass.impl:82-97) */
            v3 r = v3d_diff(mj->r, mi->r);
            double rr2 = 1 / dmax(v3_dot(r, r), mi->sR2 + mj->sR2);
            double rr = sqrt(rr2);
            double rr3 = rr * rr2;
            double tp_dphi = rr * mj->GM;
            double tp_dg = rr2 * tp_dphi;
            double rbj = v3_dot(r, mj->beta);
            double tp_rbjrr2 = rbj * rr;
            tp_rbjrr2 *= tp_rbjrr2;
            double delta1 = 4 * mi->phi + mj->phi + mi->beta2 + 2 * mj->beta2
                - 4 * v3_dot(mi->beta, mj->beta) + (v3_dot(r, mj->naccel) - 3 * tp_rbjrr2) / 2;
            v3 bv = v3_sub(mj->beta, mi->beta);
            mi->gaccel = v3_add(mi->gaccel, v3_add(v3_add(v3_scale(7 * tp_dphi / 2, mj->naccel),
                v3_scale(tp_dg * delta1, r)), v3_scale(tp_dg * (rbj - v3_dot(r, bv) * 4), bv)));
            checked_maximize(&mi->min_distance, rr);
            checked_maximize(&mi->max_influence, tp_dg);
            /* ROTATIONAL_TIDAL_DEFORMATION (mass.impl:111-116), with the reaction on mj */
            {
                v3 Cr = m3_mulv(mi->C_potential, r);
                v3 dg = v3_scale(rr3 * rr2 * mi->R2, v3_sub(v3_scale(v3_dot(r, Cr) * 5 * rr2, r), v3_add(Cr, Cr)));
                mi->daccel = v3_add(mi->daccel, v3_scale(mj->GM, dg));
                mj->daccel = v3_sub(mj->daccel, v3_scale(mi->GM, dg));
                mi->dtorque = v3_add(mi->dtorque, v3_scale(mj->GM, v3_cross(r, dg)));
            }
            /* LENSE_THIRRING (mass.impl:99-106) */
            {
                double rcr32 = 2 * mj->GM / c * rr3;
                v3 GL = v3_from_dd(mi->GL);
                v3 GLb = v3_cross(GL, bv);
                mi->daccel = v3_sub(mi->daccel, v3_scale(rcr32, v3_sub(GLb, v3_scale(3 * v3_dot(GLb, r) * rr2, r))));
                mi->dtorque = v3_sub(mi->dtorque, v3_scale(rcr32, v3_cross(GL, v3_cross(r, bv))));
                v3 GLj = v3_from_dd(mj->GL);
                mi->daccel = v3_add(mi->daccel, v3_cross(v3_scale(rcr32, v3_sub(GLj, v3_scale(3 * v3_dot(GLj, r) * rr2, r))), bv));
            }
            /* RADIATION_PRESSURE (mass.impl:108-109) */
            mi->daccel = v3_add(mi->daccel, v3_scale(mj->lum * mi->rR2G_4c * rr3 / mi->GM, r));
            /* geopotential of mi acting on mj (mass.cpp:358-363), APPLY_NONPOINT_FORCE (mass.impl:127-130) */
            if (mi->gp >= 0) {
                m3 fmis = m3_from_dd(mi->s);
                v3 lr = m3_tolocal(fmis, r);
                v3 an = m3_toworld(fmis, gp_sum(md, mi->gp, mi->R, lr));
                mj->daccel = v3_add(mj->daccel, v3_scale(mi->GM, an));
                mi->daccel = v3_sub(mi->daccel, v3_scale(mj->GM, an));
                mi->dtorque = v3_sub(mi->dtorque, v3_scale(mj->GM, v3_cross(r, an)));
            }
            /* ring of mi acting on mj (mass.cpp:365-371) */
            if (mi->ring >= 0) {
                v3 migl = v3_from_dd(mi->GL);
                v3 fx = v3_asc_node(migl), fz = v3_unit(migl);
                m3 fgls = m3_make(fx, v3_cross(fz, fx), fz);   /* mat_t(x, int, z): y = z*x (vec_t.h:281) */
                v3 lr = m3_tolocal(fgls, r);
                v3 an = m3_toworld(fgls, ring_sum(md, mi->ring, mi->R, lr));
                mj->daccel = v3_add(mj->daccel, v3_scale(mi->GM, an));
                mi->daccel = v3_sub(mi->daccel, v3_scale(mj->GM, an));
                mi->dtorque = v3_sub(mi->dtorque, v3_scale(mj->GM, v3_cross(r, an)));
            }
        }
    }
    for (int64_t i = 0; i < n; ++i) {   /* mass.cpp:389-396 */
        body *m = &b[i];
        /* FINALIZE_RELATIVITY (mass.impl:133-135) */
        m->phi *= C2;
        m->naccel = v3_scale(C2, m->naccel);
        if (m->ring >= 0) {
            /* RING_CORRECTION (mass.impl:143-152) */
            const double *rp = md->ring_param + (int64_t)m->ring * 4;
            const double GM_ratio = rp[0], GL_R2 = rp[3];
            m->daccel = v3_sub(m->daccel, v3_scale(GM_ratio, v3_add(v3_add(m->gaccel, m->daccel), m->naccel)));
            v3 mGL = v3_from_dd(m->GL);
            double rmGL = v3_normalize(&mGL);
            v3 ptorque = v3_scale(v3_dot(m->dtorque, mGL), mGL);
            v3 dtq = v3_sub(m->dtorque, ptorque);
            dtq = v3_scale(rmGL / (rmGL + GL_R2 * m->R2), dtq);
            m->dtorque = v3_add(dtq, ptorque);
        }
    }
}

void orc_accel(int64_t n, double *planes, const orc_models *models) {
    body *b = (body *)malloc(sizeof(body) * (size_t)(n ? n : 1));
    load_bodies(n, planes, b);
    accel_serial(n, b, models);
    store_bodies(n, planes, b);
    free(b);
}

/* ---------------------------------------------------------------- RK12 (RungeKutta.impl:107-194) */
static dd rk_coef(int64_t idx) {
    dd c;
    memcpy(&c.hi, &EPH_RK12_COEF_BITS[2 * idx], 8);
    memcpy(&c.lo, &EPH_RK12_COEF_BITS[2 * idx + 1], 8);
    return c;
}

static void rk12(int64_t n, body *x, const orc_models *md, double dt, int64_t n_step, dd t_eph, double *stage_acc,
                 double *stage_in, double *stage_out) {
    stage_state *x0 = (stage_state *)malloc(sizeof(stage_state) * (size_t)(n ? n : 1));
    stage_state *f = (stage_state *)malloc(sizeof(stage_state) * (size_t)(25 * (n ? n : 1)));
    int64_t n_rec = 0;
    for (int64_t i_step = 0; i_step < n_step; ++i_step) {
        for (int64_t i = 0; i < n; ++i) {
            x0[i].r = x[i].r; x0[i].v = x[i].v; x0[i].GL = x[i].GL; x0[i].s = x[i].s; x0[i].w = x[i].w;
            x[i].Egrad = x[i].dtorque;
        }
        double dt_k;
        for (int64_t k = 1; k <= 25; ++k) {
            dt_k = 0;
            for (int64_t i = 0; i < n; ++i) {
                stage_state *fi = &f[n * (k - 1) + i];
                body *xi = &x[i];
                fi->v = xi->v;
                fi->naccel = v3_add(v3_add(xi->gaccel, xi->daccel), xi->naccel);
                fi->w = xi->w;
                fi->dtorque = xi->dtorque;
                if (k == 25) {   /* RungeKutta.impl:129-140 */
                    m3 ir = m3_inverse(xi->GI);
                    double irdet = m3_det(ir);
                    double dt2 = dt * dt;
                    v3 tq = v3_scale(dt2, xi->dtorque);
                    v3 tqdot = v3_scale(dt2, v3_sub(xi->dtorque, xi->Egrad));
                    v3 j = v3_from_dd(xi->GL), w = v3_scale(dt, xi->w);
                    v3 irtq = m3_mulv(ir, tq);
                    j = v3_scale(dt, j);
                    v3 e1 = v3_scale(v3_dot(w, j), v3_add(m3_mulv(ir, w), v3_scale(irdet, m3_mulv(xi->GI, j))));
                    v3 e2 = v3_cross(w, irtq);
                    v3 e3 = m3_mulv(ir, v3_add(v3_sub(v3_cross(j, irtq), v3_scale(2, v3_cross(w, tq))), tqdot));
                    xi->Egrad = v3_add(v3_add(e1, e2), e3);
                    xi->Egrad = v3_cross(xi->Egrad, w);
                }
                xi->v = v3d_from(v3_make(0, 0, 0));
                xi->naccel = v3_make(0, 0, 0);
                xi->w = v3_make(0, 0, 0);
                xi->dtorque = v3_make(0, 0, 0);
            }
            for (int64_t j = 0; j < k; ++j) {   /* RungeKutta.impl:148-162 */
                const dd ckj = rk_coef(k * (k - 1) / 2 + j);
                const double fckj = dd_val(ckj);
                if (ckj.hi != 0) {
                    dt_k += fckj;
                    for (int64_t i = 0; i < n; ++i) {
                        const stage_state *fi = &f[n * j + i];
                        body *xi = &x[i];
                        xi->v = v3d_add(xi->v, v3d_scale(ckj, fi->v));
                        xi->naccel = v3_add(xi->naccel, v3_scale(fckj, fi->naccel));
                        xi->w = v3_add(xi->w, v3_scale(fckj, fi->w));
                        xi->dtorque = v3_add(xi->dtorque, v3_scale(fckj, fi->dtorque));
                    }
                }
            }
            double t = dd_val(t_eph) + dt * (dt_k + (double)i_step);   /* RungeKutta.impl:164 */
            for (int64_t i = 0; i < n; ++i) {   /* RungeKutta.impl:165-186 */
                const stage_state *xi0 = &x0[i];
                body *xi = &x[i];
                xi->r = v3d_add(xi0->r, v3d_scale(dd_make(dt), xi->v));
                xi->v = v3d_add(xi0->v, v3d_from(v3_scale(dt, xi->naccel)));
                xi->w = v3_div(xi->w, dt_k);
                xi->s = xi0->s;
                v3 dw = v3_scale(2.0 / 3, v3_sub(xi->w, xi0->w));
                xi->s = m3d_add_fast(xi->s, m3_mul(v3_rotation_matrix(v3_sub(xi->w, dw), dt * dt_k / 2), m3_from_dd(xi->s)));
                xi->s = m3d_add_fast(xi->s, m3_mul(v3_rotation_matrix(v3_add(xi->w, dw), dt * dt_k / 2), m3_from_dd(xi->s)));
                xi->GL = v3d_add(xi0->GL, v3d_from(v3_scale(dt, xi->dtorque)));
                if (k == 25) {
                    xi->s = m3d_add_fast(xi->s, m3_mul(v3_rotation_matrix(xi->Egrad, 1.0 / 72), m3_from_dd(xi->s)));
                    /* mass::orthogonalize (mass.h:147-150) */
                    m3 fmis = m3_from_dd(xi->s);
                    m3 one_minus = m3_add_diag(m3_neg(m3_mul(m3_transpose(fmis), fmis)), 1);
                    xi->s = m3d_add_fast(xi->s, m3_mul(m3_scale(0.5, fmis), one_minus));
                }
                xi->GM = xi->GM0 + xi->dGM * t;
                xi->exJ2 = xi->dJ2 * t;
            }
            if (stage_in) store_bodies(n, stage_in + n_rec * (int64_t)EPH_NPLANES * n, x);
            accel_serial(n, x, md);
            if (stage_out) store_bodies(n, stage_out + n_rec * (int64_t)EPH_NPLANES * n, x);
            if (stage_acc) {
                double *o = stage_acc + n_rec * 3 * n;
                for (int64_t i = 0; i < n; ++i) {
                    v3 a = v3_add(v3_add(x[i].gaccel, x[i].daccel), x[i].naccel);
                    o[i] = a.x; o[n + i] = a.y; o[2 * n + i] = a.z;
                }
            }
            ++n_rec;
        }
    }
    free(x0);
    free(f);
}

static void integrate_impl(int64_t n, double *planes, const orc_models *models, double dt, int64_t n_step,
                           double *t_eph_hi, double *t_eph_lo, double *stage_acc, double *stage_in, double *stage_out) {
    if (n_step == 0) return;   /* mass.cpp:400-404 */
    if (n_step < 0) { n_step = -n_step; dt = -dt; }
    body *b = (body *)malloc(sizeof(body) * (size_t)(n ? n : 1));
    load_bodies(n, planes, b);
    for (int64_t i = 0; i < n; ++i) b[i].max_influence = b[i].min_distance = 0;   /* mass.cpp:406 */
    dd t_eph = {*t_eph_hi, *t_eph_lo};
    rk12(n, b, models, dt, n_step, t_eph, stage_acc, stage_in, stage_out);
    for (int64_t i = 0; i < n; ++i) b[i].min_distance = 1 / b[i].min_distance;   /* mass.cpp:416 */
    t_eph = dd_add(t_eph, dd_make(dt * (double)n_step));   /* mass.cpp:441 */
    *t_eph_hi = t_eph.hi;
    *t_eph_lo = t_eph.lo;
    store_bodies(n, planes, b);
    free(b);
}

void orc_integrate(int64_t n, double *planes, const orc_models *models, double dt, int64_t n_step,
                   double *t_eph_hi, double *t_eph_lo, double *stage_acc) {
    integrate_impl(n, planes, models, dt, n_step, t_eph_hi, t_eph_lo, stage_acc, NULL, NULL);
}
void orc_integrate_stages(int64_t n, double *planes, const orc_models *models, double dt, int64_t n_step,
                          double *t_eph_hi, double *t_eph_lo, double *stage_in, double *stage_out) {
    integrate_impl(n, planes, models, dt, n_step, t_eph_hi, t_eph_lo, NULL, stage_in, stage_out);
}
