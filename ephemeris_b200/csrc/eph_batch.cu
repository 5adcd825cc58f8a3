// eph_batch.cu - batched ensembles: many independent systems integrated in one persistent launch.
//
// Each system runs the reference's msystem::integrate (mass.cpp:399-442) on its own dt, step count and
// ephemeris time. Systems whose bodies are all point-like (no tide, rotational deformation, static
// harmonics, spin, luminosity, radiation receptance, geopotential or ring: the Newtonian + 1PN systems of
// an ensemble) run in `ensemble_kernel`: one CTA integrates one whole system, so a stage needs only
// CTA barriers, and persistent CTAs take systems from an atomic queue, heaviest (bodies^2 x steps) first.
// The bodies' stage data sit in shared memory as structure-of-arrays rows; the stage values f_j and the
// start-of-step state sit in global scratch (L2-resident for ensemble sizes), and each body's thread
// forms sum_j a_kj f_j at its state update (independent loads, ascending j as in the reference). Any other system
// of the batch (a full-physics body, or more bodies than one CTA's shared memory holds) is integrated by
// the per-system persistent kernel of eph_step.cu through a context, one after another.
//
// Physics per pair (the point-class branches of the reference):
//   pass A  phi_i -= GM_j / r, a_N,i += GM_j r / r^3, r^2 floored at sR2_i + sR2_j
//           (DAMPED_TIDAL_DEFORMATION_MATRIX_NK2, mass.impl:38-46)
//   prepare beta = v / c, beta^2, phi / c^2, a_N / c^2 (PREPARE_RELATIVITY, mass.impl:76-80)
//   pass B  EIH 1PN (RELATIVITY, mass.impl:82-97) and the per-pair maxima of 1/r and GM_j/r^3
//           (RungeKutta.cu:229-230), recomputed exactly for the extremal pair; in the mixed-precision form
//           (eph_batch_set_precision) the 1PN terms in FP32 (pair_point_b32)
//   final   phi c^2, a_N c^2 (FINALIZE_RELATIVITY, mass.impl:133-135); f = (gaccel + daccel) + naccel
// For such bodies the reference's angular velocity, G*L and harmonics stay constant (w = G*L = 0), the
// frame rotations are the identity and only the end-of-step orthogonalisation of the frame acts
// (mass.h:147-150); the RK12 combination and state update are those of RungeKutta.impl:148-186.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "eph_math.cuh"
#include "eph_plan.h"
#include "eph_rk12_host.h"
#include "eph_system.cuh"
#include "../../include/eph_b200.h"
#include "../../include/eph_planes.h"

namespace eph {
namespace {

constexpr int kBThreads = 256;          // threads per ensemble CTA
constexpr int kCluster = 4;             // CTAs of a thread-block cluster that share one large system
constexpr int kCoopMin = 96;            // default: bodies from which a system is shared by a cluster
constexpr double kCB = 299792458.0;     // src/math/basic_math.h:10,18
constexpr int kAcc = 9;                 // stored values per (body, stage): velocity dd (hi 3, lo 3), acceleration 3

__constant__ double b_rk_hi[EPH_RK12_NCOEF];
__constant__ double b_rk_lo[EPH_RK12_NCOEF];
__constant__ double b_dtk[kStages + 1];

struct BatchSys {
    int n;                // bodies
    int pad;
    long long n_step;     // steps (>= 1)
    double dt;            // signed step
    double t_eph;         // double(t_eph) at the start
    double *planes;       // [EPH_NPLANES][n], in and out
    double *acc;          // [kStages][kAcc][n] stage values f_j: velocity (hi 3, lo 3), acceleration 3
    double *x0;           // [12][n] start-of-step r, v (hi, lo)
};

// shared-memory rows of one system, stride `ld` bodies
enum BRow { BR_R_HI = 0, BR_R_LO = 3, BR_GM = 6, BR_SR2 = 7, BR_PHI = 8, BR_NACC = 9, BR_BETA = 12, BR_BETA2 = 15,
            BR_V_HI = 16, BR_V_LO = 19, BR_FA = 22, BR_GA = 25, BR_MIND = 28, BR_MAXI = 29, BR_GM0 = 30, BR_DGM = 31,
            BR_F32 = 32, BR_ROWS = 37 };
// FP32 rows of the mixed-precision form (single-precision copies of what its pass-B pair terms read of body
// j), packed two to a double row from BR_F32 on
enum FRow { F_GM = 0, F_PHI = 1, F_NACC = 2, F_BETA = 5, F_BETA2 = 8, F_ROWS = 9 };
static_assert((F_ROWS + 1) / 2 <= BR_ROWS - BR_F32, "FP32 rows do not fit");

struct BatchView {
    double *T;    // rows
    int ld;
};

__device__ __forceinline__ double &row(const BatchView &V, int r, int i) { return V.T[r * V.ld + i]; }
__device__ __forceinline__ float &frow(const BatchView &V, int r, int i) {
    return reinterpret_cast<float *>(V.T + BR_F32 * V.ld)[r * V.ld + i];
}

// pass A pair (i, j): acc = {phi, a_N}
__device__ __forceinline__ void pair_point_a(const BatchView &V, int i, int j, double acc[4]) {
    const v3 r = mk(sep_diff(row(V, BR_R_HI + 0, j), row(V, BR_R_LO + 0, j), row(V, BR_R_HI + 0, i), row(V, BR_R_LO + 0, i)),
                    sep_diff(row(V, BR_R_HI + 1, j), row(V, BR_R_LO + 1, j), row(V, BR_R_HI + 1, i), row(V, BR_R_LO + 1, i)),
                    sep_diff(row(V, BR_R_HI + 2, j), row(V, BR_R_LO + 2, j), row(V, BR_R_HI + 2, i), row(V, BR_R_LO + 2, i)));
    const double q = dot(r, r), sm = row(V, BR_SR2, i) + row(V, BR_SR2, j);
    const double rr = rsqrt((q < sm) ? sm : q);
    const double rr2 = rr * rr;
    const double tp_dphi = rr * row(V, BR_GM, j);
    const double tp_dg = rr2 * tp_dphi;
    acc[0] -= tp_dphi;
    acc[1] += tp_dg * r.x;
    acc[2] += tp_dg * r.y;
    acc[3] += tp_dg * r.z;
}

struct PairMax {
    double m_min;            // smallest floored r^2
    double tq, tq_m, tq_gm;  // largest GM_j/r^3 seen, with its r^2 and GM_j
};

// pass B pair (i, j): acc = gaccel (EIH 1PN) and the maxima bookkeeping
__device__ __forceinline__ void pair_point_b(const BatchView &V, int i, int j, double acc[3], PairMax &x) {
    const v3 r = mk(sep_diff(row(V, BR_R_HI + 0, j), row(V, BR_R_LO + 0, j), row(V, BR_R_HI + 0, i), row(V, BR_R_LO + 0, i)),
                    sep_diff(row(V, BR_R_HI + 1, j), row(V, BR_R_LO + 1, j), row(V, BR_R_HI + 1, i), row(V, BR_R_LO + 1, i)),
                    sep_diff(row(V, BR_R_HI + 2, j), row(V, BR_R_LO + 2, j), row(V, BR_R_HI + 2, i), row(V, BR_R_LO + 2, i)));
    const double GMj = row(V, BR_GM, j);
    const double q = dot(r, r), sm = row(V, BR_SR2, i) + row(V, BR_SR2, j);
    const double m = (q < sm) ? sm : q;
    const double rr = rsqrt(m);
    const double rr2 = rr * rr;
    const double tp_dphi = rr * GMj;
    const double tp_dg = rr2 * tp_dphi;
    if (x.m_min == x.m_min) x.m_min = (m != m || m < x.m_min) ? m : x.m_min;
    if (x.tq == x.tq) {
        if (tp_dg != tp_dg) x.tq = tp_dg;
        else if (tp_dg > x.tq) { x.tq = tp_dg; x.tq_m = m; x.tq_gm = GMj; }
    }
    const v3 bj = mk(row(V, BR_BETA + 0, j), row(V, BR_BETA + 1, j), row(V, BR_BETA + 2, j));
    const v3 bi = mk(row(V, BR_BETA + 0, i), row(V, BR_BETA + 1, i), row(V, BR_BETA + 2, i));
    const double rbj = dot(r, bj);
    double tp = rbj * rr;
    tp *= tp;
    const v3 naj = mk(row(V, BR_NACC + 0, j), row(V, BR_NACC + 1, j), row(V, BR_NACC + 2, j));
    const double delta1 = 4 * row(V, BR_PHI, i) + row(V, BR_PHI, j) + row(V, BR_BETA2, i) + 2 * row(V, BR_BETA2, j) -
                          4 * dot(bi, bj) + (dot(r, naj) - 3 * tp) / 2;
    const v3 b = bj - bi;
    const v3 g = (7 * tp_dphi / 2) * naj + (tp_dg * delta1) * r + (tp_dg * (rbj - dot(r, b) * 4)) * b;
    acc[0] += g.x;
    acc[1] += g.y;
    acc[2] += g.z;
}

// Mixed-precision form of the pass-B pair: the separation and its floored square stay FP64 (so the per-pair
// maxima keep the reference's exact recomputation of the extremal pair), the EIH 1PN acceleration (about
// 1e-8 of the Newtonian one for solar-system speeds and potentials, so FP32's 6e-8 relative rounding is
// ~1e-15 of the total) is formed in FP32 from FP32 copies of the pass-A outputs and summed with a
// compensated FP32 sum (Fast2Sum after each add), which the caller converts into its FP64 totals. The
// extremal pair of max_influence is chosen on the FP32 value of GM/r^3, so in a near-tie (within FP32
// rounding) another pair's value may be the one recomputed.
struct BodyF32 {   // body i's FP32 pass-B inputs
    float phi, beta2, bx, by, bz;
};
struct Comp32 {    // compensated FP32 sums of the three 1PN components
    float s[3], c[3];
};
struct PairMax32 {
    double m_min;          // smallest floored r^2 (FP64)
    float tq;              // largest FP32 GM_j/r^3 seen
    double tq_m, tq_gm;    // its r^2 and GM_j
};
__device__ __forceinline__ void comp_add(float &s, float &c, float x) {
    const float t = __fadd_rn(s, x);
    const float big = fabsf(s) >= fabsf(x) ? s : x, small = fabsf(s) >= fabsf(x) ? x : s;
    c = __fadd_rn(c, __fadd_rn(__fsub_rn(big, t), small));
    s = t;
}
__device__ __forceinline__ void pair_point_b32(const BatchView &V, int i, int j, const BodyF32 &bi, Comp32 &acc,
                                               PairMax32 &x) {
    const v3 r = mk(sep_diff(row(V, BR_R_HI + 0, j), row(V, BR_R_LO + 0, j), row(V, BR_R_HI + 0, i), row(V, BR_R_LO + 0, i)),
                    sep_diff(row(V, BR_R_HI + 1, j), row(V, BR_R_LO + 1, j), row(V, BR_R_HI + 1, i), row(V, BR_R_LO + 1, i)),
                    sep_diff(row(V, BR_R_HI + 2, j), row(V, BR_R_LO + 2, j), row(V, BR_R_HI + 2, i), row(V, BR_R_LO + 2, i)));
    const double q = dot(r, r), sm = row(V, BR_SR2, i) + row(V, BR_SR2, j);
    const double m = (q < sm) ? sm : q;
    if (x.m_min == x.m_min) x.m_min = (m != m || m < x.m_min) ? m : x.m_min;
    const float rr = rsqrtf((float)m);
    const float rr2 = rr * rr;
    const float tp_dphi = rr * frow(V, F_GM, j);
    const float tp_dg = rr2 * tp_dphi;
    if (x.tq == x.tq) {
        if (tp_dg != tp_dg) x.tq = tp_dg;
        else if (tp_dg > x.tq) { x.tq = tp_dg; x.tq_m = m; x.tq_gm = row(V, BR_GM, j); }
    }
    const float rx = (float)r.x, ry = (float)r.y, rz = (float)r.z;
    const float bjx = frow(V, F_BETA + 0, j), bjy = frow(V, F_BETA + 1, j), bjz = frow(V, F_BETA + 2, j);
    const float rbj = rx * bjx + ry * bjy + rz * bjz;
    float tp = rbj * rr;
    tp *= tp;
    const float nax = frow(V, F_NACC + 0, j), nay = frow(V, F_NACC + 1, j), naz = frow(V, F_NACC + 2, j);
    const float delta1 = 4 * bi.phi + frow(V, F_PHI, j) + bi.beta2 + 2 * frow(V, F_BETA2, j) -
                         4 * (bi.bx * bjx + bi.by * bjy + bi.bz * bjz) + ((rx * nax + ry * nay + rz * naz) - 3 * tp) / 2;
    const float bx = bjx - bi.bx, by = bjy - bi.by, bz = bjz - bi.bz;
    const float c1 = 7 * tp_dphi / 2, c2 = tp_dg * delta1, c3 = tp_dg * (rbj - (rx * bx + ry * by + rz * bz) * 4);
    comp_add(acc.s[0], acc.c[0], c1 * nax + c2 * rx + c3 * bx);
    comp_add(acc.s[1], acc.c[1], c1 * nay + c2 * ry + c3 * by);
    comp_add(acc.s[2], acc.c[2], c1 * naz + c2 * rz + c3 * bz);
}
__device__ __forceinline__ BodyF32 body_f32(const BatchView &V, int i) {
    return BodyF32{frow(V, F_PHI, i), frow(V, F_BETA2, i), frow(V, F_BETA + 0, i), frow(V, F_BETA + 1, i),
                   frow(V, F_BETA + 2, i)};
}

// Threads of a pass: with n <= blockDim bodies, G consecutive lanes of a warp share body i and split its j
// range (G = the largest power of two <= min(32, blockDim / n)); their partial sums are combined by warp
// shuffles. With more bodies than threads each thread takes whole bodies.
struct PassMap {
    int G, i, sub;
    bool grouped, active;
};
__device__ __forceinline__ PassMap pass_map(int lo, int hi) {
    const int cnt = hi - lo;
    PassMap m;
    m.grouped = cnt <= (int)blockDim.x;
    int g = 1;
    if (m.grouped)
        while (g < 32 && 2 * g * cnt <= (int)blockDim.x) g *= 2;
    m.G = g;
    m.i = lo + (int)threadIdx.x / g;
    m.sub = threadIdx.x % g;
    m.active = m.grouped && m.i < hi;
    return m;
}
// sum (or NaN-propagating maximum) over the G lanes of a group; every lane of the warp takes part
__device__ __forceinline__ double group_sum(double v, int G) {
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double group_max(double v, int G) {
    for (int o = G / 2; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        checked_maximize(v, u);
    }
    return v;
}

// pass A for body i over j ≡ sub (mod G), then PREPARE_RELATIVITY by whoever holds the total
__device__ __forceinline__ void prepare_body(const BatchView &V, int i, const double s[4]) {
    const double c2 = kCB * kCB;
    const v3 beta = vdiv(mk(dd_val(dd{row(V, BR_V_HI + 0, i), row(V, BR_V_LO + 0, i)}),
                            dd_val(dd{row(V, BR_V_HI + 1, i), row(V, BR_V_LO + 1, i)}),
                            dd_val(dd{row(V, BR_V_HI + 2, i), row(V, BR_V_LO + 2, i)})), kCB);
    row(V, BR_BETA + 0, i) = beta.x;
    row(V, BR_BETA + 1, i) = beta.y;
    row(V, BR_BETA + 2, i) = beta.z;
    row(V, BR_BETA2, i) = dot(beta, beta);
    row(V, BR_PHI, i) = s[0] / c2;
    const v3 na = vdiv(mk(s[1], s[2], s[3]), c2);
    row(V, BR_NACC + 0, i) = na.x;
    row(V, BR_NACC + 1, i) = na.y;
    row(V, BR_NACC + 2, i) = na.z;
    // FP32 copies for the mixed-precision pass B (written in both forms; unused by the FP64 one)
    frow(V, F_PHI, i) = (float)row(V, BR_PHI, i);
    frow(V, F_BETA2, i) = (float)row(V, BR_BETA2, i);
    for (int c = 0; c < 3; ++c) {
        frow(V, F_NACC + c, i) = (float)row(V, BR_NACC + c, i);
        frow(V, F_BETA + c, i) = (float)row(V, BR_BETA + c, i);
    }
}

// pass A (and PREPARE_RELATIVITY) of the bodies i in [lo, hi) against all n bodies
__device__ void pass_point_a(const BatchView &V, int n, int lo, int hi) {
    const PassMap m = pass_map(lo, hi);
    if (m.grouped) {
        // two independent pair chains per thread (j and j + G), added at the end
        double acc[4] = {0, 0, 0, 0}, acc2[4] = {0, 0, 0, 0};
        if (m.active) {
            int j = m.sub;
#pragma unroll 1
            for (; j + m.G < n; j += 2 * m.G) {
                if (j != m.i) pair_point_a(V, m.i, j, acc);
                if (j + m.G != m.i) pair_point_a(V, m.i, j + m.G, acc2);
            }
            if (j < n && j != m.i) pair_point_a(V, m.i, j, acc);
        }
        double s[4];
        for (int c = 0; c < 4; ++c) s[c] = group_sum(acc[c] + acc2[c], m.G);
        if (m.active && m.sub == 0) prepare_body(V, m.i, s);
    } else {
        // whole bodies per thread: prepare_body writes only rows pass A does not read (it reads r, GM, sR2)
#pragma unroll 1
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            double s[4] = {0, 0, 0, 0}, s2[4] = {0, 0, 0, 0};
            int j = 0;
#pragma unroll 1
            for (; j + 1 < n; j += 2) {
                if (j != i) pair_point_a(V, i, j, s);
                if (j + 1 != i) pair_point_a(V, i, j + 1, s2);
            }
            if (j < n && j != i) pair_point_a(V, i, j, s);
            for (int c = 0; c < 4; ++c) s[c] += s2[c];
            prepare_body(V, i, s);
        }
    }
    __syncthreads();
}

// finalisation of body i from its pass-B totals {gaccel, 1/r max, GM/r^3 max}
__device__ __forceinline__ void finish_body(const BatchView &V, int i, const double s[5]) {
    const double c2 = kCB * kCB;
    checked_maximize(row(V, BR_MIND, i), s[3]);
    checked_maximize(row(V, BR_MAXI, i), s[4]);
    const v3 ga = mk(s[0], s[1], s[2]);
    const v3 da = mk(0, 0, 0);
    const v3 na = c2 * mk(row(V, BR_NACC + 0, i), row(V, BR_NACC + 1, i), row(V, BR_NACC + 2, i));
    const v3 fa = (ga + da) + na;
    row(V, BR_GA + 0, i) = ga.x;
    row(V, BR_GA + 1, i) = ga.y;
    row(V, BR_GA + 2, i) = ga.z;
    row(V, BR_FA + 0, i) = fa.x;
    row(V, BR_FA + 1, i) = fa.y;
    row(V, BR_FA + 2, i) = fa.z;
}

// exact extremes with the reference's expressions (rr2 = 1/m, rr = sqrt(rr2), mass.impl:84-89)
__device__ __forceinline__ void extremes_of(const PairMax &x, double &inv_r, double &infl) {
    inv_r = sqrt(1.0 / x.m_min);   // +inf -> 0 when no pair was seen
    if (x.tq != x.tq) infl = x.tq;
    else if (x.tq > 0) {
        const double r2 = 1.0 / x.tq_m;
        infl = r2 * (sqrt(r2) * x.tq_gm);
    } else infl = 0.0;
}

// exact extremes of the mixed form's tracking (the same expressions on the tracked FP64 values)
__device__ __forceinline__ void extremes_of32(const PairMax32 &x, double &inv_r, double &infl) {
    inv_r = sqrt(1.0 / x.m_min);
    if (x.tq != x.tq) infl = (double)x.tq;
    else if (x.tq > 0) {
        const double r2 = 1.0 / x.tq_m;
        infl = r2 * (sqrt(r2) * x.tq_gm);
    } else infl = 0.0;
}

// mixed-precision pass B: two pair chains per thread like the FP64 form, FP32 1PN sums converted into FP64
__device__ void pass_point_b32(const BatchView &V, int n, int lo, int hi) {
    const PassMap m = pass_map(lo, hi);
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    auto sweep = [&](int i, int j0, int step, double s[5]) {
        const BodyF32 bi = body_f32(V, i);
        Comp32 a{{0, 0, 0}, {0, 0, 0}}, a2{{0, 0, 0}, {0, 0, 0}};
        PairMax32 x{inf, 0.0f, 0.0, 0.0}, x2{inf, 0.0f, 0.0, 0.0};
        int j = j0;
#pragma unroll 1
        for (; j + step < n; j += 2 * step) {
            if (j != i) pair_point_b32(V, i, j, bi, a, x);
            if (j + step != i) pair_point_b32(V, i, j + step, bi, a2, x2);
        }
        if (j < n && j != i) pair_point_b32(V, i, j, bi, a, x);
        for (int c = 0; c < 3; ++c)
            s[c] = ((double)a.s[c] + (double)a.c[c]) + ((double)a2.s[c] + (double)a2.c[c]);
        double f0, f1;
        extremes_of32(x, s[3], s[4]);
        extremes_of32(x2, f0, f1);
        checked_maximize(s[3], f0);
        checked_maximize(s[4], f1);
    };
    if (m.grouped) {
        double s[5] = {0, 0, 0, 0, 0};
        if (m.active) sweep(m.i, m.sub, m.G, s);
        else {
            const PairMax32 none{inf, 0.0f, 0.0, 0.0};
            extremes_of32(none, s[3], s[4]);
        }
        for (int c = 0; c < 3; ++c) s[c] = group_sum(s[c], m.G);
        s[3] = group_max(s[3], m.G);
        s[4] = group_max(s[4], m.G);
        if (m.active && m.sub == 0) finish_body(V, m.i, s);
    } else {
#pragma unroll 1
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            double s[5];
            sweep(i, 0, 1, s);
            finish_body(V, i, s);
        }
    }
    __syncthreads();
}

// pass B and finalisation of the bodies i in [lo, hi) against all n bodies
__device__ void pass_point_b(const BatchView &V, int n, int lo, int hi) {
    const PassMap m = pass_map(lo, hi);
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    if (m.grouped) {
        double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
        PairMax x{inf, 0.0, 0.0, 0.0}, x2{inf, 0.0, 0.0, 0.0};
        if (m.active) {
            int j = m.sub;
#pragma unroll 1
            for (; j + m.G < n; j += 2 * m.G) {
                if (j != m.i) pair_point_b(V, m.i, j, acc, x);
                if (j + m.G != m.i) pair_point_b(V, m.i, j + m.G, acc2, x2);
            }
            if (j < n && j != m.i) pair_point_b(V, m.i, j, acc, x);
        }
        double e0, e1, f0, f1;
        extremes_of(x, e0, e1);
        extremes_of(x2, f0, f1);
        checked_maximize(e0, f0);
        checked_maximize(e1, f1);
        double s[5];
        for (int c = 0; c < 3; ++c) s[c] = group_sum(acc[c] + acc2[c], m.G);
        s[3] = group_max(e0, m.G);
        s[4] = group_max(e1, m.G);
        if (m.active && m.sub == 0) finish_body(V, m.i, s);
    } else {
        // finish_body writes only rows pass B does not read (GA, FA, MIND, MAXI)
#pragma unroll 1
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
            PairMax x{inf, 0.0, 0.0, 0.0}, x2{inf, 0.0, 0.0, 0.0};
            int j = 0;
#pragma unroll 1
            for (; j + 1 < n; j += 2) {
                if (j != i) pair_point_b(V, i, j, acc, x);
                if (j + 1 != i) pair_point_b(V, i, j + 1, acc2, x2);
            }
            if (j < n && j != i) pair_point_b(V, i, j, acc, x);
            double s[5] = {acc[0] + acc2[0], acc[1] + acc2[1], acc[2] + acc2[2], 0, 0};
            double f0, f1;
            extremes_of(x, s[3], s[4]);
            extremes_of(x2, f0, f1);
            checked_maximize(s[3], f0);
            checked_maximize(s[4], f1);
            finish_body(V, i, s);
        }
    }
    __syncthreads();
}

// mass::orthogonalize (mass.h:147-150) of body i's frame, in place in the planes
__device__ void orthogonalize_frame(double *pl, int n, int i) {
    dd s[9];
    for (int q = 0; q < 9; ++q) s[q] = dd{pl[(size_t)(EPH_P_S_HI + q) * n + i], pl[(size_t)(EPH_P_S_LO + q) * n + i]};
    double f[9];
    for (int q = 0; q < 9; ++q) f[q] = dd_val(s[q]);
    const v3 fx = mk(f[0], f[1], f[2]), fy = mk(f[3], f[4], f[5]), fz = mk(f[6], f[7], f[8]);
    double add[9];
    for (int q = 0; q < 9; ++q) {
        const int col = q / 3, rw = q % 3;
        const v3 fc = (col == 0) ? fx : (col == 1) ? fy : fz;
        const double o0 = (col == 0 ? 1.0 : 0.0) - dot(fx, fc);
        const double o1 = (col == 1 ? 1.0 : 0.0) - dot(fy, fc);
        const double o2 = (col == 2 ? 1.0 : 0.0) - dot(fz, fc);
        add[q] = (0.5 * f[0 + rw] * o0 + 0.5 * f[3 + rw] * o1) + 0.5 * f[6 + rw] * o2;
    }
    for (int q = 0; q < 9; ++q) {
        const dd r = dd_add(s[q], dd_make(add[q]));
        pl[(size_t)(EPH_P_S_HI + q) * n + i] = r.hi;
        pl[(size_t)(EPH_P_S_LO + q) * n + i] = r.lo;
    }
}

namespace cg = cooperative_groups;

// Copy rows [row0, row0 + nrows) of the bodies [lo, hi) into the shared memory of every other CTA of the
// cluster (distributed shared memory); the cluster barrier that follows publishes them.
__device__ void broadcast_rows(const BatchView &V, int row0, int nrows, int lo, int hi, int rank) {
    cg::cluster_group cl = cg::this_cluster();
    const int cnt = hi - lo;
    for (int q = 0; q < kCluster; ++q) {
        if (q == rank) continue;
        double *peer = cl.map_shared_rank(V.T, q);
        for (int idx = threadIdx.x; idx < nrows * cnt; idx += blockDim.x) {
            const int r = row0 + idx / cnt, i = lo + idx % cnt;
            peer[r * V.ld + i] = V.T[r * V.ld + i];
        }
    }
}

// The same for FP32 rows [row0, row0 + nrows).
__device__ void broadcast_frows(const BatchView &V, int row0, int nrows, int lo, int hi, int rank) {
    cg::cluster_group cl = cg::this_cluster();
    const int cnt = hi - lo;
    float *mine = reinterpret_cast<float *>(V.T + BR_F32 * V.ld);
    for (int q = 0; q < kCluster; ++q) {
        if (q == rank) continue;
        float *peer = reinterpret_cast<float *>(cl.map_shared_rank(V.T, q) + BR_F32 * V.ld);
        for (int idx = threadIdx.x; idx < nrows * cnt; idx += blockDim.x) {
            const int r = row0 + idx / cnt, i = lo + idx % cnt;
            peer[r * V.ld + i] = mine[r * V.ld + i];
        }
    }
}

// One system on one CTA (coop = false) or on the kCluster CTAs of a cluster (coop = true), this CTA
// owning bodies [lo, hi): every CTA holds all bodies' rows, computes its own bodies' stages and passes,
// and sends the rows the other CTAs read (positions and GM after the state update, the pass-A outputs
// after pass A) to their shared memory.
template <bool MIXED>
__device__ void integrate_system(const BatchSys &Y, const BatchView &V, bool coop, int rank) {
    const int n = Y.n;
    const int lo = coop ? (int)((long long)rank * n / kCluster) : 0;
    const int hi = coop ? (int)((long long)(rank + 1) * n / kCluster) : n;
    double *pl = Y.planes;
#define PLV(p, i) pl[(size_t)(p) * n + (i)]
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            row(V, BR_R_HI + c, i) = PLV(EPH_P_R_HI + c, i);
            row(V, BR_R_LO + c, i) = PLV(EPH_P_R_LO + c, i);
            row(V, BR_V_HI + c, i) = PLV(EPH_P_V_HI + c, i);
            row(V, BR_V_LO + c, i) = PLV(EPH_P_V_LO + c, i);
            row(V, BR_NACC + c, i) = PLV(EPH_P_NACCEL + c, i);
            row(V, BR_GA + c, i) = PLV(EPH_P_GACCEL + c, i);
        }
        row(V, BR_GM, i) = PLV(EPH_P_GM, i);
        frow(V, F_GM, i) = (float)PLV(EPH_P_GM, i);
        row(V, BR_SR2, i) = PLV(EPH_P_SR2, i);
        row(V, BR_GM0, i) = PLV(EPH_P_GM0, i);
        row(V, BR_DGM, i) = PLV(EPH_P_DGM, i);
        row(V, BR_PHI, i) = PLV(EPH_P_PHI, i);
        // the loaded auxiliaries are f_0 of the first step (RungeKutta.impl:110-116)
        const v3 fa = (mk(PLV(EPH_P_GACCEL, i), PLV(EPH_P_GACCEL + 1, i), PLV(EPH_P_GACCEL + 2, i)) +
                       mk(PLV(EPH_P_DACCEL, i), PLV(EPH_P_DACCEL + 1, i), PLV(EPH_P_DACCEL + 2, i))) +
                      mk(PLV(EPH_P_NACCEL, i), PLV(EPH_P_NACCEL + 1, i), PLV(EPH_P_NACCEL + 2, i));
        row(V, BR_FA + 0, i) = fa.x;
        row(V, BR_FA + 1, i) = fa.y;
        row(V, BR_FA + 2, i) = fa.z;
        row(V, BR_MIND, i) = 0.0;   // msystem::integrate resets the maxima (mass.cpp:406)
        row(V, BR_MAXI, i) = 0.0;
    }
    __syncthreads();
    const double dt = Y.dt;
#pragma unroll 1
    for (long long step = 0; step < Y.n_step; ++step) {
#pragma unroll 1
        for (int s = 0; s < kStages; ++s) {
            // f_s of every body into the stage store; at s == 0 also x0 = x (RungeKutta.impl:113-121).
            // Each thread keeps the same bodies throughout, so what it stores it reads back itself.
            const int k = s + 1;
            const double t = Y.t_eph + dt * (b_dtk[k] + (double)step);
            const int ci0 = k * (k - 1) / 2;
#pragma unroll 1
            for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
                double *F = Y.acc + (size_t)s * kAcc * n + i;   // [stage][component][body]
                for (int c = 0; c < 3; ++c) {
                    F[(size_t)c * n] = row(V, BR_V_HI + c, i);
                    F[(size_t)(3 + c) * n] = row(V, BR_V_LO + c, i);
                    F[(size_t)(6 + c) * n] = row(V, BR_FA + c, i);
                }
                if (s == 0)
                    for (int c = 0; c < 3; ++c) {
                        Y.x0[(0 + c) * n + i] = row(V, BR_R_HI + c, i);
                        Y.x0[(3 + c) * n + i] = row(V, BR_R_LO + c, i);
                        Y.x0[(6 + c) * n + i] = row(V, BR_V_HI + c, i);
                        Y.x0[(9 + c) * n + i] = row(V, BR_V_LO + c, i);
                    }
                // state of stage k: sum_j a_kj f_j in ascending j, zero coefficients skipped
                // (RungeKutta.impl:148-162), then r = r0 + dt v, v = v0 + dt a (RungeKutta.impl:164-186)
                dd sv[3] = {dd_make(0), dd_make(0), dd_make(0)};
                double sa[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
                for (int j = 0; j < k; ++j) {
                    const dd a = dd{b_rk_hi[ci0 + j], b_rk_lo[ci0 + j]};
                    if (a.hi == 0) continue;
                    const double fa = dd_val(a);
                    const double *Fj = Y.acc + (size_t)j * kAcc * n + i;
                    for (int c = 0; c < 3; ++c) {
                        sv[c] = dd_add(sv[c], dd_mul(a, dd{Fj[(size_t)c * n], Fj[(size_t)(3 + c) * n]}));
                        sa[c] = __dadd_rn(sa[c], __dmul_rn(fa, Fj[(size_t)(6 + c) * n]));
                    }
                }
                const dd ddt = dd_make(dt);
                for (int c = 0; c < 3; ++c) {
                    const dd r = dd_add(dd{Y.x0[(0 + c) * n + i], Y.x0[(3 + c) * n + i]}, dd_mul(ddt, sv[c]));
                    const dd v = dd_add(dd{Y.x0[(6 + c) * n + i], Y.x0[(9 + c) * n + i]}, dd_make(dt * sa[c]));
                    row(V, BR_R_HI + c, i) = r.hi;
                    row(V, BR_R_LO + c, i) = r.lo;
                    row(V, BR_V_HI + c, i) = v.hi;
                    row(V, BR_V_LO + c, i) = v.lo;
                }
                row(V, BR_GM, i) = row(V, BR_GM0, i) + row(V, BR_DGM, i) * t;
                frow(V, F_GM, i) = (float)row(V, BR_GM, i);
                if (k == kStages) orthogonalize_frame(pl, n, i);
            }
            __syncthreads();
            if (coop) {
                // every CTA of the cluster has finished the previous stage's pass B, which reads these rows
                // in its own shared memory, before they are overwritten there
                cg::this_cluster().sync();
                broadcast_rows(V, BR_R_HI, BR_GM + 1 - BR_R_HI, lo, hi, rank);
                if (MIXED) broadcast_frows(V, F_GM, 1, lo, hi, rank);
                cg::this_cluster().sync();
            }
            pass_point_a(V, n, lo, hi);
            if (coop) {
                broadcast_rows(V, BR_PHI, BR_BETA2 + 1 - BR_PHI, lo, hi, rank);
                if (MIXED) broadcast_frows(V, F_PHI, F_ROWS - F_PHI, lo, hi, rank);
                cg::this_cluster().sync();
            }
            if (MIXED) pass_point_b32(V, n, lo, hi);
            else pass_point_b(V, n, lo, hi);
        }
    }
    // store (cuda_rungekutta_kernel_config::save of RungeKutta.cu:124-133); min_distance inverted (mass.cpp:436)
    const double c2 = kCB * kCB;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            PLV(EPH_P_R_HI + c, i) = row(V, BR_R_HI + c, i);
            PLV(EPH_P_R_LO + c, i) = row(V, BR_R_LO + c, i);
            PLV(EPH_P_V_HI + c, i) = row(V, BR_V_HI + c, i);
            PLV(EPH_P_V_LO + c, i) = row(V, BR_V_LO + c, i);
            PLV(EPH_P_NACCEL + c, i) = c2 * row(V, BR_NACC + c, i);
            PLV(EPH_P_GACCEL + c, i) = row(V, BR_GA + c, i);
            PLV(EPH_P_DACCEL + c, i) = 0.0;
            PLV(EPH_P_DTORQUE + c, i) = 0.0;
            PLV(EPH_P_BETA + c, i) = row(V, BR_BETA + c, i);
        }
        PLV(EPH_P_GM, i) = row(V, BR_GM, i);
        PLV(EPH_P_PHI, i) = c2 * row(V, BR_PHI, i);
        PLV(EPH_P_BETA2, i) = row(V, BR_BETA2, i);
        PLV(EPH_P_MIN_DISTANCE, i) = 1 / row(V, BR_MIND, i);
        PLV(EPH_P_MAX_INFLUENCE, i) = row(V, BR_MAXI, i);
    }
#undef PLV
    __syncthreads();
}

// Persistent CTAs in clusters of kCluster. Jobs [0, n_coop) of the queue (the large systems) are taken a
// cluster at a time and shared by its CTAs; once a cluster draws a job past them, its CTAs take the
// remaining jobs one CTA each.
template <bool MIXED>
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kBThreads, 2)
    ensemble_kernel(const BatchSys *sys, const int *order, int n_sys, int n_coop, int *next, int ld) {
    extern __shared__ __align__(16) double bsm[];
    __shared__ int s_job;
    const BatchView V{bsm, ld};
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    bool together = true;
#pragma unroll 1
    for (;;) {
        int job;
        if (together) {
            cl.sync();   // every CTA of the cluster is done with the previous job and its shared memory
            if (rank == 0 && threadIdx.x == 0) s_job = atomicAdd(next, 1);
            cl.sync();
            job = *cl.map_shared_rank(&s_job, 0);
            cl.sync();   // read by all before rank 0 may reuse s_job
            if (job >= n_sys) return;
            if (job < n_coop) {
                integrate_system<MIXED>(sys[order[job]], V, true, rank);
                continue;
            }
            together = false;
            if (rank != 0) continue;   // rank 0 keeps this job, the others draw their own
        } else {
            if (threadIdx.x == 0) s_job = atomicAdd(next, 1);
            __syncthreads();
            job = s_job;
            __syncthreads();
            if (job >= n_sys) return;
        }
        integrate_system<MIXED>(sys[order[job]], V, false, 0);
    }
}

size_t ensemble_smem(int ld) { return (size_t)BR_ROWS * ld * sizeof(double); }
constexpr size_t kBMaxSmem = 227 * 1024 - 1024;
int ensemble_max_bodies() { return (int)(kBMaxSmem / sizeof(double) / BR_ROWS) / kPad * kPad; }

bool g_batch_ready[64];
cudaError_t batch_setup(int device) {
    if (device >= 0 && device < 64 && g_batch_ready[device]) return cudaSuccess;
    double hi[EPH_RK12_NCOEF], lo[EPH_RK12_NCOEF], dtk[kStages + 1];
    rk12_expand(hi, lo, dtk);
    cudaError_t e = cudaMemcpyToSymbol(b_rk_hi, hi, sizeof(hi));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(b_rk_lo, lo, sizeof(lo));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(b_dtk, dtk, sizeof(dtk));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ensemble_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBMaxSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ensemble_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBMaxSmem);
    if (e == cudaSuccess && device >= 0 && device < 64) g_batch_ready[device] = true;
    return e;
}

}  // namespace
}  // namespace eph

using namespace eph;

struct eph_batch {
    int device = 0;
    cudaStream_t stream = nullptr;     // work stream (own_stream unless eph_batch_set_stream chose another)
    cudaStream_t own_stream = nullptr;
    int mixed = 0;                     // 1: EIH 1PN terms of the ensemble kernel in FP32 (eph_batch_set_precision)
    int coop_min = kCoopMin;           // bodies from which a system is shared by a cluster (eph_batch_set_coop_min)
    std::mutex mu;
    char err[512] = {0};
    int n_sys = 0;
    std::vector<int64_t> n_body;
    std::vector<int> point;                    // 1: ensemble kernel, 0: per-system context path
    std::vector<size_t> off;                   // offset of system s in d_planes (doubles)
    std::vector<size_t> acc_off, x0_off;       // offsets of its scratch (doubles)
    std::vector<std::vector<double>> h_full;   // host copies of the context-path systems' planes
    std::vector<std::vector<int32_t>> m_gp_nz, m_gp_nt, m_ring_nd;
    std::vector<std::vector<double>> m_gp_coef, m_ring_param, m_ring_disk;
    double *d_planes = nullptr, *d_acc = nullptr, *d_x0 = nullptr;
    BatchSys *d_sys = nullptr;
    int *d_order = nullptr, *d_next = nullptr;
    int ld = 0;                                // shared-memory row stride (largest ensemble system, padded)
    eph_ctx *ctx = nullptr;                    // context path
    int64_t launches = 0;
};

static int bfail(eph_batch *b, int code, const char *what, cudaError_t e = cudaSuccess) {
    if (b) {
        if (e != cudaSuccess) snprintf(b->err, sizeof(b->err), "%s: %s", what, cudaGetErrorString(e));
        else snprintf(b->err, sizeof(b->err), "%s", what);
    }
    return code;
}
#define BCK(call, what)                                                                                     \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return bfail(b, e_ == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, what, e_); \
    } while (0)

static void batch_free(eph_batch *b) {
    for (void *p : {(void *)b->d_planes, (void *)b->d_acc, (void *)b->d_x0, (void *)b->d_sys, (void *)b->d_order,
                    (void *)b->d_next})
        if (p) cudaFree(p);
    b->d_planes = b->d_acc = b->d_x0 = nullptr;
    b->d_sys = nullptr;
    b->d_order = b->d_next = nullptr;
    b->n_sys = 0;
}

extern "C" {

int eph_batch_create(int device, eph_batch **out) {
    if (!out) return EPH_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return EPH_ERR_ARG;
    eph_batch *b = new eph_batch();
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        batch_setup(device) != cudaSuccess) {
        delete b;
        return EPH_ERR_CUDA;
    }
    *out = b;
    return EPH_OK;
}

int eph_batch_destroy(eph_batch *b) {
    if (!b) return EPH_ERR_ARG;
    cudaSetDevice(b->device);
    batch_free(b);
    if (b->ctx) eph_ctx_destroy(b->ctx);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    else if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EPH_OK;
}

const char *eph_batch_last_error(const eph_batch *b) { return b ? b->err : "null batch"; }

int eph_batch_upload(eph_batch *b, int32_t n_sys, const int64_t *n_body, const double *const *planes,
                     const eph_models *const *models) {
    if (!b || n_sys <= 0 || !n_body || !planes) return bfail(b, EPH_ERR_ARG, "eph_batch_upload: bad arguments");
    std::lock_guard<std::mutex> lock(b->mu);
    for (int s = 0; s < n_sys; ++s) {
        if (n_body[s] <= 0 || n_body[s] > (1 << 20) || !planes[s]) return bfail(b, EPH_ERR_ARG, "eph_batch_upload: bad system");
        const eph_models *m = models ? models[s] : nullptr;
        const int n_gp = m ? m->n_gp : 0, n_ring = m ? m->n_ring : 0;
        if (n_gp < 0 || n_ring < 0 || (n_gp && (!m->gp_nz || !m->gp_nt || !m->gp_coef)) ||
            (n_ring && (!m->ring_ndisk || !m->ring_param || !m->ring_disk)))
            return bfail(b, EPH_ERR_ARG, "eph_batch_upload: bad model tables");
    }
    BCK(cudaSetDevice(b->device), "cudaSetDevice");
    batch_free(b);
    b->n_sys = n_sys;
    b->n_body.assign(n_body, n_body + n_sys);
    b->point.assign(n_sys, 0);
    b->off.assign(n_sys, 0);
    b->acc_off.assign(n_sys, 0);
    b->x0_off.assign(n_sys, 0);
    b->h_full.assign(n_sys, {});
    b->m_gp_nz.assign(n_sys, {}); b->m_gp_nt.assign(n_sys, {}); b->m_ring_nd.assign(n_sys, {});
    b->m_gp_coef.assign(n_sys, {}); b->m_ring_param.assign(n_sys, {}); b->m_ring_disk.assign(n_sys, {});
    const int nmax = ensemble_max_bodies();
    size_t tot = 0, tot_acc = 0, tot_x0 = 0;
    int ld = 0;
    for (int s = 0; s < n_sys; ++s) {
        const int n = (int)n_body[s];
        bool pt = n <= nmax;
        for (int i = 0; i < n && pt; ++i) pt = !plan_full_class(planes[s], n, i);
        b->point[s] = pt;
        if (pt) {
            b->off[s] = tot;
            b->acc_off[s] = tot_acc;
            b->x0_off[s] = tot_x0;
            tot += (size_t)EPH_NPLANES * n;
            tot_acc += (size_t)n * kStages * kAcc;
            tot_x0 += (size_t)12 * n;
            ld = std::max(ld, (n + kPad - 1) / kPad * kPad);
        } else {
            b->h_full[s].assign(planes[s], planes[s] + (size_t)EPH_NPLANES * n);
            const eph_models *m = models ? models[s] : nullptr;
            if (m && m->n_gp) {
                b->m_gp_nz[s].assign(m->gp_nz, m->gp_nz + m->n_gp);
                b->m_gp_nt[s].assign(m->gp_nt, m->gp_nt + m->n_gp);
                b->m_gp_coef[s].assign(m->gp_coef, m->gp_coef + (size_t)m->n_gp * EPH_GP_TABLE_SIZE);
            }
            if (m && m->n_ring) {
                b->m_ring_nd[s].assign(m->ring_ndisk, m->ring_ndisk + m->n_ring);
                b->m_ring_param[s].assign(m->ring_param, m->ring_param + (size_t)m->n_ring * EPH_RING_PARAMS);
                b->m_ring_disk[s].assign(m->ring_disk, m->ring_disk + (size_t)m->n_ring * EPH_RING_MAX_DISKS * 3);
            }
        }
    }
    b->ld = ld;
    if (tot) {
        BCK(cudaMalloc(&b->d_planes, tot * sizeof(double)), "cudaMalloc(batch planes)");
        BCK(cudaMalloc(&b->d_acc, tot_acc * sizeof(double)), "cudaMalloc(batch accumulators)");
        BCK(cudaMalloc(&b->d_x0, tot_x0 * sizeof(double)), "cudaMalloc(batch start states)");
        BCK(cudaMalloc(&b->d_sys, (size_t)n_sys * sizeof(BatchSys)), "cudaMalloc(batch table)");
        BCK(cudaMalloc(&b->d_order, (size_t)n_sys * sizeof(int)), "cudaMalloc(batch order)");
        BCK(cudaMalloc(&b->d_next, sizeof(int)), "cudaMalloc(batch queue)");
        for (int s = 0; s < n_sys; ++s)
            if (b->point[s])
                BCK(cudaMemcpyAsync(b->d_planes + b->off[s], planes[s], (size_t)EPH_NPLANES * n_body[s] * sizeof(double),
                                    cudaMemcpyHostToDevice, b->stream), "upload batch planes");
        BCK(cudaStreamSynchronize(b->stream), "upload batch planes");
    }
    return EPH_OK;
}

int eph_batch_integrate(eph_batch *b, const double *dt, const int64_t *n_step, double *t_eph_hi, double *t_eph_lo) {
    if (!b || !dt || !n_step || !t_eph_hi || !t_eph_lo) return bfail(b, EPH_ERR_ARG, "eph_batch_integrate: bad arguments");
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b->n_sys) return bfail(b, EPH_ERR_STATE, "no batch uploaded");
    BCK(cudaSetDevice(b->device), "cudaSetDevice");
    const int n_sys = b->n_sys;
    std::vector<BatchSys> tab(n_sys);
    std::vector<int> order;
    std::vector<double> work(n_sys, 0.0);
    for (int s = 0; s < n_sys; ++s) {
        if (!b->point[s] || n_step[s] == 0) continue;
        BatchSys &Y = tab[s];
        const int n = (int)b->n_body[s];
        Y.n = n;
        Y.pad = 0;
        // msystem::integrate: a negative step count integrates backwards (mass.cpp:401-404)
        Y.n_step = n_step[s] < 0 ? -n_step[s] : n_step[s];
        Y.dt = n_step[s] < 0 ? -dt[s] : dt[s];
        Y.t_eph = t_eph_hi[s] + t_eph_lo[s];
        Y.planes = b->d_planes + b->off[s];
        Y.acc = b->d_acc + b->acc_off[s];
        Y.x0 = b->d_x0 + b->x0_off[s];
        work[s] = (double)n * (double)n * (double)Y.n_step;
        order.push_back(s);
    }
    // the large systems (shared by a cluster) first, then the others; each group heaviest first, so the
    // last systems to start are short ones
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        const bool ca = b->n_body[a] >= b->coop_min, cc = b->n_body[c] >= b->coop_min;
        if (ca != cc) return ca;
        return work[a] > work[c];
    });
    int n_coop = 0;
    for (int s : order) n_coop += b->n_body[s] >= b->coop_min;
    if (!order.empty()) {
        BCK(cudaMemcpyAsync(b->d_sys, tab.data(), (size_t)n_sys * sizeof(BatchSys), cudaMemcpyHostToDevice, b->stream),
            "upload batch table");
        BCK(cudaMemcpyAsync(b->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream),
            "upload batch order");
        BCK(cudaMemsetAsync(b->d_next, 0, sizeof(int), b->stream), "reset batch queue");
        const size_t smem = ensemble_smem(b->ld);
        int per_sm = 0, sms = 0;
        BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ensemble_kernel<false>, kBThreads, smem), "occupancy");
        BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "SM count");
        // whole clusters; clusters that find no room start when others finish (no CTA waits on another cluster)
        int grid = std::min((int)order.size() * kCluster, std::max(per_sm * sms, kCluster));
        grid = std::max(kCluster, grid / kCluster * kCluster);
        const int nj = (int)order.size();
        if (b->mixed)
            ensemble_kernel<true><<<grid, kBThreads, smem, b->stream>>>(b->d_sys, b->d_order, nj, n_coop, b->d_next, b->ld);
        else
            ensemble_kernel<false><<<grid, kBThreads, smem, b->stream>>>(b->d_sys, b->d_order, nj, n_coop, b->d_next, b->ld);
        BCK(cudaGetLastError(), "launch ensemble kernel");
        b->launches++;
    }
    // the other systems through the per-system kernel, while the ensemble kernel runs
    for (int s = 0; s < n_sys; ++s) {
        if (b->point[s]) continue;
        if (!b->ctx) {
            const int rc = eph_ctx_create(b->device, &b->ctx);
            if (rc) return bfail(b, rc, "context for full-physics systems");
        }
        eph_models m{};
        m.n_gp = (int32_t)b->m_gp_nz[s].size();
        m.gp_nz = b->m_gp_nz[s].data();
        m.gp_nt = b->m_gp_nt[s].data();
        m.gp_coef = b->m_gp_coef[s].data();
        m.n_ring = (int32_t)b->m_ring_nd[s].size();
        m.ring_ndisk = b->m_ring_nd[s].data();
        m.ring_param = b->m_ring_param[s].data();
        m.ring_disk = b->m_ring_disk[s].data();
        int rc = eph_upload_system(b->ctx, b->n_body[s], b->h_full[s].data(), &m);
        double th = t_eph_hi[s], tl = t_eph_lo[s];
        if (!rc) rc = eph_integrate(b->ctx, dt[s], n_step[s], &th, &tl);
        if (!rc) rc = eph_download_system(b->ctx, b->h_full[s].data());
        if (rc) return bfail(b, rc, eph_last_error(b->ctx));
        b->launches++;
        t_eph_hi[s] = th;
        t_eph_lo[s] = tl;
    }
    BCK(cudaStreamSynchronize(b->stream), "ensemble kernel");
    // t_eph += dt*n_step in double-double (mass.cpp:441)
    for (int s : order) {
        const double d = n_step[s] < 0 ? -dt[s] : dt[s];
        const double a = t_eph_hi[s], c = d * (double)(n_step[s] < 0 ? -n_step[s] : n_step[s]);
        const double sum = a + c, t = sum - a;
        double e = (a - (sum - t)) + (c - t);
        e = e + (t_eph_lo[s] + 0.0);
        const double hi = sum + e;
        t_eph_lo[s] = e - (hi - sum);
        t_eph_hi[s] = hi;
    }
    return EPH_OK;
}

int eph_batch_download(eph_batch *b, double *const *planes) {
    if (!b || !planes) return bfail(b, EPH_ERR_ARG, "eph_batch_download: bad arguments");
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b->n_sys) return bfail(b, EPH_ERR_STATE, "no batch uploaded");
    BCK(cudaSetDevice(b->device), "cudaSetDevice");
    for (int s = 0; s < b->n_sys; ++s) {
        if (!planes[s]) return bfail(b, EPH_ERR_ARG, "eph_batch_download: null planes");
        const size_t bytes = (size_t)EPH_NPLANES * b->n_body[s] * sizeof(double);
        if (b->point[s])
            BCK(cudaMemcpyAsync(planes[s], b->d_planes + b->off[s], bytes, cudaMemcpyDeviceToHost, b->stream), "download batch");
        else
            memcpy(planes[s], b->h_full[s].data(), bytes);
    }
    BCK(cudaStreamSynchronize(b->stream), "download batch");
    return EPH_OK;
}

int eph_batch_set_stream(eph_batch *b, void *stream) {
    if (!b) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b->own_stream) b->own_stream = b->stream;
    b->stream = stream ? (cudaStream_t)stream : b->own_stream;
    return EPH_OK;
}

int eph_batch_set_coop_min(eph_batch *b, int bodies) {
    if (!b || bodies < 0) return bfail(b, EPH_ERR_ARG, "eph_batch_set_coop_min: bad arguments");
    std::lock_guard<std::mutex> lock(b->mu);
    b->coop_min = bodies == 0 ? kCoopMin : bodies;
    return EPH_OK;
}

int eph_batch_autotune(eph_batch *b, const double *dt, const int64_t *n_step, double step_frac, int *coop_min,
                       double *ms_tuned, double *ms_default) {
    if (!b || !dt || !n_step || !(step_frac > 0 && step_frac <= 1) || !coop_min || !ms_tuned || !ms_default)
        return bfail(b, EPH_ERR_ARG, "eph_batch_autotune: bad arguments");
    int n_sys = 0;
    size_t planes_doubles = 0;
    {
        std::lock_guard<std::mutex> lock(b->mu);
        if (!b->n_sys) return bfail(b, EPH_ERR_STATE, "no batch uploaded");
        n_sys = b->n_sys;
        for (int s = 0; s < n_sys; ++s) planes_doubles = std::max(planes_doubles, b->off[s] + (size_t)EPH_NPLANES * b->n_body[s]);
    }
    BCK(cudaSetDevice(b->device), "cudaSetDevice");
    // every trial runs the shared launch from the uploaded state with step counts scaled by step_frac (the
    // members keep their relative durations); the systems of the per-system path are left out
    std::vector<int64_t> steps(n_sys);
    for (int s = 0; s < n_sys; ++s) {
        const int64_t k = n_step[s] < 0 ? -n_step[s] : n_step[s];
        const int64_t t = k == 0 ? 0 : std::max<int64_t>(1, (int64_t)std::llround((double)k * step_frac));
        steps[s] = n_step[s] < 0 ? -t : t;
    }
    double *d_save = nullptr;
    BCK(cudaMalloc(&d_save, planes_doubles * sizeof(double)), "cudaMalloc(autotune)");
    BCK(cudaMemcpy(d_save, b->d_planes, planes_doubles * sizeof(double), cudaMemcpyDeviceToDevice), "save planes");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<double> th(n_sys), tl(n_sys);
    const int saved_coop = b->coop_min;
    for (int s = 0; s < n_sys; ++s) if (!b->point[s]) steps[s] = 0;   // ensemble members only
    int rc = EPH_OK;
    auto trial = [&](int cm, double *ms) {
        double best = 1e300;
        for (int rep = 0; rep < 2 && rc == EPH_OK; ++rep) {
            b->coop_min = cm;
            if (cudaMemcpy(b->d_planes, d_save, planes_doubles * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess) {
                rc = bfail(b, EPH_ERR_CUDA, "restore planes");
                break;
            }
            std::fill(th.begin(), th.end(), 0.0);
            std::fill(tl.begin(), tl.end(), 0.0);
            cudaEventRecord(e0, b->stream);
            rc = eph_batch_integrate(b, dt, steps.data(), th.data(), tl.data());
            cudaEventRecord(e1, b->stream);
            float t = 0;
            if (rc == EPH_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess)
                best = std::min(best, (double)t);
        }
        *ms = best;
    };
    double t_def = 1e300, t_best = 1e300;
    int best = saved_coop;
    trial(saved_coop, &t_def);
    t_best = t_def;
    for (int cm : {48, 64, 128, 192, 1 << 30}) {
        if (rc || cm == saved_coop) continue;
        double t = 1e300;
        trial(cm, &t);
        if (rc == EPH_OK && t < t_best) { t_best = t; best = cm; }
    }
    b->coop_min = rc ? saved_coop : best;
    if (cudaMemcpy(b->d_planes, d_save, planes_doubles * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess && !rc)
        rc = bfail(b, EPH_ERR_CUDA, "restore planes");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_save);
    if (rc) return rc;
    *coop_min = best;
    *ms_tuned = t_best;
    *ms_default = t_def;
    return EPH_OK;
}

int eph_batch_set_precision(eph_batch *b, int mode) {
    if (!b || (mode != EPH_PREC_FP64 && mode != EPH_PREC_MIXED)) return bfail(b, EPH_ERR_ARG, "eph_batch_set_precision: unknown mode");
    std::lock_guard<std::mutex> lock(b->mu);
    b->mixed = mode == EPH_PREC_MIXED;
    return EPH_OK;
}

int eph_batch_info(const eph_batch *b, int32_t *n_ensemble, int64_t *launches) {
    if (!b || !n_ensemble || !launches) return EPH_ERR_ARG;
    int k = 0;
    for (int s = 0; s < b->n_sys; ++s) k += b->point[s];
    *n_ensemble = k;
    *launches = b->launches;
    return EPH_OK;
}

}  // extern "C"
