// eph_serve.cu - second-stage small-body serving: massless particles integrated with adaptive RK12
// against perturbers read from a device-resident B-spline ephemeris.
//
// * Ephemeris. M perturbers, each fitted (eph_bspline_fit, src/math/interp.h:68-150) with degree-d
//   B-splines of uniform knot spacing `knot` seconds over [t0, t0 + n knot], 10 channels per body:
//   position (3), velocity (3), Newtonian acceleration / c^2 (3), potential / c^2 (1). The last four are
//   what the EIH 1PN term of a particle needs of each perturber (mass.impl:82-97); fitting them avoids an
//   O(M^2) sweep per stage, and their interpolation error enters the particle's acceleration below
//   1e-20 of it. Coefficients live in HBM as [M][n + d][10]; a stage evaluation reads, per body and
//   channel, the d + 1 coefficients of the interval and combines them with the basis values
//   B[d, x - i] (the Chebyshev form of eph_bspline_cheb_coef), as the reference's sampling does
//   (src/math/interp.h:263-280).
// * Requests. A request is P particles (double-double position and velocity), a time span and a
//   tolerance. It runs as one kernel launch of ceil(P G / 256) CTAs on one of the server's streams, G
//   lanes per particle: the smallest power of two (at most 32) that spreads the request over one block per
//   SM, so that a request's latency is that of one block's sequential stages (G = 32 below ~1200
//   particles; 16 at 4096). Each CTA integrates its particles with
//   a shared adaptive step: one RK12 step of h and two of h/2 (step doubling); the error is the largest
//   |r_h - r_h/2| / |r_h/2 - r_0| over the CTA's particles (body 0 of the ephemeris is the central star);
//   a step is accepted when it is at most tol, and the two half steps are kept; the next step is
//   h * clamp(0.9 (tol / err)^(1/13), 0.2, 4). The reference has no adaptive integrator (its RK12 table
//   has no embedded pair, RungeKutta.impl:38-104); step doubling with the same 25-stage method is the
//   estimator.
// * Admission. Requests queue on the host and launch while their device memory (state, stage store)
//   fits: by default while the device's free memory (cudaMemGetInfo at admission) stays above a 1 GiB
//   reserve, or within a fixed budget set by the caller; finished requests release their memory when their
//   results are collected.
// * Particle acceleration: Newtonian + EIH 1PN against every perturber, one sweep (the 4 phi_i term of
//   mass.impl:90 factored out as 4 phi_i a_N,i), the stage combination in the second-order form of
//   eph_particles.cu (only stage accelerations stored).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <vector>

#include "eph_bspline.h"
#include "eph_math.cuh"
#include "eph_rk12_host.h"
#include "eph_system.cuh"
#include "../../include/eph_b200.h"
#include "../../include/eph_planes.h"

namespace eph {
void ctx_record_stages(eph_ctx *ctx, double *d_buf, long long base);
long long ctx_size(const eph_ctx *ctx);
}

namespace eph {
namespace {

constexpr int kSThreads = 256;
constexpr size_t kFreeReserve = 1ull << 30;   // device memory kept free when admitting by free memory
constexpr int kSmemSlots = 64;   // particles per block whose stage store fits shared memory
constexpr int kSStreams = 128;   // requests in flight at once (the device runs up to 128 kernels concurrently)
constexpr int kChan = EPH_EPHEM_CHANNELS;   // x y z vx vy vz aN/c^2 (3) phi/c^2
constexpr double kCS = 299792458.0;         // src/math/basic_math.h:10,18
constexpr long long kMaxAttempts = 1ll << 22;
constexpr unsigned long long kRequestNs = 300ull * 1000000000ull;   // device-time limit of one request
enum SRow { S_RX = 0, S_RY, S_RZ, S_BX, S_BY, S_BZ, S_B2, S_PHI, S_NX, S_NY, S_NZ, S_GM, S_SR2, kSRows };
enum SStatus { SS_OK = 0, SS_STEP_UNDERFLOW = 1, SS_ATTEMPTS = 2, SS_DEADLINE = 3 };

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__constant__ double q_a[EPH_RK12_NCOEF];
__constant__ double q_abar[EPH_RK12_NCOEF];
__constant__ double q_c[kStages + 1];

struct ServeArgs {
    // ephemeris
    const double *coef;        // [M][n + d][kChan]
    const double *gm, *sr2;    // [M]
    const double *cheb;        // [(d + 1)^2]: c(d, k, j)
    int M, Mpad, d;
    long long n;
    double t0, knot;
    // request
    double *state;             // [12][P] in place: r hi, r lo, v hi, v lo
    double *fstore;            // [grid][kStages][3][S] (blocks of more than kSmemSlots particles)
    int P, G;
    double t_start, t_end, tol, h0, hmin;
    long long *stats;          // [grid][2]: accepted, rejected
    int *status;               // [grid]
    double *hlog;              // accepted step sizes of CTA 0, or null
    int hlog_cap;
};

__device__ __forceinline__ double group_sum(double v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// channel values of all perturbers from the interval's coefficients and the basis values b. D > 0: degree
// known at compile time, four items per pass with all their coefficient loads issued before any is used
// (they come from L2); D = 0: any degree, one item at a time.
template <int D>
__device__ __forceinline__ void eval_items(const ServeArgs &A, double *PR, const double *cheb, double u, long long xi) {
    const int d = D > 0 ? D : A.d;
    // basis values B[d, x - (xi + k)], k = 0..d, at u = 2 (x - xi) - 1 from their Chebyshev form
    constexpr int NB = D > 0 ? D + 1 : EPH_BSPLINE_MAX_DEGREE + 1;
    double b[NB];
    const double u2 = 2 * u;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (k > d) break;
        const double *c = cheb + k * (d + 1);
        double sum = c[0] + c[1] * u, tm, tt = 1, tp = u;
        for (int j = 2; j <= d; ++j) {
            tm = tt;
            tt = tp;
            tp = u2 * tt - tm;
            sum += c[j] * tp;
        }
        b[k] = sum;
    }
    const long long stride = A.n + d;
    const int total = A.M * kChan;
    constexpr int U = D > 0 ? 4 : 1;
    constexpr int NK = D > 0 ? D + 1 : EPH_BSPLINE_MAX_DEGREE + 1;
#pragma unroll 1
    for (int item0 = threadIdx.x; item0 < total; item0 += U * blockDim.x) {
        double cf[U][NK];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int item = item0 + u * blockDim.x;
            const int it = item < total ? item : total - 1;
            const double *c = A.coef + ((size_t)(it / kChan) * stride + xi) * kChan + it % kChan;
            if (D > 0) {
#pragma unroll
                for (int k = 0; k < NK; ++k) cf[u][k] = __ldg(c + (size_t)k * kChan);
            } else {
                for (int k = 0; k <= d; ++k) cf[u][k] = __ldg(c + (size_t)k * kChan);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int item = item0 + u * blockDim.x;
            if (item >= total) break;
            const int body = item / kChan, ch = item % kChan;
            double v = 0;
            if (D > 0) {
#pragma unroll
                for (int k = 0; k < NK; ++k) v += b[k] * cf[u][k];
            } else {
                for (int k = 0; k <= d; ++k) v += b[k] * cf[u][k];
            }
            const int row = ch < 3 ? S_RX + ch : ch < 6 ? S_BX + (ch - 3) : ch < 9 ? S_NX + (ch - 6) : S_PHI;
            PR[row * A.Mpad + body] = (ch >= 3 && ch < 6) ? v / kCS : v;
        }
    }
}

// all perturbers at time t into the shared rows (every thread of the CTA calls it)
__device__ void eval_perturbers(const ServeArgs &A, double *PR, const double *cheb, double t) {
    __syncthreads();   // the previous stage's readers are done
    const double x = (t - A.t0) / A.knot;
    long long xi = (long long)floor(x);
    xi = xi < 0 ? 0 : (xi > A.n - 1 ? A.n - 1 : xi);
    const double u = 2 * (x - (double)xi) - 1;
    if (A.d == 3) eval_items<3>(A, PR, cheb, u, xi);
    else eval_items<0>(A, PR, cheb, u, xi);
    __syncthreads();
    for (int j = threadIdx.x; j < A.M; j += blockDim.x) {
        const double bx = PR[S_BX * A.Mpad + j], by = PR[S_BY * A.Mpad + j], bz = PR[S_BZ * A.Mpad + j];
        PR[S_B2 * A.Mpad + j] = bx * bx + by * by + bz * bz;
    }
    __syncthreads();
}

// acceleration of a particle; the G lanes of its group split the perturbers and all get the total
__device__ v3 serve_accel(const ServeArgs &A, const double *PR, const dd r[3], const dd v[3], int lane, int G) {
    const int Mp = A.Mpad;
    const double c2 = kCS * kCS;
    const v3 bi = vdiv(mk(dd_val(v[0]), dd_val(v[1]), dd_val(v[2])), kCS);
    const double beta2 = dot(bi, bi);
    double phi = 0;
    v3 na = mk(0, 0, 0), ga = mk(0, 0, 0);
#pragma unroll 1
    for (int j = lane; j < A.M; j += G) {
        const v3 d = mk(sep_diff(PR[S_RX * Mp + j], 0.0, r[0].hi, r[0].lo), sep_diff(PR[S_RY * Mp + j], 0.0, r[1].hi, r[1].lo),
                        sep_diff(PR[S_RZ * Mp + j], 0.0, r[2].hi, r[2].lo));
        const double q = dot(d, d), sm = PR[S_SR2 * Mp + j];
        const double rr = rsqrt((q < sm) ? sm : q);
        const double tp_dphi = rr * PR[S_GM * Mp + j];
        const double tp_dg = rr * rr * tp_dphi;
        phi -= tp_dphi;
        na += tp_dg * d;
        const v3 bj = mk(PR[S_BX * Mp + j], PR[S_BY * Mp + j], PR[S_BZ * Mp + j]);
        const double rbj = dot(d, bj);
        double tp = rbj * rr;
        tp *= tp;
        const v3 naj = mk(PR[S_NX * Mp + j], PR[S_NY * Mp + j], PR[S_NZ * Mp + j]);
        const double delta1 = PR[S_PHI * Mp + j] + beta2 + 2 * PR[S_B2 * Mp + j] - 4 * dot(bi, bj) +
                              (dot(d, naj) - 3 * tp) / 2;
        const v3 b = bj - bi;
        ga += (7 * tp_dphi / 2) * naj + (tp_dg * delta1) * d + (tp_dg * (rbj - dot(d, b) * 4)) * b;
    }
    if (G > 1) {
        phi = group_sum(phi, G);
        na = mk(group_sum(na.x, G), group_sum(na.y, G), group_sum(na.z, G));
        ga = mk(group_sum(ga.x, G), group_sum(ga.y, G), group_sum(ga.z, G));
    }
    phi = phi / c2;
    ga += (4 * phi) * na;
    na = vdiv(na, c2);
    return ga + c2 * na;
}

// One RK12 step of size h from the state in Xin (shared rows [12][S]) at time t, stage accelerations in F
// (f_0 given). kFull: write the end state (r, v) to Xout and return f at it; otherwise write only the end
// position (dd, rows [6][S]) to Xout and skip the last acceleration. Xout may be Xin.
template <bool kFull>
__device__ __noinline__ v3 rk_step(const ServeArgs &A, double *PR, const double *cheb, const double *Xin, double *Xout, double *F,
                      int S, int slot, int lane, bool live, double t, double h, v3 f0) {
    const int G = A.G;
    if (lane == 0) {
        F[0] = f0.x; F[S] = f0.y; F[2 * S] = f0.z;
    }
    __syncwarp();
    dd r[3], v[3];
    v3 fa = f0;
#pragma unroll 1
    for (int k = 1; k <= kStages; ++k) {
        const int row = k * (k - 1) / 2;
        double s1[3] = {0.0, 0.0, 0.0}, s2[3] = {0.0, 0.0, 0.0};
        if (k < kStages) {
#pragma unroll 4
            for (int l = 0; l < k; ++l) {
                const double ab = q_abar[row + l], a = q_a[row + l];
                const double *Fl = F + (size_t)l * 3 * S;
                for (int c = 0; c < 3; ++c) {
                    const double f = Fl[(size_t)c * S];
                    s1[c] = __fma_rn(ab, f, s1[c]);
                    s2[c] = __fma_rn(a, f, s2[c]);
                }
            }
            const double ck = q_c[k];
            for (int c = 0; c < 3; ++c) {
                r[c] = dd_add(dd{Xin[c * S + slot], Xin[(3 + c) * S + slot]},
                              dd_make(h * __fma_rn(ck, Xin[(6 + c) * S + slot], h * s1[c])));
                v[c] = dd_add(dd{Xin[(6 + c) * S + slot], Xin[(9 + c) * S + slot]}, dd_make(h * s2[c]));
            }
        } else {
#pragma unroll 1
            for (int l = 0; l < k; ++l) {
                const double ab = q_abar[row + l], a = q_a[row + l];
                const double *Fl = F + (size_t)l * 3 * S;
                for (int c = 0; c < 3; ++c) {
                    const double f = Fl[(size_t)c * S];
                    s1[c] = __fma_rn(ab, f, s1[c]);
                    if (a != 0) s2[c] = __dadd_rn(s2[c], __dmul_rn(a, f));
                }
            }
            const dd ck = dd_make(q_c[k]), dh = dd_make(h);
            for (int c = 0; c < 3; ++c) {
                const dd v0 = dd{Xin[(6 + c) * S + slot], Xin[(9 + c) * S + slot]};
                const dd sv = dd_add(dd_mul(ck, v0), dd_make(h * s1[c]));
                r[c] = dd_add(dd{Xin[c * S + slot], Xin[(3 + c) * S + slot]}, dd_mul(dh, sv));
                v[c] = dd_add(v0, dd_make(h * s2[c]));
            }
            __syncwarp();   // every lane of the group has read Xin before lane 0 overwrites it
            if (lane == 0) {
                for (int c = 0; c < 3; ++c) {
                    Xout[c * S + slot] = r[c].hi;
                    Xout[(3 + c) * S + slot] = r[c].lo;
                    if (kFull) {
                        Xout[(6 + c) * S + slot] = v[c].hi;
                        Xout[(9 + c) * S + slot] = v[c].lo;
                    }
                }
            }
            __syncwarp();
            if (!kFull) return fa;
        }
        eval_perturbers(A, PR, cheb, t + q_c[k] * h);
        const v3 fk = serve_accel(A, PR, r, v, lane, G);   // every lane: the group sums shuffle over full warps
        if (live) fa = fk;
        if (k < kStages && lane == 0) {
            double *Fk = F + (size_t)k * 3 * S;
            Fk[0] = fa.x; Fk[S] = fa.y; Fk[2 * S] = fa.z;
        }
        __syncwarp();
    }
    return fa;
}

__global__ void __launch_bounds__(kSThreads, 2) serve_kernel(ServeArgs A) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double cheb[(EPH_BSPLINE_MAX_DEGREE + 1) * (EPH_BSPLINE_MAX_DEGREE + 1)];
    __shared__ double red[kSThreads / 32];
    const int G = A.G, S = blockDim.x / G;
    const int slot = threadIdx.x / G, lane = threadIdx.x % G;
    double *PR = sm;                          // [kSRows][Mpad]
    double *X0 = PR + kSRows * A.Mpad;        // [12][S]
    double *X1 = X0 + 12 * S;                 // [12][S]
    double *RF = X1 + 12 * S;                 // [6][S]
    // stage store [kStages][3][S]: shared memory for blocks of up to kSmemSlots particles, else global
    double *F = (S <= kSmemSlots ? RF + 6 * S : A.fstore + (size_t)blockIdx.x * kStages * 3 * S) + slot;
    const int ip = blockIdx.x * S + slot;
    const bool live = ip < A.P;
    for (int q = threadIdx.x; q < (A.d + 1) * (A.d + 1); q += blockDim.x) cheb[q] = A.cheb[q];
    for (int j = threadIdx.x; j < A.M; j += blockDim.x) {
        PR[S_GM * A.Mpad + j] = A.gm[j];
        PR[S_SR2 * A.Mpad + j] = A.sr2[j];
    }
    if (lane == 0)
        for (int q = 0; q < 12; ++q) X0[q * S + slot] = live ? A.state[(size_t)q * A.P + ip] : (q < 3 ? 1e30 : 0.0);
    __syncthreads();
    const double dir = A.t_end >= A.t_start ? 1.0 : -1.0;
    double t = A.t_start;
    // f at the start state
    eval_perturbers(A, PR, cheb, t);
    v3 f0 = mk(0, 0, 0);
    {
        dd r[3], v[3];
        for (int c = 0; c < 3; ++c) {
            r[c] = dd{X0[c * S + slot], X0[(3 + c) * S + slot]};
            v[c] = dd{X0[(6 + c) * S + slot], X0[(9 + c) * S + slot]};
        }
        const v3 fs = serve_accel(A, PR, r, v, lane, G);
        if (live) f0 = fs;
    }
    double h = fabs(A.h0);
    bool just_rejected = false;
    long long accepted = 0, rejected = 0;
    int status = SS_OK;
    __shared__ unsigned long long s_t0;
    __shared__ int s_late;
    if (threadIdx.x == 0) s_t0 = now_ns();
    __syncthreads();
#pragma unroll 1
    for (long long attempt = 0; dir * (A.t_end - t) > 0; ++attempt) {
        if (attempt >= kMaxAttempts) { status = SS_ATTEMPTS; break; }
        if (threadIdx.x == 0) s_late = now_ns() - s_t0 > kRequestNs;
        __syncthreads();
        if (s_late) { status = SS_DEADLINE; break; }
        const double remaining = dir * (A.t_end - t);
        const bool last = h >= remaining;
        const double hs = dir * (last ? remaining : h);
        rk_step<false>(A, PR, cheb, X0, RF, F, S, slot, lane, live, t, hs, f0);
        const v3 fm = rk_step<true>(A, PR, cheb, X0, X1, F, S, slot, lane, live, t, hs / 2, f0);
        const v3 fe = rk_step<true>(A, PR, cheb, X1, X1, F, S, slot, lane, live, t + hs / 2, hs / 2, fm);
        // error of the particle: |r_h - r_h/2| / |r_h/2 - r_star(t + h)| (the last stage evaluated the
        // ephemeris at t + h)
        double e = 0;
        if (live && lane == 0) {
            double num = 0, den = 0;
            for (int c = 0; c < 3; ++c) {
                const double dr = (X1[c * S + slot] - RF[c * S + slot]) + (X1[(3 + c) * S + slot] - RF[(3 + c) * S + slot]);
                const double rs = (X1[c * S + slot] - PR[(S_RX + c) * A.Mpad]) + X1[(3 + c) * S + slot];
                num += dr * dr;
                den += rs * rs;
            }
            e = sqrt(num / den);
        }
        // CTA maximum, NaN-propagating
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(0xffffffffu, e, o);
            e = (e != e || u > e || u != u) ? ((e != e) ? e : u) : e;
        }
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
        __syncthreads();
        double err = red[0];
        for (int w = 1; w < (int)(blockDim.x / 32); ++w) {
            const double u = red[w];
            err = (err != err || u > err || u != u) ? ((err != err) ? err : u) : err;
        }
        const double hused = fabs(hs);
        if (err <= A.tol) {   // accept the two half steps
            if (lane == 0)
                for (int q = 0; q < 12; ++q) X0[q * S + slot] = X1[q * S + slot];
            if (A.hlog && blockIdx.x == 0 && threadIdx.x == 0 && accepted < A.hlog_cap) A.hlog[accepted] = hs;
            f0 = fe;
            t = last ? A.t_end : t + hs;
            ++accepted;
        } else {
            ++rejected;
        }
        // next step: 0.8 (tol / err)^(1/13) within [0.25, 2], no growth right after a rejection
        // (the factor only steers the step size: single precision is ample)
        double fac = (err == 0) ? 2.0 : (err != err) ? 0.25 : 0.8 * (double)powf((float)(A.tol / err), 1.0f / 13.0f);
        fac = fac < 0.25 ? 0.25 : (fac > 2.0 ? 2.0 : fac);
        if (just_rejected && fac > 1.0) fac = 1.0;
        just_rejected = !(err <= A.tol);
        h = hused * fac;
        if (h < A.hmin && dir * (A.t_end - t) > 0) { status = SS_STEP_UNDERFLOW; break; }
        __syncwarp();
    }
    __syncthreads();
    if (live && lane == 0)
        for (int q = 0; q < 12; ++q) A.state[(size_t)q * A.P + ip] = X0[q * S + slot];
    if (threadIdx.x == 0) {
        A.stats[2 * blockIdx.x] = accepted;
        A.stats[2 * blockIdx.x + 1] = rejected;
        A.status[blockIdx.x] = status;
    }
}

// the ephemeris at time t into out[M][kChan] (one CTA)
__global__ void __launch_bounds__(kSThreads) eval_kernel(ServeArgs A, double t, double *out) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double cheb[(EPH_BSPLINE_MAX_DEGREE + 1) * (EPH_BSPLINE_MAX_DEGREE + 1)];
    for (int q = threadIdx.x; q < (A.d + 1) * (A.d + 1); q += blockDim.x) cheb[q] = A.cheb[q];
    eval_perturbers(A, sm, cheb, t);
    for (int item = threadIdx.x; item < A.M * kChan; item += blockDim.x) {
        const int body = item / kChan, ch = item % kChan;
        const int row = ch < 3 ? S_RX + ch : ch < 6 ? S_BX + (ch - 3) : ch < 9 ? S_NX + (ch - 6) : S_PHI;
        const double v = sm[row * A.Mpad + body];
        out[item] = (ch >= 3 && ch < 6) ? v * kCS : v;
    }
}

// step-end stage records of sampled steps into [samples][M][kChan]
__global__ void gather_samples(const double *traj, int M, int n_take, long long first_step, int stride, double *out) {
    // sample q of this chunk is the end of local step (first_step + q * stride); its record slot is
    // 1 + local_step * kStages + (kStages - 1)
    const long long total = (long long)n_take * M;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long q = i / M;
        const int j = (int)(i % M);
        const long long local = first_step + q * stride;
        const double *rec = traj + ((size_t)(1 + local * kStages + (kStages - 1)) * M + j) * kTrajRec;
        double *o = out + (size_t)i * kChan;
        for (int c = 0; c < 3; ++c) {
            o[c] = rec[TR_R_HI + c] + rec[TR_R_LO + c];
            o[3 + c] = rec[TR_BETA + c] * kCS;
            o[6 + c] = rec[TR_NACC + c];
        }
        o[9] = rec[TR_PHI];
    }
}

// Batch B-spline fit: right-hand side and the two banded substitutions of one (series, channel) per
// thread, with the grid's factorization from bspline_factor (eph_bspline.h). The double-double operations
// are those of the host fit (eph_bspline.cpp) in the same order, so the coefficients are bit-identical.
__global__ void bspline_solve_kernel(int d, long long m, int J, int channels, long long n_series, long long series_stride,
                                     const double *__restrict__ samples, const long long *__restrict__ jmin,
                                     const int *__restrict__ cnt, const double *__restrict__ bval,
                                     const double *__restrict__ rw, const double *__restrict__ lu,
                                     const double *__restrict__ rd, double *__restrict__ y, double *__restrict__ coefs) {
    const long long T = n_series * channels;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= T) return;
    const long long sidx = t / channels;
    const int c = (int)(t % channels);
    const int w = 2 * d + 1;
    const double *smp = samples + sidx * series_stride + c;
    // y[i] (hi, lo) at y[(2 i) * T + t], y[(2 i + 1) * T + t]
#pragma unroll 1
    for (long long i = 0; i < m; ++i) {
        dd yi = dd_make(0);
        const long long j0 = jmin[i];
#pragma unroll 1
        for (int q = 0; q < cnt[i]; ++q)
            yi = dd_add(yi, dd_mul(dd_make(smp[(j0 + q) * channels]), dd_make(bval[i * J + q])));
        yi = dd_mul(yi, dd{rw[2 * i], rw[2 * i + 1]});
#pragma unroll 1
        for (long long k = i - d < 0 ? 0 : i - d; k < i; ++k) {
            const long long qq = i * w + (k - i + d);
            yi = dd_sub(yi, dd_mul(dd{lu[2 * qq], lu[2 * qq + 1]}, dd{y[(2 * k) * T + t], y[(2 * k + 1) * T + t]}));
        }
        y[(2 * i) * T + t] = yi.hi;
        y[(2 * i + 1) * T + t] = yi.lo;
    }
#pragma unroll 1
    for (long long i = m - 1; i >= 0; --i) {
        dd yi = dd{y[(2 * i) * T + t], y[(2 * i + 1) * T + t]};
        const long long hi = i + d < m - 1 ? i + d : m - 1;
#pragma unroll 1
        for (long long j = i + 1; j <= hi; ++j) {
            const long long qq = i * w + (j - i + d);
            yi = dd_sub(yi, dd_mul(dd{lu[2 * qq], lu[2 * qq + 1]}, dd{y[(2 * j) * T + t], y[(2 * j + 1) * T + t]}));
        }
        yi = dd_mul(yi, dd{rd[2 * i], rd[2 * i + 1]});
        y[(2 * i) * T + t] = yi.hi;
        y[(2 * i + 1) * T + t] = yi.lo;
        coefs[(sidx * m + i) * channels + c] = __dadd_rn(yi.hi, yi.lo);
    }
}

bool g_serve_ready[64];
cudaError_t serve_setup(int device) {
    if (device >= 0 && device < 64 && g_serve_ready[device]) return cudaSuccess;
    double hi[EPH_RK12_NCOEF], lo[EPH_RK12_NCOEF], dtk[kStages + 1];
    rk12_expand(hi, lo, dtk);
    double a[EPH_RK12_NCOEF], abar[EPH_RK12_NCOEF] = {0};
    for (int q = 0; q < EPH_RK12_NCOEF; ++q) a[q] = hi[q] + lo[q];
    for (int k = 1; k <= kStages; ++k)
        for (int l = 0; l < k; ++l) {   // Abar = A A (second-order form), long double accumulation
            long double acc = 0;
            for (int j = l + 1; j < k; ++j)
                acc += ((long double)hi[k * (k - 1) / 2 + j] + lo[k * (k - 1) / 2 + j]) *
                       ((long double)hi[j * (j - 1) / 2 + l] + lo[j * (j - 1) / 2 + l]);
            abar[k * (k - 1) / 2 + l] = (double)acc;
        }
    cudaError_t e = cudaMemcpyToSymbol(q_a, a, sizeof(a));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(q_abar, abar, sizeof(abar));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(q_c, dtk, sizeof(dtk));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess && device >= 0 && device < 64) g_serve_ready[device] = true;
    return e;
}

size_t serve_smem(int Mpad, int S) {
    return (size_t)(kSRows * Mpad + 30 * S + (S <= kSmemSlots ? kStages * 3 * S : 0)) * sizeof(double);
}

}  // namespace
}  // namespace eph

using namespace eph;

struct eph_serve {
    int device = 0;
    std::mutex mu;
    char err[512] = {0};
    cudaStream_t streams[kSStreams] = {};
    int next_stream = 0;
    int sms = 148;
    int M = 0, Mpad = 0, d = 0;
    long long n = 0;
    double t0 = 0, knot = 0;
    double *d_coef = nullptr, *d_gm = nullptr, *d_sr2 = nullptr, *d_cheb = nullptr;
    size_t budget = 0, in_use = 0;
    int64_t log_cap = 0;
    struct Req {
        int P = 0, G = 1, grid = 0, block = kSThreads;
        double t_start = 0, t_end = 0, tol = 0, h0 = 0;
        std::vector<double> host_in;
        double *d_state = nullptr, *d_fstore = nullptr, *d_hlog = nullptr;
        long long *d_stats = nullptr;
        int *d_status = nullptr;
        cudaEvent_t done = nullptr;
        int stream = 0;
        bool launched = false;
        size_t bytes = 0;
        int64_t log_cap = 0;
    };
    std::map<int64_t, Req> reqs;
    std::deque<int64_t> pending;
    int64_t next_id = 1;
    int64_t launches = 0;
};

static int sfail(eph_serve *s, int code, const char *what, cudaError_t e = cudaSuccess) {
    if (s) {
        if (e != cudaSuccess) snprintf(s->err, sizeof(s->err), "%s: %s", what, cudaGetErrorString(e));
        else snprintf(s->err, sizeof(s->err), "%s", what);
    }
    return code;
}
#define SCK(call, what)                                                                                     \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return sfail(s, e_ == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, what, e_); \
    } while (0)

static size_t req_bytes(const eph_serve::Req &r) {
    const int S = r.block / r.G;
    return (size_t)12 * r.P * sizeof(double) + (S > kSmemSlots ? (size_t)r.grid * kStages * 3 * S * sizeof(double) : 0) +
           (size_t)r.grid * (2 * sizeof(long long) + sizeof(int)) + (size_t)r.log_cap * sizeof(double);
}

static void req_free(eph_serve::Req &r, cudaStream_t st) {
    for (void *q : {(void *)r.d_state, (void *)r.d_fstore, (void *)r.d_stats, (void *)r.d_status, (void *)r.d_hlog})
        if (q) cudaFreeAsync(q, st);
    r.d_state = r.d_fstore = r.d_hlog = nullptr;
    r.d_stats = nullptr;
    r.d_status = nullptr;
}

// launch queued requests, oldest first, while their memory fits the budget
static int pump(eph_serve *s) {
    while (!s->pending.empty()) {
        auto &r = s->reqs[s->pending.front()];
        if (s->in_use > 0) {
            if (s->budget > 0) {
                if (s->in_use + r.bytes > s->budget) break;
            } else {   // admission by free device memory
                size_t free_b = 0, total_b = 0;
                if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < r.bytes + kFreeReserve) break;
            }
        }
        cudaStream_t st = s->streams[r.stream];
        const int S = r.block / r.G;
        cudaError_t e = cudaMallocAsync((void **)&r.d_state, (size_t)12 * r.P * sizeof(double), st);
        if (e == cudaSuccess && S > kSmemSlots)
            e = cudaMallocAsync((void **)&r.d_fstore, (size_t)r.grid * kStages * 3 * S * sizeof(double), st);
        if (e == cudaSuccess) e = cudaMallocAsync((void **)&r.d_stats, (size_t)r.grid * 2 * sizeof(long long), st);
        if (e == cudaSuccess) e = cudaMallocAsync((void **)&r.d_status, (size_t)r.grid * sizeof(int), st);
        if (e == cudaSuccess && r.log_cap > 0) e = cudaMallocAsync((void **)&r.d_hlog, (size_t)r.log_cap * sizeof(double), st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(r.d_state, r.host_in.data(), r.host_in.size() * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {   // the request stays queued, holding nothing
            req_free(r, st);
            return sfail(s, e == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, "admit request", e);
        }
        ServeArgs A;
        A.coef = s->d_coef; A.gm = s->d_gm; A.sr2 = s->d_sr2; A.cheb = s->d_cheb;
        A.M = s->M; A.Mpad = s->Mpad; A.d = s->d; A.n = s->n; A.t0 = s->t0; A.knot = s->knot;
        A.state = r.d_state; A.fstore = r.d_fstore; A.P = r.P; A.G = r.G;
        A.t_start = r.t_start; A.t_end = r.t_end; A.tol = r.tol; A.h0 = r.h0;
        A.hmin = std::max(1e-9 * std::fabs(r.t_end - r.t_start), 1e-3);
        A.stats = r.d_stats; A.status = r.d_status; A.hlog = r.d_hlog; A.hlog_cap = (int)r.log_cap;
        serve_kernel<<<r.grid, r.block, serve_smem(s->Mpad, S), st>>>(A);
        SCK(cudaGetLastError(), "launch serve kernel");
        SCK(cudaEventRecord(r.done, st), "record event");
        r.launched = true;
        s->in_use += r.bytes;
        ++s->launches;
        r.host_in.clear();
        r.host_in.shrink_to_fit();
        s->pending.pop_front();
    }
    return EPH_OK;
}

extern "C" {

int eph_serve_create(int device, int64_t n_pert, const double *gm, const double *sr2, int degree, int64_t n_intervals,
                     double t0, double knot, const double *coefs, eph_serve **out) {
    if (!out) return EPH_ERR_ARG;
    *out = nullptr;
    if (n_pert < 1 || n_pert > EPH_SERVE_MAX_PERTURBERS || !gm || degree < 1 || degree > EPH_BSPLINE_MAX_DEGREE ||
        n_intervals < 1 || !(knot > 0) || !coefs)
        return EPH_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return EPH_ERR_ARG;
    eph_serve *s = new eph_serve();
    s->device = device;
    s->M = (int)n_pert;
    s->Mpad = (int)((n_pert + 1) / 2 * 2);
    s->d = degree;
    s->n = n_intervals;
    s->t0 = t0;
    s->knot = knot;
    auto bail = [&](int code, const char *what, cudaError_t e) {
        sfail(s, code, what, e);
        eph_serve_destroy(s);
        return code;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = serve_setup(device);
    for (int i = 0; i < kSStreams && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(EPH_ERR_CUDA, "serve setup", e);
    const size_t ncoef = (size_t)n_pert * (n_intervals + degree) * kChan;
    std::vector<double> cheb((degree + 1) * (degree + 1)), zeros(n_pert, 0.0);
    for (int k = 0; k <= degree; ++k)
        for (int j = 0; j <= degree; ++j) cheb[k * (degree + 1) + j] = eph_bspline_cheb_coef(degree, k, j);
    if ((e = cudaMalloc(&s->d_coef, ncoef * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_gm, n_pert * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_sr2, n_pert * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_cheb, cheb.size() * sizeof(double))) != cudaSuccess)
        return bail(e == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, "cudaMalloc(ephemeris)", e);
    if ((e = cudaMemcpy(s->d_coef, coefs, ncoef * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_gm, gm, n_pert * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_sr2, sr2 ? sr2 : zeros.data(), n_pert * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_cheb, cheb.data(), cheb.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(EPH_ERR_CUDA, "upload ephemeris", e);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    s->budget = 0;   // admission by free device memory
    *out = s;
    return EPH_OK;
}

int eph_serve_destroy(eph_serve *s) {
    if (!s) return EPH_ERR_ARG;
    cudaSetDevice(s->device);
    for (auto &kv : s->reqs) {
        if (kv.second.done) cudaEventSynchronize(kv.second.done);
        req_free(kv.second, s->streams[kv.second.stream]);
        if (kv.second.done) cudaEventDestroy(kv.second.done);
    }
    for (int i = 0; i < kSStreams; ++i)
        if (s->streams[i]) {
            cudaStreamSynchronize(s->streams[i]);
            cudaStreamDestroy(s->streams[i]);
        }
    for (void *q : {(void *)s->d_coef, (void *)s->d_gm, (void *)s->d_sr2, (void *)s->d_cheb})
        if (q) cudaFree(q);
    delete s;
    return EPH_OK;
}

const char *eph_serve_last_error(const eph_serve *s) { return s ? s->err : "null server"; }

int eph_serve_set_budget(eph_serve *s, int64_t bytes) {
    if (!s || bytes < 0) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    s->budget = (size_t)bytes;
    return EPH_OK;
}

int eph_serve_set_step_log(eph_serve *s, int64_t cap) {
    if (!s || cap < 0 || cap > (1 << 24)) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    s->log_cap = cap;
    return EPH_OK;
}

int eph_serve_submit(eph_serve *s, int64_t n_part, const double *part_state, double t_start, double t_end, double tol,
                     double h0, int64_t *id) {
    if (!s || !part_state || !id || n_part < 1 || n_part > (1 << 24) || !(tol > 0) || !(h0 > 0) ||
        !std::isfinite(t_start) || !std::isfinite(t_end))
        return sfail(s, EPH_ERR_ARG, "eph_serve_submit: bad arguments");
    std::lock_guard<std::mutex> lock(s->mu);
    const double lo = s->t0, hi = s->t0 + (double)s->n * s->knot;
    if (std::min(t_start, t_end) < lo || std::max(t_start, t_end) > hi)
        return sfail(s, EPH_ERR_ARG, "eph_serve_submit: span outside the ephemeris");
    SCK(cudaSetDevice(s->device), "cudaSetDevice");
    eph_serve::Req r;
    r.P = (int)n_part;
    // lanes per particle: split the perturber sweep until the request spans one block per SM (its latency
    // is one block's sequential stage count), at most a warp per particle
    int G = 1;
    while (G < 32 && (n_part * G + kSThreads - 1) / kSThreads < s->sms) G *= 2;
    r.G = G;
    // small requests take a smaller block (whole warps): one warp for a single particle
    r.block = (int)std::min<int64_t>(kSThreads, (n_part * G + 31) / 32 * 32);
    r.grid = (int)((n_part * G + r.block - 1) / r.block);
    r.t_start = t_start; r.t_end = t_end; r.tol = tol; r.h0 = h0;
    r.host_in.assign(part_state, part_state + (size_t)12 * n_part);
    r.stream = s->next_stream;
    s->next_stream = (s->next_stream + 1) % kSStreams;
    r.log_cap = s->log_cap;
    r.bytes = req_bytes(r);
    SCK(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming), "cudaEventCreate");
    const int64_t rid = s->next_id++;
    s->reqs.emplace(rid, std::move(r));
    s->pending.push_back(rid);
    *id = rid;
    return pump(s);
}

int eph_serve_poll(eph_serve *s, int64_t id, int *state) {
    if (!s || !state) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    SCK(cudaSetDevice(s->device), "cudaSetDevice");
    int rc = pump(s);
    if (rc) return rc;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(s, EPH_ERR_ARG, "unknown request");
    if (!it->second.launched) { *state = 0; return EPH_OK; }
    const cudaError_t e = cudaEventQuery(it->second.done);
    if (e == cudaSuccess) *state = 2;
    else if (e == cudaErrorNotReady) *state = 1;
    else return sfail(s, EPH_ERR_CUDA, "request", e);
    return EPH_OK;
}

int eph_serve_result(eph_serve *s, int64_t id, double *part_state, int64_t *n_accepted, int64_t *n_rejected,
                     double *step_log, int64_t *n_logged) {
    if (!s) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    SCK(cudaSetDevice(s->device), "cudaSetDevice");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(s, EPH_ERR_ARG, "unknown request");
    if (!it->second.launched)   // collect finished requests first: their memory admits the queue
        return sfail(s, EPH_ERR_STATE, "request is still queued for device memory");
    eph_serve::Req &r = it->second;
    SCK(cudaEventSynchronize(r.done), "request");
    cudaStream_t st = s->streams[r.stream];
    std::vector<long long> stats((size_t)r.grid * 2);
    std::vector<int> status(r.grid);
    SCK(cudaMemcpyAsync(stats.data(), r.d_stats, stats.size() * sizeof(long long), cudaMemcpyDeviceToHost, st), "stats");
    SCK(cudaMemcpyAsync(status.data(), r.d_status, status.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    if (part_state)
        SCK(cudaMemcpyAsync(part_state, r.d_state, (size_t)12 * r.P * sizeof(double), cudaMemcpyDeviceToHost, st), "results");
    std::vector<double> hl;
    if (r.d_hlog) {
        hl.resize(r.log_cap);
        SCK(cudaMemcpyAsync(hl.data(), r.d_hlog, hl.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "step log");
    }
    SCK(cudaStreamSynchronize(st), "results");
    long long acc = 0, rej = 0;   // particle-steps: each block's step counts times its particles
    int bad = 0;
    const int S = r.block / r.G;
    for (int g = 0; g < r.grid; ++g) {
        const long long live = std::min<long long>(S, (long long)r.P - (long long)g * S);
        acc += stats[2 * g] * live;
        rej += stats[2 * g + 1] * live;
        bad = bad ? bad : status[g];
    }
    if (n_accepted) *n_accepted = acc;
    if (n_rejected) *n_rejected = rej;
    if (step_log && n_logged) {
        const int64_t k = std::min<int64_t>(stats[0], r.log_cap);   // block 0's accepted steps
        std::copy(hl.begin(), hl.begin() + k, step_log);
        *n_logged = k;
    }
    req_free(r, st);
    cudaEventDestroy(r.done);
    s->in_use -= std::min(s->in_use, r.bytes);
    s->reqs.erase(it);
    const int rc = pump(s);
    if (bad)
        return sfail(s, EPH_ERR_STEP, bad == SS_STEP_UNDERFLOW ? "adaptive step fell below the minimum"
                                      : bad == SS_ATTEMPTS ? "too many step attempts" : "request exceeded its device-time limit");
    return rc;
}

int eph_serve_eval(eph_serve *s, double t, double *out) {
    if (!s || !out) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    if (!(t >= s->t0 && t <= s->t0 + (double)s->n * s->knot)) return sfail(s, EPH_ERR_ARG, "time outside the ephemeris");
    SCK(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t st = s->streams[0];
    double *d_out = nullptr;
    SCK(cudaMallocAsync((void **)&d_out, (size_t)s->M * kChan * sizeof(double), st), "cudaMallocAsync(eval)");
    ServeArgs A{};
    A.coef = s->d_coef; A.gm = s->d_gm; A.sr2 = s->d_sr2; A.cheb = s->d_cheb;
    A.M = s->M; A.Mpad = s->Mpad; A.d = s->d; A.n = s->n; A.t0 = s->t0; A.knot = s->knot;
    eval_kernel<<<1, kSThreads, (size_t)kSRows * s->Mpad * sizeof(double), st>>>(A, t, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, (size_t)s->M * kChan * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_out, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return sfail(s, EPH_ERR_CUDA, "ephemeris evaluation", e);
    return EPH_OK;
}

int eph_serve_request_shape(eph_serve *s, int64_t id, int *lanes, int *particles_per_block, int *blocks) {
    if (!s || !lanes || !particles_per_block || !blocks) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return sfail(s, EPH_ERR_ARG, "unknown request");
    *lanes = it->second.G;
    *particles_per_block = it->second.block / it->second.G;
    *blocks = it->second.grid;
    return EPH_OK;
}

int eph_serve_info(const eph_serve *s, int64_t *launches, int64_t *queued, int64_t *bytes_in_use) {
    if (!s || !launches || !queued || !bytes_in_use) return EPH_ERR_ARG;
    *launches = s->launches;
    *queued = (int64_t)s->pending.size();
    *bytes_in_use = (int64_t)s->in_use;
    return EPH_OK;
}

int eph_bspline_fit_batch(int device, int d, int64_t n, int64_t mn, int channels, int64_t n_series,
                          const double *samples, double *coefs) {
    if (channels < 1 || n_series < 1 || !samples || !coefs) return EPH_ERR_ARG;
    eph::BsplineFactor f;
    if (eph::bspline_factor(d, n, mn, f)) return EPH_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return EPH_ERR_ARG;
    const long long m = f.m, T = n_series * channels;
    auto pack = [](const std::vector<double> &h, const std::vector<double> &l) {
        std::vector<double> o(2 * h.size());
        for (size_t i = 0; i < h.size(); ++i) { o[2 * i] = h[i]; o[2 * i + 1] = l[i]; }
        return o;
    };
    const std::vector<double> rw = pack(f.rw_hi, f.rw_lo), lu = pack(f.lu_hi, f.lu_lo), rd = pack(f.rd_hi, f.rd_lo);
    const size_t n_smp = (size_t)n_series * (mn + 1) * channels, n_coef = (size_t)n_series * m * channels;
    double *d_smp = nullptr, *d_coef = nullptr, *d_y = nullptr, *d_bval = nullptr, *d_rw = nullptr, *d_lu = nullptr, *d_rd = nullptr;
    long long *d_jmin = nullptr;
    int *d_cnt = nullptr;
    int rc = EPH_OK;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    alloc((void **)&d_smp, n_smp * sizeof(double));
    alloc((void **)&d_coef, n_coef * sizeof(double));
    alloc((void **)&d_y, (size_t)2 * m * T * sizeof(double));
    alloc((void **)&d_bval, f.bval.size() * sizeof(double));
    alloc((void **)&d_rw, rw.size() * sizeof(double));
    alloc((void **)&d_lu, lu.size() * sizeof(double));
    alloc((void **)&d_rd, rd.size() * sizeof(double));
    alloc((void **)&d_jmin, f.jmin.size() * sizeof(long long));
    alloc((void **)&d_cnt, f.cnt.size() * sizeof(int));
    if (e != cudaSuccess) rc = e == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA;
    if (!rc) {
        std::vector<long long> jm(f.jmin.begin(), f.jmin.end());
        if ((e = cudaMemcpy(d_smp, samples, n_smp * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_bval, f.bval.data(), f.bval.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_rw, rw.data(), rw.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_lu, lu.data(), lu.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_rd, rd.data(), rd.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_jmin, jm.data(), jm.size() * sizeof(long long), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_cnt, f.cnt.data(), f.cnt.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess)
            rc = EPH_ERR_CUDA;
    }
    if (!rc) {
        const int threads = 128;
        bspline_solve_kernel<<<(unsigned)((T + threads - 1) / threads), threads>>>(
            d, m, f.J, channels, n_series, (long long)(mn + 1) * channels, d_smp, d_jmin, d_cnt, d_bval, d_rw, d_lu, d_rd,
            d_y, d_coef);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpy(coefs, d_coef, n_coef * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess)
            rc = EPH_ERR_CUDA;
    }
    for (void *p : {(void *)d_smp, (void *)d_coef, (void *)d_y, (void *)d_bval, (void *)d_rw, (void *)d_lu, (void *)d_rd,
                    (void *)d_jmin, (void *)d_cnt})
        if (p) cudaFree(p);
    return rc;
}

// Ephemeris samples from a context: integrates n_step steps of dt from t_eph (advanced), and writes the
// state at the start and after every `stride` steps: out[(n_step / stride) + 1][n][EPH_EPHEM_CHANNELS]
// (position, velocity, Newtonian acceleration / c^2, potential / c^2 of every body, caller order).
int eph_record_samples(eph_ctx *ctx, double dt, int64_t n_step, int64_t stride, double *t_eph_hi, double *t_eph_lo,
                       double *out) {
    if (!ctx || n_step < 0 || stride < 1 || n_step % stride != 0 || !t_eph_hi || !t_eph_lo || !out) return EPH_ERR_ARG;
    const int64_t n = ctx_size(ctx);
    if (n < 1) return EPH_ERR_STATE;
    int rc = EPH_OK;
    const size_t rec_step = (size_t)kStages * n * kTrajRec * sizeof(double);
    const int64_t chunk = std::max<int64_t>(stride, std::min<int64_t>(n_step, (int64_t)((512ull << 20) / rec_step) / stride * stride));
    double *d_traj = nullptr, *d_out = nullptr;
    const int64_t per_chunk = chunk / stride;
    if (cudaMalloc(&d_traj, (size_t)(1 + kStages * std::max<int64_t>(chunk, 1)) * n * kTrajRec * sizeof(double)) != cudaSuccess)
        return EPH_ERR_OOM;
    if (cudaMalloc(&d_out, (size_t)std::max<int64_t>(per_chunk, 1) * n * kChan * sizeof(double)) != cudaSuccess) {
        cudaFree(d_traj);
        return EPH_ERR_OOM;
    }
    // the start: from the planes (their auxiliaries are the loader's accel of this state)
    {
        std::vector<double> pl((size_t)EPH_NPLANES * n);
        rc = eph_download_system(ctx, pl.data());
        if (rc) { cudaFree(d_traj); cudaFree(d_out); return rc; }
        const double c2 = kCS * kCS;
        for (int64_t j = 0; j < n; ++j) {
            auto P = [&](int q) { return pl[(size_t)q * n + j]; };
            double *o = out + (size_t)j * kChan;
            for (int c = 0; c < 3; ++c) {
                o[c] = P(EPH_P_R_HI + c) + P(EPH_P_R_LO + c);
                o[3 + c] = P(EPH_P_V_HI + c) + P(EPH_P_V_LO + c);
                o[6 + c] = P(EPH_P_NACCEL + c) / c2;
            }
            o[9] = P(EPH_P_PHI) / c2;
        }
    }
    int64_t written = 1;
    for (int64_t done = 0; done < n_step && rc == 0;) {
        const int64_t c = std::min<int64_t>(chunk, n_step - done);
        ctx_record_stages(ctx, d_traj, 1);
        rc = eph_rk12(ctx, dt, c, *t_eph_hi, *t_eph_lo);
        ctx_record_stages(ctx, nullptr, 0);
        if (rc) break;
        const int take = (int)(c / stride);
        gather_samples<<<256, 256>>>(d_traj, (int)n, take, stride - 1, (int)stride, d_out);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(out + (size_t)written * n * kChan, d_out, (size_t)take * n * kChan * sizeof(double),
                                             cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { rc = EPH_ERR_CUDA; break; }
        written += take;
        // t_eph += dt * c in double-double (mass.cpp:441)
        const double a = *t_eph_hi, b = dt * (double)c, s = a + b, tt = s - a;
        double er = (a - (s - tt)) + (b - tt);
        er = er + (*t_eph_lo + 0.0);
        const double hsum = s + er;
        *t_eph_lo = er - (hsum - s);
        *t_eph_hi = hsum;
        done += c;
    }
    cudaFree(d_traj);
    cudaFree(d_out);
    return rc;
}

}  // extern "C"
