// eph_particles.cu - massless test particles integrated against massive perturbers.
//
// A particle feels the perturbers and nothing else, and the perturbers do not feel it, so the two
// integrations separate: the perturbers run through the single-system kernel (eph_step.cu), which records
// every stage evaluation of every perturber (position, potential, Newtonian acceleration, velocity/c,
// harmonics, spin, frames: the TrajField record); then `particle_kernel` integrates each particle on its
// own thread through the same 25 stage times, reading the perturber records of each stage from shared
// memory. Per particle and stage (the reference's terms for a point-like body i and perturber j):
//   pass A  phi_i, a_N,i of mass.impl:38-46 (floored at sR2_j: the particle has no radius)
//   prepare beta_i = v_i / c, beta_i^2, phi_i / c^2, a_N,i / c^2 (mass.impl:76-80)
//   pass B  EIH 1PN (mass.impl:82-97) with the perturbers' own prepared values; j's deformation force and
//           j's Lense-Thirring field on i (mass.impl:99-125, the j-side terms)
//   fields  geopotential and ring fields of the extended perturbers at i (mass.cpp:358-371; the reaction
//           on the perturber is GM_i times the field, zero for a massless particle)
//   final   f_i = (gaccel + daccel) + naccel (mass.cpp:389-396)
// The RK12 step is RungeKutta.impl:107-194's in second-order form (only the stage accelerations are
// stored; see particle_kernel), with its state update's arithmetic. The reference has no massless bodies;
// bodies of negligible mass
// (GM = 1e-20 m^3/s^2) in one system with the perturbers are its equivalent, and the tests compare with
// exactly that.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "eph_math.cuh"
#include "eph_models.cuh"
#include "eph_rk12_host.h"
#include "eph_system.cuh"
#include "../../include/eph_b200.h"
#include "../../include/eph_planes.h"

namespace eph {
void ctx_record_stages(eph_ctx *ctx, double *d_buf, long long base);
}

namespace eph {
namespace {

constexpr int kPThreads = 256;          // particles per CTA
constexpr int kPMaxPert = 32;           // perturbers (their stage records live in shared memory)
constexpr size_t kPRecordBytes = 1ull << 30;   // stage records of one round of perturbers then particles
constexpr double kCP = 299792458.0;     // src/math/basic_math.h:10,18
constexpr int kPF = 3;                  // stored values per (particle, stage): the acceleration

// The Feagin table as the particle kernel uses it, rows k = 1..25 at k(k-1)/2: a_kj (hi + lo rounded), the
// second-order rows Abar = A A, and the nodes c_k.
__constant__ double p_a[EPH_RK12_NCOEF];
__constant__ double p_abar[EPH_RK12_NCOEF];
__constant__ double p_c[kStages + 1];

struct PertInfo {
    int gp, ring;   // model indices, or -1
    int full;       // its deformation / spin act on others (full-class body)
    int pad;
};

struct PartArgs {
    int n_part, n_pert;
    long long n_step;
    double dt;
    const double *traj;         // [1 + kStages * n_step][n_pert][kTrajRec]
    int start_accel;            // 1: form f_0 from record slot 0 (first round); 0: f_0 is in the state
    double *state;              // [15][n_part]: r hi, r lo, v hi, v lo, f
    double *fstore;             // [gridDim][kStages][kPF][kPThreads]: stage accelerations
    const PertInfo *info;
    const int *gp_nz, *gp_nt;
    const double *gp_coef;
    const int *ring_nd;
    const double *ring_disk;
    int *next;                  // particle-block queue
};

// Field of a purely zonal geopotential (Nt = 0), inline: the Cunningham recursion of gp_core with its two
// columns (m = 0 and m = 1, the only ones zonal terms read) advanced together in one loop over the degree,
// V_k0 for a_z and V_k1 + i W_k1 for a_x, a_y, in a handful of registers, so the particle kernel keeps its
// occupancy when its only extended perturber is zonal:
//   a_z += k J_{k-1} V_k0,  a_x += J_{k-1} V_k1,  a_y += J_{k-1} W_k1   (k - 1 = 2 .. Nz), all / R^2.
__device__ __forceinline__ v3 gp_zonal(const double *__restrict__ c_table, int Nz, double R, v3 r) {
    if (Nz < 2) return mk(0, 0, 0);
    double xs, ys, zs, rho2, v00;
    gp_setup(R, r.x, r.y, r.z, xs, ys, zs, rho2, v00);
    double a0 = v00, a0p = 0;            // column 0 at degrees k, k - 1
    double b1 = xs * v00, c1 = ys * v00; // column 1 (V, W) at degree k = 1 (the diagonal)
    double b1p = 0, c1p = 0;
    a0p = a0;
    a0 = zs * v00;                       // V_10
    double ax = 0, ay = 0, az = 0;
#pragma unroll 1
    for (int k = 2; k <= Nz + 1; ++k) {
        const double kd = (double)k, f = 2 * kd - 1;
        const double n0 = (f * zs * a0 - (kd - 1) * rho2 * a0p) * __ldg(GP_RCP + k);
        const double rc = __ldg(GP_RCP + (k - 1));
        const double nb = (f * zs * b1 - kd * rho2 * b1p) * rc, nc = (f * zs * c1 - kd * rho2 * c1p) * rc;
        a0p = a0; a0 = n0;
        b1p = b1; b1 = nb;
        c1p = c1; c1 = nc;
        if (k >= 3) {
            const double J = __ldg(c_table + ((k - 1) * (k - 1) - 4));
            az += kd * (J * a0);
            ax += J * b1;
            ay += J * c1;
        }
    }
    const double s = 1.0 / (R * R);
    return mk(ax * s, ay * s, az * s);
}

// Mixed precision: the perturber fields that the FP32 form reads, as floats, kPF32 per perturber.
constexpr int kPF32 = 8;
enum F32Field { F_BETA = 0, F_NACC = 3, F_PHI = 6, F_BETA2 = 7, kF32Used = 8 };
__device__ __forceinline__ int f32_source(int k) {   // TrajField of float field k
    return k < 3 ? TR_BETA + k : k < 6 ? TR_NACC + (k - 3) : k == 6 ? TR_PHI : TR_BETA2;
}
struct f3 { float x, y, z; };
__device__ __forceinline__ f3 fk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 tof(v3 a) { return f3{(float)a.x, (float)a.y, (float)a.z}; }
__device__ __forceinline__ v3 tod(f3 a) { return v3{(double)a.x, (double)a.y, (double)a.z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 &operator+=(f3 &a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// acceleration of particle (r, v) at the stage whose perturber records are in P. One sweep over the
// perturbers: pass B's 4 phi_i term (mass.impl:90) is sum_j GM_j/r^3 * 4 phi_i * d = 4 phi_i * a_N,i, so it
// is added once after the sweep instead of waiting for phi_i; the other terms are the reference's.
// kGeneral = false: the field loop handles zonal geopotentials only (gp_zonal, inline); true: any model
// (gp_field, ring_sum: calls, whose register saves cost the kernel some spilling).
// kMixed: the EIH 1PN terms in FP32 from the float records Pf (their sum is ~(v/c)^2 ~ 1e-8 of the
// Newtonian acceleration for solar-system speeds, so FP32 rounding is ~1e-15 of it); the separations, 1/r,
// the Newtonian terms and the deformation and Lense-Thirring terms (which can reach 1e-3 of the Newtonian
// acceleration near an oblate planet) stay FP64.
template <bool kGeneral, bool kMixed>
__device__ __forceinline__ v3 particle_accel(const PartArgs &A, const double *P, const float *Pf,
                                             const PertInfo *info, const dd r[3], const dd v[3]) {
    const int np = A.n_pert;
    const double c2 = kCP * kCP;
#define PR(j, f) P[(j) * kTrajRec + (f)]
    const v3 bi = vdiv(mk(dd_val(v[0]), dd_val(v[1]), dd_val(v[2])), kCP);   // PREPARE_RELATIVITY
    const double beta2 = dot(bi, bi);
    double phi = 0;
    v3 na = mk(0, 0, 0), ga = mk(0, 0, 0), da = mk(0, 0, 0);
    const f3 bif = tof(bi);
    const float beta2f = (float)beta2;
    f3 gaf = fk(0, 0, 0);
#pragma unroll 2
    for (int j = 0; j < np; ++j) {
        const v3 d = mk(sep_diff(PR(j, TR_R_HI + 0), PR(j, TR_R_LO + 0), r[0].hi, r[0].lo),
                        sep_diff(PR(j, TR_R_HI + 1), PR(j, TR_R_LO + 1), r[1].hi, r[1].lo),
                        sep_diff(PR(j, TR_R_HI + 2), PR(j, TR_R_LO + 2), r[2].hi, r[2].lo));
        const double GMj = PR(j, TR_GM);
        const double q = dot(d, d), sm = PR(j, TR_SR2);
        const double rr = rsqrt((q < sm) ? sm : q);
        const double rr2 = rr * rr;
        const double tp_dphi = rr * GMj;
        const double tp_dg = rr2 * tp_dphi;
        phi -= tp_dphi;                                            // pass A (mass.impl:38-46)
        na += tp_dg * d;
        if (kMixed) {
            const float *Q = Pf + j * kPF32;
            const f3 df = tof(d);
            const float tpf = (float)tp_dphi, tgf = (float)tp_dg;
            const f3 bj = fk(Q[F_BETA + 0], Q[F_BETA + 1], Q[F_BETA + 2]);
            const float rbj = dot(df, bj);
            float tp = rbj * (float)rr;
            tp *= tp;
            const f3 naj = fk(Q[F_NACC + 0], Q[F_NACC + 1], Q[F_NACC + 2]);
            const float delta1 = Q[F_PHI] + beta2f + 2 * Q[F_BETA2] - 4 * dot(bif, bj) + (dot(df, naj) - 3 * tp) / 2;
            const f3 b = bj - bif;
            gaf += (7 * tpf / 2) * naj + (tgf * delta1) * df + (tgf * (rbj - dot(df, b) * 4)) * b;
            if (!info[j].full) continue;
        }
        const v3 bj = mk(PR(j, TR_BETA + 0), PR(j, TR_BETA + 1), PR(j, TR_BETA + 2));
        const v3 b = bj - bi;
        if (!kMixed) {
            const double rbj = dot(d, bj);
            double tp = rbj * rr;
            tp *= tp;
            const v3 naj = mk(PR(j, TR_NACC + 0), PR(j, TR_NACC + 1), PR(j, TR_NACC + 2));
            const double delta1 = PR(j, TR_PHI) + beta2 + 2 * PR(j, TR_BETA2) - 4 * dot(bi, bj) +
                                  (dot(d, naj) - 3 * tp) / 2;             // mass.impl:82-97 less 4 phi_i
            ga += (7 * tp_dphi / 2) * naj + (tp_dg * delta1) * d + (tp_dg * (rbj - dot(d, b) * 4)) * b;
            if (!info[j].full) continue;
        }
        const double rr3 = rr * rr2;                               // j's deformation and spin (mass.impl:99-125)
        const m3 Cj = m3{mk(PR(j, TR_CPOT + 0), PR(j, TR_CPOT + 1), PR(j, TR_CPOT + 2)),
                         mk(PR(j, TR_CPOT + 3), PR(j, TR_CPOT + 4), PR(j, TR_CPOT + 5)),
                         mk(PR(j, TR_CPOT + 6), PR(j, TR_CPOT + 7), PR(j, TR_CPOT + 8))};
        const v3 Cjr = mul(Cj, d);
        v3 dj = (GMj * rr3 * rr2 * PR(j, TR_R2)) * ((dot(d, Cjr) * 5 * rr2) * d - (Cjr + Cjr));
        const double rcr32 = 2 * GMj / kCP * rr3;
        const v3 GLj = mk(PR(j, TR_GL + 0), PR(j, TR_GL + 1), PR(j, TR_GL + 2));
        dj += cross(rcr32 * (GLj - (3 * dot(GLj, d) * rr2) * d), b);
        da += dj;
    }
    if (kMixed) ga = tod(gaf);
    phi = phi / c2;
    ga += (4 * phi) * na;
    na = vdiv(na, c2);
    // fields of the extended perturbers, r = r_particle - r_host (mass.cpp:184,198)
#pragma unroll 1
    for (int j = 0; j < np; ++j) {
        const int gp = info[j].gp, rg = info[j].ring;
        if (gp < 0 && rg < 0) continue;
        const v3 re = mk(dd_diff(r[0].hi, r[0].lo, PR(j, TR_R_HI + 0), PR(j, TR_R_LO + 0)),
                         dd_diff(r[1].hi, r[1].lo, PR(j, TR_R_HI + 1), PR(j, TR_R_LO + 1)),
                         dd_diff(r[2].hi, r[2].lo, PR(j, TR_R_HI + 2), PR(j, TR_R_LO + 2)));
        if (gp >= 0) {
            const m3 f = m3{mk(PR(j, TR_FRAME + 0), PR(j, TR_FRAME + 1), PR(j, TR_FRAME + 2)),
                            mk(PR(j, TR_FRAME + 3), PR(j, TR_FRAME + 4), PR(j, TR_FRAME + 5)),
                            mk(PR(j, TR_FRAME + 6), PR(j, TR_FRAME + 7), PR(j, TR_FRAME + 8))};
            const double *tab = A.gp_coef + (size_t)gp * EPH_GP_TABLE_SIZE;
            const int nz = A.gp_nz[gp], nt = A.gp_nt[gp];
            const v3 rl = tolocal(f, re);
            const v3 an = toworld(f, (!kGeneral || nt == 0) ? gp_zonal(tab, nz, PR(j, TR_RADIUS), rl)
                                                            : gp_field(tab, nz, nt, PR(j, TR_RADIUS), rl));
            da += PR(j, TR_GM) * an;
        }
        if (kGeneral && rg >= 0) {
            const m3 f = m3{mk(PR(j, TR_RFRAME + 0), PR(j, TR_RFRAME + 1), PR(j, TR_RFRAME + 2)),
                            mk(PR(j, TR_RFRAME + 3), PR(j, TR_RFRAME + 4), PR(j, TR_RFRAME + 5)),
                            mk(PR(j, TR_RFRAME + 6), PR(j, TR_RFRAME + 7), PR(j, TR_RFRAME + 8))};
            const v3 an = toworld(f, ring_sum(A.ring_disk + (size_t)rg * EPH_RING_MAX_DISKS * 3, A.ring_nd[rg],
                                              PR(j, TR_RADIUS), tolocal(f, re)));
            da += PR(j, TR_GM) * an;
        }
    }
#undef PR
    return (ga + da) + c2 * na;
}

template <bool kMixed>
__device__ __forceinline__ void load_records(const PartArgs &A, double *P, float *Pf, long long slot) {
    const double *src = A.traj + (size_t)slot * A.n_pert * kTrajRec;
    __syncthreads();   // everyone is done with the previous stage's records
    for (int q = threadIdx.x; q < A.n_pert * kTrajRec; q += blockDim.x) P[q] = src[q];
    if (kMixed)
        for (int q = threadIdx.x; q < A.n_pert * kF32Used; q += blockDim.x) {
            const int j = q / kF32Used, k = q % kF32Used;
            Pf[j * kPF32 + k] = (float)src[j * kTrajRec + f32_source(k)];
        }
    __syncthreads();
}

// Stage combination in second-order (Runge-Kutta-Nystrom) form. A particle's stage velocities are
// themselves combinations of its stage accelerations, v_j = v0 + dt sum_l a_jl f_l, so
//   sum_j a_kj v_j = c_k v0 + dt sum_l Abar_kl f_l,   Abar = A A (strictly lower triangular),
// and only f_l (3 doubles per stage) is stored: a third of the velocity-and-acceleration store, small enough
// to stay in L2. Stage k < 25 (dense rows, fused multiply-adds):
//   r_k = r0 + dt (c_k v0 + dt sum_l Abar_kl f_l),   v_k = v0 + dt sum_l a_kl f_l.
// The state update (row 25) keeps RungeKutta.impl:166-186's arithmetic where it sets the result's
// precision: v = v0 + dt sum_j b_j f_j summed term by term in ascending j over nonzero b_j, and
// r = r0 + dt (sum_j b_j v_j) in double-double with sum_j b_j v_j = c_25 v0 + dt sum_l Abar_25,l f_l. The
// rearranged sums differ from the reference's in rounding at ~1e-16 of the stage increment.
template <bool kGeneral, bool kMixed>
__global__ void __launch_bounds__(kPThreads, 2) particle_kernel(PartArgs A) {
    __shared__ double P[kPMaxPert * kTrajRec];
    __shared__ float Pf[kMixed ? kPMaxPert * kPF32 : 1];
    __shared__ double X0[12][kPThreads];    // the step's start state: r hi, r lo, v hi, v lo
    __shared__ PertInfo info[kPMaxPert];
    __shared__ int s_blk;
    const int t = threadIdx.x;
    for (int j = t; j < A.n_pert; j += blockDim.x) info[j] = A.info[j];
    double *F = A.fstore + (size_t)blockIdx.x * kStages * kPF * kPThreads + t;   // [stage][3] stride kPThreads
    const int nb = (A.n_part + kPThreads - 1) / kPThreads;
#pragma unroll 1
    for (;;) {
        __syncthreads();
        if (t == 0) s_blk = atomicAdd(A.next, 1);
        __syncthreads();
        const int blk = s_blk;
        if (blk >= nb) return;
        const int ip = blk * kPThreads + t;
        const bool live = ip < A.n_part;
        const int n = A.n_part;
        dd r[3], v[3];
        v3 fa = mk(0, 0, 0);
        for (int c = 0; c < 3; ++c) {
            r[c] = live ? dd{A.state[(0 + c) * n + ip], A.state[(3 + c) * n + ip]} : dd_make(1e30);
            v[c] = live ? dd{A.state[(6 + c) * n + ip], A.state[(9 + c) * n + ip]} : dd_make(0);
            X0[c][t] = r[c].hi; X0[3 + c][t] = r[c].lo;
            X0[6 + c][t] = v[c].hi; X0[9 + c][t] = v[c].lo;
        }
        if (live) fa = mk(A.state[12 * n + ip], A.state[13 * n + ip], A.state[14 * n + ip]);
        if (A.start_accel) {   // f_0 at the start state (the reference's loader runs accel(), mass_loader.cpp:555)
            load_records<kMixed>(A, P, Pf, 0);
            if (live) fa = particle_accel<kGeneral, kMixed>(A, P, Pf, info, r, v);
        }
        F[0] = fa.x;
        F[kPThreads] = fa.y;
        F[2 * kPThreads] = fa.z;
        const double dt = A.dt;
        const dd ddt = dd_make(dt);
#pragma unroll 1
        for (long long step = 0; step < A.n_step; ++step) {
#pragma unroll 1
            for (int s = 0; s < kStages; ++s) {
                const int k = s + 1, row = k * (k - 1) / 2;
                double s1[3] = {0.0, 0.0, 0.0}, s2[3] = {0.0, 0.0, 0.0};
                double *Fk;
                if (k < kStages) {
#pragma unroll 4
                    for (int l = 0; l < k; ++l) {
                        const double ab = p_abar[row + l], a = p_a[row + l];
                        const double *Fl = F + (size_t)l * kPF * kPThreads;
                        for (int c = 0; c < 3; ++c) {
                            const double f = Fl[(size_t)c * kPThreads];
                            s1[c] = __fma_rn(ab, f, s1[c]);
                            s2[c] = __fma_rn(a, f, s2[c]);
                        }
                    }
                    const double ck = p_c[k];
                    for (int c = 0; c < 3; ++c) {
                        r[c] = dd_add(dd{X0[c][t], X0[3 + c][t]}, dd_make(dt * __fma_rn(ck, X0[6 + c][t], dt * s1[c])));
                        v[c] = dd_add(dd{X0[6 + c][t], X0[9 + c][t]}, dd_make(dt * s2[c]));
                    }
                    Fk = F + (size_t)k * kPF * kPThreads;
                } else {
#pragma unroll 1
                    for (int l = 0; l < k; ++l) {
                        const double ab = p_abar[row + l], a = p_a[row + l];
                        const double *Fl = F + (size_t)l * kPF * kPThreads;
                        for (int c = 0; c < 3; ++c) {
                            const double f = Fl[(size_t)c * kPThreads];
                            s1[c] = __fma_rn(ab, f, s1[c]);
                            if (a != 0) s2[c] = __dadd_rn(s2[c], __dmul_rn(a, f));
                        }
                    }
                    const dd c25 = dd_make(p_c[k]);
                    for (int c = 0; c < 3; ++c) {
                        const dd v0 = dd{X0[6 + c][t], X0[9 + c][t]};
                        const dd sv = dd_add(dd_mul(c25, v0), dd_make(dt * s1[c]));
                        r[c] = dd_add(dd{X0[c][t], X0[3 + c][t]}, dd_mul(ddt, sv));
                        v[c] = dd_add(v0, dd_make(dt * s2[c]));
                        X0[c][t] = r[c].hi; X0[3 + c][t] = r[c].lo;
                        X0[6 + c][t] = v[c].hi; X0[9 + c][t] = v[c].lo;
                    }
                    Fk = F;   // the new state is stage 0 of the next step
                }
                load_records<kMixed>(A, P, Pf, 1 + step * kStages + s);
                if (live) fa = particle_accel<kGeneral, kMixed>(A, P, Pf, info, r, v);
                Fk[0] = fa.x;
                Fk[kPThreads] = fa.y;
                Fk[2 * kPThreads] = fa.z;
            }
        }
        if (live) {
            for (int c = 0; c < 3; ++c) {
                A.state[(0 + c) * n + ip] = X0[c][t];
                A.state[(3 + c) * n + ip] = X0[3 + c][t];
                A.state[(6 + c) * n + ip] = X0[6 + c][t];
                A.state[(9 + c) * n + ip] = X0[9 + c][t];
            }
            A.state[12 * n + ip] = fa.x;
            A.state[13 * n + ip] = fa.y;
            A.state[14 * n + ip] = fa.z;
        }
    }
}

using PartKernel = void (*)(PartArgs);
PartKernel kernel_of(bool general, bool mixed) {
    return general ? (mixed ? particle_kernel<true, true> : particle_kernel<true, false>)
                   : (mixed ? particle_kernel<false, true> : particle_kernel<false, false>);
}

bool g_part_ready[64];
cudaError_t particles_setup(int device) {
    if (device >= 0 && device < 64 && g_part_ready[device]) return cudaSuccess;
    double hi[EPH_RK12_NCOEF], lo[EPH_RK12_NCOEF], dtk[kStages + 1];
    rk12_expand(hi, lo, dtk);
    // Abar_kl = sum_{l<j<k} a_kj a_jl, accumulated in long double from the double-double coefficients
    double a[EPH_RK12_NCOEF], abar[EPH_RK12_NCOEF] = {0};
    for (int q = 0; q < EPH_RK12_NCOEF; ++q) a[q] = hi[q] + lo[q];
    for (int k = 1; k <= kStages; ++k)
        for (int l = 0; l < k; ++l) {
            long double acc = 0;
            for (int j = l + 1; j < k; ++j)
                acc += ((long double)hi[k * (k - 1) / 2 + j] + lo[k * (k - 1) / 2 + j]) *
                       ((long double)hi[j * (j - 1) / 2 + l] + lo[j * (j - 1) / 2 + l]);
            abar[k * (k - 1) / 2 + l] = (double)acc;
        }
    cudaError_t e = cudaMemcpyToSymbol(p_a, a, sizeof(a));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(p_abar, abar, sizeof(abar));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(p_c, dtk, sizeof(dtk));
    if (e == cudaSuccess && device >= 0 && device < 64) g_part_ready[device] = true;
    return e;
}

}  // namespace
}  // namespace eph

using namespace eph;

struct eph_particles {
    int device = 0;
    cudaStream_t stream = nullptr;     // work stream (own_stream unless eph_particles_set_stream chose another)
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t launches = 0;              // kernels launched (step kernel, particle kernel)
    double kernel_ms = 0;              // particle_kernel device time, summed
    std::mutex mu;
    char err[512] = {0};
    eph_ctx *ctx = nullptr;            // the perturbers
    eph_ctx *ctx0 = nullptr;           // scratch context for the start-state records
    int64_t n_pert = 0, n_part = 0;
    std::vector<double> h_pert;        // perturber planes as uploaded (for the start-state records)
    std::vector<int32_t> gp_nz, gp_nt, ring_nd;
    std::vector<double> gp_coef, ring_param, ring_disk;
    bool started = false;              // f_0 of the particles formed
    double *d_state = nullptr, *d_traj = nullptr, *d_fstore = nullptr;
    int *d_gp_nz = nullptr, *d_gp_nt = nullptr, *d_ring_nd = nullptr, *d_next = nullptr;
    double *d_gp_coef = nullptr, *d_ring_disk = nullptr;
    PertInfo *d_info = nullptr;
    size_t traj_cap = 0;
    int grid = 0;
    int64_t cap_part = 0, cap_pert = 0;  // sizes the device buffers hold
    int cap_grid = 0, cap_gp = 0, cap_ring = 0;
    bool general = false;              // a tesseral geopotential or a ring among the perturbers
    bool mixed = false;                // EPH_PREC_MIXED
};

static int pfail(eph_particles *p, int code, const char *what, cudaError_t e = cudaSuccess) {
    if (p) {
        if (e != cudaSuccess) snprintf(p->err, sizeof(p->err), "%s: %s", what, cudaGetErrorString(e));
        else snprintf(p->err, sizeof(p->err), "%s", what);
    }
    return code;
}
#define PCK(call, what)                                                                                     \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return pfail(p, e_ == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, what, e_); \
    } while (0)

static void part_free(eph_particles *p) {
    for (void *q : {(void *)p->d_state, (void *)p->d_traj, (void *)p->d_fstore, (void *)p->d_gp_nz, (void *)p->d_gp_nt,
                    (void *)p->d_ring_nd, (void *)p->d_next, (void *)p->d_gp_coef, (void *)p->d_ring_disk,
                    (void *)p->d_info})
        if (q) cudaFree(q);
    p->d_state = p->d_traj = p->d_fstore = nullptr;
    p->d_gp_nz = p->d_gp_nt = p->d_ring_nd = p->d_next = nullptr;
    p->d_gp_coef = p->d_ring_disk = nullptr;
    p->d_info = nullptr;
    p->traj_cap = 0;
    p->cap_part = p->cap_pert = 0;
    p->cap_grid = p->cap_gp = p->cap_ring = 0;
}

// t += d in double-double (mass.cpp:441)
static void dd_advance(double *hi, double *lo, double d) {
    const double a = *hi, s = a + d, t = s - a;
    double e = (a - (s - t)) + (d - t);
    e = e + (*lo + 0.0);
    const double h = s + e;
    *lo = e - (h - s);
    *hi = h;
}

extern "C" {

int eph_particles_create(int device, eph_particles **out) {
    if (!out) return EPH_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return EPH_ERR_ARG;
    eph_particles *p = new eph_particles();
    p->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&p->ev0) != cudaSuccess || cudaEventCreate(&p->ev1) != cudaSuccess ||
        particles_setup(device) != cudaSuccess || eph_ctx_create(device, &p->ctx) != EPH_OK ||
        eph_ctx_create(device, &p->ctx0) != EPH_OK) {
        eph_particles_destroy(p);
        return EPH_ERR_CUDA;
    }
    p->stream = p->own_stream;
    *out = p;
    return EPH_OK;
}

int eph_particles_destroy(eph_particles *p) {
    if (!p) return EPH_ERR_ARG;
    cudaSetDevice(p->device);
    part_free(p);
    if (p->ctx) eph_ctx_destroy(p->ctx);
    if (p->ctx0) eph_ctx_destroy(p->ctx0);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
    delete p;
    return EPH_OK;
}

const char *eph_particles_last_error(const eph_particles *p) { return p ? p->err : "null particle set"; }

int eph_particles_set_stream(eph_particles *p, void *stream) {
    if (!p) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(p->mu);
    p->stream = stream ? (cudaStream_t)stream : p->own_stream;
    int rc = eph_set_stream(p->ctx, stream);
    if (!rc) rc = eph_set_stream(p->ctx0, stream);
    return rc;
}

int eph_particles_set_precision(eph_particles *p, int mode) {
    if (!p || (mode != EPH_PREC_FP64 && mode != EPH_PREC_MIXED)) return pfail(p, EPH_ERR_ARG, "bad precision mode");
    std::lock_guard<std::mutex> lock(p->mu);
    p->mixed = mode == EPH_PREC_MIXED;
    return EPH_OK;
}

int eph_particles_info(const eph_particles *p, int64_t *launches, double *particle_kernel_ms) {
    if (!p || !launches || !particle_kernel_ms) return EPH_ERR_ARG;
    *launches = p->launches;
    *particle_kernel_ms = p->kernel_ms;
    return EPH_OK;
}

int eph_particles_upload(eph_particles *p, int64_t n_pert, const double *pert_planes, const eph_models *models,
                         int64_t n_part, const double *part_state) {
    if (!p || n_pert <= 0 || n_pert > kPMaxPert || !pert_planes || n_part <= 0 || n_part > (1ll << 31) / 16 || !part_state)
        return pfail(p, n_pert > kPMaxPert ? EPH_ERR_LIMIT : EPH_ERR_ARG, "eph_particles_upload: bad arguments");
    std::lock_guard<std::mutex> lock(p->mu);
    PCK(cudaSetDevice(p->device), "cudaSetDevice");
    int rc = eph_upload_system(p->ctx, n_pert, pert_planes, models);
    if (rc) return pfail(p, rc, eph_last_error(p->ctx));
    p->n_pert = n_pert;
    p->n_part = n_part;
    p->h_pert.assign(pert_planes, pert_planes + (size_t)EPH_NPLANES * n_pert);
    const int n_gp = models ? models->n_gp : 0, n_ring = models ? models->n_ring : 0;
    p->gp_nz.assign(n_gp ? models->gp_nz : nullptr, n_gp ? models->gp_nz + n_gp : nullptr);
    p->gp_nt.assign(n_gp ? models->gp_nt : nullptr, n_gp ? models->gp_nt + n_gp : nullptr);
    p->gp_coef.assign(n_gp ? models->gp_coef : nullptr, n_gp ? models->gp_coef + (size_t)n_gp * EPH_GP_TABLE_SIZE : nullptr);
    p->ring_nd.assign(n_ring ? models->ring_ndisk : nullptr, n_ring ? models->ring_ndisk + n_ring : nullptr);
    p->ring_param.assign(n_ring ? models->ring_param : nullptr, n_ring ? models->ring_param + (size_t)n_ring * 4 : nullptr);
    p->ring_disk.assign(n_ring ? models->ring_disk : nullptr,
                        n_ring ? models->ring_disk + (size_t)n_ring * EPH_RING_MAX_DISKS * 3 : nullptr);
    std::vector<PertInfo> info(n_pert);
    for (int j = 0; j < n_pert; ++j) {
        auto P = [&](int q) { return pert_planes[(size_t)q * n_pert + j]; };
        info[j].gp = (int)P(EPH_P_GP_INDEX);
        info[j].ring = (int)P(EPH_P_RING_INDEX);
        bool full = P(EPH_P_K2) != 0 || P(EPH_P_K2R) != 0 || P(EPH_P_DJ2) != 0 || P(EPH_P_LUM) != 0 ||
                    P(EPH_P_RR2G_4C) != 0 || info[j].gp >= 0 || info[j].ring >= 0;
        for (int q = 0; q < 9; ++q) full = full || P(EPH_P_C_STATIC + q) != 0;
        for (int c = 0; c < 3; ++c) full = full || P(EPH_P_W + c) != 0 || P(EPH_P_GL_HI + c) != 0 || P(EPH_P_GL_LO + c) != 0;
        info[j].full = full;
        info[j].pad = 0;
    }
    int per_sm = 0, sms = 0;
    p->general = false;
    for (int j = 0; j < n_pert; ++j)
        p->general = p->general || info[j].ring >= 0 || (info[j].gp >= 0 && p->gp_nt[info[j].gp] > 0);
    PCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_of(p->general, p->mixed), kPThreads, 0),
        "occupancy");
    PCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device), "SM count");
    const int64_t nblk = (n_part + kPThreads - 1) / kPThreads;
    p->grid = (int)std::max<int64_t>(1, std::min<int64_t>(nblk, (int64_t)per_sm * sms));
    // device buffers are kept across uploads while they are large enough (a repeated upload of the same
    // sizes allocates nothing)
    if (n_part > p->cap_part || p->grid > p->cap_grid || n_pert > p->cap_pert || std::max(n_gp, 1) > p->cap_gp ||
        std::max(n_ring, 1) > p->cap_ring) {
        part_free(p);
        p->cap_part = n_part;
        p->cap_grid = p->grid;
        p->cap_pert = n_pert;
        p->cap_gp = std::max(n_gp, 1);
        p->cap_ring = std::max(n_ring, 1);
        PCK(cudaMalloc(&p->d_state, (size_t)15 * n_part * sizeof(double)), "cudaMalloc(particles)");
        PCK(cudaMalloc(&p->d_fstore, (size_t)p->grid * kStages * kPF * kPThreads * sizeof(double)), "cudaMalloc(stage store)");
        PCK(cudaMalloc(&p->d_info, n_pert * sizeof(PertInfo)), "cudaMalloc(perturbers)");
        PCK(cudaMalloc(&p->d_next, sizeof(int)), "cudaMalloc(queue)");
        PCK(cudaMalloc(&p->d_gp_nz, p->cap_gp * sizeof(int)), "cudaMalloc(gp)");
        PCK(cudaMalloc(&p->d_gp_nt, p->cap_gp * sizeof(int)), "cudaMalloc(gp)");
        PCK(cudaMalloc(&p->d_gp_coef, (size_t)p->cap_gp * EPH_GP_TABLE_SIZE * sizeof(double)), "cudaMalloc(gp)");
        PCK(cudaMalloc(&p->d_ring_nd, p->cap_ring * sizeof(int)), "cudaMalloc(ring)");
        PCK(cudaMalloc(&p->d_ring_disk, (size_t)p->cap_ring * EPH_RING_MAX_DISKS * 3 * sizeof(double)), "cudaMalloc(ring)");
    }
    // particle state [15][n_part]: r hi, r lo, v hi, v lo straight from the caller's rows (a pinned caller
    // buffer is a DMA), then f, formed at the first integration
    PCK(cudaMemcpyAsync(p->d_state, part_state, (size_t)12 * n_part * sizeof(double), cudaMemcpyHostToDevice, p->stream),
        "upload particles");
    PCK(cudaMemsetAsync(p->d_state + (size_t)12 * n_part, 0, (size_t)3 * n_part * sizeof(double), p->stream), "clear f");
    PCK(cudaStreamSynchronize(p->stream), "upload particles");
    PCK(cudaMemcpy(p->d_info, info.data(), n_pert * sizeof(PertInfo), cudaMemcpyHostToDevice), "upload perturbers");
    if (n_gp) {
        PCK(cudaMemcpy(p->d_gp_nz, p->gp_nz.data(), n_gp * sizeof(int), cudaMemcpyHostToDevice), "upload gp");
        PCK(cudaMemcpy(p->d_gp_nt, p->gp_nt.data(), n_gp * sizeof(int), cudaMemcpyHostToDevice), "upload gp");
        PCK(cudaMemcpy(p->d_gp_coef, p->gp_coef.data(), p->gp_coef.size() * sizeof(double), cudaMemcpyHostToDevice), "upload gp");
    }
    if (n_ring) {
        PCK(cudaMemcpy(p->d_ring_nd, p->ring_nd.data(), n_ring * sizeof(int), cudaMemcpyHostToDevice), "upload ring");
        PCK(cudaMemcpy(p->d_ring_disk, p->ring_disk.data(), p->ring_disk.size() * sizeof(double), cudaMemcpyHostToDevice),
            "upload ring");
    }
    p->started = false;
    return EPH_OK;
}

int eph_particles_integrate(eph_particles *p, double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo) {
    if (!p || !t_eph_hi || !t_eph_lo) return pfail(p, EPH_ERR_ARG, "eph_particles_integrate: bad arguments");
    std::lock_guard<std::mutex> lock(p->mu);
    if (!p->n_part) return pfail(p, EPH_ERR_STATE, "no particles uploaded");
    if (n_step == 0) return EPH_OK;
    if (n_step < 0) {   // mass.cpp:401-404
        n_step = -n_step;
        dt = -dt;
    }
    PCK(cudaSetDevice(p->device), "cudaSetDevice");
    const size_t rec = (size_t)p->n_pert * kTrajRec;
    // steps per round: all of them while their stage records fit kPRecordBytes
    const int64_t chunk = std::max<int64_t>(1, (int64_t)(kPRecordBytes / (sizeof(double) * kStages * rec)));
    const size_t need = (size_t)(1 + kStages * std::min<int64_t>(n_step, chunk)) * rec;
    if (need > p->traj_cap) {
        if (p->d_traj) cudaFree(p->d_traj);
        p->d_traj = nullptr;
        PCK(cudaMalloc(&p->d_traj, need * sizeof(double)), "cudaMalloc(stage records)");
        p->traj_cap = need;
    }
    int rc;
    if (!p->started) {
        // the perturbers' records at the start state (slot 0), from a scratch copy so that their own
        // integration starts exactly from the uploaded state
        eph_models m{};
        m.n_gp = (int32_t)p->gp_nz.size();
        m.gp_nz = p->gp_nz.data(); m.gp_nt = p->gp_nt.data(); m.gp_coef = p->gp_coef.data();
        m.n_ring = (int32_t)p->ring_nd.size();
        m.ring_ndisk = p->ring_nd.data(); m.ring_param = p->ring_param.data(); m.ring_disk = p->ring_disk.data();
        rc = eph_upload_system(p->ctx0, p->n_pert, p->h_pert.data(), &m);
        ctx_record_stages(p->ctx0, p->d_traj, 0);
        if (!rc) rc = eph_accel(p->ctx0);
        ctx_record_stages(p->ctx0, nullptr, 0);
        ++p->launches;
        if (rc) return pfail(p, rc, eph_last_error(p->ctx0));
    }
    // msystem::integrate: maxima reset before, min_distance inverted after (mass.cpp:406,436)
    double *d_pl = nullptr;
    eph_device_planes(p->ctx, &d_pl);
    PCK(cudaMemset(d_pl + (size_t)EPH_P_MIN_DISTANCE * p->n_pert, 0, 2 * p->n_pert * sizeof(double)), "reset maxima");
    for (int64_t done = 0; done < n_step;) {
        const int64_t c = std::min<int64_t>(n_step - done, chunk);
        ctx_record_stages(p->ctx, p->d_traj, 1);
        rc = eph_rk12(p->ctx, dt, c, *t_eph_hi, *t_eph_lo);
        ctx_record_stages(p->ctx, nullptr, 0);
        ++p->launches;
        if (rc) return pfail(p, rc, eph_last_error(p->ctx));
        PartArgs A;
        A.n_part = (int)p->n_part;
        A.n_pert = (int)p->n_pert;
        A.n_step = c;
        A.dt = dt;
        A.traj = p->d_traj;
        A.start_accel = p->started ? 0 : 1;
        A.state = p->d_state;
        A.fstore = p->d_fstore;
        A.info = p->d_info;
        A.gp_nz = p->d_gp_nz; A.gp_nt = p->d_gp_nt; A.gp_coef = p->d_gp_coef;
        A.ring_nd = p->d_ring_nd; A.ring_disk = p->d_ring_disk;
        A.next = p->d_next;
        PCK(cudaMemsetAsync(p->d_next, 0, sizeof(int), p->stream), "reset queue");
        PCK(cudaEventRecord(p->ev0, p->stream), "event");
        kernel_of(p->general, p->mixed)<<<p->grid, kPThreads, 0, p->stream>>>(A);
        PCK(cudaGetLastError(), "launch particle kernel");
        ++p->launches;
        PCK(cudaEventRecord(p->ev1, p->stream), "event");
        PCK(cudaStreamSynchronize(p->stream), "particle kernel");
        float ms = 0;
        PCK(cudaEventElapsedTime(&ms, p->ev0, p->ev1), "event time");
        p->kernel_ms += ms;
        p->started = true;
        dd_advance(t_eph_hi, t_eph_lo, dt * (double)c);
        done += c;
    }
    std::vector<double> md(p->n_pert);
    PCK(cudaMemcpy(md.data(), d_pl + (size_t)EPH_P_MIN_DISTANCE * p->n_pert, p->n_pert * sizeof(double),
                   cudaMemcpyDeviceToHost), "maxima");
    for (auto &x : md) x = 1 / x;
    PCK(cudaMemcpy(d_pl + (size_t)EPH_P_MIN_DISTANCE * p->n_pert, md.data(), p->n_pert * sizeof(double),
                   cudaMemcpyHostToDevice), "maxima");
    return EPH_OK;
}

int eph_particles_download(eph_particles *p, double *pert_planes, double *part_state) {
    if (!p) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(p->mu);
    if (!p->n_part) return pfail(p, EPH_ERR_STATE, "no particles uploaded");
    PCK(cudaSetDevice(p->device), "cudaSetDevice");
    if (pert_planes) {
        const int rc = eph_download_system(p->ctx, pert_planes);
        if (rc) return pfail(p, rc, eph_last_error(p->ctx));
    }
    if (part_state) {
        PCK(cudaMemcpyAsync(part_state, p->d_state, (size_t)12 * p->n_part * sizeof(double), cudaMemcpyDeviceToHost,
                            p->stream), "download particles");
        PCK(cudaStreamSynchronize(p->stream), "download particles");
    }
    return EPH_OK;
}

}  // extern "C"
