// eph_step.cu - the RK12 step of one system of bodies as a single persistent cooperative kernel.
//
// Reference path replaced: msystem::Cuda_RungeKutta12 / Cuda_RungeKutta_Kernel
// (src/integrators/RungeKutta.cu:391-412, RungeKutta.impl:107-194) and msystem::Cuda_accel
// (RungeKutta.cu:348-375,414-438). The physics is that of the CPU integrator (src/physics/mass.cpp:78-397,
// mass.impl:1-152); the schedule is new:
//
//   * every CTA owns up to kOwnMax bodies for the whole launch and keeps their private state (start of
//     step, the 25 RK12 stage accumulators, auxiliaries) in shared memory;
//   * one stage evaluation is two O(N^2) sweeps separated by grid barriers:
//       pass A  - potential, Newtonian acceleration and tidal matrix of each owned body, summed over all
//                 bodies j by the CTA's threads (threads stride over j; pair sums stay in registers for
//                 up to kRegBodies owned bodies so each j is loaded once), reduced with warp shuffles;
//                 then the harmonics update and the angular-velocity fixed point per body (mass.impl:48-80);
//       pass B  - 1PN, deformation, Lense-Thirring, radiation and extended-body forces, reduced the same way,
//                 followed by the finalisation, the RK12 stage combination and the state update of the
//                 owned bodies (all private, so no barrier is needed between them);
//   * the stage state other CTAs read is double-buffered (ping-pong), so pass B of stage k and the state
//     update for stage k+1 need no barrier between them: 2 barriers per stage, 50 per step;
//   * the RK12 combination sum_j a_kj f_j is accumulated incrementally: when f_j is known it is added into
//     the accumulators of every later stage k, in ascending j, which is the reference's summation order.
//
// The grid barrier waits are bounded (kBarrierTimeoutNs): on timeout the kernel records
// ST_BARRIER_TIMEOUT in the status word and returns; it never traps.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "eph_math.cuh"
#include "eph_models.cuh"
#include "eph_system.cuh"
#include "../../include/eph_planes.h"
#include "../../include/eph_rk12_table.h"

namespace eph {

constexpr double kC = 299792458.0;                      // src/math/basic_math.h:10,18
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;

__constant__ double c_rk_hi[EPH_RK12_NCOEF];            // a_kj, double-double
__constant__ double c_rk_lo[EPH_RK12_NCOEF];
__constant__ double c_dtk[kStages + 1];                 // c_k = sum of nonzero a_kj, summed in j order

// ------------------------------------------------------------------ owned-body private state (shared memory)
struct Own {
    int idx, kind, gp, ring;          // kind: 0 point Newtonian (k2 == 0), 1 undelayed tide, 2 delayed tide
    int converged, swept, pad0, pad1;
    double GM0, dGM, dJ2, R, R2, A, k2, k2r, td, sR2, rR2G4c;
    double Cst[9];
    double ring_GM_ratio, ring_GL_R2;
    // current stage state
    dd r[3], v[3], GL[3], s[9];
    double w[3], GM, exJ2;
    // start of step
    dd r0[3], v0[3], GL0[3], s0[9];
    double w0[3];
    // auxiliaries
    double phi, nacc[3], C[9], GI[9], beta[3], beta2;
    double gacc[3], dacc[3], dtq[3], Egrad[3], mind, maxi;
    double sumA[13];
    double fa[3];                     // f_s acceleration of the current stage
    double gpf[9], rgf[9];            // geopotential frame (rounded s) and ring frame, fixed within a pass
    int gl_fixed, pad2;
    // RK12 accumulators of stages k = 1..25 (index k-1)
    dd accv[kStages][3];
    double acca[kStages][3], accw[kStages][3], acct[kStages][3];
};

struct Scratch {
    double red[kThreads / 32][kRegBodies][13];
    double ext[kOwnMax][kMaxExt][3];
    unsigned long long t_last, t_phase[kPhases];
    int flag;
};

__device__ __forceinline__ unsigned long long global_ns();

// Optional phase timers: thread 0 charges the time since the previous mark to phase `ph`. Marks sit
// right after a __syncthreads(), so they bound the whole CTA's work of the phase.
__device__ __forceinline__ void mark(const SysDev &S, Scratch &sc, int ph) {
    if (S.timers && threadIdx.x == 0) {
        unsigned long long t = global_ns();
        sc.t_phase[ph] += t - sc.t_last;
        sc.t_last = t;
    }
}

// ------------------------------------------------------------------ small helpers
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Barrier over all CTAs of the launch (co-resident by the cooperative launch). Returns false when the
// wait timed out here or elsewhere (status word set); the caller then leaves the kernel.
__device__ bool grid_sync(const SysDev &S, Scratch &sc) {
    __syncthreads();
    if (gridDim.x == 1) return true;
    if (threadIdx.x == 0) {
        unsigned *count = S.bar, *gen = S.bar + 1;
        unsigned g = ld_acquire(gen);
        __threadfence();
        unsigned prev = atomicAdd(count, 1u);
        int fail = 0;
        if (prev == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            unsigned long long t0 = global_ns();
            while (ld_acquire(gen) == g) {
                if (global_ns() - t0 > kBarrierTimeoutNs) {
                    atomicExch(S.status, (int)ST_BARRIER_TIMEOUT);
                    fail = 1;
                    break;
                }
            }
        }
        __threadfence();
        if (*(volatile int *)S.status != ST_OK) fail = 1;
        sc.flag = fail;
    }
    __syncthreads();
    return sc.flag == 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_cmax(double v) {   // NaN-propagating maximum
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double u = __shfl_xor_sync(0xffffffffu, v, o);
        checked_maximize(v, u);
    }
    return v;
}

__device__ __forceinline__ v3 ld3(const double *p, int n, int i) {
    return mk(__ldcg(p + i), __ldcg(p + n + i), __ldcg(p + 2 * n + i));
}
__device__ __forceinline__ m3 ld9(const double *p, int n, int i) {
    return m3{ld3(p, n, i), ld3(p + 3 * n, n, i), ld3(p + 6 * n, n, i)};
}
__device__ __forceinline__ v3 fast3(const dd *a) { return mk(dd_val(a[0]), dd_val(a[1]), dd_val(a[2])); }
__device__ __forceinline__ m3 fast9(const dd *a) { return m3{fast3(a), fast3(a + 3), fast3(a + 6)}; }
__device__ __forceinline__ v3 ldv(const double *a) { return mk(a[0], a[1], a[2]); }
__device__ __forceinline__ void stv(double *a, v3 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }
__device__ __forceinline__ m3 ldm(const double *a) { return m3{ldv(a), ldv(a + 3), ldv(a + 6)}; }
__device__ __forceinline__ void stm(double *a, m3 m) { stv(a, m.x); stv(a + 3, m.y); stv(a + 6, m.z); }

// ring frame of a host: x = ascending node of G*L, z = unit G*L, y = z x x (mass.cpp:366-368, vec_t.h:281)
__device__ __forceinline__ m3 ring_frame(v3 gl) {
    v3 p = mk(-gl.y, gl.x, 0);
    normalize2(p.y, p.x);
    v3 z = gl;
    normalize(z);
    return m3{p, cross(z, p), z};
}

// ------------------------------------------------------------------ load / publish / store
__device__ void load_own(const SysDev &S, Own *own, int nb, const StepParams &P) {
    const int n = S.n;
    const double *pl = S.planes;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &o = own[b];
        const int i = o.idx;
#define PLV(p) pl[(size_t)(p) * n + i]
        o.GM0 = PLV(EPH_P_GM0); o.dGM = PLV(EPH_P_DGM); o.dJ2 = PLV(EPH_P_DJ2); o.R = PLV(EPH_P_RADIUS);
        o.R2 = PLV(EPH_P_R2); o.A = PLV(EPH_P_A); o.k2 = PLV(EPH_P_K2); o.k2r = PLV(EPH_P_K2R);
        o.td = PLV(EPH_P_TIDE_DELAY); o.sR2 = PLV(EPH_P_SR2); o.rR2G4c = PLV(EPH_P_RR2G_4C);
        for (int q = 0; q < 9; ++q) o.Cst[q] = PLV(EPH_P_C_STATIC + q);
        o.kind = (o.k2 != 0) ? ((o.td != 0) ? 2 : 1) : 0;
        o.gp = (int)PLV(EPH_P_GP_INDEX);
        o.ring = (int)PLV(EPH_P_RING_INDEX);
        o.ring_GM_ratio = o.ring >= 0 ? S.ring_param[o.ring * 4 + 0] : 0.0;
        o.ring_GL_R2 = o.ring >= 0 ? S.ring_param[o.ring * 4 + 3] : 0.0;
        for (int c = 0; c < 3; ++c) {
            o.r[c] = dd{PLV(EPH_P_R_HI + c), PLV(EPH_P_R_LO + c)};
            o.v[c] = dd{PLV(EPH_P_V_HI + c), PLV(EPH_P_V_LO + c)};
            o.GL[c] = dd{PLV(EPH_P_GL_HI + c), PLV(EPH_P_GL_LO + c)};
            o.w[c] = PLV(EPH_P_W + c);
            o.nacc[c] = PLV(EPH_P_NACCEL + c);
            o.dacc[c] = PLV(EPH_P_DACCEL + c);
            o.gacc[c] = PLV(EPH_P_GACCEL + c);
            o.dtq[c] = PLV(EPH_P_DTORQUE + c);
            o.beta[c] = PLV(EPH_P_BETA + c);
        }
        for (int q = 0; q < 9; ++q) {
            o.s[q] = dd{PLV(EPH_P_S_HI + q), PLV(EPH_P_S_LO + q)};
            o.C[q] = PLV(EPH_P_C_POTENTIAL + q);
            o.GI[q] = PLV(EPH_P_GI + q);
        }
        o.GM = PLV(EPH_P_GM);
        o.exJ2 = PLV(EPH_P_EXJ2);
        o.phi = PLV(EPH_P_PHI);
        o.beta2 = PLV(EPH_P_BETA2);
        o.mind = P.reset_minmax ? 0.0 : PLV(EPH_P_MIN_DISTANCE);
        o.maxi = P.reset_minmax ? 0.0 : PLV(EPH_P_MAX_INFLUENCE);
#undef PLV
    }
}

__device__ void store_own(const SysDev &S, const Own *own, int nb, bool deform_only) {
    const int n = S.n;
    double *pl = S.planes;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const Own &o = own[b];
        const int i = o.idx;
#define PLV(p) pl[(size_t)(p) * n + i]
        for (int q = 0; q < 9; ++q) {
            PLV(EPH_P_C_POTENTIAL + q) = o.C[q];
            PLV(EPH_P_GI + q) = o.GI[q];
        }
        PLV(EPH_P_PHI) = o.phi;
        for (int c = 0; c < 3; ++c) PLV(EPH_P_NACCEL + c) = o.nacc[c];
        if (deform_only) continue;
        for (int c = 0; c < 3; ++c) {
            PLV(EPH_P_R_HI + c) = o.r[c].hi; PLV(EPH_P_R_LO + c) = o.r[c].lo;
            PLV(EPH_P_V_HI + c) = o.v[c].hi; PLV(EPH_P_V_LO + c) = o.v[c].lo;
            PLV(EPH_P_GL_HI + c) = o.GL[c].hi; PLV(EPH_P_GL_LO + c) = o.GL[c].lo;
            PLV(EPH_P_W + c) = o.w[c];
            PLV(EPH_P_DACCEL + c) = o.dacc[c];
            PLV(EPH_P_GACCEL + c) = o.gacc[c];
            PLV(EPH_P_DTORQUE + c) = o.dtq[c];
            PLV(EPH_P_BETA + c) = o.beta[c];
        }
        for (int q = 0; q < 9; ++q) { PLV(EPH_P_S_HI + q) = o.s[q].hi; PLV(EPH_P_S_LO + q) = o.s[q].lo; }
        PLV(EPH_P_GM) = o.GM;
        PLV(EPH_P_EXJ2) = o.exJ2;
        PLV(EPH_P_BETA2) = o.beta2;
        PLV(EPH_P_MIN_DISTANCE) = o.mind;
        PLV(EPH_P_MAX_INFLUENCE) = o.maxi;
#undef PLV
    }
}

// publish the stage state of owned body b into public buffer `buf`
__device__ void publish_body(const SysDev &S, const Own &o, int buf) {
    const int n = S.n, i = o.idx;
    double *pub = S.pub + (size_t)buf * PUB_NPLANES * n;
    for (int c = 0; c < 3; ++c) {
        pub[(PUB_R_HI + c) * n + i] = o.r[c].hi;
        pub[(PUB_R_LO + c) * n + i] = o.r[c].lo;
        pub[(PUB_V_HI + c) * n + i] = o.v[c].hi;
        pub[(PUB_V_LO + c) * n + i] = o.v[c].lo;
    }
    v3 gl = fast3(o.GL);
    pub[(PUB_GL + 0) * n + i] = gl.x;
    pub[(PUB_GL + 1) * n + i] = gl.y;
    pub[(PUB_GL + 2) * n + i] = gl.z;
    pub[PUB_GM * n + i] = o.GM;
    if (o.gp >= 0) {
        for (int q = 0; q < 9; ++q) pub[(PUB_FRAME + q) * n + i] = dd_val(o.s[q]);
    }
    if (o.ring >= 0) {
        m3 f = ring_frame(gl);
        double t[9];
        stm(t, f);
        for (int q = 0; q < 9; ++q) pub[(PUB_RFRAME + q) * n + i] = t[q];
    }
}

// ------------------------------------------------------------------ pass A: deform_by + angular velocity
// One ordered pair (i = owned body o, j) of DAMPED_TIDAL_DEFORMATION_MATRIX / _NDELAY / _NK2
// (mass.impl:1-46), accumulated into acc = {phi, naccel[3], C[9]}.
__device__ __forceinline__ void pair_a(const Own &o, const double rjh[3], const double rjl[3],
                                       const double vjh[3], const double vjl[3], double GMj, double sR2j,
                                       double tdfj, double acc[13]) {
    v3 r = mk(dd_diff(rjh[0], rjl[0], o.r[0].hi, o.r[0].lo), dd_diff(rjh[1], rjl[1], o.r[1].hi, o.r[1].lo),
              dd_diff(rjh[2], rjl[2], o.r[2].hi, o.r[2].lo));
    double q = dot(r, r), sm = o.sR2 + sR2j;
    double rr2 = 1.0 / ((q < sm) ? sm : q);
    double rr = sqrt(rr2);
    double tp_dphi = rr * GMj;
    double tp_dg = rr2 * tp_dphi;
    acc[0] -= tp_dphi;
    acc[1] += tp_dg * r.x;
    acc[2] += tp_dg * r.y;
    acc[3] += tp_dg * r.z;
    if (o.kind == 0) return;
    double fk = (-3 * tp_dg) * o.k2;
    m3 T;
    if (o.kind == 2) {
        v3 v = mk(dd_diff(vjh[0], vjl[0], o.v[0].hi, o.v[0].lo), dd_diff(vjh[1], vjl[1], o.v[1].hi, o.v[1].lo),
                  dd_diff(vjh[2], vjl[2], o.v[2].hi, o.v[2].lo));
        v3 w = mk(o.w[0], o.w[1], o.w[2]);
        v3 dw = rr2 * cross(r, cross(w, r) - v);
        double dwt = normalize(dw);
        dwt *= o.td * tdfj;
        double ecwt2 = 1 + 4 * dwt * dwt, secwt2 = sqrt(ecwt2);
        double x0 = sqrt((1 + secwt2) / (2 * ecwt2));
        double y0 = dwt * sqrt(2 / (ecwt2 * (1 + secwt2)));
        double z02 = dwt * dwt * (2 / (ecwt2 + secwt2));
        v3 dr = x0 * r + y0 * cross(dw, r);
        T = add_diag(outer(rr2 * dr, dr) - outer(z02 * dw, dw), z02 - 1.0 / 3);
    } else {
        T = add_diag(outer(rr2 * r, r), -(1.0 / 3));
    }
    acc[4] -= fk * T.x.x; acc[5] -= fk * T.x.y; acc[6] -= fk * T.x.z;
    acc[7] -= fk * T.y.x; acc[8] -= fk * T.y.y; acc[9] -= fk * T.y.z;
    acc[10] -= fk * T.z.x; acc[11] -= fk * T.z.y; acc[12] -= fk * T.z.z;
}

// UPDATE_HARMONICS (mass.impl:48-61) from the pass-A sums of owned body o
__device__ void update_harmonics(Own &o) {
    o.phi = o.sumA[0];
    o.nacc[0] = o.sumA[1]; o.nacc[1] = o.sumA[2]; o.nacc[2] = o.sumA[3];
    m3 C = ldm(o.sumA + 4);
    v3 w = ldv(o.w);
    double w2 = dot(w, w);
    C = add_diag(C, w2 * o.k2r / 3);
    C = C - outer(o.k2r * w, w);
    C = (o.R * o.R2 / (2 * o.GM)) * C;
    m3 fmis = fast9(o.s);
    m3 mc = ldm(o.Cst);
    mc.x.x += o.exJ2 / 2;
    mc.y.y += o.exJ2 / 2;
    mc.z.z -= o.exJ2;
    mc = toworld(fmis, mc);
    C = C + mc;
    stm(o.C, C);
    stm(o.GI, ((-2.0) / 3 * o.R2) * add_diag(C, -o.A));
}

// UPDATE_ANGULAR_VELOCITY (mass.impl:63-72); returns should_break
__device__ bool update_angular_velocity(Own &o) {
    bool finite = true;
    for (int c = 0; c < 3; ++c) finite = finite && dd_finite(o.GL[c]);
    m3 GI = ldm(o.GI);
    v3 w = ldv(o.w);
    if (finite) {
        v3 nw = mul(inverse(GI), fast3(o.GL));
        stv(o.w, nw);
        v3 d = nw - w;
        return dot(d, d) < 1e-18 * dot(w, w);
    }
    v3 gl = mul(GI, w);
    o.GL[0] = dd_make(gl.x); o.GL[1] = dd_make(gl.y); o.GL[2] = dd_make(gl.z);
    o.gl_fixed = 1;
    return true;
}

template <int NV>
__device__ __forceinline__ void block_reduce(double (&acc)[kRegBodies][13], unsigned mask, Scratch &sc,
                                             double *out /* [kRegBodies][13] */, int max_from) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int bb = 0; bb < kRegBodies; ++bb) {
        if (!((mask >> bb) & 1)) continue;
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            double v = (c >= max_from) ? warp_cmax(acc[bb][c]) : warp_sum(acc[bb][c]);
            if (lane == 0) sc.red[warp][bb][c] = v;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kRegBodies * NV; idx += blockDim.x) {
        int bb = idx / NV, c = idx % NV;
        if (!((mask >> bb) & 1)) continue;
        double s = sc.red[0][bb][c];
        for (int w = 1; w < kThreads / 32; ++w) {
            if (c >= max_from) checked_maximize(s, sc.red[w][bb][c]);
            else s += sc.red[w][bb][c];
        }
        out[bb * 13 + c] = s;
    }
    __syncthreads();
}

__device__ void pass_a(const SysDev &S, Own *own, int nb, int buf, bool deform_only, Scratch &sc,
                       double *red_out) {
    const int n = S.n;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * n;
    const double *cst = S.cst;
    if (threadIdx.x < nb) { own[threadIdx.x].converged = 0; own[threadIdx.x].gl_fixed = 0; }
    __syncthreads();
    const int max_iter = deform_only ? 1 : 4;   // MAX_ANGULAR_VELOCITY_ITER (mass.impl:74)
    for (int it = 0; it < max_iter; ++it) {
        for (int c0 = 0; c0 < nb; c0 += kRegBodies) {
            unsigned mask = 0;
            bool any_delay = false;
            for (int bb = 0; bb < kRegBodies && c0 + bb < nb; ++bb) {
                const Own &o = own[c0 + bb];
                // the pair sums depend on the angular velocity only for delayed tides
                bool need = (it == 0) || (!o.converged && o.kind == 2);
                if (need) { mask |= 1u << bb; any_delay |= (o.kind == 2); }
            }
            if (!mask) continue;
            double acc[kRegBodies][13];
#pragma unroll
            for (int bb = 0; bb < kRegBodies; ++bb)
#pragma unroll
                for (int c = 0; c < 13; ++c) acc[bb][c] = 0;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double rjh[3], rjl[3], vjh[3] = {0, 0, 0}, vjl[3] = {0, 0, 0};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    rjh[c] = __ldcg(pub + (PUB_R_HI + c) * n + j);
                    rjl[c] = __ldcg(pub + (PUB_R_LO + c) * n + j);
                }
                if (any_delay) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        vjh[c] = __ldcg(pub + (PUB_V_HI + c) * n + j);
                        vjl[c] = __ldcg(pub + (PUB_V_LO + c) * n + j);
                    }
                }
                const double GMj = __ldcg(pub + PUB_GM * n + j);
                const double sR2j = __ldg(cst + CST_SR2 * n + j);
                const double tdfj = __ldg(cst + CST_TDF * n + j);
#pragma unroll
                for (int bb = 0; bb < kRegBodies; ++bb) {
                    if (!((mask >> bb) & 1)) continue;
                    const Own &o = own[c0 + bb];
                    if (o.idx == j) continue;
                    pair_a(o, rjh, rjl, vjh, vjl, GMj, sR2j, tdfj, acc[bb]);
                }
            }
            block_reduce<13>(acc, mask, sc, red_out, 13);
            if (threadIdx.x < kRegBodies && ((mask >> threadIdx.x) & 1)) {
                Own &o = own[c0 + threadIdx.x];
                for (int c = 0; c < 13; ++c) o.sumA[c] = red_out[threadIdx.x * 13 + c];
            }
            __syncthreads();
        }
        mark(S, sc, PH_A_SWEEP);
        if (threadIdx.x < nb) {
            Own &o = own[threadIdx.x];
            if (!o.converged) {
                update_harmonics(o);
                o.converged = deform_only ? 1 : (update_angular_velocity(o) ? 1 : 0);
            }
        }
        __syncthreads();
        mark(S, sc, PH_A_UPDATE);
        int all = 1;
        for (int b = 0; b < nb; ++b) all &= own[b].converged;
        if (all) break;
        __syncthreads();
    }
    if (deform_only) return;
    // PREPARE_RELATIVITY (mass.impl:76-80) and the pass-A outputs other CTAs read in pass B
    const double c2 = kC * kC;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &o = own[b];
        v3 beta = vdiv(fast3(o.v), kC);
        stv(o.beta, beta);
        o.beta2 = dot(beta, beta);
        o.phi = o.phi / c2;
        stv(o.nacc, vdiv(ldv(o.nacc), c2));
        for (int c = 0; c < 3; ++c) { o.dacc[c] = 0; o.dtq[c] = 0; o.gacc[c] = 0; }
        const int i = o.idx;
        double *aux = S.aux;
        aux[AUX_PHI * n + i] = o.phi;
        for (int c = 0; c < 3; ++c) {
            aux[(AUX_NACC + c) * n + i] = o.nacc[c];
            aux[(AUX_BETA + c) * n + i] = o.beta[c];
        }
        aux[AUX_BETA2 * n + i] = o.beta2;
        for (int q = 0; q < 9; ++q) aux[(AUX_CPOT + q) * n + i] = o.C[q];
        // a non-finite G*L was replaced by GI*w: republish it for pass B
        if (o.gl_fixed) publish_body(S, o, buf);
    }
    __syncthreads();
    mark(S, sc, PH_A_UPDATE);
}

// ------------------------------------------------------------------ pass B: main force
// One ordered pair of RELATIVITY, the per-pair maxima, ROTATIONAL_TIDAL_DEFORMATION_NANTI_FORCE,
// LENSE_THIRRING and RADIATION_PRESSURE (mass.impl:82-125, mass.cpp:147-155), plus the reaction of
// owned body o's own geopotential / ring on j (mass.cpp:358-371, APPLY_NONPOINT_FORCE mass.impl:127-130).
struct JB {
    double rh[3], rl[3], gl[3], GM, phi, nacc[3], beta[3], beta2, C[9], R2, lum, sR2;
};

__device__ __forceinline__ void pair_b(const SysDev &S, const Own &o, const JB &J, double acc[13]) {
    v3 r = mk(dd_diff(J.rh[0], J.rl[0], o.r[0].hi, o.r[0].lo), dd_diff(J.rh[1], J.rl[1], o.r[1].hi, o.r[1].lo),
              dd_diff(J.rh[2], J.rl[2], o.r[2].hi, o.r[2].lo));
    double q = dot(r, r), sm = o.sR2 + J.sR2;
    double rr2 = 1.0 / ((q < sm) ? sm : q);
    double rr = sqrt(rr2);
    double rr3 = rr * rr2;
    double tp_dphi = rr * J.GM;
    double tp_dg = rr2 * tp_dphi;
    v3 bj = mk(J.beta[0], J.beta[1], J.beta[2]);
    v3 bi = ldv(o.beta);
    double rbj = dot(r, bj);
    double tp = rbj * rr;
    tp *= tp;
    v3 naj = mk(J.nacc[0], J.nacc[1], J.nacc[2]);
    double delta1 = 4 * o.phi + J.phi + o.beta2 + 2 * J.beta2 - 4 * dot(bi, bj) + (dot(r, naj) - 3 * tp) / 2;
    v3 b = bj - bi;
    v3 g = (7 * tp_dphi / 2) * naj + (tp_dg * delta1) * r + (tp_dg * (rbj - dot(r, b) * 4)) * b;
    acc[0] += g.x; acc[1] += g.y; acc[2] += g.z;
    checked_maximize(acc[9], rr);
    checked_maximize(acc[10], tp_dg);
    // deformation of i and of j (no reaction written to j: recomputed by j's owner)
    m3 Ci = ldm(o.C);
    v3 Cr = mul(Ci, r);
    v3 dg = (J.GM * rr3 * rr2 * o.R2) * ((dot(r, Cr) * 5 * rr2) * r - (Cr + Cr));
    v3 da = dg;
    v3 dt = cross(r, dg);
    m3 Cj = m3{mk(J.C[0], J.C[1], J.C[2]), mk(J.C[3], J.C[4], J.C[5]), mk(J.C[6], J.C[7], J.C[8])};
    v3 Cjr = mul(Cj, r);
    da += (J.GM * rr3 * rr2 * J.R2) * ((dot(r, Cjr) * 5 * rr2) * r - (Cjr + Cjr));
    // Lense-Thirring
    double rcr32 = 2 * J.GM / kC * rr3;
    v3 GL = fast3(o.GL);
    v3 GLb = cross(GL, b);
    da -= rcr32 * (GLb - (3 * dot(GLb, r) * rr2) * r);
    dt -= rcr32 * cross(GL, cross(r, b));
    v3 GLj = mk(J.gl[0], J.gl[1], J.gl[2]);
    da += cross(rcr32 * (GLj - (3 * dot(GLj, r) * rr2) * r), b);
    // radiation pressure
    da += (J.lum * o.rR2G4c * rr3 / o.GM) * r;
    acc[3] += da.x; acc[4] += da.y; acc[5] += da.z;
    acc[6] += dt.x; acc[7] += dt.y; acc[8] += dt.z;
}

__device__ __forceinline__ void nonpoint_i(const SysDev &S, const Own &o, const JB &J, double acc[13]) {
    const m3 gpf = ldm(o.gpf), rgf = ldm(o.rgf);
    v3 r = mk(dd_diff(J.rh[0], J.rl[0], o.r[0].hi, o.r[0].lo), dd_diff(J.rh[1], J.rl[1], o.r[1].hi, o.r[1].lo),
              dd_diff(J.rh[2], J.rl[2], o.r[2].hi, o.r[2].lo));
    v3 da = mk(0, 0, 0), dt = mk(0, 0, 0);
    if (o.gp >= 0) {
        v3 an = toworld(gpf, gp_sum(S.gp_coef + (size_t)o.gp * EPH_GP_TABLE_SIZE, __ldg(S.gp_nz + o.gp),
                                    __ldg(S.gp_nt + o.gp), o.R, tolocal(gpf, r)));
        da -= J.GM * an;
        dt -= J.GM * cross(r, an);
    }
    if (o.ring >= 0) {
        v3 an = toworld(rgf, ring_sum(S.ring_disk + (size_t)o.ring * EPH_RING_MAX_DISKS * 3,
                                      __ldg(S.ring_nd + o.ring), o.R, tolocal(rgf, r)));
        da -= J.GM * an;
        dt -= J.GM * cross(r, an);
    }
    acc[3] += da.x; acc[4] += da.y; acc[5] += da.z;
    acc[6] += dt.x; acc[7] += dt.y; acc[8] += dt.z;
}

__device__ void pass_b(const SysDev &S, Own *own, int nb, int buf, Scratch &sc, double *red_out) {
    const int n = S.n;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * n;
    const double *aux = S.aux, *cst = S.cst;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &o = own[b];
        if (o.gp >= 0) stm(o.gpf, fast9(o.s));
        if (o.ring >= 0) stm(o.rgf, ring_frame(fast3(o.GL)));
    }
    __syncthreads();
    for (int c0 = 0; c0 < nb; c0 += kRegBodies) {
        unsigned mask = 0;
        bool any_ext = false;
        for (int bb = 0; bb < kRegBodies && c0 + bb < nb; ++bb) {
            mask |= 1u << bb;
            any_ext |= (own[c0 + bb].gp >= 0 || own[c0 + bb].ring >= 0);
        }
        double acc[kRegBodies][13];
#pragma unroll
        for (int bb = 0; bb < kRegBodies; ++bb)
#pragma unroll
            for (int c = 0; c < 13; ++c) acc[bb][c] = 0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            JB J;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                J.rh[c] = __ldcg(pub + (PUB_R_HI + c) * n + j);
                J.rl[c] = __ldcg(pub + (PUB_R_LO + c) * n + j);
                J.gl[c] = __ldcg(pub + (PUB_GL + c) * n + j);
                J.nacc[c] = __ldcg(aux + (AUX_NACC + c) * n + j);
                J.beta[c] = __ldcg(aux + (AUX_BETA + c) * n + j);
            }
            J.GM = __ldcg(pub + PUB_GM * n + j);
            J.phi = __ldcg(aux + AUX_PHI * n + j);
            J.beta2 = __ldcg(aux + AUX_BETA2 * n + j);
#pragma unroll
            for (int q = 0; q < 9; ++q) J.C[q] = __ldcg(aux + (AUX_CPOT + q) * n + j);
            J.R2 = __ldg(cst + CST_R2 * n + j);
            J.lum = __ldg(cst + CST_LUM * n + j);
            J.sR2 = __ldg(cst + CST_SR2 * n + j);
#pragma unroll
            for (int bb = 0; bb < kRegBodies; ++bb) {
                if (!((mask >> bb) & 1)) continue;
                const Own &o = own[c0 + bb];
                if (o.idx == j) continue;
                pair_b(S, o, J, acc[bb]);
            }
            if (any_ext) {
                for (int bb = 0; bb < kRegBodies; ++bb) {
                    if (!((mask >> bb) & 1)) continue;
                    const Own &o = own[c0 + bb];
                    if (o.idx == j || (o.gp < 0 && o.ring < 0)) continue;
                    nonpoint_i(S, o, J, acc[bb]);
                }
            }
        }
        block_reduce<11>(acc, mask, sc, red_out, 9);
        if (threadIdx.x < kRegBodies && ((mask >> threadIdx.x) & 1)) {
            Own &o = own[c0 + threadIdx.x];
            const double *rr = red_out + threadIdx.x * 13;
            for (int c = 0; c < 3; ++c) { o.gacc[c] = rr[c]; o.dacc[c] = rr[3 + c]; o.dtq[c] = rr[6 + c]; }
            checked_maximize(o.mind, rr[9]);
            checked_maximize(o.maxi, rr[10]);
        }
        __syncthreads();
    }
    mark(S, sc, PH_B_SWEEP);
    // forces of the other extended bodies' geopotentials and rings on the owned bodies
    // (the `mj.daccel += mi.GM*an` half of APPLY_NONPOINT_FORCE, mass.impl:127-128)
    const int n_ext = S.n_ext;
    for (int item = threadIdx.x; item < nb * n_ext; item += blockDim.x) {
        const int b = item / n_ext, e = item % n_ext;
        const Own &o = own[b];
        const int E = __ldg(S.ext_body + e);
        v3 add3 = mk(0, 0, 0);
        if (E != o.idx) {
            v3 r = mk(dd_diff(o.r[0].hi, o.r[0].lo, __ldcg(pub + PUB_R_HI * n + E), __ldcg(pub + PUB_R_LO * n + E)),
                      dd_diff(o.r[1].hi, o.r[1].lo, __ldcg(pub + (PUB_R_HI + 1) * n + E), __ldcg(pub + (PUB_R_LO + 1) * n + E)),
                      dd_diff(o.r[2].hi, o.r[2].lo, __ldcg(pub + (PUB_R_HI + 2) * n + E), __ldcg(pub + (PUB_R_LO + 2) * n + E)));
            const double GME = __ldcg(pub + PUB_GM * n + E);
            const double RE = __ldg(cst + CST_R * n + E);
            const int gpE = (int)__ldg(cst + CST_GP * n + E), ringE = (int)__ldg(cst + CST_RING * n + E);
            if (gpE >= 0) {
                m3 f = ld9(pub + PUB_FRAME * n, n, E);
                v3 an = toworld(f, gp_sum(S.gp_coef + (size_t)gpE * EPH_GP_TABLE_SIZE, __ldg(S.gp_nz + gpE),
                                          __ldg(S.gp_nt + gpE), RE, tolocal(f, r)));
                add3 += GME * an;
            }
            if (ringE >= 0) {
                m3 f = ld9(pub + PUB_RFRAME * n, n, E);
                v3 an = toworld(f, ring_sum(S.ring_disk + (size_t)ringE * EPH_RING_MAX_DISKS * 3,
                                            __ldg(S.ring_nd + ringE), RE, tolocal(f, r)));
                add3 += GME * an;
            }
        }
        sc.ext[b][e][0] = add3.x; sc.ext[b][e][1] = add3.y; sc.ext[b][e][2] = add3.z;
    }
    __syncthreads();
    mark(S, sc, PH_B_EXT);
    // finalisation (mass.cpp:389-396): FINALIZE_RELATIVITY and RING_CORRECTION
    const double c2 = kC * kC;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &o = own[b];
        v3 da = ldv(o.dacc);
        for (int e = 0; e < n_ext; ++e) da += mk(sc.ext[b][e][0], sc.ext[b][e][1], sc.ext[b][e][2]);
        o.phi *= c2;
        v3 na = c2 * ldv(o.nacc);
        stv(o.nacc, na);
        v3 ga = ldv(o.gacc);
        v3 tq = ldv(o.dtq);
        if (o.ring >= 0) {
            da = da - o.ring_GM_ratio * ((ga + da) + na);
            v3 mGL = fast3(o.GL);
            double rmGL = normalize(mGL);
            v3 ptorque = dot(tq, mGL) * mGL;
            v3 dtq = tq - ptorque;
            dtq = (rmGL / (rmGL + o.ring_GL_R2 * o.R2)) * dtq;
            tq = dtq + ptorque;
        }
        stv(o.dacc, da);
        stv(o.dtq, tq);
        stv(o.fa, (ga + da) + na);
    }
    __syncthreads();
    mark(S, sc, PH_B_FINAL);
}

// ------------------------------------------------------------------ RK12 stage combination and update
// Called with f_s known for all owned bodies (s = 0..24). Adds a_{k,s} f_s into the accumulators of
// stages k = s+1..25 (RungeKutta.impl:148-162 in incremental form), then forms the state of stage s+1
// (RungeKutta.impl:164-186) and publishes it to buffer `buf_out`.
__device__ void rk_stage(const SysDev &S, Own *own, int nb, int s, long long i_step, const StepParams &P,
                         int buf_out) {
    const double dt = P.dt;
    if (threadIdx.x < nb) {
        Own &o = own[threadIdx.x];
        if (s == 0) {   // start of a step: x0 = x; Egrad = dtorque (RungeKutta.impl:113-116)
            for (int c = 0; c < 3; ++c) { o.r0[c] = o.r[c]; o.v0[c] = o.v[c]; o.GL0[c] = o.GL[c]; o.w0[c] = o.w[c]; }
            for (int q = 0; q < 9; ++q) o.s0[q] = o.s[q];
            for (int c = 0; c < 3; ++c) o.Egrad[c] = o.dtq[c];
        }
        if (s == kStages - 1) {   // rotational end-of-step correction (RungeKutta.impl:129-140)
            m3 GI = ldm(o.GI);
            m3 ir = inverse(GI);
            double irdet = det(ir);
            double dt2 = dt * dt;
            v3 dtq = ldv(o.dtq);
            v3 tq = dt2 * dtq;
            v3 tqdot = dt2 * (dtq - ldv(o.Egrad));
            v3 j = fast3(o.GL), w = dt * ldv(o.w);
            v3 irtq = mul(ir, tq);
            j = dt * j;
            v3 e1 = dot(w, j) * (mul(ir, w) + irdet * mul(GI, j));
            v3 e2 = cross(w, irtq);
            v3 e3 = mul(ir, (cross(j, irtq) - 2 * cross(w, tq)) + tqdot);
            v3 eg = (e1 + e2) + e3;
            stv(o.Egrad, cross(eg, w));
        }
    }
    __syncthreads();
    // incremental combination: 12 components (velocity as double-double) per later stage
    const int nk = kStages - s;   // stages s+1..25
    for (int item = threadIdx.x; item < nb * nk * 12; item += blockDim.x) {
        const int b = item / (nk * 12);
        const int rem = item % (nk * 12);
        const int k = s + 1 + rem / 12;
        const int c = rem % 12;
        Own &o = own[b];
        const int ci = k * (k - 1) / 2 + s;
        const dd a = dd{c_rk_hi[ci], c_rk_lo[ci]};
        const bool nz = a.hi != 0;
        if (c < 3) {
            dd cur = (s == 0) ? dd_make(0) : o.accv[k - 1][c];
            if (nz) cur = dd_add(cur, dd_mul(a, o.v[c]));
            o.accv[k - 1][c] = cur;
        } else {
            const double fa = dd_val(a);
            double *slot;
            double f;
            if (c < 6) { slot = &o.acca[k - 1][c - 3]; f = o.fa[c - 3]; }
            else if (c < 9) { slot = &o.accw[k - 1][c - 6]; f = o.w[c - 6]; }
            else { slot = &o.acct[k - 1][c - 9]; f = o.dtq[c - 9]; }
            double cur = (s == 0) ? 0.0 : *slot;
            if (nz) cur = __dadd_rn(cur, __dmul_rn(fa, f));
            *slot = cur;
        }
    }
    __syncthreads();
    // state of stage k = s+1
    const int k = s + 1;
    const double dt_k = c_dtk[k];
    const double t = P.t_eph + dt * (dt_k + (double)i_step);
    if (threadIdx.x < nb) {
        Own &o = own[threadIdx.x];
        const dd ddt = dd_make(dt);
        for (int c = 0; c < 3; ++c) {
            o.r[c] = dd_add(o.r0[c], dd_mul(ddt, o.accv[k - 1][c]));
            o.v[c] = dd_add(o.v0[c], dd_make(dt * o.acca[k - 1][c]));
            o.GL[c] = dd_add(o.GL0[c], dd_make(dt * o.acct[k - 1][c]));
        }
        v3 w = vdiv(ldv(o.accw[k - 1]), dt_k);
        stv(o.w, w);
        v3 dw = (2.0 / 3) * (w - ldv(o.w0));
        for (int q = 0; q < 9; ++q) o.s[q] = o.s0[q];
        double st[9];
        m3 R1 = rotation_matrix(w - dw, dt * dt_k / 2);
        stm(st, mul(R1, fast9(o.s)));
        for (int q = 0; q < 9; ++q) o.s[q] = dd_add(o.s[q], dd_make(st[q]));
        m3 R2 = rotation_matrix(w + dw, dt * dt_k / 2);
        stm(st, mul(R2, fast9(o.s)));
        for (int q = 0; q < 9; ++q) o.s[q] = dd_add(o.s[q], dd_make(st[q]));
        if (k == kStages) {
            m3 R3 = rotation_matrix(ldv(o.Egrad), 1.0 / 72);
            stm(st, mul(R3, fast9(o.s)));
            for (int q = 0; q < 9; ++q) o.s[q] = dd_add(o.s[q], dd_make(st[q]));
            // mass::orthogonalize (mass.h:147-150)
            m3 fmis = fast9(o.s);
            m3 one_minus = add_diag((-1.0) * mul(transpose(fmis), fmis), 1.0);
            stm(st, mul(0.5 * fmis, one_minus));
            for (int q = 0; q < 9; ++q) o.s[q] = dd_add(o.s[q], dd_make(st[q]));
        }
        o.GM = o.GM0 + o.dGM * t;
        o.exJ2 = o.dJ2 * t;
        publish_body(S, o, buf_out);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ the kernel
__global__ void __launch_bounds__(kThreads, 1) step_kernel(SysDev S, StepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Own *own = reinterpret_cast<Own *>(smem_raw);
    Scratch &sc = *reinterpret_cast<Scratch *>(smem_raw + sizeof(Own) * kOwnMax);
    __shared__ double red_out[kRegBodies * 13];

    if (threadIdx.x == 0) {
        sc.t_last = global_ns();
        for (int p = 0; p < kPhases; ++p) sc.t_phase[p] = 0;
    }
    int nb = 0;
    for (int b = 0; b < kOwnMax; ++b) {
        int id = S.own_list[blockIdx.x * kOwnMax + b];
        if (id < 0) break;
        if (threadIdx.x == 0) own[b].idx = id;
        ++nb;
    }
    __syncthreads();
    load_own(S, own, nb, P);
    __syncthreads();
    if (threadIdx.x < nb) publish_body(S, own[threadIdx.x], 0);
    auto sync = [&]() {
        bool ok = grid_sync(S, sc);
        mark(S, sc, PH_BARRIER);
        return ok;
    };
    auto finish = [&](bool deform_only) {
        store_own(S, own, nb, deform_only);
        __syncthreads();
        mark(S, sc, PH_IO);
        if (S.timers && threadIdx.x == 0)
            for (int p = 0; p < kPhases; ++p) S.timers[blockIdx.x * kPhases + p] = sc.t_phase[p];
    };
    mark(S, sc, PH_IO);

    if (P.mode == MODE_DEFORM || P.mode == MODE_ACCEL) {
        if (!sync()) return;
        pass_a(S, own, nb, 0, P.mode == MODE_DEFORM, sc, red_out);
        if (P.mode == MODE_ACCEL) {
            if (!sync()) return;
            pass_b(S, own, nb, 0, sc, red_out);
        }
        finish(P.mode == MODE_DEFORM);
        return;
    }
    // MODE_INTEGRATE: the loaded auxiliaries are f_0 of the first step
    if (threadIdx.x < nb) {
        Own &o = own[threadIdx.x];
        stv(o.fa, (ldv(o.gacc) + ldv(o.dacc)) + ldv(o.nacc));
    }
    __syncthreads();
    int buf = 0;
    for (long long step = 0; step < P.n_step; ++step) {
        for (int s = 0; s < kStages; ++s) {
            rk_stage(S, own, nb, s, step, P, buf ^ 1);
            mark(S, sc, PH_RK);
            buf ^= 1;
            if (!sync()) return;
            pass_a(S, own, nb, buf, false, sc, red_out);
            if (!sync()) return;
            pass_b(S, own, nb, buf, sc, red_out);
        }
    }
    if (P.invert_min && threadIdx.x < nb) own[threadIdx.x].mind = 1 / own[threadIdx.x].mind;
    __syncthreads();
    finish(false);
}

}  // namespace eph

// ------------------------------------------------------------------ host launcher
namespace eph {

size_t step_smem_bytes() { return sizeof(Own) * kOwnMax + sizeof(Scratch); }

static bool g_consts_ready[64];

cudaError_t upload_constants(int device) {
    if (device >= 0 && device < 64 && g_consts_ready[device]) return cudaSuccess;
    double hi[EPH_RK12_NCOEF], lo[EPH_RK12_NCOEF], dtk[kStages + 1];
    for (int q = 0; q < EPH_RK12_NCOEF; ++q) {
        memcpy(&hi[q], &EPH_RK12_COEF_BITS[2 * q], 8);
        memcpy(&lo[q], &EPH_RK12_COEF_BITS[2 * q + 1], 8);
    }
    // c_k accumulated exactly as RungeKutta.impl:118-152: skip zero coefficients, add hi+lo in j order
    dtk[0] = 0;
    for (int k = 1; k <= kStages; ++k) {
        double acc = 0;
        for (int j = 0; j < k; ++j) {
            const int ci = k * (k - 1) / 2 + j;
            if (hi[ci] != 0) acc += hi[ci] + lo[ci];
        }
        dtk[k] = acc;
    }
    cudaError_t e = cudaMemcpyToSymbol(c_rk_hi, hi, sizeof(hi));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rk_lo, lo, sizeof(lo));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_dtk, dtk, sizeof(dtk));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)step_smem_bytes());
    if (e == cudaSuccess && device >= 0 && device < 64) g_consts_ready[device] = true;
    return e;
}

cudaError_t launch_step(const SysDev &S, const StepParams &P, int grid, cudaStream_t stream) {
    void *args[] = {(void *)&S, (void *)&P};
    return cudaLaunchCooperativeKernel((void *)step_kernel, dim3(grid), dim3(kThreads), args, step_smem_bytes(),
                                       stream);
}

int max_coresident_ctas(int device, int *out) {
    int per_sm = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel, kThreads, step_smem_bytes());
    if (e != cudaSuccess) return (int)e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return (int)e;
    *out = per_sm * sms;
    return 0;
}

}  // namespace eph
