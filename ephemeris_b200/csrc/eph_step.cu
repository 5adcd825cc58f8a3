// eph_step.cu - the RK12 step of one system of bodies as a single persistent cooperative kernel.
//
// Reference path replaced: msystem::Cuda_RungeKutta12 / Cuda_RungeKutta_Kernel
// (src/integrators/RungeKutta.cu:391-412, RungeKutta.impl:107-194) and msystem::Cuda_accel
// (RungeKutta.cu:348-375,414-438). The physics is that of the CPU integrator (src/physics/mass.cpp:78-397,
// mass.impl:1-152); the schedule is new:
//
//   * every CTA owns up to kOwnMax bodies for the whole launch and keeps their private state (start of
//     step, the 25 RK12 stage accumulators, auxiliaries) in shared memory;
//   * one stage evaluation is two O(N^2) sweeps separated by grid barriers. Before each sweep the
//     planes of all bodies j that the pair terms read are staged into a shared-memory tile by the
//     bulk-copy engine (cp.async.bulk, completion on an mbarrier); the CTA's warps are split into one
//     group per owned body, each group strides over j in the tile, accumulates that body's pair sums
//     in registers and reduces them with warp shuffles;
//       pass A  - potential, Newtonian acceleration and tidal matrix (mass.impl:1-46), then the harmonics
//                 update and the angular-velocity fixed point per body (mass.impl:48-80); meanwhile the
//                 other warps evaluate every geopotential / ring host's field at the owned bodies, once
//                 per (host, body) pair: the force on the body stays in shared memory, the reaction on
//                 the host goes to a global table its owner sums in pass B (APPLY_NONPOINT_FORCE,
//                 mass.impl:127-130). A CTA that owns a delayed tide hands its bodies' field items to
//                 CTAs that own none (field_handoff), so that its fixed-point sweeps run on every warp;
//       pass B  - 1PN, deformation, Lense-Thirring and radiation (mass.impl:82-125), the hosts' reaction
//                 sums, finalisation (mass.cpp:389-396), then the RK12 stage combination and the state
//                 update of the owned bodies;
//   * the stage state other CTAs read is double-buffered (ping-pong), so pass B of stage k and the state
//     update for stage k+1 need no barrier between them: 2 barriers per stage, 50 per step;
//   * the RK12 combination sum_j a_kj f_j is accumulated incrementally: when f_j is known it is added into
//     the accumulators of every later stage k, in ascending j, which is the reference's summation order.
//
// All waits are bounded (S.wait_ns, 2 s by default): a grid-barrier or copy wait that runs out records a status
// word and the kernel returns (after waiting, again bounded, for its own copies in flight); it never traps.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "eph_math.cuh"
#include "eph_models.cuh"
#include "eph_system.cuh"
#include "../../include/eph_planes.h"
#include "eph_rk12_host.h"

namespace eph {

constexpr double kC = 299792458.0;                      // src/math/basic_math.h:10,18

__constant__ double c_rk_hi[EPH_RK12_NCOEF];            // a_kj, double-double
__constant__ double c_rk_lo[EPH_RK12_NCOEF];
__constant__ double c_dtk[kStages + 1];                 // c_k = sum of nonzero a_kj, summed in j order

// ------------------------------------------------------------------ owned-body private state (shared memory)
struct Own {
    int idx, kind, gp, ring;          // kind: 0 point Newtonian (k2 == 0), 1 undelayed tide, 2 delayed tide
    int converged, ext_slot, gl_fixed, full;   // ext_slot: index in the extended-body list, or -1
    int orig, pad1, pad2, pad3;               // orig: index in the caller's plane arrays
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
    double Cs[9];                     // s (C_static + exJ2 terms) s^T of the stage (fixed during the fixed point)
    double fa[3];                     // f_s acceleration of the current stage
    double wnew[3], dw[3];            // stage angular velocity and its 2/3 increment (state update)
    // RK12 accumulators of stages k = 1..25 (index k-1)
    dd accv[kStages][3];
    double acca[kStages][3], accw[kStages][3], acct[kStages][3];
};

// An extended body (geopotential and/or ring host): fixed for the launch, read by every field item
struct HostInfo {
    int E;                            // body index
    short gp, ring;                   // model indices, or -1
    unsigned char nz, nt, nd, pad;    // geopotential zonal / tesseral degree, ring disks
};

// A body whose fields this CTA evaluates: one of its own, or one handed over by a CTA that owns a delayed
// tide (`slot` < 0). Filled at the start of every pass A.
constexpr int kForeignMax = 4;                   // bodies one CTA evaluates the fields of for other CTAs
constexpr int kFieldMax = kOwnMax + kForeignMax;
struct FieldBody {
    int idx, slot;                    // body index; owned-body slot, or -1
    dd r[3];                          // stage position
    double GM;
};

struct Scratch {
    double part[kWarps][16];          // per-warp partial sums
    int split_a0[kOwnMax + 1];        // warp groups of the first pass-A sweep (all owned bodies, weighted)
    int split_b[kOwnMax + 1];         // warp groups of the pass-B sweep (all owned bodies, weighted)
    int nw_b;                         // warps of the pass-B sweep (the last one sums host reactions meanwhile)
    double ext[kOwnMax][kMaxExt][3];  // other hosts' fields on the owned bodies (geopotential, or ring)
    double ext2[kOwnMax][kMaxExt][3]; // ring half of a host that has both models
    double react[kOwnMax][6];         // summed reactions of owned hosts
    HostInfo host[kMaxExt];           // the extended bodies
    unsigned char gp_list[kMaxExt], ring_list[kMaxExt];   // extended-body slots with a geopotential / a ring
    int n_gp_e, n_ring_e, ring_dmax;
    int ext_overlap;                  // geopotential items on warps [kWarps - kExtWarps, kWarps - 1) beside the pass-A sweeps
    int ring_side;                    // ring items on the last warp beside the pass-A sweeps
    int has_delayed;                  // the CTA owns a delayed tide
    int fields_away;                  // this CTA's field items are evaluated by other CTAs (hand-off)
    int n_foreign, foreign[kForeignMax];   // bodies of other CTAs whose field items this CTA evaluates
    int nfb;                          // field bodies of the stage: nb owned ones, then the foreign ones
    FieldBody fb[kFieldMax];
    int nw_a;                         // warps of the pass-A sweeps (fields computed)
    double gp_x[kGpSmem][kGpX];                     // expanded tables of the first kGpSmem geopotential models
    double gp_rcp[EPH_GP_MAX_DEGREE + 2];          // 1/k of the degree recursion
    double rk_hi[EPH_RK12_NCOEF], rk_lo[EPH_RK12_NCOEF];   // a_kj (lane-divergent reads: shared, not constant, memory)
    unsigned long long t_last, t_phase[kPhases];
    unsigned long long mbar;          // mbarrier of the tile copies
    unsigned long long bar_target;    // grid-barrier arrivals that complete the next barrier
    long long traj_slot;              // stage-record slot of the current stage evaluation
    int flag, pad;
};

// Shared memory: the owned bodies, the scratch, then the staging tile of kTileRows rows. The tile's row stride
// kTileW is fixed at compile time (the widest tile that fits), so that every tile access is a fixed offset
// from the body's column; a system of n <= kTileW bodies is staged in one tile, a larger one in chunks.
constexpr int kMaxSmem = 227 * 1024 - 4096;   // the 227 KB per-CTA maximum less room for static arrays
constexpr size_t kFixedSmem = ((sizeof(Own) * kOwnMax + sizeof(Scratch) + 127) / 128) * 128;
constexpr int kTileW = (int)((kMaxSmem - kFixedSmem) / (kTileRows * sizeof(double))) / kPad * kPad;
static_assert(kTileW >= 512, "the staging tile must hold a 512-body system in one piece");

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
__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// Optional phase timers: thread 0 charges the time since the previous mark to phase `ph`. Marks sit
// right after a __syncthreads(), so they bound the whole CTA's work of the phase.
__device__ __forceinline__ void mark(const SysDev &S, Scratch &sc, int ph) {
    if (S.timers && threadIdx.x == 0) {
        unsigned long long t = global_ns();
        sc.t_phase[ph] += t - sc.t_last;
        sc.t_last = t;
    }
}

// Barrier over all CTAs of the launch (co-resident by the cooperative launch). The arrival counter is a
// 64-bit word zeroed before the launch that only grows: barrier number k of the launch is complete when it
// reaches k * gridDim.x, so every CTA announces its arrival with one acquire-release add (which carries the
// CTA's writes, ordered before it by the CTA barrier) and polls the counter only if its add was not the
// last one; no CTA has to reset or flip anything. Returns false when the wait timed out here, or when the
// status word, read in flight with every poll (no dependent load once the barrier completes), shows that
// another CTA failed; the caller then leaves the kernel. A CTA that failed arrives at no later barrier, so
// the others see its status while they wait there.
__device__ bool grid_sync(const SysDev &S, Scratch &sc) {
    __syncthreads();
    if (gridDim.x == 1) return true;
    if (threadIdx.x == 0) {
        unsigned long long *count = reinterpret_cast<unsigned long long *>(S.bar);
        // (S.stall_barrier: a self-test asks for one arrival more than the launch has, so every wait runs out)
        const unsigned long long target = (sc.bar_target += gridDim.x + (S.stall_barrier ? 1u : 0u));
        unsigned long long old;
        asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], 1;" : "=l"(old) : "l"(count) : "memory");
        int fail = 0;
        unsigned long long t0 = 0;
        for (unsigned it = 0; old + 1 < target; ++it) {   // the last arrival does not wait
            // the status word is read before the counter, so that both loads are in flight together
            const int st = *(volatile const int *)S.status;
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(count) : "memory");
            if (v >= target) break;
            if (st != ST_OK) {   // another CTA failed: leave at once
                fail = 1;
                break;
            }
            if ((it & 15) == 15) {
                const unsigned long long t = global_ns();
                if (t0 == 0) t0 = t;
                else if (t - t0 > (unsigned long long)S.wait_ns) {
                    atomicExch(S.status, (int)ST_BARRIER_TIMEOUT);
                    fail = 1;
                    break;
                }
            }
        }
        sc.flag = fail;
    }
    __syncthreads();
    return sc.flag == 0;
}

// ------------------------------------------------------------------ bulk copies into the staging tile
struct TileState {
    unsigned parity;   // phase parity of the mbarrier for the next completion
};

__device__ __forceinline__ void mbar_init(Scratch &sc) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&sc.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// Copy `rows` planes (row r from src[r] + j0, `count` bodies rounded up to kPad; rows from `tail_from` on
// `count_tail` bodies; a null src[r] keeps tile row r as it is) into tile rows of `stride` doubles. Every
// thread waits for completion (bounded). Returns false on timeout.
__device__ bool load_tile(const SysDev &S, Scratch &sc, TileState &ts, double *tile, int stride,
                                       const double *const *src, int rows, int j0, int count, int count_tail,
                                       int tail_from) {
    __syncthreads();   // the previous sweep's reads of the tile are done
    const int cpad = (count + kPad - 1) / kPad * kPad;
    const int tpad = (count_tail + kPad - 1) / kPad * kPad;
    const unsigned bytes = (unsigned)cpad * 8u, tbytes = (unsigned)tpad * 8u;
    unsigned total = 0;
    for (int r = 0; r < rows; ++r)
        if (src[r]) total += r < tail_from ? bytes : tbytes;
    const unsigned mb = smem_addr(&sc.mbar);
    if (threadIdx.x == 0) {
        // order the generic-proxy accesses (tile reads, other CTAs' global stores) before the copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("fence.proxy.async.global;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(total) : "memory");
        for (int r = 0; r < rows; ++r) {
            const unsigned nbytes = r < tail_from ? bytes : tbytes;
            if (nbytes == 0 || !src[r]) continue;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(tile + (size_t)r * stride)),
                "l"(src[r] + j0), "r"(nbytes), "r"(mb)
                : "memory");
        }
    }
    const unsigned parity = ts.parity;
    ts.parity ^= 1u;
    unsigned long long t0 = 0;
    for (unsigned it = 0;; ++it) {
        unsigned done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(mb), "r"(parity)
            : "memory");
        if (done) break;
        if ((it & 63) == 0) {
            unsigned long long t = global_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > (unsigned long long)S.wait_ns) {
                if (threadIdx.x == 0) atomicExch(S.status, (int)ST_COPY_TIMEOUT);
                // give the copies in flight one more bounded wait before the CTA leaves
                const unsigned long long t1 = global_ns();
                for (;;) {
                    asm volatile(
                        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                        : "=r"(done)
                        : "r"(mb), "r"(parity)
                        : "memory");
                    if (done || global_ns() - t1 > (unsigned long long)S.wait_ns) break;
                }
                return false;
            }
        }
    }
    mark(S, sc, PH_IO);   // tile staging (and load/store) time
    return true;
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

__device__ __forceinline__ v3 ld3(const double *p, int ld, int i) {
    return mk(__ldcg(p + i), __ldcg(p + ld + i), __ldcg(p + 2 * ld + i));
}
__device__ __forceinline__ m3 ld9(const double *p, int ld, int i) {
    return m3{ld3(p, ld, i), ld3(p + 3 * ld, ld, i), ld3(p + 6 * ld, ld, i)};
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

// Split the first `nw` warps of the CTA into one group of consecutive warps per active body, in
// proportion to the bodies' weights (the relative cost of their pair terms), each body at least one warp
// (na <= nw): the body with the heaviest pair terms gets the most lanes, so the groups finish together.
// Computed once per launch by one thread: active body a owns warps [first[a], first[a+1]).
__device__ void split_warps(const int *wt, int na, int nw, int *first) {
    int cnt[kOwnMax], tot = 0;
    for (int a = 0; a < na; ++a) tot += wt[a];
    const int spare = nw - na;
    int used = 0;
    for (int a = 0; a < na; ++a) {
        cnt[a] = 1 + spare * wt[a] / tot;
        used += cnt[a];
    }
    // leftover warps to the heaviest bodies first (ties: lower index), one each
    for (int lvl_max = 0x7fffffff; used < nw;) {
        int lvl = -1;
        for (int a = 0; a < na; ++a)
            if (wt[a] < lvl_max && wt[a] > lvl) lvl = wt[a];
        if (lvl < 0) { lvl_max = 0x7fffffff; continue; }
        for (int a = 0; a < na && used < nw; ++a)
            if (wt[a] == lvl) { ++cnt[a]; ++used; }
        lvl_max = lvl;
    }
    first[0] = 0;
    for (int a = 0; a < na; ++a) first[a + 1] = first[a] + cnt[a];
}

struct Group {
    int slot;   // index into the active list
    int tid;    // thread index inside the group
    int size;   // threads in the group
};
__device__ __forceinline__ Group group_of(const int *first, int na) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int a = 0;
    while (a + 1 < na && w >= first[a + 1]) ++a;
    Group g;
    g.slot = a;
    g.tid = (w - first[a]) * 32 + lane;
    g.size = (first[a + 1] - first[a]) * 32;
    return g;
}

// Barrier over the first `nthreads` threads (named barrier 1), or the whole CTA.
__device__ __forceinline__ void part_sync(int nthreads) {
    if (nthreads == (int)blockDim.x) __syncthreads();
    else asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

__device__ __forceinline__ double combine(double a, double b, bool is_max) {
    if (is_max) {
        checked_maximize(a, b);
        return a;
    }
    return a + b;
}

// Reduce-scatter of 16 per-lane values over the warp: afterwards lanes 2c and 2c+1 hold the warp sum of
// value c. 16 shuffles (8 + 4 + 2 + 1 + 1) instead of 5 per value.
__device__ __forceinline__ double warp_reduce_scatter16(double (&v)[16], int lane) {
#pragma unroll
    for (int h = 8, bit = 16; h >= 1; h >>= 1, bit >>= 1) {
        const bool up = (lane & bit) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const double send = up ? v[k] : v[k + h];
            const double keep = up ? v[k + h] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
        }
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// Sum NV per-thread values over each group of the first `nw` warps (a warp reduce-scatter, then the
// group's warps in order, four interleaved partial sums) into out[slot][0..NV); entries c >= max_from are
// NaN-propagating maxima (reduced across the warp with shuffles of their own).
template <int NV>
__device__ __forceinline__ void group_reduce(const double (&acc)[NV], const int *first, int na, int nw, Scratch &sc,
                                             double (*out)[16], int max_from) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    {
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = (c < NV && c < max_from) ? acc[c] : 0.0;
        const double r = warp_reduce_scatter16(v, lane);
        if ((lane & 1) == 0 && (lane >> 1) < min(NV, max_from)) sc.part[w][lane >> 1] = r;
    }
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        if (c < max_from) continue;
        const double v = warp_cmax(acc[c]);
        if (lane == 0) sc.part[w][c] = v;
    }
    part_sync(nw * 32);
    #pragma unroll 1
    for (int idx = threadIdx.x; idx < na * NV; idx += nw * 32) {
        const int slot = idx / NV, c = idx % NV;
        const int w0 = first[slot], w1 = first[slot + 1];
        const bool mx = c >= max_from;
        // four interleaved partial sums over the group's warps (w0 + 4m + q), then combined in q order
        double s0 = sc.part[w0][c], s1 = 0, s2 = 0, s3 = 0;
        const bool h1 = w0 + 1 < w1, h2 = w0 + 2 < w1, h3 = w0 + 3 < w1;
        if (h1) s1 = sc.part[w0 + 1][c];
        if (h2) s2 = sc.part[w0 + 2][c];
        if (h3) s3 = sc.part[w0 + 3][c];
        for (int ww = w0 + 4; ww < w1; ww += 4) {
            s0 = combine(s0, sc.part[ww][c], mx);
            if (ww + 1 < w1) s1 = combine(s1, sc.part[ww + 1][c], mx);
            if (ww + 2 < w1) s2 = combine(s2, sc.part[ww + 2][c], mx);
            if (ww + 3 < w1) s3 = combine(s3, sc.part[ww + 3][c], mx);
        }
        double r = s0;
        if (h1) r = combine(r, s1, mx);
        if (h2) r = combine(r, s2, mx);
        if (h3) r = combine(r, s3, mx);
        out[slot][c] = r;
    }
    part_sync(nw * 32);
}

// ------------------------------------------------------------------ load / publish / store
__device__ void load_own(const SysDev &S, Own *own, int nb, const StepParams &P) {
    const int n = S.n;
    const double *pl = S.planes;
    #pragma unroll 1
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &o = own[b];
        const int i = o.orig;
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
        o.ext_slot = -1;
        for (int e = 0; e < S.n_ext; ++e)
            if (S.ext_body[e] == o.idx) o.ext_slot = e;
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
    #pragma unroll 1
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const Own &o = own[b];
        const int i = o.orig;
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

// publish the stage state of owned body o into public buffer `buf` (one thread)
__device__ void publish_body(const SysDev &S, const Own &o, int buf) {
    const int ld = S.ld, i = o.idx;
    double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    for (int c = 0; c < 3; ++c) {
        pub[(PUB_R_HI + c) * ld + i] = o.r[c].hi;
        pub[(PUB_R_LO + c) * ld + i] = o.r[c].lo;
        pub[(PUB_V_HI + c) * ld + i] = o.v[c].hi;
        pub[(PUB_V_LO + c) * ld + i] = o.v[c].lo;
    }
    v3 gl = fast3(o.GL);
    pub[(PUB_GL + 0) * ld + i] = gl.x;
    pub[(PUB_GL + 1) * ld + i] = gl.y;
    pub[(PUB_GL + 2) * ld + i] = gl.z;
    pub[PUB_GM * ld + i] = o.GM;
    if (o.gp >= 0) {
        for (int q = 0; q < 9; ++q) pub[(PUB_FRAME + q) * ld + i] = dd_val(o.s[q]);
    }
    if (o.ring >= 0) {
        double t[9];
        stm(t, ring_frame(gl));
        for (int q = 0; q < 9; ++q) pub[(PUB_RFRAME + q) * ld + i] = t[q];
    }
}

// publish_body spread over the lanes of one warp
__device__ void publish_body_warp(const SysDev &S, const Own &o, int buf, int lane) {
    const int ld = S.ld, i = o.idx;
    double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    if (lane < 3) {
        const int c = lane;
        pub[(PUB_R_HI + c) * ld + i] = o.r[c].hi;
        pub[(PUB_R_LO + c) * ld + i] = o.r[c].lo;
        pub[(PUB_V_HI + c) * ld + i] = o.v[c].hi;
        pub[(PUB_V_LO + c) * ld + i] = o.v[c].lo;
        pub[(PUB_GL + c) * ld + i] = dd_val(o.GL[c]);
    } else if (lane == 3) {
        pub[PUB_GM * ld + i] = o.GM;
    } else if (lane == 4 && o.ring >= 0) {
        double t[9];
        stm(t, ring_frame(fast3(o.GL)));
        for (int q = 0; q < 9; ++q) pub[(PUB_RFRAME + q) * ld + i] = t[q];
    }
    if (o.gp >= 0 && lane >= 8 && lane < 17) pub[(PUB_FRAME + lane - 8) * ld + i] = dd_val(o.s[lane - 8]);
}

// ------------------------------------------------------------------ pass A: deform_by + angular velocity
// One ordered pair (i = owned body o, j from the tile) of DAMPED_TIDAL_DEFORMATION_MATRIX / _NDELAY /
// _NK2 (mass.impl:1-46), accumulated into acc = {phi, naccel[3], C[9]}.
__device__ __forceinline__ void pair_a(const Own &o, const double *T, int j, double acc[13]) {
    constexpr int ts = kTileW;
    v3 r = mk(sep_diff(T[(TA_R_HI + 0) * ts + j], T[(TA_R_LO + 0) * ts + j], o.r[0].hi, o.r[0].lo),
              sep_diff(T[(TA_R_HI + 1) * ts + j], T[(TA_R_LO + 1) * ts + j], o.r[1].hi, o.r[1].lo),
              sep_diff(T[(TA_R_HI + 2) * ts + j], T[(TA_R_LO + 2) * ts + j], o.r[2].hi, o.r[2].lo));
    const double GMj = T[TA_GM * ts + j], sR2j = T[TA_SR2 * ts + j];
    double q = dot(r, r), sm = o.sR2 + sR2j;
    double rr = rsqrt((q < sm) ? sm : q);   // 1/r within 1 ulp; rr2 = rr^2
    double rr2 = rr * rr;
    double tp_dphi = rr * GMj;
    double tp_dg = rr2 * tp_dphi;
    acc[0] -= tp_dphi;
    acc[1] += tp_dg * r.x;
    acc[2] += tp_dg * r.y;
    acc[3] += tp_dg * r.z;
    if (o.kind == 0) return;
    double fk = (-3 * tp_dg) * o.k2;
    m3 M;
    if (o.kind == 2) {
        v3 v = mk(sep_diff(T[(TA_V_HI + 0) * ts + j], T[(TA_V_LO + 0) * ts + j], o.v[0].hi, o.v[0].lo),
                  sep_diff(T[(TA_V_HI + 1) * ts + j], T[(TA_V_LO + 1) * ts + j], o.v[1].hi, o.v[1].lo),
                  sep_diff(T[(TA_V_HI + 2) * ts + j], T[(TA_V_LO + 2) * ts + j], o.v[2].hi, o.v[2].lo));
        v3 w = mk(o.w[0], o.w[1], o.w[2]);
        v3 dw = rr2 * cross(r, cross(w, r) - v);
        double dwt;
        const double dw2 = dot(dw, dw);
        if (dw2 > 0x1p-960 && dw2 < 0x1p960) {   // inside the range where normalize needs no rescaling
            const double rn = rsqrt(dw2);
            dwt = dw2 * rn;
            dw = rn * dw;
        } else {
            dwt = normalize(dw);
        }
        dwt *= o.td * T[TA_TDF * ts + j];
        // x0, y0, z02 of the damped deformation (mass.impl:16-20) from two reciprocal square roots: with
        // e = 1 + 4 dwt^2, s = sqrt(e), u = 1 + s, re = 1/s and ru = 1/sqrt(u/2),
        //   x0 = sqrt(u / (2e)) = (u/2) ru re,  y0 = dwt sqrt(2 / (e u)) = dwt ru re,
        //   z02 = 2 dwt^2 / (e + s) = dwt^2 re ru^2.
        const double e = 1 + 4 * dwt * dwt;
        const double re = rsqrt(e);
        const double hu = 0.5 * (1 + e * re);
        const double ru = rsqrt(hu);
        const double rue = ru * re;
        const double x0 = hu * rue, y0 = dwt * rue, z02 = (dwt * dwt) * (rue * ru);
        v3 dr = x0 * r + y0 * cross(dw, r);
        M = add_diag(outer(rr2 * dr, dr) - outer(z02 * dw, dw), z02 - 1.0 / 3);
    } else {
        M = add_diag(outer(rr2 * r, r), -(1.0 / 3));
    }
    acc[4] -= fk * M.x.x; acc[5] -= fk * M.x.y; acc[6] -= fk * M.x.z;
    acc[7] -= fk * M.y.x; acc[8] -= fk * M.y.y; acc[9] -= fk * M.y.z;
    acc[10] -= fk * M.z.x; acc[11] -= fk * M.z.y; acc[12] -= fk * M.z.z;
}

// UPDATE_HARMONICS followed by UPDATE_ANGULAR_VELOCITY (mass.impl:48-72) for owned body o, on one thread,
// from the pass-A sums in o.sumA. The first iteration of a stage (`first`) also sets the potential and the
// Newtonian acceleration and rotates the static harmonics into the world frame once for the stage (they do
// not depend on the angular velocity). Sets o.converged: the reference's convergence test, or an iteration
// that reproduces w exactly (a fixed point: every further iteration of the reference's loop recomputes the
// same sums, harmonics and w, so stopping leaves the identical state; needed for w = 0, where
// 0 < 1e-18 * 0 never passes). Small and branch-light on purpose: it runs once per fixed-point iteration on
// the critical path of the stage.
__device__ void update_body(Own &o, bool first, bool deform_only) {
    if (first) {
        o.phi = o.sumA[0];
        o.nacc[0] = o.sumA[1]; o.nacc[1] = o.sumA[2]; o.nacc[2] = o.sumA[3];
        m3 mc = ldm(o.Cst);
        mc.x.x += o.exJ2 / 2;
        mc.y.y += o.exJ2 / 2;
        mc.z.z -= o.exJ2;
        stm(o.Cs, toworld(fast9(o.s), mc));
    }
    const v3 w = ldv(o.w);
    m3 C = ldm(o.sumA + 4);
    C = add_diag(C, dot(w, w) * o.k2r / 3);
    C = C - outer(o.k2r * w, w);
    C = (o.R * o.R2 / (2 * o.GM)) * C;
    C = C + ldm(o.Cs);
    stm(o.C, C);
    const m3 GI = ((-2.0) / 3 * o.R2) * add_diag(C, -o.A);
    stm(o.GI, GI);
    if (deform_only) { o.converged = 1; return; }
    bool finite = true;
    for (int c = 0; c < 3; ++c) finite = finite && dd_finite(o.GL[c]);
    if (!finite) {   // UPDATE_ANGULAR_VELOCITY's else-branch: G*L = GI w
        const v3 gl = mul(GI, w);
        o.GL[0] = dd_make(gl.x); o.GL[1] = dd_make(gl.y); o.GL[2] = dd_make(gl.z);
        o.gl_fixed = 1;
        o.converged = 1;
        return;
    }
    const v3 nw = mul(inverse(GI), fast3(o.GL));
    stv(o.w, nw);
    const v3 d = nw - w;
    const bool same = nw.x == w.x && nw.y == w.y && nw.z == w.z;
    o.converged = (same || dot(d, d) < 1e-18 * dot(w, w)) ? 1 : 0;
}

// Sources of the pass-A tile rows. Only a delayed tide reads the velocities and tidal delay factors of the
// bodies j: a CTA without one leaves those rows out of the copy (null source).
__device__ __forceinline__ void tile_a_rows(const SysDev &S, const double *pub, bool need_v, const double *(&src)[TA_ROWS]) {
    const int ld = S.ld;
    for (int c = 0; c < 3; ++c) {
        src[TA_R_HI + c] = pub + (PUB_R_HI + c) * ld;
        src[TA_R_LO + c] = pub + (PUB_R_LO + c) * ld;
        src[TA_V_HI + c] = need_v ? pub + (PUB_V_HI + c) * ld : nullptr;
        src[TA_V_LO + c] = need_v ? pub + (PUB_V_LO + c) * ld : nullptr;
    }
    src[TA_GM] = pub + PUB_GM * ld;
    src[TA_SR2] = S.cst + CST_SR2 * ld;
    src[TA_TDF] = need_v ? S.cst + CST_TDF * ld : nullptr;
}

// Pair sums of pass A for the owned bodies in `mask` over all bodies j, by the first `nw` warps (tile
// already staged when the whole system fits in one tile; otherwise tiles are streamed, which needs the
// whole CTA, nw == kWarps). Results land in own[b].sumA. One pair per iteration: a second pair chain in
// flight per thread spills registers at the kernel's 128 per thread.
__device__ bool sweep_a(const SysDev &S, Own *own, int nb, unsigned mask, int buf, Scratch &sc, TileState &ts,
                        double *tile, bool staged, int nw, const int *first_all) {
    const int na = __popc(mask);
    if (na == 0) return true;
    const int ld = S.ld, n = S.n, T = S.tile;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    // Warp groups: the first sweep of a stage covers every owned body (`first_all`, weighted, fixed per
    // launch); a re-sweep covers the unconverged delayed tides, which all cost the same, so the nw warps are
    // split equally: slot a owns warps [ceil(a nw / na), ceil((a + 1) nw / na)), i.e. warp w is in slot
    // floor(w na / nw). Every thread works its group out itself: no shared list, no barrier.
    auto bounds = [&](int slot, int &w0, int &w1) {
        if (first_all) { w0 = first_all[slot]; w1 = first_all[slot + 1]; }
        else { w0 = (slot * nw + na - 1) / na; w1 = ((slot + 1) * nw + na - 1) / na; }
    };
    auto body_of = [&](int slot) {   // the slot-th set bit of mask
        unsigned m = mask;
        for (int k = 0; k < slot; ++k) m &= m - 1;
        return __ffs(m) - 1;
    };
    const int warp = threadIdx.x >> 5;
    int my_slot;
    if (first_all) { my_slot = 0; while (my_slot + 1 < na && warp >= first_all[my_slot + 1]) ++my_slot; }
    else my_slot = (warp * na) / nw;
    int gw0, gw1;
    bounds(my_slot, gw0, gw1);
    const Group g{my_slot, (warp - gw0) * 32 + (int)(threadIdx.x & 31), (gw1 - gw0) * 32};
    const Own &o = own[body_of(my_slot)];
    double acc[13];
#pragma unroll
    for (int c = 0; c < 13; ++c) acc[c] = 0;
    #pragma unroll 1
    for (int j0 = 0; j0 < n; j0 += T) {
        const int cnt = min(T, n - j0);
        if (!staged) {
            const double *src[TA_ROWS];
            tile_a_rows(S, pub, sc.has_delayed, src);
            if (!load_tile(S, sc, ts, tile, kTileW, src, TA_ROWS, j0, cnt, cnt, TA_ROWS)) return false;
        }
        const int self = o.idx - j0;
#pragma unroll 1
        for (int jj = g.tid; jj < cnt; jj += g.size)
            if (jj != self) pair_a(o, tile, jj, acc);
    }
    // sums over each body's warp group: a warp reduce-scatter, then the group's warps in ascending order
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = c < 13 ? acc[c] : 0.0;
        const double r = warp_reduce_scatter16(v, lane);
        if ((lane & 1) == 0 && (lane >> 1) < 13) sc.part[w][lane >> 1] = r;
    }
    part_sync(nw * 32);
    #pragma unroll 1
    for (int idx = threadIdx.x; idx < na * 13; idx += nw * 32) {
        const int slot = idx / 13, c = idx % 13;
        int w0, w1;
        bounds(slot, w0, w1);
        double p[kWarps];   // every load first, then the sum in warp order
#pragma unroll
        for (int k = 0; k < kWarps; ++k) p[k] = w0 + k < w1 ? sc.part[w0 + k][c] : 0.0;
        double sum = p[0];
#pragma unroll
        for (int k = 1; k < kWarps; ++k)
            if (w0 + k < w1) sum += p[k];
        own[body_of(slot)].sumA[c] = sum;
    }
    part_sync(nw * 32);
    return true;
}

// Reactions of the field items before the CTA's ordered sum, per (host slot e, owned body b, model half):
// six values (force, torque). They stay in the pass-A tile's free rows when those hold them, else they go
// through the global table S.react.
struct ReactStage {
    double *smem;   // [n_ext][nb][2][6] in shared memory, or null
    int nb;
    __device__ __forceinline__ double *slot(const SysDev &S, int e, int b, int idx, int half) const {
        return smem ? smem + ((size_t)(e * nb + b) * 2 + half) * 6 : S.react + (((size_t)e * S.ld + idx) * 2 + half) * 6;
    }
    __device__ __forceinline__ double get(const double *p) const { return smem ? *p : __ldcg(p); }
};
constexpr int kRingTerms = kFieldMax * kRingPar * kRingDiskPar * 3;   // per-disk ring terms, [f][h][d][3]

// Geopotential items (field body b, geopotential host slot e) on `nthr` threads (t = this
// thread's index), G lanes per item: every item's lanes evaluate it together (gp_field_lanes on the
// expanded table in shared memory, columns of the recursion split over the lanes) and the group's first
// lane stores it; a model beyond the shared-memory copies runs gp_field on that lane alone.
template <int G, typename Put>
__device__ __forceinline__ void gp_items(const SysDev &S, const FieldBody *fb, int nb, const double *pub, const Scratch &sc,
                                         int t, int nthr, const Put &put) {
    const int ld = S.ld, ng = sc.n_gp_e;
    const int q = t & (G - 1), lane = threadIdx.x & 31;
    const unsigned mask = G == 1 ? (1u << lane) : (((1u << G) - 1u) << (lane & ~(G - 1)));
    #pragma unroll 1
    for (int item = t / G; item < nb * ng; item += nthr / G) {
        const int b = item / ng, e = sc.gp_list[item % ng];
        const FieldBody &o = fb[b];
        const HostInfo h = sc.host[e];
        const bool live = h.E != o.idx;
        v3 r = mk(0, 0, 0), an = mk(0, 0, 0);
        double GME = 0;
        if (live) {   // uniform over the group
            const int E = h.E;
            r = mk(dd_diff(o.r[0].hi, o.r[0].lo, __ldcg(pub + PUB_R_HI * ld + E), __ldcg(pub + PUB_R_LO * ld + E)),
                   dd_diff(o.r[1].hi, o.r[1].lo, __ldcg(pub + (PUB_R_HI + 1) * ld + E), __ldcg(pub + (PUB_R_LO + 1) * ld + E)),
                   dd_diff(o.r[2].hi, o.r[2].lo, __ldcg(pub + (PUB_R_HI + 2) * ld + E), __ldcg(pub + (PUB_R_LO + 2) * ld + E)));
            GME = __ldcg(pub + PUB_GM * ld + E);
            const m3 f = ld9(pub + PUB_FRAME * ld, ld, E);
            const double R = __ldg(S.cst + CST_R * ld + E);
            v3 al = mk(0, 0, 0);
            if (G == 1 && h.gp < kGpSmem && gp_fits_columns(h.nz, h.nt))
                al = gp_field_columns<kGpColK, kGpColM>(sc.gp_x[h.gp], sc.gp_rcp, R, tolocal(f, r));
            else if (h.gp < kGpSmem) al = gp_field_lanes<G>(sc.gp_x[h.gp], sc.gp_rcp, h.nz, h.nt, R, tolocal(f, r), q, mask);
            else if (q == 0) al = gp_field(S.gp_coef + (size_t)h.gp * EPH_GP_TABLE_SIZE, h.nz, h.nt, R, tolocal(f, r));
            an = toworld(f, al);
        }
        if (q == 0) put(0, b, e, o, r, an, GME, live);
    }
}

// Fields of the geopotential / ring hosts at the field bodies, once per (host, body) item: the force on an
// owned body goes to sc.ext (geopotential) / sc.ext2 (ring), on a body of another CTA to the global
// table S.react (its slots [host][body][half][0..2], read by the owner in pass B), the host's reaction to
// the staging `st` (APPLY_NONPOINT_FORCE, mass.impl:127-130; r = r_body - r_host as `mj.r - mi.r` with mi
// the host, mass.cpp:358-371). Only the halves of a host's models are written: the readers skip the half a
// host does not have.
struct FieldPut {
    const SysDev &S;
    Scratch &sc;
    const ReactStage &st;
    __device__ void operator()(int half, int b, int e, const FieldBody &o, v3 r, v3 an, double GME, bool live) const {
        v3 add3 = mk(0, 0, 0), da = mk(0, 0, 0), dt = mk(0, 0, 0);
        if (live) {
            add3 = GME * an;
            da = -(o.GM * an);
            dt = -(o.GM * cross(r, an));
        }
        double *f;
        if (o.slot >= 0) f = (half ? sc.ext2 : sc.ext)[o.slot][e];
        else f = S.react + (((size_t)e * S.ld + o.idx) * 2 + half) * 6;
        f[0] = add3.x; f[1] = add3.y; f[2] = add3.z;
        double *rc = st.slot(S, e, b, o.idx, half);
        rc[0] = da.x; rc[1] = da.y; rc[2] = da.z; rc[3] = dt.x; rc[4] = dt.y; rc[5] = dt.z;
    }
};

__device__ __forceinline__ v3 body_sep(const FieldBody &o, const double *pub, int ld, int E) {   // r_body - r_host (mass.cpp:184,198)
    return mk(dd_diff(o.r[0].hi, o.r[0].lo, __ldcg(pub + PUB_R_HI * ld + E), __ldcg(pub + PUB_R_LO * ld + E)),
              dd_diff(o.r[1].hi, o.r[1].lo, __ldcg(pub + (PUB_R_HI + 1) * ld + E), __ldcg(pub + (PUB_R_LO + 1) * ld + E)),
              dd_diff(o.r[2].hi, o.r[2].lo, __ldcg(pub + (PUB_R_HI + 2) * ld + E), __ldcg(pub + (PUB_R_LO + 2) * ld + E)));
}

// Geopotential items on warps [w_lo, w_hi), as many lanes per item as one round over the items allows
// (more lanes: shorter chains).
__device__ void ext_gp(const SysDev &S, const FieldBody *own, int nb, int buf, Scratch &sc, const ReactStage &st, int w_lo,
                       int w_hi) {
    if (sc.n_gp_e == 0) return;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * S.ld;
    const FieldPut put{S, sc, st};
    const int nthr = (w_hi - w_lo) * 32, t = threadIdx.x - w_lo * 32;
    const int items = nb * sc.n_gp_e;
    if (items * 8 <= nthr) gp_items<8>(S, own, nb, pub, sc, t, nthr, put);
    else if (items * 4 <= nthr) gp_items<4>(S, own, nb, pub, sc, t, nthr, put);
    else if (items * 2 <= nthr) gp_items<2>(S, own, nb, pub, sc, t, nthr, put);
    else gp_items<1>(S, own, nb, pub, sc, t, nthr, put);
}

// Ring items on the calling warp. With few hosts and disks each lane takes one (body, host, disk) term and
// the terms are added in disk order afterwards (ring.impl:2122-2192, staged in `rterm`); otherwise one lane
// per (body, host) runs ring::sum whole.
__device__ void ext_ring(const SysDev &S, const FieldBody *own, int nb, int buf, Scratch &sc, const ReactStage &st,
                         double *rterm) {
    const int ld = S.ld, lane = threadIdx.x & 31;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    const FieldPut put{S, sc, st};
    const int nr = sc.n_ring_e, dmax = sc.ring_dmax;
    if (nr == 0) return;
    if (nr > kRingPar || dmax > kRingDiskPar) {
        #pragma unroll 1
        for (int item = lane; item < nb * nr; item += 32) {
            const int b = item / nr, e = sc.ring_list[item % nr];
            const FieldBody &o = own[b];
            const HostInfo h = sc.host[e];
            const bool live = h.E != o.idx;
            v3 r = mk(0, 0, 0), an = mk(0, 0, 0);
            double GME = 0;
            if (live) {
                r = body_sep(o, pub, ld, h.E);
                GME = __ldcg(pub + PUB_GM * ld + h.E);
                m3 f = ld9(pub + PUB_RFRAME * ld, ld, h.E);
                an = toworld(f, ring_sum(S.ring_disk + (size_t)h.ring * EPH_RING_MAX_DISKS * 3, h.nd,
                                         __ldg(S.cst + CST_R * ld + h.E), tolocal(f, r)));
            }
            put(1, b, e, o, r, an, GME, live);
        }
        return;
    }
    #pragma unroll 1
    for (int item = lane; item < nb * nr * dmax; item += 32) {
        const int b = item / (nr * dmax), hh = (item / dmax) % nr, d = item % dmax;
        const FieldBody &o = own[b];
        const HostInfo h = sc.host[sc.ring_list[hh]];
        v3 t = mk(0, 0, 0);
        if (h.E != o.idx && d < h.nd) {
            m3 f = ld9(pub + PUB_RFRAME * ld, ld, h.E);
            const RingGeom g = ring_geom(tolocal(f, body_sep(o, pub, ld, h.E)));
            t = ring_disk_term(S.ring_disk + ((size_t)h.ring * EPH_RING_MAX_DISKS + d) * 3, __ldg(S.cst + CST_R * ld + h.E), g);
        }
        double *rt = rterm + ((b * kRingPar + hh) * kRingDiskPar + d) * 3;
        rt[0] = t.x; rt[1] = t.y; rt[2] = t.z;
    }
    __syncwarp();
    #pragma unroll 1
    for (int item = lane; item < nb * nr; item += 32) {
        const int b = item / nr, hh = item % nr, e = sc.ring_list[hh];
        const FieldBody &o = own[b];
        const HostInfo h = sc.host[e];
        const bool live = h.E != o.idx;
        v3 r = mk(0, 0, 0), an = mk(0, 0, 0);
        double GME = 0;
        if (live) {
            r = body_sep(o, pub, ld, h.E);
            GME = __ldcg(pub + PUB_GM * ld + h.E);
            m3 f = ld9(pub + PUB_RFRAME * ld, ld, h.E);
            const RingGeom g = ring_geom(tolocal(f, r));
            v3 ret = mk(0, 0, 0);
            const double *rt = rterm + (b * kRingPar + hh) * kRingDiskPar * 3;
            for (int d = 0; d < h.nd; ++d) ret += mk(rt[3 * d], rt[3 * d + 1], rt[3 * d + 2]);
            if (g.psign) ret.z = -ret.z;
            an = toworld(f, ret);
        }
        put(1, b, e, o, r, an, GME, live);
    }
}

// This CTA's share of every host's reaction on threads [t0, t0 + nthr): the sum over its owned bodies (in
// ownership order) of both model halves, S.react_cta[host][CTA][6], so that a host's owner adds one value per
// CTA in pass B instead of one per body.
__device__ void ext_react(const SysDev &S, const FieldBody *own, int nb, const Scratch &sc, const ReactStage &st, int t0,
                          int nthr) {
    const int ld = S.ld;
    #pragma unroll 1
    for (int item = threadIdx.x - t0; item < S.n_ext * 6; item += nthr) {
        const int e = item / 6, c = item % 6;
        const HostInfo h = sc.host[e];
        double sum = 0;
        for (int b = 0; b < nb; ++b) {
            const double *rc = st.slot(S, e, b, own[b].idx, 0);   // halves at rc[0..5] and rc[6..11]
            const double g = h.gp >= 0 ? st.get(rc + c) : 0.0;
            const double r = h.ring >= 0 ? st.get(rc + 6 + c) : 0.0;
            sum += g + r;
        }
        S.react_cta[((size_t)e * ld + blockIdx.x) * 6 + c] = sum;
    }
}

// The stage record of owned body o for massless particles (TrajField layout), in the caller's body order.
__device__ __noinline__ void record_body(const SysDev &S, const Own &o, long long slot) {
    double *t = S.traj + ((size_t)slot * S.n + o.orig) * kTrajRec;
    for (int c = 0; c < 3; ++c) {
        t[TR_R_HI + c] = o.r[c].hi;
        t[TR_R_LO + c] = o.r[c].lo;
        t[TR_NACC + c] = o.nacc[c];
        t[TR_BETA + c] = o.beta[c];
    }
    t[TR_GM] = o.GM;
    t[TR_PHI] = o.phi;
    t[TR_BETA2] = o.beta2;
    for (int q = 0; q < 9; ++q) t[TR_CPOT + q] = o.C[q];
    t[TR_R2] = o.R2;
    const v3 gl = fast3(o.GL);
    t[TR_GL + 0] = gl.x; t[TR_GL + 1] = gl.y; t[TR_GL + 2] = gl.z;
    for (int q = 0; q < 9; ++q) t[TR_FRAME + q] = dd_val(o.s[q]);
    t[TR_RADIUS] = o.R;
    t[TR_SR2] = o.sR2;
    double rf[9];
    stm(rf, ring_frame(gl));
    for (int q = 0; q < 9; ++q) t[TR_RFRAME + q] = o.ring >= 0 ? rf[q] : 0.0;
}

__device__ bool pass_a(const SysDev &S, Own *own, int nb, int buf, bool deform_only, Scratch &sc, TileState &ts,
                       double *tile) {
    const int ld = S.ld;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    if (threadIdx.x < nb) { own[threadIdx.x].converged = 0; own[threadIdx.x].gl_fixed = 0; }
    // the bodies whose fields this CTA evaluates: its own (ordered before their use by load_tile's CTA
    // barrier), then those handed over to it (filled by the field warps below)
    if (threadIdx.x < nb) {
        FieldBody &f = sc.fb[threadIdx.x];
        const Own &o = own[threadIdx.x];
        f.idx = o.idx; f.slot = threadIdx.x; f.GM = o.GM;
        for (int c = 0; c < 3; ++c) f.r[c] = o.r[c];
    }
    const bool one_tile = S.n <= S.tile;
    if (one_tile) {
        const double *src[TA_ROWS];
        tile_a_rows(S, pub, sc.has_delayed, src);
        if (!load_tile(S, sc, ts, tile, kTileW, src, TA_ROWS, 0, S.n, S.n, TA_ROWS)) return false;
    } else {
        __syncthreads();
    }
    // The extended bodies' fields do not depend on the angular velocity, so they run beside the pass-A sweeps
    // (one tile only: streaming tiles needs every warp): the ring items on the last warp, the geopotential
    // items (sc.ext_overlap) on the kExtWarps - 1 warps before it. With streaming tiles they run on every warp
    // after the sweeps. The per-disk ring terms and, when they fit, the reactions are staged in the rows of
    // the pass-A tile that pass A does not use.
    const bool fields = !deform_only && S.n_ext > 0 && !sc.fields_away;
    const bool ring_side = fields && sc.ring_side;
    const bool gp_side = fields && sc.ext_overlap;
    const int max_iter = deform_only ? 1 : 4;   // MAX_ANGULAR_VELOCITY_ITER (mass.impl:74)
    const int nw = deform_only ? kWarps : sc.nw_a;
    double *xa = tile + (size_t)TA_ROWS * kTileW;
    const int nf = sc.nfb;
    const ReactStage st{kRingTerms + nf * S.n_ext * 12 <= (kTileRows - TA_ROWS) * kTileW ? xa + kRingTerms : nullptr, nf};
    const int warp = threadIdx.x >> 5;
    if (warp < nw) {
        #pragma unroll 1
        for (int it = 0; it < max_iter; ++it) {
            unsigned mask = 0;
            for (int b = 0; b < nb; ++b) {
                // the pair sums depend on the angular velocity only for delayed tides
                if (it == 0 || (!own[b].converged && own[b].kind == 2)) mask |= 1u << b;
            }
            if (!sweep_a(S, own, nb, mask, buf, sc, ts, tile, one_tile, nw, it == 0 ? sc.split_a0 : nullptr)) return false;
            if (S.timers && threadIdx.x == 0) sc.t_phase[PH_A_COUNT] += 1;
            mark(S, sc, PH_A_SWEEP);   // thread 0 sits in a sweep warp
            // harmonics and angular velocity of the owned bodies: lane 0 of warp b updates body b
            if (warp < nb && (threadIdx.x & 31) == 0 && !own[warp].converged) update_body(own[warp], it == 0, deform_only);
            part_sync(nw * 32);
            mark(S, sc, PH_A_UPDATE);
            int all = 1;
            for (int b = 0; b < nb; ++b) all &= own[b].converged;
            if (all) break;
        }
    }
    // the field items: phase 0 beside the sweeps (warps >= nw), phase 1 after them on every warp; one call
    // site per evaluator, so that each is compiled once
    const bool ring_after = fields && !ring_side && sc.n_ring_e > 0;
    // handed-over bodies (only with the fields beside the sweeps): their stage position and GM from the
    // published state, loaded by the field warps once the tile copies are under way
    if (warp >= nw && sc.n_foreign > 0) {
        const int k = threadIdx.x - nw * 32;
        if (k < sc.n_foreign) {
            FieldBody &f = sc.fb[nb + k];
            const int j = sc.foreign[k];
            f.idx = j; f.slot = -1; f.GM = __ldcg(pub + PUB_GM * ld + j);
            for (int c = 0; c < 3; ++c) f.r[c] = dd{__ldcg(pub + (PUB_R_HI + c) * ld + j), __ldcg(pub + (PUB_R_LO + c) * ld + j)};
        }
        asm volatile("bar.sync 2, %0;" ::"r"((kWarps - nw) * 32) : "memory");
    }
    #pragma unroll 1
    for (int ph = 0; ph < 2; ++ph) {
        if (ph == 1) {
            __syncthreads();
            if (!fields || (gp_side && !ring_after)) break;
        }
        const bool ring_here = warp == kWarps - 1 && (ph == 0 ? ring_side : ring_after);
        const bool gp_here = ph == 0 ? (gp_side && warp >= nw) : !gp_side;
        const int gp_lo = ph == 0 ? kWarps - kExtWarps : 0;
        const int gp_hi = (ph == 0 ? ring_side : ring_after) ? kWarps - 1 : kWarps;
        if (ring_here) ext_ring(S, sc.fb, nf, buf, sc, st, xa);
        else if (gp_here && warp >= gp_lo && warp < gp_hi) ext_gp(S, sc.fb, nf, buf, sc, st, gp_lo, gp_hi);
    }
    if (fields) {
        __syncthreads();
        ext_react(S, sc.fb, nf, sc, st, 0, blockDim.x);
        __syncthreads();
    }
    mark(S, sc, PH_B_EXT);   // the fields beyond the sweeps and updates
    if (deform_only) return true;
    // PREPARE_RELATIVITY (mass.impl:76-80) and the pass-A outputs other CTAs read in pass B
    const double c2 = kC * kC;
    #pragma unroll 1
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
        aux[AUX_PHI * ld + i] = o.phi;
        for (int c = 0; c < 3; ++c) {
            aux[(AUX_NACC + c) * ld + i] = o.nacc[c];
            aux[(AUX_BETA + c) * ld + i] = o.beta[c];
        }
        aux[AUX_BETA2 * ld + i] = o.beta2;
        for (int q = 0; q < 9; ++q) aux[(AUX_CPOT + q) * ld + i] = o.C[q];
        // a non-finite G*L was replaced by GI*w: republish it for pass B
        if (o.gl_fixed) publish_body(S, o, buf);
        if (S.traj) record_body(S, o, sc.traj_slot);
    }
    __syncthreads();
    mark(S, sc, PH_A_UPDATE);
    return true;
}

// ------------------------------------------------------------------ pass B: main force
// Extremal pairs of the per-pair maxima (RungeKutta.cu:229-230; min_distance tracks 1/r, max_influence
// GM/r^3). The sweep uses a 1-ulp reciprocal square root; the extremes are recomputed afterwards with
// the reference's own expressions rr2 = 1/m, rr = sqrt(rr2) (mass.impl:84-89) from the tracked pair.
struct Extremes {
    double m_min;           // smallest max(r^2, sR2_i + sR2_j): the largest 1/r
    double tq, tq_m, tq_gm; // largest GM/r^3 seen (approximate), with its m and GM_j
};
__device__ __forceinline__ void track(Extremes &x, double m, double tp_dg, double GMj) {
    if (x.m_min == x.m_min) x.m_min = (m != m || m < x.m_min) ? m : x.m_min;   // NaN sticks
    if (x.tq == x.tq) {
        if (tp_dg != tp_dg) x.tq = tp_dg;
        else if (tp_dg > x.tq) { x.tq = tp_dg; x.tq_m = m; x.tq_gm = GMj; }
    }
}

// One ordered pair of RELATIVITY, ROTATIONAL_TIDAL_DEFORMATION_NANTI_FORCE, LENSE_THIRRING and
// RADIATION_PRESSURE (mass.impl:82-125, mass.cpp:147-155) into acc = {gaccel[3], daccel[3], dtorque[3]}.
// IF / JF: body i / body j of the full class. For a point-like body the deformation matrix, G*L,
// luminosity and receptance are all zero, so the terms they multiply are exactly zero and skipped.
template <bool IF, bool JF>
__device__ __forceinline__ void pair_b(const Own &o, const double *T, int j, double acc[9], Extremes &x) {
    constexpr int ts = kTileW;
    v3 r = mk(sep_diff(T[(TB_R_HI + 0) * ts + j], T[(TB_R_LO + 0) * ts + j], o.r[0].hi, o.r[0].lo),
              sep_diff(T[(TB_R_HI + 1) * ts + j], T[(TB_R_LO + 1) * ts + j], o.r[1].hi, o.r[1].lo),
              sep_diff(T[(TB_R_HI + 2) * ts + j], T[(TB_R_LO + 2) * ts + j], o.r[2].hi, o.r[2].lo));
    const double GMj = T[TB_GM * ts + j];
    const double q = dot(r, r), sm = o.sR2 + T[TB_SR2 * ts + j];
    const double m = (q < sm) ? sm : q;
    const double rr = rsqrt(m);
    const double rr2 = rr * rr;
    const double rr3 = rr * rr2;
    const double tp_dphi = rr * GMj;
    const double tp_dg = rr2 * tp_dphi;
    track(x, m, tp_dg, GMj);
    v3 bj = mk(T[(TB_BETA + 0) * ts + j], T[(TB_BETA + 1) * ts + j], T[(TB_BETA + 2) * ts + j]);
    v3 bi = ldv(o.beta);
    double rbj = dot(r, bj);
    double tp = rbj * rr;
    tp *= tp;
    v3 naj = mk(T[(TB_NACC + 0) * ts + j], T[(TB_NACC + 1) * ts + j], T[(TB_NACC + 2) * ts + j]);
    double delta1 = 4 * o.phi + T[TB_PHI * ts + j] + o.beta2 + 2 * T[TB_BETA2 * ts + j] - 4 * dot(bi, bj) +
                    (dot(r, naj) - 3 * tp) / 2;
    v3 b = bj - bi;
    v3 g = (7 * tp_dphi / 2) * naj + (tp_dg * delta1) * r + (tp_dg * (rbj - dot(r, b) * 4)) * b;
    acc[0] += g.x; acc[1] += g.y; acc[2] += g.z;
    if (!IF && !JF) return;
    v3 da = mk(0, 0, 0), dt = mk(0, 0, 0);
    const double rcr32 = 2 * GMj / kC * rr3;
    if (IF) {
        // deformation of i, Lense-Thirring of i's spin, radiation received by i
        m3 Ci = ldm(o.C);
        v3 Cr = mul(Ci, r);
        v3 dg = (GMj * rr3 * rr2 * o.R2) * ((dot(r, Cr) * 5 * rr2) * r - (Cr + Cr));
        da = dg;
        dt = cross(r, dg);
        v3 GL = fast3(o.GL);
        v3 GLb = cross(GL, b);
        da -= rcr32 * (GLb - (3 * dot(GLb, r) * rr2) * r);
        dt -= rcr32 * cross(GL, cross(r, b));
    }
    if (JF) {
        // deformation of j (no reaction written to j: recomputed by j's owner), j's spin, j's light
        const double *Cjp = T + TB_CPOT * ts + j;
        m3 Cj = m3{mk(Cjp[0], Cjp[ts], Cjp[2 * ts]), mk(Cjp[3 * ts], Cjp[4 * ts], Cjp[5 * ts]),
                   mk(Cjp[6 * ts], Cjp[7 * ts], Cjp[8 * ts])};
        v3 Cjr = mul(Cj, r);
        da += (GMj * rr3 * rr2 * T[TB_R2 * ts + j]) * ((dot(r, Cjr) * 5 * rr2) * r - (Cjr + Cjr));
        v3 GLj = mk(T[(TB_GL + 0) * ts + j], T[(TB_GL + 1) * ts + j], T[(TB_GL + 2) * ts + j]);
        da += cross(rcr32 * (GLj - (3 * dot(GLj, r) * rr2) * r), b);
        if (IF) da += (T[TB_LUM * ts + j] * o.rR2G4c * rr3 / o.GM) * r;
    }
    acc[3] += da.x; acc[4] += da.y; acc[5] += da.z;
    acc[6] += dt.x; acc[7] += dt.y; acc[8] += dt.z;
}

template <bool IF, bool JF>
__device__ __forceinline__ void sweep_b_range(const Own &o, const double *tile, int lo, int hi, int self,
                                              const Group &g, double acc[9], Extremes &x) {
#pragma unroll 1
    for (int jj = lo + g.tid; jj < hi; jj += g.size)
        if (jj != self) pair_b<IF, JF>(o, tile, jj, acc, x);
}

__device__ bool pass_b(const SysDev &S, Own *own, int nb, int buf, Scratch &sc, TileState &ts, double *tile) {
    const int ld = S.ld, n = S.n, T = S.tile;
    const double *pub = S.pub + (size_t)buf * PUB_NPLANES * ld;
    const double *aux = S.aux, *cst = S.cst;
    const int nwb = sc.nw_b;
    const bool sweeper = (threadIdx.x >> 5) < nwb;
    const Group g = group_of(sc.split_b, nb);
    const Own &o = own[g.slot];
    double acc[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[c] = 0;
    Extremes x{__longlong_as_double(0x7ff0000000000000ll), 0.0, 0.0, 0.0};   // m_min = +inf
    #pragma unroll 1
    for (int j0 = 0; j0 < n; j0 += T) {
        const int cnt = min(T, n - j0);
        const int cnt_full = max(0, min(cnt, S.n_full - j0));
        // rows every body needs, then rows only full-class bodies need; with one tile the positions, GM
        // and sR2 are still in the tile from pass A of this stage (`reuse`)
        const bool reuse = n <= T;
        const double *src[TB_ROWS] = {
            reuse ? nullptr : pub + (PUB_R_HI + 0) * ld, reuse ? nullptr : pub + (PUB_R_HI + 1) * ld,
            reuse ? nullptr : pub + (PUB_R_HI + 2) * ld, reuse ? nullptr : pub + (PUB_R_LO + 0) * ld,
            reuse ? nullptr : pub + (PUB_R_LO + 1) * ld, reuse ? nullptr : pub + (PUB_R_LO + 2) * ld,
            aux + (AUX_NACC + 0) * ld, aux + (AUX_NACC + 1) * ld, aux + (AUX_NACC + 2) * ld,
            aux + (AUX_BETA + 0) * ld, aux + (AUX_BETA + 1) * ld, aux + (AUX_BETA + 2) * ld,
            reuse ? nullptr : pub + PUB_GM * ld, reuse ? nullptr : cst + CST_SR2 * ld,
            aux + AUX_PHI * ld, aux + AUX_BETA2 * ld,
            pub + (PUB_GL + 0) * ld, pub + (PUB_GL + 1) * ld, pub + (PUB_GL + 2) * ld,
            aux + (AUX_CPOT + 0) * ld, aux + (AUX_CPOT + 1) * ld, aux + (AUX_CPOT + 2) * ld,
            aux + (AUX_CPOT + 3) * ld, aux + (AUX_CPOT + 4) * ld, aux + (AUX_CPOT + 5) * ld,
            aux + (AUX_CPOT + 6) * ld, aux + (AUX_CPOT + 7) * ld, aux + (AUX_CPOT + 8) * ld,
            cst + CST_R2 * ld, cst + CST_LUM * ld};
        if (!load_tile(S, sc, ts, tile, kTileW, src, TB_ROWS, j0, cnt, cnt_full, kTileBFullRows)) return false;
        const int self = o.idx - j0;
        if (!sweeper) continue;
        if (o.full) {
            sweep_b_range<true, true>(o, tile, 0, cnt_full, self, g, acc, x);
            sweep_b_range<true, false>(o, tile, cnt_full, cnt, self, g, acc, x);
        } else {
            sweep_b_range<false, true>(o, tile, 0, cnt_full, self, g, acc, x);
            sweep_b_range<false, false>(o, tile, cnt_full, cnt, self, g, acc, x);
        }
    }
    __shared__ double red[kOwnMax][16];
    if (sweeper) {
        // exact extremes with the reference's expressions
        double red_in[11];
#pragma unroll
        for (int c = 0; c < 9; ++c) red_in[c] = acc[c];
        {
            const double rr2 = 1.0 / x.m_min;
            red_in[9] = sqrt(rr2);                                // +inf -> 0 when no pair was seen
            if (x.tq != x.tq) red_in[10] = x.tq;
            else if (x.tq > 0) {
                const double r2 = 1.0 / x.tq_m;
                red_in[10] = r2 * (sqrt(r2) * x.tq_gm);
            } else red_in[10] = 0.0;
        }
        group_reduce<11>(red_in, sc.split_b, nb, nwb, sc, red, 9);
        if (threadIdx.x < nb) {
            Own &ob = own[threadIdx.x];
            const double *rr = red[threadIdx.x];
            for (int c = 0; c < 3; ++c) { ob.gacc[c] = rr[c]; ob.dacc[c] = rr[3 + c]; ob.dtq[c] = rr[6 + c]; }
            checked_maximize(ob.mind, rr[9]);
            checked_maximize(ob.maxi, rr[10]);
        }
    } else {
        // the last warp: reactions of the owned extended bodies, the sum over all CTAs of their shares
        // written in pass A (lane-strided over the CTAs, then a butterfly over the warp)
        const int lane = threadIdx.x & 31;
        #pragma unroll 1
        for (int b = 0; b < nb; ++b) {
            const int e = own[b].ext_slot;
            if (e < 0) continue;
            double part[6] = {0, 0, 0, 0, 0, 0};
            const double *rc = S.react_cta + (size_t)e * ld * 6;   // [CTA][6]
            #pragma unroll 4
            for (int g = lane; g < (int)gridDim.x; g += 32)
                for (int c = 0; c < 6; ++c) part[c] += __ldcg(rc + (size_t)g * 6 + c);
            for (int c = 0; c < 6; ++c) {
                const double v = warp_sum(part[c]);
                if (lane == c) sc.react[b][c] = v;
            }
        }
    }
    __syncthreads();
    mark(S, sc, PH_B_SWEEP);
    // reactions of the owned extended bodies, when every warp swept: the sum over all CTAs of their shares
    // written in pass A
    #pragma unroll 1
    for (int b = 0; b < (nwb == kWarps ? nb : 0); ++b) {
        const int e = own[b].ext_slot;
        if (e < 0) continue;   // uniform over the CTA
        double part[6] = {0, 0, 0, 0, 0, 0};
        const double *rc = S.react_cta + (size_t)e * ld * 6;   // [CTA][6]
        #pragma unroll 1
        for (int g = threadIdx.x; g < (int)gridDim.x; g += blockDim.x)
            for (int c = 0; c < 6; ++c) part[c] += __ldcg(rc + (size_t)g * 6 + c);
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int c = 0; c < 6; ++c) {
            double v = warp_sum(part[c]);
            if (lane == 0) sc.part[w][c] = v;
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            double s = 0;
            for (int ww = 0; ww < kWarps; ++ww) s += sc.part[ww][threadIdx.x];
            sc.react[b][threadIdx.x] = s;
        }
        __syncthreads();
    }
    mark(S, sc, PH_B_FINAL);   // host reaction sums
    // finalisation (mass.cpp:389-396): FINALIZE_RELATIVITY and RING_CORRECTION
    const double c2 = kC * kC;
    const int n_ext = S.n_ext;
    // the extended bodies' fields on the owned bodies, added to the deformation sum in host order, one thread
    // per (body, component): the halves of each host's models (a missing half adds zero), from shared memory
    // or, when other CTAs evaluated this CTA's fields, from their slots in the global table
    if (n_ext > 0) {
        if (threadIdx.x < nb * 3) {
            const int b = threadIdx.x / 3, c = threadIdx.x - 3 * b;
            Own &ob = own[b];
            double da = ob.dacc[c];
            if (sc.fields_away) {
                const double *g = S.react + (size_t)ob.idx * 12 + c;
                #pragma unroll 4
                for (int e = 0; e < n_ext; ++e) {
                    const HostInfo h = sc.host[e];
                    const double a0 = __ldcg(g + (size_t)e * S.ld * 12), a1 = __ldcg(g + (size_t)e * S.ld * 12 + 6);
                    da += h.gp >= 0 ? a0 : 0.0;
                    da += h.ring >= 0 ? a1 : 0.0;
                }
            } else {
                #pragma unroll 4
                for (int e = 0; e < n_ext; ++e) {
                    const HostInfo h = sc.host[e];
                    const double a0 = sc.ext[b][e][c], a1 = sc.ext2[b][e][c];
                    da += h.gp >= 0 ? a0 : 0.0;
                    da += h.ring >= 0 ? a1 : 0.0;
                }
            }
            ob.dacc[c] = da;
        }
        __syncthreads();
    }
    #pragma unroll 1
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        Own &ob = own[b];
        v3 da = ldv(ob.dacc);
        v3 tq = ldv(ob.dtq);
        if (ob.ext_slot >= 0) {
            da += mk(sc.react[b][0], sc.react[b][1], sc.react[b][2]);
            tq += mk(sc.react[b][3], sc.react[b][4], sc.react[b][5]);
        }
        ob.phi *= c2;
        v3 na = c2 * ldv(ob.nacc);
        stv(ob.nacc, na);
        v3 ga = ldv(ob.gacc);
        if (ob.ring >= 0) {
            da = da - ob.ring_GM_ratio * ((ga + da) + na);
            v3 mGL = fast3(ob.GL);
            double rmGL = normalize(mGL);
            v3 ptorque = dot(tq, mGL) * mGL;
            v3 dtq = tq - ptorque;
            dtq = (rmGL / (rmGL + ob.ring_GL_R2 * ob.R2)) * dtq;
            tq = dtq + ptorque;
        }
        stv(ob.dacc, da);
        stv(ob.dtq, tq);
        stv(ob.fa, (ga + da) + na);
    }
    __syncthreads();
    mark(S, sc, PH_B_FINAL);
    return true;
}

// ------------------------------------------------------------------ RK12 stage combination and update
// Adds a_{k,s} f_s into the accumulators of stages k = k_lo..k_hi (RungeKutta.impl:148-162 in incremental
// form: every accumulator receives its terms in ascending s, the reference's summation order); 12
// components per stage, the velocity as double-double.
__device__ void combine_stage(Own *own, int nb, int s, int k_lo, int k_hi, const Scratch &sc) {
    const int nk = k_hi - k_lo + 1;
    if (nk <= 0) return;
    #pragma unroll 1
    for (int item = threadIdx.x; item < nb * nk * 12; item += blockDim.x) {
        const int b = item / (nk * 12);
        const int rem = item % (nk * 12);
        const int k = k_lo + rem / 12;
        const int c = rem % 12;
        Own &o = own[b];
        const int ci = k * (k - 1) / 2 + s;
        const dd a = dd{sc.rk_hi[ci], sc.rk_lo[ci]};
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
}

// Frame of stage k = s + 1 for body o on its warp (RungeKutta.impl:170-186): s = s0, then s += R % fast(s)
// for the passes R0 (w - dw), R1 (w + dw) and, at the last stage, R2 (Egrad), element (col, row) =
// sum_m R[m][row] * s[col][m]; the increment matrices depend only on w, dw and Egrad, so every lane builds
// the one of its pass (lanes 9p .. 9p+8 apply pass p) at the same time and the passes are applied in
// order. At the last stage mass::orthogonalize follows (mass.h:147-150).
__device__ void rotate_frame(Own &o, int lane, int s, double dt) {
    const int k = s + 1;
    const double dt_k = c_dtk[k];
    if (lane < 9) o.s[lane] = o.s0[lane];
    __syncwarp();
    const v3 wv = ldv(o.wnew), dwv = ldv(o.dw), eg = ldv(o.Egrad);
    // A body that does not rotate (w, its stage change and Egrad all exactly zero) has zero rotation
    // increments R (rotation_matrix of a zero vector), so its frame keeps s0 exactly: skip the passes.
    const bool still = wv.x == 0 && wv.y == 0 && wv.z == 0 && dwv.x == 0 && dwv.y == 0 && dwv.z == 0 &&
                       (k != kStages || (eg.x == 0 && eg.y == 0 && eg.z == 0));
    const int npass = still ? 0 : (k == kStages ? 3 : 2);
    if (npass) {
        const int my = min(lane / 9, 2);
        // one evaluation per lane on its pass's arguments (one copy of the code, no divergence)
        const v3 axis = my == 0 ? wv - dwv : my == 1 ? wv + dwv : eg;
        const m3 R = rotation_matrix(axis, my < 2 ? dt * dt_k / 2 : 1.0 / 72);
        const double *Rr = &R.x.x;   // R column m at Rr[3m]
        const int q = lane - 9 * my, col = q / 3, row = q % 3;
        #pragma unroll 1
        for (int pass = 0; pass < npass; ++pass) {
            const bool mine = my == pass && q < 9;
            double add = 0;
            if (mine) {
                const v3 sc = fast3(o.s + 3 * col);
                add = (Rr[0 + row] * sc.x + Rr[3 + row] * sc.y) + Rr[6 + row] * sc.z;
            }
            __syncwarp();
            if (mine) o.s[q] = dd_add(o.s[q], dd_make(add));
            __syncwarp();
        }
    }
    if (k == kStages) {
        // s += 0.5 fmis % (1 - fmis^T % fmis)
        double add = 0;
        if (lane < 9) {
            const int col = lane / 3, row = lane % 3;
            const m3 f = fast9(o.s);
            // column `col` of (1 - f^T f): entries m = (1 if m == col) - dot(f[m], f[col])
            const v3 fc = (col == 0) ? f.x : (col == 1) ? f.y : f.z;
            const double o0 = (col == 0 ? 1.0 : 0.0) - dot(f.x, fc);
            const double o1 = (col == 1 ? 1.0 : 0.0) - dot(f.y, fc);
            const double o2 = (col == 2 ? 1.0 : 0.0) - dot(f.z, fc);
            const double *fr = &f.x.x;
            add = (0.5 * fr[0 + row] * o0 + 0.5 * fr[3 + row] * o1) + 0.5 * fr[6 + row] * o2;
        }
        __syncwarp();
        if (lane < 9) o.s[lane] = dd_add(o.s[lane], dd_make(add));
        __syncwarp();
    }
}

// Called with f_s known for all owned bodies (s = 0..24). Adds a_{k,s} f_s into the accumulators of
// stages k = s+1..25, then forms the state of stage s+1 (RungeKutta.impl:164-186) and publishes it to
// buffer `buf_out`. The state update of body b runs on warp b: lanes 0..2 take the vector components,
// lanes 0..8 the 3x3 frame elements.
__device__ void rk_stage(const SysDev &S, Own *own, int nb, int s, long long i_step, const StepParams &P,
                         int buf_out, const Scratch &sc) {
    const double dt = P.dt;
    if (s == 0) {   // start of a step: x0 = x; Egrad = dtorque (RungeKutta.impl:113-116), 24 items per body
        #pragma unroll 1
        for (int item = threadIdx.x; item < nb * 24; item += blockDim.x) {
            Own &o = own[item / 24];
            const int f = item % 24;
            if (f < 3) o.r0[f] = o.r[f];
            else if (f < 6) o.v0[f - 3] = o.v[f - 3];
            else if (f < 9) o.GL0[f - 6] = o.GL[f - 6];
            else if (f < 18) o.s0[f - 9] = o.s[f - 9];
            else if (f < 21) o.w0[f - 18] = o.w[f - 18];
            else o.Egrad[f - 21] = o.dtq[f - 21];
        }
    }
    if (threadIdx.x < nb) {
        Own &o = own[threadIdx.x];
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
    combine_stage(own, nb, s, s + 1, kStages, sc);
    __syncthreads();
    // state of stage k = s+1, warp b for body b
    const int k = s + 1;
    const double dt_k = c_dtk[k];
    const double t = P.t_eph + dt * (dt_k + (double)i_step);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < nb) {
        Own &o = own[w];
        if (lane < 3) {
            const int c = lane;
            const dd ddt = dd_make(dt);
            o.r[c] = dd_add(o.r0[c], dd_mul(ddt, o.accv[k - 1][c]));
            o.v[c] = dd_add(o.v0[c], dd_make(dt * o.acca[k - 1][c]));
            o.GL[c] = dd_add(o.GL0[c], dd_make(dt * o.acct[k - 1][c]));
            const double wc = o.accw[k - 1][c] * (1.0 / dt_k);   // xi.w /= dt_k (vec_t.h:197-203)
            o.wnew[c] = wc;
            o.dw[c] = (2.0 / 3) * (wc - o.w0[c]);
        }
        __syncwarp();
        rotate_frame(o, lane, s, dt);
        if (lane == 0) {
            stv(o.w, ldv(o.wnew));
            o.GM = o.GM0 + o.dGM * t;
            o.exJ2 = o.dJ2 * t;
        }
        __syncwarp();
        publish_body_warp(S, o, buf_out, lane);
    }
    __syncthreads();
}

// Field hand-off, decided once per launch by every CTA alike: a CTA that owns a delayed tide iterates
// pass A up to four times, and every warp it can give the sweeps shortens each iteration (one pair per
// thread for a whole system of up to 512 bodies instead of two), so the field items of its bodies are
// evaluated by the CTAs that own no delayed tide, each taking at most kForeignMax of them, dealt in CTA
// order round-robin. The forces on the handed-over bodies travel through the global table S.react (its
// reaction-staging slots, free when every CTA stages its reactions in shared memory, which the hand-off
// requires) and the CTAs that handed over their fields report zero reactions. Uses the staging tile, not
// yet filled, as scratch; ends with a CTA barrier.
constexpr int kPlanCtas = 1024;   // CTAs the hand-off plan handles (grids are at most the SM count)
__device__ void field_handoff(const SysDev &S, const StepParams &P, const Own *own, int nb, Scratch &sc, double *tile) {
    int *cta_del = reinterpret_cast<int *>(tile);   // [grid]: the CTA owns a delayed tide
    int *cta_nb = cta_del + kPlanCtas;              // [grid]: bodies of the CTA
    const bool possible = P.mode != MODE_DEFORM && S.n_ext > 0 && S.n <= S.tile && gridDim.x <= kPlanCtas &&
                          kRingTerms + kFieldMax * S.n_ext * 12 <= (kTileRows - TA_ROWS) * kTileW;
    const int n = S.n;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += blockDim.x) {
        int d = 0, k = 0;
        for (int b = 0; b < kOwnMax; ++b) {
            const int id = S.own_list[c * kOwnMax + b];
            if (id < 0) break;
            ++k;
            const int o = S.orig[id];   // kind 2 of load_own: k2 != 0 and a tide delay
            d |= S.planes[(size_t)EPH_P_K2 * n + o] != 0 && S.planes[(size_t)EPH_P_TIDE_DELAY * n + o] != 0;
        }
        cta_del[c] = d;
        cta_nb[c] = k;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int n_recv = 0, n_give = 0, my_rank = -1;
        for (int c = 0; c < (int)gridDim.x; ++c) {
            if (cta_del[c]) n_give += cta_nb[c];
            else {
                if (c == (int)blockIdx.x) my_rank = n_recv;
                ++n_recv;
            }
        }
        const bool on = possible && n_recv > 0 && n_give > 0 && (n_give + n_recv - 1) / n_recv <= kForeignMax;
        sc.fields_away = on && cta_del[blockIdx.x];
        sc.n_foreign = 0;
        if (on && my_rank >= 0) {   // handed-over body k (CTA order) goes to receiver k % n_recv
            int k = 0;
            for (int c = 0; c < (int)gridDim.x; ++c) {
                if (!cta_del[c]) continue;
                for (int b = 0; b < cta_nb[c]; ++b, ++k)
                    if (k % n_recv == my_rank) sc.foreign[sc.n_foreign++] = S.own_list[c * kOwnMax + b];
            }
        }
        sc.nfb = sc.fields_away ? 0 : nb + sc.n_foreign;
    }
    __syncthreads();
    if (sc.fields_away)   // this CTA's share of every host's reaction is evaluated elsewhere
        for (int q = threadIdx.x; q < S.n_ext * 6; q += blockDim.x)
            S.react_cta[((size_t)(q / 6) * S.ld + blockIdx.x) * 6 + q % 6] = 0.0;
}

// ------------------------------------------------------------------ the kernel
__global__ void __launch_bounds__(kThreads, 1) step_kernel(SysDev S, StepParams P) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Own *own = reinterpret_cast<Own *>(smem_raw);
    Scratch &sc = *reinterpret_cast<Scratch *>(smem_raw + sizeof(Own) * kOwnMax);
    double *tile = reinterpret_cast<double *>(smem_raw + ((sizeof(Own) * kOwnMax + sizeof(Scratch) + 127) / 128) * 128);
    TileState ts{0u};

    if (threadIdx.x == 0) {
        sc.t_last = global_ns();
        for (int p = 0; p < kPhases; ++p) sc.t_phase[p] = 0;
        sc.bar_target = 0;
    }
    for (int q = threadIdx.x; q < EPH_RK12_NCOEF; q += blockDim.x) {
        sc.rk_hi[q] = c_rk_hi[q];
        sc.rk_lo[q] = c_rk_lo[q];
    }
    for (int k = 0; k < min(S.n_gp, kGpSmem); ++k)
        gp_expand(S.gp_coef + (size_t)k * EPH_GP_TABLE_SIZE, S.gp_nz[k], S.gp_nt[k], sc.gp_x[k], threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < EPH_GP_MAX_DEGREE + 2; q += blockDim.x) sc.gp_rcp[q] = GP_RCP[q];
    for (int e = threadIdx.x; e < S.n_ext; e += blockDim.x) {   // the extended bodies and their models
        HostInfo h;
        h.E = S.ext_body[e];
        const int gp = (int)S.cst[CST_GP * S.ld + h.E], rg = (int)S.cst[CST_RING * S.ld + h.E];
        h.gp = (short)gp;
        h.ring = (short)rg;
        h.nz = gp >= 0 ? (unsigned char)S.gp_nz[gp] : 0;
        h.nt = gp >= 0 ? (unsigned char)S.gp_nt[gp] : 0;
        h.nd = rg >= 0 ? (unsigned char)S.ring_nd[rg] : 0;
        h.pad = 0;
        sc.host[e] = h;
    }
    mbar_init(sc);
    if (threadIdx.x == 0) {
        int ng = 0, nr = 0, dmax = 0;
        for (int e = 0; e < S.n_ext; ++e) {
            if (sc.host[e].gp >= 0) sc.gp_list[ng++] = (unsigned char)e;
            if (sc.host[e].ring >= 0) {
                sc.ring_list[nr++] = (unsigned char)e;
                dmax = max(dmax, (int)sc.host[e].nd);
            }
        }
        sc.n_gp_e = ng;
        sc.n_ring_e = nr;
        sc.ring_dmax = dmax;
    }
    int nb = 0;
    for (int b = 0; b < kOwnMax; ++b) {
        int id = S.own_list[blockIdx.x * kOwnMax + b];
        if (id < 0) break;
        if (threadIdx.x == 0) {
            own[b].idx = id;
            own[b].orig = S.orig[id];
            own[b].full = id < S.n_full;
        }
        ++nb;
    }
    __syncthreads();
    load_own(S, own, nb, P);
    field_handoff(S, P, own, nb, sc, tile);
    __syncthreads();
    if (threadIdx.x < nb) publish_body(S, own[threadIdx.x], 0);
    if (threadIdx.x == 32) {
        // warp groups of the sweeps over all owned bodies: delayed-tide pass-A pairs cost ~8x a point pair,
        // full-class pass-B pairs ~2x. During the pass-A sweeps the last warp evaluates the ring items and
        // the kExtWarps - 1 warps before it the geopotential items.
        int wt[kOwnMax];
        bool delayed = false;
        for (int b = 0; b < nb; ++b) delayed |= own[b].kind == 2;
        sc.has_delayed = delayed;
        const bool side = P.mode != MODE_DEFORM && S.n_ext > 0 && S.n <= S.tile && !sc.fields_away;
        sc.ext_overlap = side;
        sc.ring_side = side && sc.n_ring_e > 0;
        sc.nw_a = sc.ext_overlap ? kWarps - kExtWarps : sc.ring_side ? kWarps - 1 : kWarps;
        for (int b = 0; b < nb; ++b) wt[b] = own[b].kind == 2 ? 8 : 1;
        split_warps(wt, nb, P.mode == MODE_DEFORM ? kWarps : sc.nw_a, sc.split_a0);
        for (int b = 0; b < nb; ++b) wt[b] = own[b].full ? 2 : 1;
        // a CTA that owns geopotential / ring hosts sums their reactions on its last warp during the
        // pass-B sweep (one tile only: streaming tiles needs every warp for the copies)
        bool host = false;
        for (int b = 0; b < nb; ++b) host |= own[b].ext_slot >= 0;
        sc.nw_b = (host && S.n <= S.tile && nb < kWarps) ? kWarps - 1 : kWarps;
        split_warps(wt, nb, sc.nw_b, sc.split_b);
    }
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
        if (threadIdx.x == 0) sc.traj_slot = S.traj_base;
        if (!pass_a(S, own, nb, 0, P.mode == MODE_DEFORM, sc, ts, tile)) return;
        if (P.mode == MODE_ACCEL) {
            if (!sync()) return;
            if (!pass_b(S, own, nb, 0, sc, ts, tile)) return;
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
    #pragma unroll 1
    for (long long step = 0; step < P.n_step; ++step) {
        #pragma unroll 1
        for (int s = 0; s < kStages; ++s) {
            rk_stage(S, own, nb, s, step, P, buf ^ 1, sc);
            mark(S, sc, PH_RK);
            buf ^= 1;
            if (!sync()) return;
            if (threadIdx.x == 0) sc.traj_slot = S.traj_base + step * kStages + s;
            if (!pass_a(S, own, nb, buf, false, sc, ts, tile)) return;
            if (!sync()) return;
            if (!pass_b(S, own, nb, buf, sc, ts, tile)) return;
        }
    }
    if (P.invert_min && threadIdx.x < nb) own[threadIdx.x].mind = 1 / own[threadIdx.x].mind;
    __syncthreads();
    finish(false);
}

}  // namespace eph

// ------------------------------------------------------------------ host launcher
namespace eph {

size_t step_fixed_smem_bytes() { return kFixedSmem; }
// the tile is always allocated at its full stride; `tile` (bodies staged per chunk) does not change the size
size_t step_smem_bytes(int tile) { (void)tile; return kFixedSmem + (size_t)kTileRows * kTileW * sizeof(double); }

// Largest tile (bodies, multiple of kPad): the tile's stride.
int max_tile() { return kTileW; }

// Per-device "constants uploaded" flags. Contexts (each under its own lock) and the fixed-scratch entry
// point (under its own) may set a device up at the same time: one mutex of its own orders the uploads.
static std::atomic<bool> g_consts_ready[64];
static std::mutex g_consts_mu;

cudaError_t upload_constants(int device) {
    if (device >= 0 && device < 64 && g_consts_ready[device].load(std::memory_order_acquire)) return cudaSuccess;
    std::lock_guard<std::mutex> lock(g_consts_mu);
    if (device >= 0 && device < 64 && g_consts_ready[device].load(std::memory_order_relaxed)) return cudaSuccess;
    double hi[EPH_RK12_NCOEF], lo[EPH_RK12_NCOEF], dtk[kStages + 1];
    rk12_expand(hi, lo, dtk);
    cudaError_t e = cudaMemcpyToSymbol(c_rk_hi, hi, sizeof(hi));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rk_lo, lo, sizeof(lo));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_dtk, dtk, sizeof(dtk));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
    if (e == cudaSuccess && device >= 0 && device < 64) g_consts_ready[device].store(true, std::memory_order_release);
    return e;
}

cudaError_t launch_step(const SysDev &S, const StepParams &P, int grid, cudaStream_t stream) {
    void *args[] = {(void *)&S, (void *)&P};
    return cudaLaunchCooperativeKernel((void *)step_kernel, dim3(grid), dim3(kThreads), args, step_smem_bytes(S.tile),
                                       stream);
}

int max_coresident_ctas(int device, int tile, int *out) {
    int per_sm = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel, kThreads, step_smem_bytes(tile));
    if (e != cudaSuccess) return (int)e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return (int)e;
    *out = per_sm * sms;
    return 0;
}

}  // namespace eph
