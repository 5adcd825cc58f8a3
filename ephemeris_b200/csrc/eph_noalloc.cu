// eph_noalloc.cu - eph_integrate_noalloc: the RK12 integration of eph_integrate for callers that cannot
// allocate device memory.
//
// Who needs it: a host program whose device memory is owned by someone else - an application that hands
// this library a slice of its own pool and forbids further cudaMalloc (allocation would fragment or
// overrun that pool), a plug-in that runs inside a process with a fixed memory budget per device, or code
// that must not trigger an allocation (and the implicit synchronisation cudaMalloc / cudaFree bring) in
// the middle of its own stream work. Such a caller brings the system's planes in device memory it already
// has and calls one function; the library allocates nothing, on the device or through any library.
//
// The step kernel's working memory (public stage state, pass-A outputs, constants, extended-body
// reactions, ownership lists, model tables, barrier and status words) lives in one file-scope
// __device__ array, g_noalloc_scratch, sized for at most EPH_NOALLOC_MAX_BODIES bodies,
// EPH_NOALLOC_MAX_EXT extended bodies, EPH_NOALLOC_MAX_GP geopotential and EPH_NOALLOC_MAX_RING ring
// models (about 3.2 MB). The array is part of the library's device image: every GPU on which the library
// is loaded holds it from module load until the process exits. In host code `g_noalloc_scratch` names a
// host-side stand-in for the symbol, not a device address; the device address comes from
// cudaGetSymbolAddress, once per device, in noalloc_setup().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "eph_plan.h"
#include "eph_system.cuh"
#include "../../include/eph_b200.h"

namespace eph {
int max_tile();
cudaError_t upload_constants(int device);
cudaError_t launch_step(const SysDev &S, const StepParams &P, int grid, cudaStream_t stream);
int max_coresident_ctas(int device, int tile, int *out);
}  // namespace eph

using namespace eph;

namespace {

constexpr int kNB = EPH_NOALLOC_MAX_BODIES;   // plane stride of the scratch regions (a multiple of kPad)
constexpr int kNE = EPH_NOALLOC_MAX_EXT;
constexpr int kNGP = EPH_NOALLOC_MAX_GP;
constexpr int kNRing = EPH_NOALLOC_MAX_RING;
static_assert(kNB % kPad == 0, "scratch plane stride must be a multiple of the plane padding");
static_assert(kNE <= kMaxExt, "extended-body limit above the kernel's own");

// Scratch regions, in doubles, each rounded up to 256 bytes (32 doubles). The integer regions are counted
// in doubles too (two ints per double).
constexpr size_t r32(size_t d) { return (d + 31) / 32 * 32; }
constexpr size_t kOffPub = 0;
constexpr size_t kOffAux = kOffPub + r32((size_t)2 * PUB_NPLANES * kNB);
constexpr size_t kOffCst = kOffAux + r32((size_t)AUX_NPLANES * kNB);
constexpr size_t kOffReact = kOffCst + r32((size_t)CST_NPLANES * kNB);
constexpr size_t kOffReactCta = kOffReact + r32((size_t)kNE * kNB * 12);
constexpr size_t kOffGpCoef = kOffReactCta + r32((size_t)kNE * kNB * 6);
constexpr size_t kOffRingParam = kOffGpCoef + r32((size_t)kNGP * EPH_GP_TABLE_SIZE);
constexpr size_t kOffRingDisk = kOffRingParam + r32((size_t)kNRing * EPH_RING_PARAMS);
constexpr size_t kOffOrig = kOffRingDisk + r32((size_t)kNRing * EPH_RING_MAX_DISKS * 3);
constexpr size_t kOffOwn = kOffOrig + r32(kNB / 2);
constexpr size_t kOffExt = kOffOwn + r32((size_t)kNB * kOwnMax / 2);
constexpr size_t kOffGpNz = kOffExt + r32(kNE / 2 + 1);
constexpr size_t kOffGpNt = kOffGpNz + r32(kNGP / 2 + 1);
constexpr size_t kOffRingNd = kOffGpNt + r32(kNGP / 2 + 1);
constexpr size_t kOffWords = kOffRingNd + r32(kNRing / 2 + 1);   // 64-bit barrier arrival counter, status
constexpr size_t kScratchDoubles = kOffWords + 32;

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Per-device set-up state and the host staging buffers of one call. One lock serialises every call in
// the process, so the host buffers are never shared by two calls and the device scratch is never used by
// two calls at once.
std::mutex g_mu;
double *g_dev_scratch[64];   // device address of g_noalloc_scratch per device (null until set up)
double g_h_planes[(size_t)EPH_NPLANES * kNB];
double g_h_cst[(size_t)CST_NPLANES * kNB];
int g_h_orig[kNB], g_h_ext[kNE], g_h_own[(size_t)kNB * kOwnMax], g_h_order[kNB], g_h_cnt[kNB];
double g_h_cost[kNB], g_h_load[kNB];

// Once per device, with that device current: the scratch array's device address and the RK12 tables.
cudaError_t noalloc_setup(int device, double **out) {
    if (g_dev_scratch[device]) {
        *out = g_dev_scratch[device];
        return cudaSuccess;
    }
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = upload_constants(device);
    if (e != cudaSuccess) return e;
    g_dev_scratch[device] = (double *)p;
    *out = (double *)p;
    return cudaSuccess;
}

struct DeviceGuard {   // restores the caller's current device
    int prev = -1;
    DeviceGuard() { cudaGetDevice(&prev); }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

int body(int device, cudaStream_t stream, int n, double *d_planes, const eph_models *models, double dt,
         int64_t n_step, double *t_eph_hi, double *t_eph_lo) {
#define NA_CK(call)                                      \
    do {                                                 \
        if ((call) != cudaSuccess) return EPH_ERR_CUDA;  \
    } while (0)
    NA_CK(cudaSetDevice(device));
    double *scr = nullptr;
    NA_CK(noalloc_setup(device, &scr));
    const int n_gp = models ? models->n_gp : 0, n_ring = models ? models->n_ring : 0;
    const int ld = (n + kPad - 1) / kPad * kPad;

    // the caller's planes, for the body classes, constants and the model-index checks
    NA_CK(cudaMemcpyAsync(g_h_planes, d_planes, (size_t)EPH_NPLANES * n * sizeof(double), cudaMemcpyDeviceToHost,
                          stream));
    NA_CK(cudaStreamSynchronize(stream));
    const double *pl = g_h_planes;
    for (int i = 0; i < n; ++i) {
        const double g = pl[(size_t)EPH_P_GP_INDEX * n + i], r = pl[(size_t)EPH_P_RING_INDEX * n + i];
        if (!(g >= -1 && g < n_gp) || !(r >= -1 && r < n_ring)) return EPH_ERR_ARG;
    }
    // device order (full class first), constant planes, extended bodies, work estimates: the same rules as
    // eph_upload_system
    int n_full = 0, k = 0;
    for (int i = 0; i < n; ++i)
        if (plan_full_class(pl, n, i)) g_h_orig[k++] = i;
    n_full = k;
    for (int i = 0; i < n; ++i)
        if (!plan_full_class(pl, n, i)) g_h_orig[k++] = i;
    std::fill(g_h_cst, g_h_cst + (size_t)CST_NPLANES * ld, 0.0);
    int n_ext = 0;
    for (k = 0; k < n; ++k) {
        const int i = g_h_orig[k];
        auto P = [&](int p) { return pl[(size_t)p * n + i]; };
        g_h_cst[CST_SR2 * ld + k] = P(EPH_P_SR2);
        g_h_cst[CST_TDF * ld + k] = P(EPH_P_TIDE_DELAY_FACTOR);
        g_h_cst[CST_R2 * ld + k] = P(EPH_P_R2);
        g_h_cst[CST_LUM * ld + k] = P(EPH_P_LUM);
        g_h_cst[CST_R * ld + k] = P(EPH_P_RADIUS);
        g_h_cst[CST_GP * ld + k] = P(EPH_P_GP_INDEX);
        g_h_cst[CST_RING * ld + k] = P(EPH_P_RING_INDEX);
        if (P(EPH_P_GP_INDEX) >= 0 || P(EPH_P_RING_INDEX) >= 0) {
            if (n_ext == kNE) return EPH_ERR_LIMIT;
            g_h_ext[n_ext++] = k;
        }
        g_h_cost[k] = plan_cost(pl, n, i, k < n_full);
    }

    // launch shape and ownership split: the automatic choice of eph_upload_system
    const int tile = std::min(max_tile(), ld);
    int maxc = 0, grid = 0, per = 0;
    if (max_coresident_ctas(device, tile, &maxc) != 0 || maxc <= 0) return EPH_ERR_CUDA;
    if (!plan_shape(n, maxc, 0, 0, &grid, &per)) return EPH_ERR_LIMIT;
    plan_ownership(g_h_cost, n, grid, per, g_h_order, g_h_load, g_h_cnt, g_h_own);

    // scratch contents: the previous call's are stale, so everything the kernel reads before writing is
    // either uploaded here or cleared to zero
    auto I = [&](size_t off) { return (int *)(scr + off); };
    NA_CK(cudaMemsetAsync(scr + kOffPub, 0, (size_t)2 * PUB_NPLANES * ld * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(scr + kOffAux, 0, (size_t)AUX_NPLANES * ld * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(scr + kOffReact, 0, (size_t)std::max(n_ext, 1) * ld * 12 * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(scr + kOffWords, 0, 32 * sizeof(double), stream));
    NA_CK(cudaMemcpyAsync(scr + kOffCst, g_h_cst, (size_t)CST_NPLANES * ld * sizeof(double), cudaMemcpyHostToDevice,
                          stream));
    NA_CK(cudaMemcpyAsync(I(kOffOrig), g_h_orig, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, stream));
    NA_CK(cudaMemcpyAsync(I(kOffOwn), g_h_own, (size_t)grid * kOwnMax * sizeof(int), cudaMemcpyHostToDevice, stream));
    if (n_ext)
        NA_CK(cudaMemcpyAsync(I(kOffExt), g_h_ext, (size_t)n_ext * sizeof(int), cudaMemcpyHostToDevice, stream));
    if (n_gp) {
        NA_CK(cudaMemcpyAsync(I(kOffGpNz), models->gp_nz, n_gp * sizeof(int), cudaMemcpyHostToDevice, stream));
        NA_CK(cudaMemcpyAsync(I(kOffGpNt), models->gp_nt, n_gp * sizeof(int), cudaMemcpyHostToDevice, stream));
        NA_CK(cudaMemcpyAsync(scr + kOffGpCoef, models->gp_coef, (size_t)n_gp * EPH_GP_TABLE_SIZE * sizeof(double),
                              cudaMemcpyHostToDevice, stream));
    }
    if (n_ring) {
        NA_CK(cudaMemcpyAsync(I(kOffRingNd), models->ring_ndisk, n_ring * sizeof(int), cudaMemcpyHostToDevice, stream));
        NA_CK(cudaMemcpyAsync(scr + kOffRingParam, models->ring_param, (size_t)n_ring * EPH_RING_PARAMS * sizeof(double),
                              cudaMemcpyHostToDevice, stream));
        NA_CK(cudaMemcpyAsync(scr + kOffRingDisk, models->ring_disk,
                              (size_t)n_ring * EPH_RING_MAX_DISKS * 3 * sizeof(double), cudaMemcpyHostToDevice, stream));
    }

    SysDev S;
    S.n = n;
    S.n_full = n_full;
    S.ld = ld;
    S.n_ext = n_ext;
    S.tile = tile;
    S.orig = I(kOffOrig);
    S.pub = scr + kOffPub;
    S.aux = scr + kOffAux;
    S.cst = scr + kOffCst;
    S.react = scr + kOffReact;
    S.react_cta = scr + kOffReactCta;
    S.planes = d_planes;
    S.ext_body = I(kOffExt);
    S.n_gp = n_gp;
    S.gp_nz = I(kOffGpNz);
    S.gp_nt = I(kOffGpNt);
    S.gp_coef = scr + kOffGpCoef;
    S.ring_nd = I(kOffRingNd);
    S.ring_param = scr + kOffRingParam;
    S.ring_disk = scr + kOffRingDisk;
    S.own_list = I(kOffOwn);
    S.bar = (unsigned *)(scr + kOffWords);
    S.status = I(kOffWords) + 2;
    S.timers = nullptr;
    S.traj = nullptr;
    S.traj_base = 0;
    S.wait_ns = kWaitDefaultNs;
    S.stall_barrier = 0;
    if (n_step < 0) {   // mass.cpp:401-404
        n_step = -n_step;
        dt = -dt;
    }
    StepParams P{MODE_INTEGRATE, 1, 1, (long long)n_step, dt, *t_eph_hi + *t_eph_lo};
    NA_CK(launch_step(S, P, grid, stream));
    int status = 0;
    NA_CK(cudaMemcpyAsync(&status, S.status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    // a bounded grid-barrier or tile-copy wait gave up (as the context path maps it); anything else is a fault
    if (status == ST_BARRIER_TIMEOUT || status == ST_COPY_TIMEOUT) return EPH_ERR_TIMEOUT;
    if (status != ST_OK) return EPH_ERR_CUDA;
    // t_eph += dt*n_step in double-double (mass.cpp:441)
    double a = *t_eph_hi, b = dt * (double)n_step;
    double s = a + b, t = s - a;
    double e = (a - (s - t)) + (b - t);
    e = e + (*t_eph_lo + 0.0);
    const double hi = s + e;
    *t_eph_lo = e - (hi - s);
    *t_eph_hi = hi;
    return EPH_OK;
#undef NA_CK
}

}  // namespace

extern "C" int eph_integrate_noalloc(int device, void *stream, int64_t n, double *d_planes, const eph_models *models,
                                     double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo) {
    if (!d_planes || !t_eph_hi || !t_eph_lo || n <= 0 || device < 0 || device >= 64) return EPH_ERR_ARG;
    const int n_gp = models ? models->n_gp : 0, n_ring = models ? models->n_ring : 0;
    if (n_gp < 0 || n_ring < 0 || (n_gp && (!models->gp_nz || !models->gp_nt || !models->gp_coef)) ||
        (n_ring && (!models->ring_ndisk || !models->ring_param || !models->ring_disk)))
        return EPH_ERR_ARG;
    if (n > kNB || n_gp > kNGP || n_ring > kNRing) return EPH_ERR_LIMIT;
    for (int k = 0; k < n_ring; ++k)
        if (models->ring_ndisk[k] < 0 || models->ring_ndisk[k] > EPH_RING_MAX_DISKS) return EPH_ERR_ARG;
    for (int k = 0; k < n_gp; ++k)
        if (models->gp_nz[k] < 0 || models->gp_nz[k] > EPH_GP_MAX_DEGREE || models->gp_nt[k] > models->gp_nz[k])
            return EPH_ERR_ARG;
    if (n_step == 0) return EPH_OK;   // mass.cpp:400
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceGuard guard;
    return body(device, (cudaStream_t)stream, (int)n, d_planes, models, dt, n_step, t_eph_hi, t_eph_lo);
}
