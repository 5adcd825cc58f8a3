// eph_capi.cu - context management and the extern "C" entry points of include/eph_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <numeric>
#include <vector>

#include "eph_plan.h"
#include "eph_system.cuh"
#include "../../include/eph_b200.h"

namespace eph {
size_t step_smem_bytes(int tile);
int max_tile();
cudaError_t upload_constants(int device);
cudaError_t launch_step(const SysDev &S, const StepParams &P, int grid, cudaStream_t stream);
int max_coresident_ctas(int device, int tile, int *out);
}  // namespace eph

using namespace eph;
static_assert(kOwnMax == EPH_MAX_BODIES_PER_CTA, "the C ABI states the per-CTA body limit");

struct eph_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;       // work stream (own_stream unless eph_set_stream chose another)
    cudaStream_t own_stream = nullptr;
    std::mutex mu;
    char err[512] = {0};
    // system
    int n = 0, n_gp = 0, n_ring = 0, n_ext = 0;
    size_t cap_n = 0;
    int cap_gp = 0, cap_ring = 0;
    double *d_planes = nullptr, *d_pub = nullptr, *d_aux = nullptr, *d_cst = nullptr, *d_react = nullptr;
    int ld = 0, tile = 0;                // plane stride (n rounded up to kPad), bodies per smem tile
    int n_full = 0;                      // full-class bodies (device order)
    int *d_orig = nullptr;               // [n] device order -> caller order
    int *d_ext = nullptr, *d_own = nullptr, *d_status = nullptr;
    unsigned *d_bar = nullptr;
    int *d_gp_nz = nullptr, *d_gp_nt = nullptr, *d_ring_nd = nullptr;
    double *d_gp_coef = nullptr, *d_ring_param = nullptr, *d_ring_disk = nullptr;
    std::vector<double> h_cost;          // per-body work estimate for the ownership split (device order)
    std::vector<double> cost_override;   // caller-order work estimates from eph_set_body_costs (empty: built-in)
    std::vector<int> h_orig;             // device order -> caller order
    std::vector<int> h_own;              // current ownership [grid][kOwnMax] (device order, -1 padded)
    int grid = 0, per_cta = 0;           // current launch shape
    int req_grid = 0, req_per_cta = 0;   // requested by eph_set_launch (0 = automatic)
    int64_t launches = 0;
    unsigned long long *d_timers = nullptr;   // phase timers of the last launch, when profiling
    int timers_grid = 0;
    double *d_traj = nullptr;            // stage records for massless particles (caller-owned), or null
    long long traj_base = 0;
    long long wait_ns = kWaitDefaultNs;  // limit of the kernel's bounded waits
    int stall_barrier = 0;               // set only for the duration of eph_selftest_wait_timeout
};

namespace eph {
// Stage records of the following launches go to d_buf, starting at slot `base` (null: off).
void ctx_record_stages(eph_ctx *ctx, double *d_buf, long long base) {
    ctx->d_traj = d_buf;
    ctx->traj_base = base;
}
long long ctx_size(const eph_ctx *ctx) { return ctx ? (long long)ctx->n : 0; }
}  // namespace eph

static int fail(eph_ctx *c, int code, const char *what, cudaError_t e = cudaSuccess) {
    if (c) {
        if (e != cudaSuccess)
            snprintf(c->err, sizeof(c->err), "%s: %s", what, cudaGetErrorString(e));
        else
            snprintf(c->err, sizeof(c->err), "%s", what);
    }
    return code;
}
#define CK(call, what)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA, what, e_); \
    } while (0)

static void free_system(eph_ctx *ctx) {
    void *ptrs[] = {ctx->d_planes, ctx->d_pub, ctx->d_aux, ctx->d_cst, ctx->d_react, ctx->d_ext, ctx->d_own, ctx->d_orig,
                    ctx->d_gp_nz, ctx->d_gp_nt, ctx->d_ring_nd, ctx->d_gp_coef, ctx->d_ring_param,
                    ctx->d_ring_disk};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    ctx->d_planes = ctx->d_pub = ctx->d_aux = ctx->d_cst = ctx->d_react = nullptr;
    ctx->d_ext = ctx->d_own = ctx->d_orig = nullptr;
    ctx->d_gp_nz = ctx->d_gp_nt = ctx->d_ring_nd = nullptr;
    ctx->d_gp_coef = ctx->d_ring_param = ctx->d_ring_disk = nullptr;
    ctx->cap_n = 0;
    ctx->cap_gp = ctx->cap_ring = 0;
    ctx->n = 0;
    ctx->grid = 0;
}

extern "C" {

int eph_ctx_create(int device, eph_ctx **out) {
    if (!out) return EPH_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return EPH_ERR_ARG;
    eph_ctx *ctx = new eph_ctx();
    ctx->device = device;
    CK(cudaSetDevice(device), "cudaSetDevice");
    CK(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx->stream = ctx->own_stream;
    CK(cudaMalloc(&ctx->d_bar, 2 * sizeof(unsigned)), "cudaMalloc(barrier)");
    CK(cudaMalloc(&ctx->d_status, sizeof(int)), "cudaMalloc(status)");
    CK(upload_constants(device), "upload RK12 constants");
    *out = ctx;
    return EPH_OK;
}

int eph_ctx_destroy(eph_ctx *ctx) {
    if (!ctx) return EPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    free_system(ctx);
    if (ctx->d_timers) cudaFree(ctx->d_timers);
    if (ctx->d_bar) cudaFree(ctx->d_bar);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return EPH_OK;
}

const char *eph_last_error(const eph_ctx *ctx) { return ctx ? ctx->err : "null context"; }

}  // extern "C"

static int choose_shape(eph_ctx *ctx) {
    int maxc = 0;
    ctx->tile = std::min(max_tile(), ctx->ld);
    if (max_coresident_ctas(ctx->device, ctx->tile, &maxc) != 0 || maxc <= 0) return fail(ctx, EPH_ERR_CUDA, "occupancy query failed");
    const int n = ctx->n;
    int grid = 0, per = 0;
    if (!plan_shape(n, maxc, ctx->req_grid, ctx->req_per_cta, &grid, &per))
        return fail(ctx, EPH_ERR_ARG, "launch shape exceeds co-resident CTAs (bodies_per_cta too small)");
    std::vector<int> own((size_t)grid * kOwnMax), order(n), cnt(grid);
    std::vector<double> load(grid);
    plan_ownership(ctx->h_cost.data(), n, grid, per, order.data(), load.data(), cnt.data(), own.data());
    cudaError_t e = cudaMemcpy(ctx->d_own, own.data(), own.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(ctx, EPH_ERR_CUDA, "upload ownership", e);
    ctx->h_own = own;
    ctx->grid = grid;
    ctx->per_cta = per;
    return EPH_OK;
}

static int prepare_constants(eph_ctx *ctx, const double *h_planes) {
    const int n = ctx->n;
    const int ld = ctx->ld;
    // device order: full-class bodies first, each class in the caller's order
    std::vector<int> orig;
    orig.reserve(n);
    for (int i = 0; i < n; ++i)
        if (plan_full_class(h_planes, n, i)) orig.push_back(i);
    ctx->n_full = (int)orig.size();
    for (int i = 0; i < n; ++i)
        if (!plan_full_class(h_planes, n, i)) orig.push_back(i);
    std::vector<double> cst((size_t)CST_NPLANES * ld, 0.0);
    std::vector<int> ext;
    ctx->h_cost.assign(n, 0.0);
    for (int k = 0; k < n; ++k) {
        const int i = orig[k];
        auto P = [&](int p) { return h_planes[(size_t)p * n + i]; };
        cst[CST_SR2 * ld + k] = P(EPH_P_SR2);
        cst[CST_TDF * ld + k] = P(EPH_P_TIDE_DELAY_FACTOR);
        cst[CST_R2 * ld + k] = P(EPH_P_R2);
        cst[CST_LUM * ld + k] = P(EPH_P_LUM);
        cst[CST_R * ld + k] = P(EPH_P_RADIUS);
        cst[CST_GP * ld + k] = P(EPH_P_GP_INDEX);
        cst[CST_RING * ld + k] = P(EPH_P_RING_INDEX);
        const bool gp = P(EPH_P_GP_INDEX) >= 0, ring = P(EPH_P_RING_INDEX) >= 0;
        if (gp || ring) ext.push_back(k);
        ctx->h_cost[k] = (int)ctx->cost_override.size() == n ? ctx->cost_override[i]
                                                              : plan_cost(h_planes, n, i, k < ctx->n_full);
    }
    ctx->h_orig = orig;
    if ((int)ext.size() > kMaxExt) return fail(ctx, EPH_ERR_ARG, "too many bodies with geopotential or ring models");
    ctx->n_ext = (int)ext.size();
    cudaError_t e = cudaMemcpy(ctx->d_cst, cst.data(), cst.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !ext.empty())
        e = cudaMemcpy(ctx->d_ext, ext.data(), ext.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->d_orig, orig.data(), orig.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(ctx, EPH_ERR_CUDA, "upload constants", e);
    return EPH_OK;
}

extern "C" {

int eph_upload_system(eph_ctx *ctx, int64_t n64, const double *planes, const eph_models *models) {
    if (!ctx || !planes || n64 <= 0 || n64 > (1 << 20)) return fail(ctx, EPH_ERR_ARG, "eph_upload_system: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int n = (int)n64;
    const int n_gp = models ? models->n_gp : 0, n_ring = models ? models->n_ring : 0;
    if (n_gp < 0 || n_ring < 0 || (n_gp && (!models->gp_nz || !models->gp_nt || !models->gp_coef)) ||
        (n_ring && (!models->ring_ndisk || !models->ring_param || !models->ring_disk)))
        return fail(ctx, EPH_ERR_ARG, "eph_upload_system: bad model tables");
    for (int k = 0; k < n_ring; ++k)
        if (models->ring_ndisk[k] < 0 || models->ring_ndisk[k] > EPH_RING_MAX_DISKS)
            return fail(ctx, EPH_ERR_ARG, "eph_upload_system: ring disk count out of range");
    for (int k = 0; k < n_gp; ++k)
        if (models->gp_nz[k] < 0 || models->gp_nz[k] > EPH_GP_MAX_DEGREE || models->gp_nt[k] > models->gp_nz[k])
            return fail(ctx, EPH_ERR_ARG, "eph_upload_system: geopotential degree out of range");
    for (int i = 0; i < n; ++i) {
        const double g = planes[(size_t)EPH_P_GP_INDEX * n + i], r = planes[(size_t)EPH_P_RING_INDEX * n + i];
        if (!(g >= -1 && g < n_gp) || !(r >= -1 && r < n_ring))
            return fail(ctx, EPH_ERR_ARG, "eph_upload_system: model index out of range");
    }
    if ((size_t)n > ctx->cap_n) {
        free_system(ctx);
        CK(cudaMalloc(&ctx->d_planes, (size_t)EPH_NPLANES * n * sizeof(double)), "cudaMalloc(planes)");
        const int ld = (n + kPad - 1) / kPad * kPad;
        CK(cudaMalloc(&ctx->d_pub, (size_t)2 * PUB_NPLANES * ld * sizeof(double)), "cudaMalloc(public state)");
        CK(cudaMalloc(&ctx->d_aux, (size_t)AUX_NPLANES * ld * sizeof(double)), "cudaMalloc(aux)");
        CK(cudaMalloc(&ctx->d_react, (size_t)kMaxExt * ld * 18 * sizeof(double)), "cudaMalloc(reactions)");
        CK(cudaMalloc(&ctx->d_cst, (size_t)CST_NPLANES * ld * sizeof(double)), "cudaMalloc(constants)");
        CK(cudaMemset(ctx->d_aux, 0, (size_t)AUX_NPLANES * ld * sizeof(double)), "cudaMemset");
        CK(cudaMemset(ctx->d_react, 0, (size_t)kMaxExt * ld * 18 * sizeof(double)), "cudaMemset");
        CK(cudaMalloc(&ctx->d_ext, (size_t)kMaxExt * sizeof(int)), "cudaMalloc(ext)");
        CK(cudaMalloc(&ctx->d_own, (size_t)n * kOwnMax * sizeof(int)), "cudaMalloc(ownership)");
        CK(cudaMalloc(&ctx->d_orig, (size_t)n * sizeof(int)), "cudaMalloc(order)");
        CK(cudaMemset(ctx->d_pub, 0, (size_t)2 * PUB_NPLANES * ld * sizeof(double)), "cudaMemset");
        ctx->ld = ld;
        ctx->cap_n = n;
    }
    // model tables: reallocated only when a larger table set arrives
    if (!ctx->d_gp_nz || n_gp > ctx->cap_gp) {
        for (int **p : {&ctx->d_gp_nz, &ctx->d_gp_nt}) { if (*p) cudaFree(*p); *p = nullptr; }
        if (ctx->d_gp_coef) cudaFree(ctx->d_gp_coef);
        ctx->d_gp_coef = nullptr;
        ctx->cap_gp = std::max(n_gp, 1);
        CK(cudaMalloc(&ctx->d_gp_nz, ctx->cap_gp * sizeof(int)), "cudaMalloc(gp)");
        CK(cudaMalloc(&ctx->d_gp_nt, ctx->cap_gp * sizeof(int)), "cudaMalloc(gp)");
        CK(cudaMalloc(&ctx->d_gp_coef, ctx->cap_gp * EPH_GP_TABLE_SIZE * sizeof(double)), "cudaMalloc(gp)");
    }
    if (!ctx->d_ring_nd || n_ring > ctx->cap_ring) {
        if (ctx->d_ring_nd) cudaFree(ctx->d_ring_nd);
        for (double **p : {&ctx->d_ring_param, &ctx->d_ring_disk}) { if (*p) cudaFree(*p); *p = nullptr; }
        ctx->d_ring_nd = nullptr;
        ctx->cap_ring = std::max(n_ring, 1);
        CK(cudaMalloc(&ctx->d_ring_nd, ctx->cap_ring * sizeof(int)), "cudaMalloc(ring)");
        CK(cudaMalloc(&ctx->d_ring_param, ctx->cap_ring * 4 * sizeof(double)), "cudaMalloc(ring)");
        CK(cudaMalloc(&ctx->d_ring_disk, ctx->cap_ring * EPH_RING_MAX_DISKS * 3 * sizeof(double)), "cudaMalloc(ring)");
    }
    const bool same_n = (ctx->n == n);
    ctx->n = n;
    ctx->n_gp = n_gp;
    ctx->n_ring = n_ring;
    if (n_gp) {
        CK(cudaMemcpy(ctx->d_gp_nz, models->gp_nz, n_gp * sizeof(int), cudaMemcpyHostToDevice), "upload gp");
        CK(cudaMemcpy(ctx->d_gp_nt, models->gp_nt, n_gp * sizeof(int), cudaMemcpyHostToDevice), "upload gp");
        CK(cudaMemcpy(ctx->d_gp_coef, models->gp_coef, (size_t)n_gp * EPH_GP_TABLE_SIZE * sizeof(double),
                      cudaMemcpyHostToDevice), "upload gp");
    }
    if (n_ring) {
        CK(cudaMemcpy(ctx->d_ring_nd, models->ring_ndisk, n_ring * sizeof(int), cudaMemcpyHostToDevice), "upload ring");
        CK(cudaMemcpy(ctx->d_ring_param, models->ring_param, (size_t)n_ring * 4 * sizeof(double),
                      cudaMemcpyHostToDevice), "upload ring");
        CK(cudaMemcpy(ctx->d_ring_disk, models->ring_disk, (size_t)n_ring * EPH_RING_MAX_DISKS * 3 * sizeof(double),
                      cudaMemcpyHostToDevice), "upload ring");
    }
    CK(cudaMemcpy(ctx->d_planes, planes, (size_t)EPH_NPLANES * n * sizeof(double), cudaMemcpyHostToDevice),
       "upload planes");
    std::vector<double> old_cost = ctx->h_cost;
    int rc = prepare_constants(ctx, planes);
    if (rc) return rc;
    if (same_n && ctx->grid > 0 && old_cost == ctx->h_cost) return EPH_OK;   // same ownership plan
    return choose_shape(ctx);
}

int eph_upload_planes_device(eph_ctx *ctx, const double *d_planes) {
    if (!ctx || !d_planes) return fail(ctx, EPH_ERR_ARG, "eph_upload_planes_device: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(ctx->d_planes, d_planes, (size_t)EPH_NPLANES * ctx->n * sizeof(double),
                       cudaMemcpyDeviceToDevice, ctx->stream), "device planes copy");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return EPH_OK;
}

int eph_download_system(eph_ctx *ctx, double *planes) {
    if (!ctx || !planes) return fail(ctx, EPH_ERR_ARG, "eph_download_system: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpy(planes, ctx->d_planes, (size_t)EPH_NPLANES * ctx->n * sizeof(double), cudaMemcpyDeviceToHost),
       "download planes");
    return EPH_OK;
}

int eph_device_planes(eph_ctx *ctx, double **d_planes) {
    if (!ctx || !d_planes) return fail(ctx, EPH_ERR_ARG, "eph_device_planes: bad arguments");
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    *d_planes = ctx->d_planes;
    return EPH_OK;
}

}  // extern "C"

static int run(eph_ctx *ctx, const StepParams &P) {
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    SysDev S;
    S.n = ctx->n;
    S.n_full = ctx->n_full;
    S.orig = ctx->d_orig;
    S.ld = ctx->ld;
    S.tile = ctx->tile;
    S.react = ctx->d_react;
    S.react_cta = ctx->d_react + (size_t)kMaxExt * ctx->ld * 12;
    S.n_ext = ctx->n_ext;
    S.pub = ctx->d_pub;
    S.aux = ctx->d_aux;
    S.cst = ctx->d_cst;
    S.planes = ctx->d_planes;
    S.ext_body = ctx->d_ext;
    S.n_gp = ctx->n_gp;
    S.gp_nz = ctx->d_gp_nz;
    S.gp_nt = ctx->d_gp_nt;
    S.gp_coef = ctx->d_gp_coef;
    S.ring_nd = ctx->d_ring_nd;
    S.ring_param = ctx->d_ring_param;
    S.ring_disk = ctx->d_ring_disk;
    S.own_list = ctx->d_own;
    S.bar = ctx->d_bar;
    S.status = ctx->d_status;
    S.timers = nullptr;
    S.traj = ctx->d_traj;
    S.traj_base = ctx->traj_base;
    S.wait_ns = ctx->wait_ns;
    S.stall_barrier = ctx->stall_barrier;
    if (ctx->d_timers) {
        if (ctx->timers_grid < ctx->grid) {
            cudaFree(ctx->d_timers);
            ctx->d_timers = nullptr;
            CK(cudaMalloc(&ctx->d_timers, (size_t)ctx->grid * kPhases * sizeof(unsigned long long)), "cudaMalloc(timers)");
            ctx->timers_grid = ctx->grid;
        }
        S.timers = ctx->d_timers;
    }
    CK(cudaMemsetAsync(ctx->d_bar, 0, 2 * sizeof(unsigned), ctx->stream), "reset barrier");
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream), "reset status");
    CK(launch_step(S, P, ctx->grid, ctx->stream), "launch RK12 kernel");
    ctx->launches++;
    int status = 0;
    CK(cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "read status");
    CK(cudaStreamSynchronize(ctx->stream), "RK12 kernel");
    if (status == ST_BARRIER_TIMEOUT) return fail(ctx, EPH_ERR_TIMEOUT, "grid barrier wait timed out");
    if (status == ST_COPY_TIMEOUT) return fail(ctx, EPH_ERR_TIMEOUT, "tile copy wait timed out");
    if (status != ST_OK) return fail(ctx, EPH_ERR_CUDA, "step kernel reported an unknown status");
    return EPH_OK;
}

extern "C" {

int eph_rk12(eph_ctx *ctx, double dt, int64_t n_step, double t_eph_hi, double t_eph_lo) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n_step <= 0) return EPH_OK;   // RungeKutta.cu:392
    StepParams P{MODE_INTEGRATE, 0, 0, (long long)n_step, dt, t_eph_hi + t_eph_lo};
    return run(ctx, P);
}

int eph_integrate(eph_ctx *ctx, double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo) {
    if (!ctx || !t_eph_hi || !t_eph_lo) return fail(ctx, EPH_ERR_ARG, "eph_integrate: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n_step == 0) return EPH_OK;   // mass.cpp:400
    if (n_step < 0) {                 // mass.cpp:401-404
        n_step = -n_step;
        dt = -dt;
    }
    StepParams P{MODE_INTEGRATE, 1, 1, (long long)n_step, dt, *t_eph_hi + *t_eph_lo};
    int rc = run(ctx, P);
    if (rc) return rc;
    // t_eph += dt*n_step in double-double (mass.cpp:441, dfloat_t.h:49-55)
    double a = *t_eph_hi, b = dt * (double)n_step;
    double s = a + b, t = s - a;
    double e = (a - (s - t)) + (b - t);
    e = e + (*t_eph_lo + 0.0);
    double hi = s + e;
    double lo = e - (hi - s);
    *t_eph_hi = hi;
    *t_eph_lo = lo;
    return EPH_OK;
}

int eph_accel(eph_ctx *ctx) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    StepParams P{MODE_ACCEL, 0, 0, 0, 0.0, 0.0};
    return run(ctx, P);
}

int eph_deform(eph_ctx *ctx) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    StepParams P{MODE_DEFORM, 0, 0, 0, 0.0, 0.0};
    return run(ctx, P);
}

int eph_selftest_wait_timeout(eph_ctx *ctx, int64_t wait_ns) {
    if (!ctx || wait_ns < 100000 || wait_ns > kWaitDefaultNs) return fail(ctx, EPH_ERR_ARG, "eph_selftest_wait_timeout: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->wait_ns = wait_ns;
    ctx->stall_barrier = 1;
    StepParams P{MODE_ACCEL, 0, 0, 0, 0.0, 0.0};
    const int rc = run(ctx, P);
    ctx->wait_ns = kWaitDefaultNs;
    ctx->stall_barrier = 0;
    return rc;
}

int eph_set_stream(eph_ctx *ctx, void *stream) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return EPH_OK;
}

int eph_set_launch(eph_ctx *ctx, int grid, int bodies_per_cta) {
    if (!ctx || grid < 0 || bodies_per_cta < 0 || bodies_per_cta > kOwnMax)
        return fail(ctx, EPH_ERR_ARG, "eph_set_launch: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->req_grid = grid;
    ctx->req_per_cta = bodies_per_cta;
    if (!ctx->n) return EPH_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return choose_shape(ctx);
}

int eph_set_body_costs(eph_ctx *ctx, const double *cost) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    const int n = ctx->n;
    if (cost) {
        for (int i = 0; i < n; ++i)
            if (!(cost[i] > 0) || !std::isfinite(cost[i])) return fail(ctx, EPH_ERR_ARG, "eph_set_body_costs: costs must be positive");
        ctx->cost_override.assign(cost, cost + n);
    } else {
        ctx->cost_override.clear();
    }
    std::vector<double> h_planes((size_t)EPH_NPLANES * n);
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpy(h_planes.data(), ctx->d_planes, h_planes.size() * sizeof(double), cudaMemcpyDeviceToHost),
       "read planes");
    int rc = prepare_constants(ctx, h_planes.data());
    return rc ? rc : choose_shape(ctx);
}

int eph_get_ownership(const eph_ctx *ctx, int32_t *bodies, int *grid) {
    if (!ctx || !bodies || !grid) return EPH_ERR_ARG;
    if (!ctx->n || ctx->h_own.size() < (size_t)ctx->grid * kOwnMax) return EPH_ERR_STATE;
    for (size_t q = 0; q < (size_t)ctx->grid * kOwnMax; ++q) {
        const int k = ctx->h_own[q];
        bodies[q] = k < 0 ? -1 : ctx->h_orig[k];
    }
    *grid = ctx->grid;
    return EPH_OK;
}

// ---- autotuner: candidates of the launch shape and the ownership cost model, timed on the uploaded system
namespace {
struct TuneKey {
    int device, n, n_full, n_delayed, n_ext;
    bool operator<(const TuneKey &o) const {
        return std::tie(device, n, n_full, n_delayed, n_ext) < std::tie(o.device, o.n, o.n_full, o.n_delayed, o.n_ext);
    }
};
struct TuneChoice {
    int req_grid, req_per;
    double delayed_weight;   // 0: the built-in cost model
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune_cache;
}  // namespace

static int apply_choice(eph_ctx *ctx, const double *h_planes, const TuneChoice &c) {
    const int n = ctx->n;
    if (c.delayed_weight > 0) {
        std::vector<double> cost(n);
        for (int i = 0; i < n; ++i) {
            const bool full = plan_full_class(h_planes, n, i);
            const bool delayed = h_planes[(size_t)EPH_P_K2 * n + i] != 0 && h_planes[(size_t)EPH_P_TIDE_DELAY * n + i] != 0;
            cost[i] = delayed ? c.delayed_weight : plan_cost(h_planes, n, i, full);
        }
        ctx->cost_override = cost;
    } else {
        ctx->cost_override.clear();
    }
    ctx->req_grid = c.req_grid;
    ctx->req_per_cta = c.req_per;
    int rc = prepare_constants(ctx, h_planes);
    return rc ? rc : choose_shape(ctx);
}

int eph_autotune(eph_ctx *ctx, double dt, int n_step, int reps, int use_cache, int *grid, int *bodies_per_cta,
                 double *ms_tuned, double *ms_default) {
    if (!ctx || !(dt != 0) || n_step < 1 || reps < 1 || !grid || !bodies_per_cta || !ms_tuned || !ms_default)
        return fail(ctx, EPH_ERR_ARG, "eph_autotune: bad arguments");
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->n) return fail(ctx, EPH_ERR_STATE, "no system uploaded");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int n = ctx->n;
    std::vector<double> h_planes((size_t)EPH_NPLANES * n);
    CK(cudaMemcpy(h_planes.data(), ctx->d_planes, h_planes.size() * sizeof(double), cudaMemcpyDeviceToHost), "read planes");
    int n_delayed = 0;
    for (int i = 0; i < n; ++i)
        n_delayed += h_planes[(size_t)EPH_P_K2 * n + i] != 0 && h_planes[(size_t)EPH_P_TIDE_DELAY * n + i] != 0;
    const TuneKey key{ctx->device, n, ctx->n_full, n_delayed, ctx->n_ext};
    // every trial integrates from the uploaded state, which is restored afterwards
    double *d_save = nullptr;
    CK(cudaMalloc(&d_save, h_planes.size() * sizeof(double)), "cudaMalloc(autotune)");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = EPH_OK;
    auto time_choice = [&](const TuneChoice &c, double *ms) -> int {
        int r = apply_choice(ctx, h_planes.data(), c);
        if (r) return r;
        double best = 1e300;
        for (int q = 0; q < reps + 1 && r == EPH_OK; ++q) {   // the first run warms up
            if (cudaMemcpyAsync(ctx->d_planes, d_save, h_planes.size() * sizeof(double), cudaMemcpyDeviceToDevice,
                                ctx->stream) != cudaSuccess)
                return fail(ctx, EPH_ERR_CUDA, "autotune restore");
            cudaEventRecord(e0, ctx->stream);
            const StepParams P{MODE_INTEGRATE, 0, 0, (long long)n_step, dt, 0.0};
            r = run(ctx, P);
            cudaEventRecord(e1, ctx->stream);
            float t = 0;
            if (r == EPH_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) {
                if (q > 0) best = std::min(best, (double)t / n_step);
            }
        }
        *ms = best;
        return r;
    };
    if (cudaMemcpy(d_save, ctx->d_planes, h_planes.size() * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        rc = fail(ctx, EPH_ERR_CUDA, "autotune set-up");
    const TuneChoice heuristic{0, 0, 0.0};
    double t_def = 1e300, t_best = 1e300;
    TuneChoice best = heuristic;
    if (rc == EPH_OK) rc = time_choice(heuristic, &t_def);
    t_best = t_def;
    bool cached = false;
    if (rc == EPH_OK && use_cache) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) { best = it->second; cached = true; }
    }
    if (rc == EPH_OK && cached) {
        rc = time_choice(best, &t_best);
    } else if (rc == EPH_OK) {
        std::vector<TuneChoice> cands;
        for (int per : {1, 2, 3, 4, 6, 8}) cands.push_back(TuneChoice{0, per, 0.0});
        if (n_delayed > 0)
            for (double wd : {15.0, 25.0, 80.0})
                for (int per : {0, 4, 8}) cands.push_back(TuneChoice{0, per, wd});
        for (const TuneChoice &c : cands) {
            double t = 1e300;
            const int r = time_choice(c, &t);
            if (r == EPH_ERR_ARG) continue;   // a shape that does not fit the co-resident CTAs
            if (r) { rc = r; break; }
            if (t < t_best) { t_best = t; best = c; }
        }
        if (rc == EPH_OK) {
            std::lock_guard<std::mutex> g(g_tune_mu);
            g_tune_cache[key] = best;
        }
    }
    // leave the context on the chosen shape, with the uploaded state
    if (rc == EPH_OK) rc = apply_choice(ctx, h_planes.data(), best);
    if (cudaMemcpy(ctx->d_planes, d_save, h_planes.size() * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess && !rc)
        rc = fail(ctx, EPH_ERR_CUDA, "autotune restore");
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_save);
    if (rc) return rc;
    *grid = ctx->grid;
    *bodies_per_cta = ctx->per_cta;
    *ms_tuned = t_best;
    *ms_default = t_def;
    return EPH_OK;
}

int eph_get_launch(const eph_ctx *ctx, int *grid, int *bodies_per_cta) {
    if (!ctx || !grid || !bodies_per_cta) return EPH_ERR_ARG;
    *grid = ctx->grid;
    *bodies_per_cta = ctx->per_cta;
    return EPH_OK;
}

int64_t eph_launch_count(const eph_ctx *ctx) { return ctx ? ctx->launches : -1; }

int eph_profile_phases(eph_ctx *ctx, int enable) {
    if (!ctx) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!enable) {
        if (ctx->d_timers) cudaFree(ctx->d_timers);
        ctx->d_timers = nullptr;
        ctx->timers_grid = 0;
        return EPH_OK;
    }
    if (!ctx->d_timers) {
        const int g = std::max(ctx->grid, 1);
        CK(cudaMalloc(&ctx->d_timers, (size_t)g * kPhases * sizeof(unsigned long long)), "cudaMalloc(timers)");
        CK(cudaMemset(ctx->d_timers, 0, (size_t)g * kPhases * sizeof(unsigned long long)), "cudaMemset(timers)");
        ctx->timers_grid = g;
    }
    return EPH_OK;
}

int eph_phase_times(eph_ctx *ctx, uint64_t *out, int *grid, int *phases) {
    if (!ctx || !out || !grid || !phases) return EPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!ctx->d_timers) return fail(ctx, EPH_ERR_STATE, "phase timers are off");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpy(out, ctx->d_timers, (size_t)ctx->grid * kPhases * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
       "read timers");
    *grid = ctx->grid;
    *phases = kPhases;
    return EPH_OK;
}

}  // extern "C"
