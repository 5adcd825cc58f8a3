/*
 * ref_driver.cpp - flat C entry points over the reference's own CPU integrator.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY. This file is compiled together with the unmodified
 * reference sources (src/physics/mass.cpp, src/integrators/RungeKutta.cpp, src/modules/mass_loader.cpp,
 * ...) into oracle/_ref/libephref.so by oracle/Makefile. It lets the tests and the CPU-baseline leg
 * of bench.py drive the reference exactly as its own callers do:
 *   msystem::load(config)              src/modules/mass_loader.cpp:67-294
 *   msystem::integrate(dt, n, 0)       src/physics/mass.cpp:399-442 -> RungeKutta12 (RungeKutta.impl:107-194)
 *   msystem::accel(option)             src/physics/mass.cpp:216-397
 *   ThreadPool::thread_local_pool_alloc src/utils/threadpool.cpp:13-18
 * and exchange body state in the plane layout of include/eph_planes.h.
 *
 * Per-stage capture: the library is linked with -Wl,--wrap=_ZN7msystem5accelEi, so the ACCEL()
 * call inside RungeKutta12 (RungeKutta.impl:188) lands in __wrap_... below, which calls the real
 * accel() and then copies the stage's body planes out. No reference source is modified.
 */
#include "physics/mass.h"
#include "physics/geopotential.h"
#include "physics/ring.h"
#include "utils/threadpool.h"
#include "utils/logger.h"
#include "eph_planes.h"

#include <cstdint>
#include <cstring>
#include <vector>

// mass.h:213-215 grants friendship to ephemeris_reader; its translation unit is not linked into
// this library, so this file uses the name to reach msystem's private members.
class ephemeris_reader {
public:
    static htl::vector<mass> &bodies(msystem &m) { return m.mlist; }
    static real &t_eph(msystem &m) { return m.t_eph; }
    static fast_real &delta_t(msystem &m) { return m.delta_t; }
    static void deform(msystem &m) { m.deform(); }
};

// geopotential keeps {Nz, Nt, c_table[]} private (src/physics/geopotential.h:7-9).
struct gp_view { int64_t Nz, Nt; double c_table[1]; };

static void put3(double *pl, int64_t n, int p, int64_t i, const fast_mpvec &v) {
    pl[(p + 0) * n + i] = v.x; pl[(p + 1) * n + i] = v.y; pl[(p + 2) * n + i] = v.z;
}
static void put3dd(double *pl, int64_t n, int phi, int plo, int64_t i, const mpvec &v) {
    pl[(phi + 0) * n + i] = v.x.hi; pl[(phi + 1) * n + i] = v.y.hi; pl[(phi + 2) * n + i] = v.z.hi;
    pl[(plo + 0) * n + i] = v.x.lo; pl[(plo + 1) * n + i] = v.y.lo; pl[(plo + 2) * n + i] = v.z.lo;
}
static void put9(double *pl, int64_t n, int p, int64_t i, const fast_mpmat &m) {
    put3(pl, n, p, i, m.x); put3(pl, n, p + 3, i, m.y); put3(pl, n, p + 6, i, m.z);
}
static void put9dd(double *pl, int64_t n, int phi, int plo, int64_t i, const mpmat &m) {
    put3dd(pl, n, phi, plo, i, m.x); put3dd(pl, n, phi + 3, plo + 3, i, m.y); put3dd(pl, n, phi + 6, plo + 6, i, m.z);
}
static fast_mpvec get3(const double *pl, int64_t n, int p, int64_t i) {
    return fast_mpvec(pl[(p + 0) * n + i], pl[(p + 1) * n + i], pl[(p + 2) * n + i]);
}
static mpvec get3dd(const double *pl, int64_t n, int phi, int plo, int64_t i) {
    return mpvec(real(pl[(phi + 0) * n + i], pl[(plo + 0) * n + i]),
                 real(pl[(phi + 1) * n + i], pl[(plo + 1) * n + i]),
                 real(pl[(phi + 2) * n + i], pl[(plo + 2) * n + i]));
}
static fast_mpmat get9(const double *pl, int64_t n, int p, int64_t i) {
    return fast_mpmat(get3(pl, n, p, i), get3(pl, n, p + 3, i), get3(pl, n, p + 6, i));
}
static mpmat get9dd(const double *pl, int64_t n, int phi, int plo, int64_t i) {
    return mpmat(get3dd(pl, n, phi, plo, i), get3dd(pl, n, phi + 3, plo + 3, i), get3dd(pl, n, phi + 6, plo + 6, i));
}

static void dump_planes(msystem &ms, double *pl, uint64_t *sid) {
    auto &ml = ephemeris_reader::bodies(ms);
    const int64_t n = ml.size();
    // model indices follow body order: the k-th body with a geopotential has index k
    int64_t igp = 0, iring = 0;
    for (int64_t i = 0; i < n; ++i) {
        const mass &m = ml[i];
        put3dd(pl, n, EPH_P_R_HI, EPH_P_R_LO, i, m.r);
        put3dd(pl, n, EPH_P_V_HI, EPH_P_V_LO, i, m.v);
        put3dd(pl, n, EPH_P_GL_HI, EPH_P_GL_LO, i, m.GL);
        put9dd(pl, n, EPH_P_S_HI, EPH_P_S_LO, i, m.s);
        put3(pl, n, EPH_P_W, i, m.w);
        pl[EPH_P_GM * n + i] = m.GM;
        pl[EPH_P_EXJ2 * n + i] = m.exJ2;
        pl[EPH_P_GM0 * n + i] = m.GM0;
        pl[EPH_P_DGM * n + i] = m.dGM;
        pl[EPH_P_DJ2 * n + i] = m.dJ2;
        pl[EPH_P_RADIUS * n + i] = m.R;
        pl[EPH_P_INERTIA * n + i] = m.inertia;
        pl[EPH_P_K2 * n + i] = m.k2;
        pl[EPH_P_K2R * n + i] = m.k2r;
        pl[EPH_P_TIDE_DELAY * n + i] = m.tide_delay;
        pl[EPH_P_TIDE_DELAY_FACTOR * n + i] = m.tide_delay_factor;
        pl[EPH_P_LUM * n + i] = m.lum;
        pl[EPH_P_RECPT * n + i] = m.recpt;
        pl[EPH_P_A * n + i] = m.A;
        pl[EPH_P_R2 * n + i] = m.R2;
        pl[EPH_P_SR2 * n + i] = m.sR2;
        pl[EPH_P_RR2G_4C * n + i] = m.rR2G_4c;
        put9(pl, n, EPH_P_C_STATIC, i, m.C_static);
        pl[EPH_P_PHI * n + i] = m.phi;
        pl[EPH_P_BETA2 * n + i] = m.beta2;
        put3(pl, n, EPH_P_NACCEL, i, m.naccel);
        put3(pl, n, EPH_P_DACCEL, i, m.daccel);
        put3(pl, n, EPH_P_DTORQUE, i, m.dtorque);
        put3(pl, n, EPH_P_GACCEL, i, m.gaccel);
        put3(pl, n, EPH_P_BETA, i, m.beta);
        put9(pl, n, EPH_P_GI, i, m.GI);
        put9(pl, n, EPH_P_C_POTENTIAL, i, m.C_potential);
        pl[EPH_P_MIN_DISTANCE * n + i] = m.min_distance;
        pl[EPH_P_MAX_INFLUENCE * n + i] = m.max_influence;
        pl[EPH_P_GP_INDEX * n + i] = m.gpmodel ? (double)igp++ : -1.0;
        pl[EPH_P_RING_INDEX * n + i] = m.ringmodel ? (double)iring++ : -1.0;
        if (sid) sid[i] = m.sid;
    }
}

/* --- per-stage capture through the linker wrap of msystem::accel(int) --- */
static struct {
    msystem *ms = nullptr;
    double *buf = nullptr;
    int64_t cap = 0, count = 0;
} g_rec;

extern "C" void __real__ZN7msystem5accelEi(msystem *self, int option);
extern "C" void __wrap__ZN7msystem5accelEi(msystem *self, int option) {
    __real__ZN7msystem5accelEi(self, option);
    if (g_rec.ms == self && g_rec.count < g_rec.cap) {
        const int64_t n = ephemeris_reader::bodies(*self).size();
        dump_planes(*self, g_rec.buf + g_rec.count * (int64_t)EPH_NPLANES * n, nullptr);
        ++g_rec.count;
    }
}

extern "C" {

void *ref_load(const char *config) {
    msystem *ms = new msystem();
    if (!ms->load(config)) { delete ms; return nullptr; }
    return ms;
}
void ref_free(void *h) { delete (msystem *)h; }
void *ref_clone(void *h) { return new msystem(*(msystem *)h); }
int64_t ref_size(void *h) { return ephemeris_reader::bodies(*(msystem *)h).size(); }
void ref_get_t_eph(void *h, double *hi, double *lo) {
    const real &t = ephemeris_reader::t_eph(*(msystem *)h); *hi = t.hi; *lo = t.lo;
}
double ref_delta_t(void *h) { return ephemeris_reader::delta_t(*(msystem *)h); }
/* level: messages below it are dropped (LogLevel values, src/utils/logger.h:23-31) */
void ref_set_log_level(int level) { global_logger.set_log_levels(LogLevel((uint8_t)level)); }

/* option 1: the calling thread gets the reference's thread pool (min(16, cores) workers,
 * threadpool.h:28); 0: it is released and accel() runs its serial branch (mass.cpp:309-374). */
void ref_thread_pool(int enable) {
    if (enable) ThreadPool::thread_local_pool_alloc();
    else ThreadPool::thread_local_pool_free();
}

void ref_integrate(void *h, double dt, int64_t n_step) { ((msystem *)h)->integrate(dt, n_step, 0); }
/* msystem::integrate(dt, n, USE_GPU=1): the reference's GPU branch, i.e. whatever translation unit
 * defines msystem::Cuda_RungeKutta12 in this library (the B200 bridge in libephref_b200.so). */
void ref_integrate_gpu(void *h, double dt, int64_t n_step) { ((msystem *)h)->integrate(dt, n_step, 1); }
void ref_accel(void *h, int option) { ((msystem *)h)->accel(option); }
void ref_deform(void *h) { ephemeris_reader::deform(*(msystem *)h); }

void ref_get_planes(void *h, double *planes, uint64_t *sid) { dump_planes(*(msystem *)h, planes, sid); }

/* Overwrite the evolving state, time-variable parameters and auxiliaries from planes (the
 * constants and model links are left as loaded). */
void ref_set_planes(void *h, const double *pl) {
    auto &ml = ephemeris_reader::bodies(*(msystem *)h);
    const int64_t n = ml.size();
    for (int64_t i = 0; i < n; ++i) {
        mass &m = ml[i];
        m.r = get3dd(pl, n, EPH_P_R_HI, EPH_P_R_LO, i);
        m.v = get3dd(pl, n, EPH_P_V_HI, EPH_P_V_LO, i);
        m.GL = get3dd(pl, n, EPH_P_GL_HI, EPH_P_GL_LO, i);
        m.s = get9dd(pl, n, EPH_P_S_HI, EPH_P_S_LO, i);
        m.w = get3(pl, n, EPH_P_W, i);
        m.GM = pl[EPH_P_GM * n + i];
        m.exJ2 = pl[EPH_P_EXJ2 * n + i];
        m.phi = pl[EPH_P_PHI * n + i];
        m.beta2 = pl[EPH_P_BETA2 * n + i];
        m.naccel = get3(pl, n, EPH_P_NACCEL, i);
        m.daccel = get3(pl, n, EPH_P_DACCEL, i);
        m.dtorque = get3(pl, n, EPH_P_DTORQUE, i);
        m.gaccel = get3(pl, n, EPH_P_GACCEL, i);
        m.beta = get3(pl, n, EPH_P_BETA, i);
        m.GI = get9(pl, n, EPH_P_GI, i);
        m.C_potential = get9(pl, n, EPH_P_C_POTENTIAL, i);
        m.min_distance = pl[EPH_P_MIN_DISTANCE * n + i];
        m.max_influence = pl[EPH_P_MAX_INFLUENCE * n + i];
    }
}

/* Model tables in body order: gp_nz/gp_nt[k], gp_coef[k*EPH_GP_TABLE_SIZE + t];
 * ring_ndisk[k], ring_param[k*4 + {GM_ratio,A,J2,GL_R2}], ring_disk[(k*EPH_RING_MAX_DISKS+d)*3 + {GsR2,R_R,H_R}].
 * Returns the number of geopotential models in the low 32 bits and ring models in the high bits. */
int64_t ref_get_models(void *h, int32_t *gp_nz, int32_t *gp_nt, double *gp_coef,
                       int32_t *ring_ndisk, double *ring_param, double *ring_disk) {
    auto &ml = ephemeris_reader::bodies(*(msystem *)h);
    int64_t ngp = 0, nring = 0;
    for (const mass &m : ml) {
        if (m.gpmodel) {
            const gp_view *g = (const gp_view *)m.gpmodel;
            if (gp_nz) {
                gp_nz[ngp] = (int32_t)g->Nz;
                gp_nt[ngp] = (int32_t)g->Nt;
                const int64_t sz = g->Nz * (g->Nz + 2) - 3;
                for (int64_t t = 0; t < EPH_GP_TABLE_SIZE; ++t)
                    gp_coef[ngp * EPH_GP_TABLE_SIZE + t] = t < sz ? g->c_table[t] : 0.0;
            }
            ++ngp;
        }
        if (m.ringmodel) {
            const ring *rg = m.ringmodel;
            if (ring_ndisk) {
                ring_ndisk[nring] = (int32_t)rg->N;
                ring_param[nring * 4 + 0] = rg->GM_ratio;
                ring_param[nring * 4 + 1] = rg->A;
                ring_param[nring * 4 + 2] = rg->J2;
                ring_param[nring * 4 + 3] = rg->GL_R2;
                for (int64_t d = 0; d < rg->N && d < EPH_RING_MAX_DISKS; ++d) {
                    double *o = ring_disk + (nring * EPH_RING_MAX_DISKS + d) * 3;
                    o[0] = rg->c_table[d].GsR2; o[1] = rg->c_table[d].R_R; o[2] = rg->c_table[d].H_R;
                }
            }
            ++nring;
        }
    }
    return ngp | (nring << 32);
}

/* Start capturing the body planes after every accel() of system h into buf
 * (cap stages of EPH_NPLANES*n doubles); h == NULL stops. Returns the stages captured so far. */
int64_t ref_capture(void *h, double *buf, int64_t cap) {
    int64_t got = g_rec.count;
    g_rec.ms = (msystem *)h; g_rec.buf = buf; g_rec.cap = cap; g_rec.count = 0;
    return got;
}
int64_t ref_capture_count(void) { return g_rec.count; }

}  // extern "C"

