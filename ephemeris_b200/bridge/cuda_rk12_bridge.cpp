// cuda_rk12_bridge.cpp - drop-in replacement for the reference's src/integrators/RungeKutta.cu.
//
// A maintainer removes RungeKutta.cu from the reference build, adds this translation unit, and links
// libeph_b200.so. It defines the two private members the reference declares for its GPU path
// (src/physics/mass.h:268,270):
//   void msystem::Cuda_RungeKutta12(fast_real dt, int_t n_step)   replaces RungeKutta.cu:391-412
//   void msystem::Cuda_accel()                                    replaces RungeKutta.cu:418-438
// so msystem::integrate(dt, n, USE_GPU=1) (mass.cpp:408-409) and msystem::accel(1) (mass.cpp:218-220)
// run the B200 kernels. Each call packs the `mass` list into the plane layout of include/eph_planes.h,
// runs eph_rk12 / eph_accel and unpacks every field the host reads afterwards, as the reference's
// kernel config load/save does (RungeKutta.cu:77-133). Calls are serialised on one mutex, as the
// reference serialises GPU work on cuda_mutex (RungeKutta.cu:25,396,410). Errors are logged and, like
// Cuda_OnError (RungeKutta.cu:379-389), end the process.
//
// Compiled against the reference's own headers (physics/mass.h, physics/geopotential.h, physics/ring.h).
#include "physics/mass.h"
#include "physics/geopotential.h"
#include "physics/ring.h"
#include "utils/logger.h"

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "eph_b200.h"

namespace {

std::mutex g_mu;
eph_ctx *g_ctx = nullptr;

// geopotential keeps {Nz, Nt, c_table[]} private (src/physics/geopotential.h:7-9)
struct gp_layout { int64_t Nz, Nt; double c_table[1]; };

void put3(double *pl, int64_t n, int p, int64_t i, const fast_mpvec &v) {
    pl[(p + 0) * n + i] = v.x; pl[(p + 1) * n + i] = v.y; pl[(p + 2) * n + i] = v.z;
}
void put3dd(double *pl, int64_t n, int ph, int plo, int64_t i, const mpvec &v) {
    const real *c[3] = {&v.x, &v.y, &v.z};
    for (int k = 0; k < 3; ++k) { pl[(ph + k) * n + i] = c[k]->hi; pl[(plo + k) * n + i] = c[k]->lo; }
}
fast_mpvec get3(const double *pl, int64_t n, int p, int64_t i) {
    return fast_mpvec(pl[(p + 0) * n + i], pl[(p + 1) * n + i], pl[(p + 2) * n + i]);
}
mpvec get3dd(const double *pl, int64_t n, int ph, int plo, int64_t i) {
    return mpvec(real(pl[(ph + 0) * n + i], pl[(plo + 0) * n + i]), real(pl[(ph + 1) * n + i], pl[(plo + 1) * n + i]),
                 real(pl[(ph + 2) * n + i], pl[(plo + 2) * n + i]));
}

struct Packed {
    std::vector<double> planes;
    std::vector<int32_t> gp_nz, gp_nt, ring_nd;
    std::vector<double> gp_coef, ring_param, ring_disk;
    eph_models models{};
};

void pack(const htl::vector<mass> &ml, Packed &pk) {
    const int64_t n = ml.size();
    pk.planes.assign((size_t)EPH_NPLANES * n, 0.0);
    double *pl = pk.planes.data();
    for (int64_t i = 0; i < n; ++i) {
        const mass &m = ml[i];
        put3dd(pl, n, EPH_P_R_HI, EPH_P_R_LO, i, m.r);
        put3dd(pl, n, EPH_P_V_HI, EPH_P_V_LO, i, m.v);
        put3dd(pl, n, EPH_P_GL_HI, EPH_P_GL_LO, i, m.GL);
        put3dd(pl, n, EPH_P_S_HI, EPH_P_S_LO, i, m.s.x);
        put3dd(pl, n, EPH_P_S_HI + 3, EPH_P_S_LO + 3, i, m.s.y);
        put3dd(pl, n, EPH_P_S_HI + 6, EPH_P_S_LO + 6, i, m.s.z);
        put3(pl, n, EPH_P_W, i, m.w);
        const double sc[] = {m.GM, m.exJ2, m.GM0, m.dGM, m.dJ2, m.R, m.inertia, m.k2, m.k2r, m.tide_delay,
                             m.tide_delay_factor, m.lum, m.recpt, m.A, m.R2, m.sR2, m.rR2G_4c};
        for (int k = 0; k < 17; ++k) pl[(EPH_P_GM + k) * n + i] = sc[k];
        put3(pl, n, EPH_P_C_STATIC, i, m.C_static.x);
        put3(pl, n, EPH_P_C_STATIC + 3, i, m.C_static.y);
        put3(pl, n, EPH_P_C_STATIC + 6, i, m.C_static.z);
        pl[EPH_P_PHI * n + i] = m.phi;
        pl[EPH_P_BETA2 * n + i] = m.beta2;
        put3(pl, n, EPH_P_NACCEL, i, m.naccel);
        put3(pl, n, EPH_P_DACCEL, i, m.daccel);
        put3(pl, n, EPH_P_DTORQUE, i, m.dtorque);
        put3(pl, n, EPH_P_GACCEL, i, m.gaccel);
        put3(pl, n, EPH_P_BETA, i, m.beta);
        put3(pl, n, EPH_P_GI, i, m.GI.x); put3(pl, n, EPH_P_GI + 3, i, m.GI.y); put3(pl, n, EPH_P_GI + 6, i, m.GI.z);
        put3(pl, n, EPH_P_C_POTENTIAL, i, m.C_potential.x);
        put3(pl, n, EPH_P_C_POTENTIAL + 3, i, m.C_potential.y);
        put3(pl, n, EPH_P_C_POTENTIAL + 6, i, m.C_potential.z);
        pl[EPH_P_MIN_DISTANCE * n + i] = m.min_distance;
        pl[EPH_P_MAX_INFLUENCE * n + i] = m.max_influence;
        pl[EPH_P_GP_INDEX * n + i] = -1;
        pl[EPH_P_RING_INDEX * n + i] = -1;
        if (m.gpmodel) {
            const gp_layout *g = (const gp_layout *)m.gpmodel;
            pl[EPH_P_GP_INDEX * n + i] = (double)pk.gp_nz.size();
            pk.gp_nz.push_back((int32_t)g->Nz);
            pk.gp_nt.push_back((int32_t)g->Nt);
            const int64_t sz = g->Nz * (g->Nz + 2) - 3;
            for (int t = 0; t < EPH_GP_TABLE_SIZE; ++t) pk.gp_coef.push_back(t < sz ? g->c_table[t] : 0.0);
        }
        if (m.ringmodel) {
            const ring *r = m.ringmodel;
            pl[EPH_P_RING_INDEX * n + i] = (double)pk.ring_nd.size();
            pk.ring_nd.push_back((int32_t)r->N);
            pk.ring_param.insert(pk.ring_param.end(), {r->GM_ratio, r->A, r->J2, r->GL_R2});
            for (int d = 0; d < EPH_RING_MAX_DISKS; ++d) {
                const bool on = d < r->N;
                pk.ring_disk.push_back(on ? r->c_table[d].GsR2 : 0.0);
                pk.ring_disk.push_back(on ? r->c_table[d].R_R : 0.0);
                pk.ring_disk.push_back(on ? r->c_table[d].H_R : 0.0);
            }
        }
    }
    pk.models.n_gp = (int32_t)pk.gp_nz.size();
    pk.models.gp_nz = pk.gp_nz.data();
    pk.models.gp_nt = pk.gp_nt.data();
    pk.models.gp_coef = pk.gp_coef.data();
    pk.models.n_ring = (int32_t)pk.ring_nd.size();
    pk.models.ring_ndisk = pk.ring_nd.data();
    pk.models.ring_param = pk.ring_param.data();
    pk.models.ring_disk = pk.ring_disk.data();
}

// write back every field the reference's kernel leaves behind (RungeKutta.cu:124-133)
void unpack(const std::vector<double> &planes, htl::vector<mass> &ml) {
    const int64_t n = ml.size();
    const double *pl = planes.data();
    for (int64_t i = 0; i < n; ++i) {
        mass &m = ml[i];
        m.r = get3dd(pl, n, EPH_P_R_HI, EPH_P_R_LO, i);
        m.v = get3dd(pl, n, EPH_P_V_HI, EPH_P_V_LO, i);
        m.GL = get3dd(pl, n, EPH_P_GL_HI, EPH_P_GL_LO, i);
        m.s.x = get3dd(pl, n, EPH_P_S_HI, EPH_P_S_LO, i);
        m.s.y = get3dd(pl, n, EPH_P_S_HI + 3, EPH_P_S_LO + 3, i);
        m.s.z = get3dd(pl, n, EPH_P_S_HI + 6, EPH_P_S_LO + 6, i);
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
        m.GI = fast_mpmat(get3(pl, n, EPH_P_GI, i), get3(pl, n, EPH_P_GI + 3, i), get3(pl, n, EPH_P_GI + 6, i));
        m.C_potential = fast_mpmat(get3(pl, n, EPH_P_C_POTENTIAL, i), get3(pl, n, EPH_P_C_POTENTIAL + 3, i),
                                   get3(pl, n, EPH_P_C_POTENTIAL + 6, i));
        m.min_distance = pl[EPH_P_MIN_DISTANCE * n + i];
        m.max_influence = pl[EPH_P_MAX_INFLUENCE * n + i];
    }
}

void on_error(int rc) {
    if (rc == EPH_OK) return;
    LogCritical("\n\nCritical Error : [B200 RK12] status %d: %s\n    The program will now exit.\n", rc,
                g_ctx ? eph_last_error(g_ctx) : "no device context");
    exit(-1);
}

void run(htl::vector<mass> &ml, bool integrate, double dt, int64_t n_step, double t_hi, double t_lo) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ctx) on_error(eph_ctx_create(0, &g_ctx));
    Packed pk;
    pack(ml, pk);
    on_error(eph_upload_system(g_ctx, (int64_t)ml.size(), pk.planes.data(), &pk.models));
    on_error(integrate ? eph_rk12(g_ctx, dt, n_step, t_hi, t_lo) : eph_accel(g_ctx));
    on_error(eph_download_system(g_ctx, pk.planes.data()));
    unpack(pk.planes, ml);
}

}  // namespace

void msystem::Cuda_RungeKutta12(fast_real dt, int_t n_step) {
    if (n_step <= 0 || mlist.empty()) return;
    run(mlist, true, dt, n_step, t_eph.hi, t_eph.lo);
}

void msystem::Cuda_accel() {
    if (mlist.empty()) return;
    run(mlist, false, 0, 0, 0, 0);
}
