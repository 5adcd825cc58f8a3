// eph_msystem.cpp - host side of the drop-in: the reference's system loading, configuration and
// integrator entry points over the device path of eph_capi.cu.
//
//   eph_msystem_load       msystem::load(config)              src/modules/mass_loader.cpp:67-294,324-561
//                          geopotential::load                 src/physics/geopotential.cpp:8-127
//                          ring::load                         src/physics/ring.cpp:15-108
//   eph_msystem_integrate  msystem::integrate(dt, n, USE_GPU) src/physics/mass.cpp:399-442
//   eph_msystem_accel      msystem::accel(parallel_option)    src/physics/mass.cpp:216-221
//
// The loader reads the same text formats with the same sscanf patterns and builds the same derived
// fields; the load-time deformation and the initial acceleration run on the GPU (eph_deform,
// eph_accel). The barycentre analysis (msystem::analyse) and checkpoints are outside this path.
// There is no CPU integrator here: USE_GPU=0 / parallel_option<=0 return EPH_ERR_UNSUPPORTED.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/eph_b200.h"
#include "../../include/eph_msystem.h"

namespace {

// ---------------------------------------------------------------- constants (src/math/basic_math.h:9-31)
constexpr double kPi = 3.1415926535897932;
constexpr double kC = 299792458;
constexpr double kG = 6.67430E-11;
constexpr double kDegree = kPi / 180;
constexpr double kObliquity = 84381.448 / 3600 * kDegree;
constexpr double kEps = 0x1p-53;
constexpr size_t kMaxLine = 1024;   // src/configs.h:5
constexpr int kMaxGpDegree = EPH_GP_MAX_DEGREE;

int g_log_level = 30;   // messages below this level are dropped (INFO 20, WARNING 30, ERROR 40)

void log_msg(int level, const char *fmt, ...) {
    if (level < g_log_level) return;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
}

// ---------------------------------------------------------------- host double-double / vectors
struct dd { double hi, lo; };
dd dd_of(double h) { return dd{h, 0.0}; }
double dval(dd a) { return a.hi + a.lo; }
dd dd_add(dd x, dd y) {
    double s = x.hi + y.hi, t = s - x.hi;
    double e = (x.hi - (s - t)) + (y.hi - t);
    e = e + (x.lo + y.lo);
    double h = s + e;
    return dd{h, e - (h - s)};
}
struct v3 { double x, y, z; };
v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
v3 operator*(double s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
struct m3 { v3 x, y, z; };   // axis columns, as mat_t (src/math/vec_t.h:270-272)
m3 operator+(m3 a, m3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
m3 operator-(m3 a, m3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
m3 operator*(double s, m3 a) { return {s * a.x, s * a.y, s * a.z}; }
m3 add_diag(m3 a, double s) { a.x.x += s; a.y.y += s; a.z.z += s; return a; }
v3 mul(m3 a, v3 b) { return (b.x * a.x + b.y * a.y) + b.z * a.z; }
v3 tmul(v3 a, m3 b) { return {dot(a, b.x), dot(a, b.y), dot(a, b.z)}; }
m3 mul(m3 a, m3 b) { return {mul(a, b.x), mul(a, b.y), mul(a, b.z)}; }
m3 transpose(m3 m) { return {{m.x.x, m.y.x, m.z.x}, {m.x.y, m.y.y, m.z.y}, {m.x.z, m.y.z, m.z.z}}; }
m3 toworld(m3 s, m3 a) {
    m3 sa = mul(s, a);
    return {(s.x.x * sa.x + s.y.x * sa.y) + s.z.x * sa.z, (s.x.y * sa.x + s.y.y * sa.y) + s.z.y * sa.z,
            (s.x.z * sa.x + s.y.z * sa.y) + s.z.z * sa.z};
}
m3 tolocal(m3 s, m3 a) {
    m3 sTa{tmul(a.x, s), tmul(a.y, s), tmul(a.z, s)};
    return mul(sTa, s);
}
double det(m3 a) { return dot(cross(a.x, a.y), a.z); }
double normsqr(m3 a) { return dot(a.x, a.x) + dot(a.y, a.y) + dot(a.z, a.z); }
m3 from_harmonics(double j2, double c21, double c22, double s21, double s22) {   // vec_t.h:522-530
    m3 m;
    m.x.x = 3 * c22 + j2 / 2;
    m.y.x = m.x.y = 3 * s22;
    m.z.x = m.x.z = 3 * c21 / 2;
    m.y.y = -3 * c22 + j2 / 2;
    m.z.y = m.y.z = 3 * s21 / 2;
    m.z.z = -j2;
    return m;
}
void to_harmonics(const m3 &m, double &j2, double &c21, double &c22, double &s21, double &s22) {  // vec_t.h:531-537
    j2 = -m.z.z;
    c21 = (m.x.z + m.z.x) / 3;
    c22 = (m.x.x - m.y.y) / 6;
    s21 = (m.y.z + m.z.y) / 3;
    s22 = (m.x.y + m.y.x) / 6;
}
double hypot_normalize3(double &a, double &b, double &c) {   // hypot_t::normalize, vec_t.h:54-81
    const double high = 0x1p960, mulv = 0x1p768, divv = 0x1p-768, low = 0x1p-960;
    double x = a, y = b, z = c, r = x * x + y * y + z * z, back = 1;
    if (r < low) {
        x *= mulv; y *= mulv; z *= mulv;
        r = x * x + y * y + z * z;
        if (r == 0) { a = 0; b = 0; c = 1; return 0; }
        back = divv;
    } else if (!(r < high)) {
        x *= divv; y *= divv; z *= divv;
        r = x * x + y * y + z * z;
        back = mulv;
    }
    double s = std::sqrt(r), rs = 1 / s;
    a = x * rs; b = y * rs; c = z * rs;
    return back * s;
}
m3 rotation_matrix(v3 w, double t) {   // vec_t.h:540-559
    double x = w.x, y = w.y, z = w.z;
    double wt = hypot_normalize3(x, y, z) * t;
    double st = std::sin(wt), st222 = std::sin(wt / 2);
    st222 *= 2 * st222;
    m3 dr{{x * x - 1, x * y, x * z}, {x * y, y * y - 1, y * z}, {x * z, y * z, z * z - 1}};
    dr = st222 * dr;
    dr.x.y += z * st; dr.y.x -= z * st;
    dr.x.z -= y * st; dr.z.x += y * st;
    dr.y.z += x * st; dr.z.y -= x * st;
    return dr;
}
v3 from_theta_phi(double theta, double phi) {   // vec_t.h:112-115
    double c = std::sin(theta);
    return {c * std::cos(phi), c * std::sin(phi), std::cos(theta)};
}
void rotx(v3 &v, double b) {   // vec_t.h:129-134
    double s = std::sin(b), c = std::cos(b), ny = v.y * c - v.z * s;
    v.z = v.z * c + v.y * s;
    v.y = ny;
}

// ---------------------------------------------------------------- text input (MFILE::readline, memio.cpp:257-301)
struct LineReader {
    FILE *f = nullptr;
    explicit LineReader(const std::string &path) {
        std::string p = path;
        for (char &ch : p)
            if (ch == '\\') ch = '/';
        f = fopen(p.c_str(), "rb");
    }
    ~LineReader() { if (f) fclose(f); }
    // next non-empty line not starting with '#'; "\r" and "\n" both end a line; false at EOF
    bool next(std::string &out) {
        for (;;) {
            out.clear();
            int c;
            bool any = false;
            while ((c = fgetc(f)) != EOF) {
                any = true;
                if (c == '\r' || c == '\n') break;
                out.push_back((char)c);
            }
            if (!out.empty() && out[0] == '#') out.clear();
            if (!out.empty()) return true;
            if (c == EOF && !any) return false;
            if (c == EOF) return false;
        }
    }
};

std::string join(const std::string &dir, const std::string &name) { return dir + "/" + name; }

// ---------------------------------------------------------------- model files
struct Gp { int nz, nt; double coef[EPH_GP_TABLE_SIZE]; };
struct Ring { int n; double param[4]; double disk[EPH_RING_MAX_DISKS][3]; };

// geopotential::load(file, ref_radius_factor, N_start=3) (geopotential.cpp:8-127)
bool load_geopotential(const std::string &file, double rrf, Gp &gp) {
    const int N_start = 3;
    LineReader in(file);
    if (!in.f) { log_msg(40, "%s : Error opening harmonics model\n", file.c_str()); return false; }
    long long Nz = -1, Nt = 0;
    long long Nzmax = 0, Ntmax = 0;
    std::string line;
    bool ok = false;
    memset(gp.coef, 0, sizeof(gp.coef));
    while (in.next(line)) {
        if (Nz < 0) {
            if (2 != sscanf(line.c_str(), "%lld%lld", &Nz, &Nt)) {
                log_msg(40, "%s : Error reading max numbers of zonal/tesseral degrees\n", file.c_str());
                return false;
            }
            if (Nt < 0) Nt = 0;
            if (Nz < Nt) Nz = Nt;
            if (Nz > kMaxGpDegree) { Nz = kMaxGpDegree; if (Nt > kMaxGpDegree) Nt = kMaxGpDegree; }
            if (Nz < N_start) { log_msg(30, "%s : Geopotential degree too low. Ignored.\n", file.c_str()); return false; }
            ok = true;
            continue;
        }
        long long n = 0, m = 0;
        double Cnm = 0, Snm = 0;
        int nr = sscanf(line.c_str(), "%lld%lld%lf%lf", &n, &m, &Cnm, &Snm);
        if (nr < 3 || n < 2 || m < 0 || m > n || (nr == 3 && m != 0) || (m == 0 && Snm != 0)) {
            log_msg(40, "%s : %s : malformed geopotential line\n", file.c_str(), line.c_str());
            return false;
        }
        if (n < N_start) continue;
        if (n > Nz || (n > Nt && m > 0)) continue;
        double f = std::pow(rrf, (double)n);
        Cnm *= f;
        Snm *= f;
        const long long J = n * n - 4;
        if (m == 0) {
            gp.coef[J] += Cnm;
        } else {
            gp.coef[J + 2 * m - 1] += Cnm;
            gp.coef[J + 2 * m] += Snm;
            if (n > Ntmax) Ntmax = n;
        }
        if (n > Nzmax) Nzmax = n;
    }
    if (!ok) return false;
    if (!Nzmax) { log_msg(30, "%s : No valid geopotential terms. Ignored.\n", file.c_str()); return false; }
    if (Nzmax < Nz) Nz = Nzmax;
    if (Ntmax < Nt) Nt = Ntmax;
    gp.nz = (int)Nz;
    gp.nt = (int)Nt;
    return true;
}

// ring::load(file, ref_GM, ref_R, direction_mass_factor) (ring.cpp:15-108); returns -1 on error,
// 0 when the file holds no disk, 1 when loaded
int load_ring(const std::string &file, double ref_GM, double ref_R, double dmf, Ring &rg) {
    LineReader in(file);
    if (!in.f) { log_msg(40, "%s : Error opening ring model\n", file.c_str()); return -1; }
    struct Disk { double Gs, R, H; };
    std::vector<Disk> disks;
    auto adddisk = [&](double Gs, double R, double H) {
        for (auto &d : disks)
            if (d.R == R && d.H == H) { d.Gs += Gs; return; }
        disks.push_back({Gs, R, H});
    };
    std::string line;
    char rname[kMaxLine];
    while (in.next(line)) {
        if (line.size() >= kMaxLine) { log_msg(40, "%s : line too long\n", file.c_str()); return -1; }
        double rin, rout, thick, GM;
        if (5 != sscanf(line.c_str(), "%[^\t]%lf%lf%lf%lf", rname, &rin, &rout, &thick, &GM)) {
            log_msg(40, "%s : Line Length Error: %s\n", file.c_str(), line.c_str());
            return -1;
        }
        GM *= std::abs(dmf);
        rin *= 1000;
        rout *= 1000;
        thick *= 1000;
        double Gs = GM / (kPi * (rout - rin) * (rout + rin));
        adddisk(-Gs, rin, thick);
        adddisk(Gs, rout, thick);
    }
    if ((int)disks.size() > EPH_RING_MAX_DISKS) { log_msg(40, "%s : too many disks\n", file.c_str()); return -1; }
    rg.n = (int)disks.size();
    if (!rg.n) return 0;
    double GM_ratio = 0, A = 0, J2 = 0, GL_R2 = 0;
    double ref_R2 = ref_R * ref_R, ref_GMR2 = ref_GM * ref_R2;
    for (int i = 0; i < rg.n; ++i) {
        const Disk &d = disks[i];
        double R2 = d.R * d.R, H2 = d.H * d.H, GM = kPi * R2 * d.Gs;
        GM_ratio += GM;
        A += GM * (6 * R2 + H2) / (12 * ref_GMR2);
        J2 += GM * (3 * R2 - H2) / (12 * ref_GMR2);
        GL_R2 += 4 * GM * std::sqrt(ref_GM * d.R) / (5 * ref_GMR2);
        rg.disk[i][0] = d.Gs / ref_GM * ref_R2;
        rg.disk[i][1] = d.R / ref_R;
        rg.disk[i][2] = d.H / ref_R;
    }
    GM_ratio = 1 / (1 + ref_GM / GM_ratio);
    if (dmf < 0) GL_R2 *= -1;
    rg.param[0] = GM_ratio; rg.param[1] = A; rg.param[2] = J2; rg.param[3] = GL_R2;
    return 1;
}

// ---------------------------------------------------------------- body record used while loading
struct Body {
    uint64_t sid = 0;
    dd r[3], v[3], GL[3], s[9];
    v3 w{0, 0, 0};
    double GM = 0, exJ2 = 0, GM0 = 0, dGM = 0, dJ2 = 0, R = 0, inertia = 0, k2 = 0, k2r = 0, td = 0, tdf = 0;
    double lum = 0, recpt = 0, A = 0, R2 = 0, sR2 = 0, rR2G_4c = 0;
    m3 C_static{};
    int gp = -1, ring = -1;
};

m3 fast_s(const Body &b) {
    auto col = [&](int o) { return v3{dval(b.s[o]), dval(b.s[o + 1]), dval(b.s[o + 2])}; };
    return m3{col(0), col(3), col(6)};
}
void add_to_s(Body &b, const m3 &d) {
    const double *p = &d.x.x;
    for (int q = 0; q < 9; ++q) b.s[q] = dd_add(b.s[q], dd_of(p[q]));
}

// mass::sanity (mass_loader.cpp:18-65)
bool sanity(const Body &m, const std::string &name, bool has_gp, bool has_ring) {
    std::vector<const char *> errs;
    constexpr double eps2 = kEps * kEps, large = 1 / eps2;
    v3 r{dval(m.r[0]), dval(m.r[1]), dval(m.r[2])}, v{dval(m.v[0]), dval(m.v[1]), dval(m.v[2])};
    if (!(dot(r, r) < large * large) || !(dot(v, v) < kC * kC)) errs.push_back("position/velocity not finite");
    m3 f = fast_s(m);
    if (!(normsqr(add_diag((-1.0) * mul(transpose(f), f), 1.0)) < 64 * eps2) || !(det(f) > 0))
        errs.push_back("rotation not normalized");
    if (!(dot(m.w, m.w) * m.R2 < kC * kC)) errs.push_back("rotation too fast");
    if (!(eps2 < m.GM0 && m.GM0 < large)) errs.push_back("invalid gravititional parameter");
    if (!(2 * m.GM0 < kC * kC * std::abs(m.R))) errs.push_back("invalid radius");
    if (!(eps2 < m.inertia && m.inertia <= 1)) errs.push_back("invalid inertia factor");
    if (!(0 <= m.k2 && m.k2 <= 1.5 && 0 <= m.k2r && m.k2r <= 1.5)) errs.push_back("invalid tidal/rotational deformation factor");
    if (!(0 <= m.td && m.td < large && 0 <= m.tdf && m.tdf <= large)) errs.push_back("invalid tidal delay time/factor");
    double j2, c21, c22, s21, s22;
    to_harmonics(m.C_static, j2, c21, c22, s21, s22);
    if (!(0 <= j2 && j2 + 6 * std::abs(c22) < 3 * m.inertia && std::abs(c21) < m.inertia && std::abs(s21) < m.inertia &&
          std::abs(s22) * 2 < m.inertia))
        errs.push_back("invalid static harmonics");
    if (m.R < 0 && (m.k2 || m.k2r || j2 || m.dJ2 || c21 || c22 || s21 || s22 || has_gp || has_ring || m.td))
        errs.push_back("soft mass shall not have non-point components");
    for (const char *e : errs) log_msg(40, "Error when loading <%s>: %s\n", name.c_str(), e);
    return errs.empty();
}

}  // namespace

struct eph_msystem {
    eph_ctx *ctx = nullptr;
    int64_t n = 0;
    dd t_eph{0, 0};
    double delta_t = 300, data_cadence = 7200, max_ephm_length = 631152000, combined_delta_t = 28800;
    int integrator = 2;   // COMBINED_RK12 default (mass_loader.cpp:300)
    std::vector<uint64_t> sid;
    std::vector<std::string> names;
    std::vector<Gp> gps;
    std::vector<Ring> rings;
    std::vector<int32_t> gp_nz, gp_nt, ring_nd;
    std::vector<double> gp_coef, ring_param, ring_disk;
    eph_models models{};
    char err[256] = {0};
};

namespace {

void fill_models(eph_msystem *ms) {
    ms->gp_nz.clear(); ms->gp_nt.clear(); ms->gp_coef.clear();
    ms->ring_nd.clear(); ms->ring_param.clear(); ms->ring_disk.clear();
    for (const Gp &g : ms->gps) {
        ms->gp_nz.push_back(g.nz);
        ms->gp_nt.push_back(g.nt);
        ms->gp_coef.insert(ms->gp_coef.end(), g.coef, g.coef + EPH_GP_TABLE_SIZE);
    }
    for (const Ring &r : ms->rings) {
        ms->ring_nd.push_back(r.n);
        ms->ring_param.insert(ms->ring_param.end(), r.param, r.param + 4);
        for (int d = 0; d < EPH_RING_MAX_DISKS; ++d)
            for (int c = 0; c < 3; ++c) ms->ring_disk.push_back(d < r.n ? r.disk[d][c] : 0.0);
    }
    ms->models.n_gp = (int32_t)ms->gps.size();
    ms->models.gp_nz = ms->gp_nz.data();
    ms->models.gp_nt = ms->gp_nt.data();
    ms->models.gp_coef = ms->gp_coef.data();
    ms->models.n_ring = (int32_t)ms->rings.size();
    ms->models.ring_ndisk = ms->ring_nd.data();
    ms->models.ring_param = ms->ring_param.data();
    ms->models.ring_disk = ms->ring_disk.data();
}

void to_planes(const std::vector<Body> &bodies, std::vector<double> &pl) {
    const size_t n = bodies.size();
    pl.assign((size_t)EPH_NPLANES * n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        const Body &b = bodies[i];
        auto P = [&](int p) -> double & { return pl[(size_t)p * n + i]; };
        for (int c = 0; c < 3; ++c) {
            P(EPH_P_R_HI + c) = b.r[c].hi; P(EPH_P_R_LO + c) = b.r[c].lo;
            P(EPH_P_V_HI + c) = b.v[c].hi; P(EPH_P_V_LO + c) = b.v[c].lo;
            P(EPH_P_GL_HI + c) = b.GL[c].hi; P(EPH_P_GL_LO + c) = b.GL[c].lo;
        }
        for (int q = 0; q < 9; ++q) { P(EPH_P_S_HI + q) = b.s[q].hi; P(EPH_P_S_LO + q) = b.s[q].lo; }
        P(EPH_P_W) = b.w.x; P(EPH_P_W + 1) = b.w.y; P(EPH_P_W + 2) = b.w.z;
        P(EPH_P_GM) = b.GM; P(EPH_P_EXJ2) = b.exJ2; P(EPH_P_GM0) = b.GM0; P(EPH_P_DGM) = b.dGM;
        P(EPH_P_DJ2) = b.dJ2; P(EPH_P_RADIUS) = b.R; P(EPH_P_INERTIA) = b.inertia; P(EPH_P_K2) = b.k2;
        P(EPH_P_K2R) = b.k2r; P(EPH_P_TIDE_DELAY) = b.td; P(EPH_P_TIDE_DELAY_FACTOR) = b.tdf;
        P(EPH_P_LUM) = b.lum; P(EPH_P_RECPT) = b.recpt; P(EPH_P_A) = b.A; P(EPH_P_R2) = b.R2;
        P(EPH_P_SR2) = b.sR2; P(EPH_P_RR2G_4C) = b.rR2G_4c;
        const double *cs = &b.C_static.x.x;
        for (int q = 0; q < 9; ++q) P(EPH_P_C_STATIC + q) = cs[q];
        P(EPH_P_GP_INDEX) = b.gp;
        P(EPH_P_RING_INDEX) = b.ring;
    }
}

m3 get9(const std::vector<double> &pl, size_t n, int p, size_t i) {
    auto g = [&](int q) { return pl[(size_t)(p + q) * n + i]; };
    return m3{{g(0), g(1), g(2)}, {g(3), g(4), g(5)}, {g(6), g(7), g(8)}};
}
void put9(std::vector<double> &pl, size_t n, int p, size_t i, const m3 &m) {
    const double *s = &m.x.x;
    for (int q = 0; q < 9; ++q) pl[(size_t)(p + q) * n + i] = s[q];
}

int set_err(eph_msystem *ms, int code, const char *msg) {
    snprintf(ms->err, sizeof(ms->err), "%s", msg);
    return code;
}

// msystem::load(fbase, fext, gppath, ringpath) (mass_loader.cpp:324-561)
int load_bodies(eph_msystem *ms, const std::string &fbase, const std::string *fext, const std::string &gppath,
                const std::string &ringpath, std::vector<Body> &bodies) {
    LineReader in(fbase);
    if (!in.f) return set_err(ms, EPH_ERR_LOAD, ("File Not Exist: " + fbase).c_str());
    std::map<uint64_t, int> midx;
    std::string line;
    while (in.next(line)) {
        if (line.size() >= kMaxLine) return set_err(ms, EPH_ERR_LOAD, "Line Too Long in initial file");
        char sname[kMaxLine], ssid[kMaxLine];
        double GM, R, inertia, k2, k2r, td, j2, c21, c22, s21, s22, tdf, gprf, ringmf;
        double ra, dec, W, p;
        v3 r, v, x, z, w;
        int nf = sscanf(line.c_str(),
                        "%[^\t]%s%lf%lf"
                        "%lf%lf%lf%lf"
                        "%lf%lf%lf%lf%lf"
                        "%lf%lf%lf"
                        "%lf%lf%lf%lf%lf%lf"
                        "%lf%lf%lf%lf"
                        "%lf%lf%lf%lf%lf%lf%lf%lf%lf",
                        sname, ssid, &GM, &R, &inertia, &k2, &k2r, &td, &j2, &c21, &c22, &s21, &s22, &tdf, &gprf,
                        &ringmf, &r.x, &r.y, &r.z, &v.x, &v.y, &v.z, &ra, &dec, &W, &p, &x.x, &x.y, &x.z, &z.x,
                        &z.y, &z.z, &w.x, &w.y, &w.z);
        if (!(nf == 35 || nf == 26)) return set_err(ms, EPH_ERR_LOAD, ("Line Length Error: " + line).c_str());
        Body m;
        size_t sidlen = strlen(ssid);
        if (sidlen >= 8) return set_err(ms, EPH_ERR_LOAD, "sid Too Long");
        memcpy(&m.sid, ssid, sidlen);
        if (!midx.emplace(m.sid, (int)bodies.size()).second) return set_err(ms, EPH_ERR_LOAD, "Duplicate sid");
        m.GM = GM;
        m.R = R * 1000;
        m.inertia = inertia; m.k2 = k2; m.k2r = k2r; m.td = td; m.tdf = tdf;
        m.GM0 = m.GM;
        if (gprf != 0) {
            Gp g;
            if (!load_geopotential(join(gppath, std::string(ssid) + ".txt"), gprf, g))
                return set_err(ms, EPH_ERR_LOAD, "geopotential model failed to load");
            m.gp = (int)ms->gps.size();
            ms->gps.push_back(g);
        }
        if (ringmf != 0) {
            Ring rg;
            int rc = load_ring(join(ringpath, std::string(ssid) + ".txt"), m.GM, m.R, ringmf, rg);
            if (rc < 0) return set_err(ms, EPH_ERR_LOAD, "ring model failed to load");
            if (rc > 0) {
                m.ring = (int)ms->rings.size();
                ms->rings.push_back(rg);
            }
        }
        if (nf == 26) {   // rotation from IAU angles (mass_loader.cpp:441-451)
            z = from_theta_phi((90 - dec) * kDegree, ra * kDegree);
            x = from_theta_phi(90 * kDegree, (ra + 90) * kDegree);
            x = x + mul(rotation_matrix(z, W * kDegree), x);
            rotx(x, -kObliquity);
            rotx(z, -kObliquity);
            w = (2 * kPi / (p * 3600)) * z;
        }
        v3 y = cross(z, x);
        const double *ax[3] = {&x.x, &y.x, &z.x};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) m.s[3 * a + c] = dd_of(ax[a][c]);
        {   // mass::orthogonalize (mass.h:147-150)
            m3 f = fast_s(m);
            add_to_s(m, mul(0.5 * f, add_diag((-1.0) * mul(transpose(f), f), 1.0)));
        }
        const double *rv = &r.x, *vv = &v.x;
        for (int c = 0; c < 3; ++c) { m.r[c] = dd_of(rv[c]); m.v[c] = dd_of(vv[c]); }
        m.w = w;
        m.A = 3 * m.inertia / 2;
        m.R2 = m.R * m.R;
        m.sR2 = m.R < 0 ? m.R2 : 0;
        m.rR2G_4c = 0;
        m.C_static = from_harmonics(j2, c21, c22, s21, s22);
        m3 GI = ((-2.0) / 3 * m.R2) * add_diag(toworld(fast_s(m), m.C_static), -m.A);
        v3 GL = mul(GI, m.w);
        m.GL[0] = dd_of(GL.x); m.GL[1] = dd_of(GL.y); m.GL[2] = dd_of(GL.z);
        bodies.push_back(m);
        ms->names.push_back(sname);
    }
    if (fext) {   // Extra file (mass_loader.cpp:475-538)
        LineReader ex(*fext);
        if (!ex.f) return set_err(ms, EPH_ERR_LOAD, ("File Not Exist: " + *fext).c_str());
        while (ex.next(line)) {
            if (line.size() >= kMaxLine) return set_err(ms, EPH_ERR_LOAD, "Line Too Long in extra file");
            char ssid[kMaxLine], sname[kMaxLine];
            double param;
            if (3 != sscanf(line.c_str(), "%s%s%lf", ssid, sname, &param))
                return set_err(ms, EPH_ERR_LOAD, ("Line Length Error: " + line).c_str());
            uint64_t key = 0;
            size_t len = strlen(ssid);
            memcpy(&key, ssid, len < 8 ? len : 8);
            auto it = len < 8 ? midx.find(key) : midx.end();
            if (it == midx.end()) { log_msg(30, "Ignoring %s of non-existing sid %s\n", sname, ssid); continue; }
            Body &m = bodies[it->second];
            if (!strcmp(sname, "MassRate")) m.dGM = param;
            else if (!strcmp(sname, "Luminosity")) m.lum = param;
            else if (!strcmp(sname, "Receptance")) { m.recpt = param; m.rR2G_4c = m.recpt * m.R2 * (kG / (4 * kC)); }
            else if (!strcmp(sname, "J2Rate")) m.dJ2 = param;
            else return set_err(ms, EPH_ERR_LOAD, (std::string("Unknown Parameter: ") + sname).c_str());
        }
    }
    return EPH_OK;
}

bool parse_double(const std::string &s, double &out) {
    if (s.empty()) return false;
    out = atof(s.c_str());
    return true;
}

}  // namespace

extern "C" {

void eph_set_log_level(int level) { g_log_level = level; }

int eph_msystem_load(const char *fconfig, int device, eph_msystem **out) {
    if (!fconfig || !out) return EPH_ERR_ARG;
    *out = nullptr;
    eph_msystem *ms = new eph_msystem();
    auto bail = [&](int code) {
        if (ms->err[0]) log_msg(40, "eph_msystem_load: %s\n", ms->err);
        if (ms->ctx) eph_ctx_destroy(ms->ctx);
        delete ms;
        return code;
    };
    // config file (mass_loader.cpp:67-160)
    std::string sip = fconfig;
    size_t spos = 1 + sip.find_last_of("/\\");
    std::string dir = spos ? sip.substr(0, spos - 1) : ".";
    std::string fname = sip.substr(spos);
    if (fname.empty()) return bail(EPH_ERR_ARG);
    static const char *keys[] = {"Initial", "Extra", "Geopotentials", "Rings", "TDB", "Integrator", "Delta_t",
                                 "Cadence", "Max_Ephemeris_Length", "Combined_Delta_t_Max", "Combined_GM_Max_Parent",
                                 "Combined_GM_Max_Child", "Combined_GM_Max_Tiny", "Combined_Period_Max_Child"};
    std::map<std::string, std::string> cfg;
    for (const char *k : keys) cfg[k] = "";
    {
        LineReader in(join(dir, fname));
        if (!in.f) { set_err(ms, EPH_ERR_LOAD, "config file not found"); return bail(EPH_ERR_LOAD); }
        std::string line;
        while (in.next(line)) {
            if (line.size() >= kMaxLine) { set_err(ms, EPH_ERR_LOAD, "Line Too Long in config"); return bail(EPH_ERR_LOAD); }
            char k[kMaxLine], v[kMaxLine];
            if (2 != sscanf(line.c_str(), "%s%s", k, v)) { set_err(ms, EPH_ERR_LOAD, "config line length error"); return bail(EPH_ERR_LOAD); }
            auto it = cfg.find(k);
            if (it == cfg.end()) { set_err(ms, EPH_ERR_LOAD, "Unknown config parameter"); return bail(EPH_ERR_LOAD); }
            if (!it->second.empty()) { set_err(ms, EPH_ERR_LOAD, "Duplicate config parameter"); return bail(EPH_ERR_LOAD); }
            it->second = v;
        }
    }
    if (cfg["Initial"].empty()) { set_err(ms, EPH_ERR_LOAD, "Missing Parameter: Initial"); return bail(EPH_ERR_LOAD); }
    std::string fext = cfg["Extra"].empty() ? "" : join(dir, cfg["Extra"]);
    std::string gppath = cfg["Geopotentials"].empty() ? "." : join(dir, cfg["Geopotentials"]);
    std::string ringpath = cfg["Rings"].empty() ? "." : join(dir, cfg["Rings"]);
    if (cfg["Geopotentials"].empty()) gppath = ".";
    if (cfg["Rings"].empty()) ringpath = ".";

    std::vector<Body> bodies;
    int rc = load_bodies(ms, join(dir, cfg["Initial"]), fext.empty() ? nullptr : &fext, gppath, ringpath, bodies);
    if (rc) return bail(rc);
    if (bodies.empty()) { set_err(ms, EPH_ERR_LOAD, "no bodies"); return bail(EPH_ERR_LOAD); }
    ms->n = (int64_t)bodies.size();
    for (const Body &b : bodies) ms->sid.push_back(b.sid);
    fill_models(ms);

    // load-time deformation on the device (mass_loader.cpp:540-551)
    rc = eph_ctx_create(device, &ms->ctx);
    if (rc) { set_err(ms, rc, "eph_ctx_create failed"); return bail(rc); }
    std::vector<double> pl;
    to_planes(bodies, pl);
    const size_t n = bodies.size();
    if ((rc = eph_upload_system(ms->ctx, ms->n, pl.data(), &ms->models)) ||
        (rc = eph_deform(ms->ctx)) || (rc = eph_download_system(ms->ctx, pl.data()))) {
        set_err(ms, rc, eph_last_error(ms->ctx));
        return bail(rc);
    }
    bool failed = false;
    for (size_t i = 0; i < n; ++i) {
        m3 f = fast_s(bodies[i]);
        m3 Cst = get9(pl, n, EPH_P_C_STATIC, i);
        m3 Cpot = get9(pl, n, EPH_P_C_POTENTIAL, i);
        m3 ncp = toworld(f, Cst);
        Cst = Cst - (tolocal(f, Cpot) - Cst);
        put9(pl, n, EPH_P_C_STATIC, i, Cst);
        put9(pl, n, EPH_P_C_POTENTIAL, i, ncp);
        bodies[i].C_static = Cst;
        if (!sanity(bodies[i], ms->names[i], bodies[i].gp >= 0, bodies[i].ring >= 0)) failed = true;
    }
    if (failed) { set_err(ms, EPH_ERR_LOAD, "sanity check failed"); return bail(EPH_ERR_LOAD); }
    // initial acceleration (mass_loader.cpp:555)
    if ((rc = eph_upload_system(ms->ctx, ms->n, pl.data(), &ms->models)) || (rc = eph_accel(ms->ctx))) {
        set_err(ms, rc, eph_last_error(ms->ctx));
        return bail(rc);
    }
    // integrator and numeric keys (mass_loader.cpp:185-245)
    const std::string &integ = cfg["Integrator"];
    if (!integ.empty()) {
        if (integ == "CPU_RK12") ms->integrator = 0;
        else if (integ == "GPU_RK12") ms->integrator = 1;
        else if (integ == "COMBINED_RK12") ms->integrator = 2;
        else { set_err(ms, EPH_ERR_LOAD, "Invalid Integrator"); return bail(EPH_ERR_LOAD); }
    }
    double tdb = 0;
    if (parse_double(cfg["TDB"], tdb)) ms->t_eph = dd_of(tdb);
    parse_double(cfg["Delta_t"], ms->delta_t);
    parse_double(cfg["Cadence"], ms->data_cadence);
    parse_double(cfg["Max_Ephemeris_Length"], ms->max_ephm_length);
    if (ms->integrator == 2) parse_double(cfg["Combined_Delta_t_Max"], ms->combined_delta_t);
    if ((double)(long long)ms->t_eph.hi != ms->t_eph.hi || ms->t_eph.lo != 0) {
        set_err(ms, EPH_ERR_LOAD, "TDB should be an integer");
        return bail(EPH_ERR_LOAD);
    }
    // time-variable parameters referred to t_eph = 0 (mass_loader.cpp:233-239)
    if ((rc = eph_download_system(ms->ctx, pl.data()))) { set_err(ms, rc, eph_last_error(ms->ctx)); return bail(rc); }
    for (size_t i = 0; i < n; ++i) {
        auto P = [&](int p) -> double & { return pl[(size_t)p * n + i]; };
        P(EPH_P_GM0) = P(EPH_P_GM) - P(EPH_P_DGM) * ms->t_eph.hi;
        P(EPH_P_EXJ2) = P(EPH_P_DJ2) * ms->t_eph.hi;
        P(EPH_P_C_STATIC + 0) -= P(EPH_P_EXJ2) / 2;
        P(EPH_P_C_STATIC + 4) -= P(EPH_P_EXJ2) / 2;
        P(EPH_P_C_STATIC + 8) += P(EPH_P_EXJ2);
    }
    auto ok_dt = [](double d) { return d > 0 && d != INFINITY; };
    if (!ok_dt(ms->delta_t) || !ok_dt(ms->data_cadence) || !ok_dt(ms->max_ephm_length) || !ok_dt(ms->combined_delta_t)) {
        set_err(ms, EPH_ERR_LOAD, "Delta_t/Cadence/Max_Ephemeris_Length/Combined_Delta_t_Max must be finite and positive");
        return bail(EPH_ERR_LOAD);
    }
    if ((rc = eph_upload_system(ms->ctx, ms->n, pl.data(), &ms->models))) { set_err(ms, rc, eph_last_error(ms->ctx)); return bail(rc); }
    *out = ms;
    return EPH_OK;
}

int eph_msystem_free(eph_msystem *ms) {
    if (!ms) return EPH_ERR_ARG;
    if (ms->ctx) eph_ctx_destroy(ms->ctx);
    delete ms;
    return EPH_OK;
}

int64_t eph_msystem_size(const eph_msystem *ms) { return ms ? ms->n : -1; }
eph_ctx *eph_msystem_ctx(eph_msystem *ms) { return ms ? ms->ctx : nullptr; }
const char *eph_msystem_error(const eph_msystem *ms) { return ms ? ms->err : "null system"; }

int eph_msystem_t_eph(const eph_msystem *ms, double *hi, double *lo) {
    if (!ms || !hi || !lo) return EPH_ERR_ARG;
    *hi = ms->t_eph.hi;
    *lo = ms->t_eph.lo;
    return EPH_OK;
}
double eph_msystem_delta_t(const eph_msystem *ms) { return ms ? ms->delta_t : 0; }
int eph_msystem_integrator(const eph_msystem *ms) { return ms ? ms->integrator : -1; }

int eph_msystem_models(const eph_msystem *ms, eph_models *out) {
    if (!ms || !out) return EPH_ERR_ARG;
    *out = ms->models;
    return EPH_OK;
}
int eph_msystem_sids(const eph_msystem *ms, uint64_t *out) {
    if (!ms || !out) return EPH_ERR_ARG;
    for (size_t i = 0; i < ms->sid.size(); ++i) out[i] = ms->sid[i];
    return EPH_OK;
}

int eph_msystem_get_planes(eph_msystem *ms, double *planes) {
    if (!ms || !planes) return EPH_ERR_ARG;
    return eph_download_system(ms->ctx, planes);
}
int eph_msystem_set_planes(eph_msystem *ms, const double *planes) {
    if (!ms || !planes) return EPH_ERR_ARG;
    return eph_upload_system(ms->ctx, ms->n, planes, &ms->models);
}

// msystem::integrate(dt, n_step, USE_GPU) (mass.cpp:399-442)
int eph_msystem_integrate(eph_msystem *ms, double dt, int64_t n_step, int use_gpu) {
    if (!ms) return EPH_ERR_ARG;
    if (!use_gpu) return set_err(ms, EPH_ERR_UNSUPPORTED, "the CPU integrator is not part of this library");
    if (n_step == 0) return EPH_OK;
    double hi = ms->t_eph.hi, lo = ms->t_eph.lo;
    int rc = eph_integrate(ms->ctx, dt, n_step, &hi, &lo);
    if (rc) return set_err(ms, rc, eph_last_error(ms->ctx));
    if (g_log_level <= 40) {   // collision and step-size checks (mass.cpp:411-439)
        std::vector<double> pl((size_t)EPH_NPLANES * ms->n);
        if (!eph_download_system(ms->ctx, pl.data())) {
            const double adt = std::abs(dt), dt2 = adt * adt;
            for (int64_t i = 0; i < ms->n; ++i) {
                const double mind = pl[(size_t)EPH_P_MIN_DISTANCE * ms->n + i];
                const double maxi = pl[(size_t)EPH_P_MAX_INFLUENCE * ms->n + i];
                const double R = pl[(size_t)EPH_P_RADIUS * ms->n + i];
                if (R > mind)
                    log_msg(40, "Catastrophy: at ephemeris time %lld s, another body entered the radius of <%s>: %.16e m < %.16e m\n",
                            (long long)(ms->t_eph.hi + ms->t_eph.lo), ms->names[i].c_str(), mind, R);
                if (maxi * dt2 > 0.01)
                    log_msg(30, "Warning: at ephemeris time %lld s, time step too large for <%s>: %.16e s > %.16e s\n",
                            (long long)(ms->t_eph.hi + ms->t_eph.lo), ms->names[i].c_str(), adt, std::sqrt(0.01 / maxi));
            }
        }
    }
    ms->t_eph = dd{hi, lo};
    return EPH_OK;
}

// msystem::accel(parallel_option) (mass.cpp:216-221): only the device branch exists here
int eph_msystem_accel(eph_msystem *ms, int parallel_option) {
    if (!ms) return EPH_ERR_ARG;
    if (parallel_option <= 0) return set_err(ms, EPH_ERR_UNSUPPORTED, "the CPU accel() is not part of this library");
    int rc = eph_accel(ms->ctx);
    if (rc) return set_err(ms, rc, eph_last_error(ms->ctx));
    return EPH_OK;
}

}  // extern "C"
