// eph_models.cuh - device evaluation of the extended-body force models.
//
//   gp_field : spherical-harmonic field of degree 2..8 (zonal up to Nz, tesseral up to Nt) in the
//              body frame, per unit GM of the extended body: what geopotential::sum computes
//              (src/physics/geopotential.impl:26-106), by Cunningham's Cartesian recursion instead of
//              the reference's spherical-coordinate Legendre recursion (method below).
//   ring_sum : field of a cylindrical annulus built from signed uniform disks, per unit GM of the
//              host, in the ring frame. Same Pade series, angle formula and fp32 bicubic correction
//              table as ring::sum (src/physics/ring.impl:2070-2195).
#pragma once
#include "eph_math.cuh"
#include "../../include/eph_planes.h"
#include "../../include/eph_ring_table.h"

namespace eph {

// 1/k for the degree recursion (k = 1 .. EPH_GP_MAX_DEGREE + 1); index 0 unused. Global memory, not
// constant memory: the lanes of one evaluation group read different entries. The step kernel keeps a copy
// in shared memory next to its copies of the coefficient tables (the recursion's loads sit on its chain).
__device__ const double GP_RCP[EPH_GP_MAX_DEGREE + 2] = {
    0.0, 1.0, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9};

// Gradient of the spherical-harmonic potential of an extended body, per unit GM of the body, at the
// body-frame position r = (x, y, z):
//   U / GM = 1/r sum_{n>=2} (R/r)^n [ -J_n P_n(sin lat) + sum_{m=1..n} P_nm(sin lat) (C_nm cos m lon + S_nm sin m lon) ],
// with unnormalised associated Legendre functions without the Condon-Shortley phase (the convention of the
// model files the loader reads; the coefficient of (n, m) sits at n^2-4 (J_n), n^2-4+2m-1 (C_nm),
// n^2-4+2m (S_nm), geopotential.impl:21-24). Degrees 2..Nz are zonal, tesseral orders only for n <= Nt.
//
// Method: Cunningham's Cartesian recursion of the solid harmonics
//   V_km + i W_km = (R/r)^(k+1) P_km(sin lat) e^(i m lon)
// (Cunningham 1970; Montenbruck & Gill, Satellite Orbits, 2000, sec. 3.2.4-3.2.5), whose gradient terms
// are again solid harmonics of one degree higher:
//   a_x = 1/R^2 sum [ m=0: -C_n0 V_{n+1,1};  m>0: ( -C V_{n+1,m+1} - S W_{n+1,m+1}
//                     + (n-m+2)(n-m+1) (C V_{n+1,m-1} + S W_{n+1,m-1}) ) / 2 ]
//   a_y = 1/R^2 sum [ m=0: -C_n0 W_{n+1,1};  m>0: ( -C W_{n+1,m+1} + S V_{n+1,m+1}
//                     + (n-m+2)(n-m+1) (-C W_{n+1,m-1} + S V_{n+1,m-1}) ) / 2 ]
//   a_z = 1/R^2 sum (n-m+1) ( -C V_{n+1,m} - S W_{n+1,m} ).
// No angle, square root of rho or division by cos(lat) is needed, so the poles are regular points. The
// table of V, W is never stored: column m (orders) is walked upwards in degree k with the three-term
// recursion, starting from the diagonal V_mm, W_mm, and every value is consumed at once by the (up to)
// three gradient terms that read it: a_z of (k-1, m), a_x / a_y of (k-1, m-1) and of (k-1, m+1). Column 0
// and 1 run to degree Nz + 1 (zonal terms), higher columns to Nt + 1; with kZonal only columns 0 and 1
// run. T is double (plain FP64) or float (mixed precision; the caller scales far fields into range).
// Column m of the recursion, from its diagonal value (vd, wd) = (V_mm, W_mm), adding every gradient term
// that reads a value of the column to (ax, ay, az) (unscaled by 1/R^2).
template <typename T, bool kZonal>
__device__ __forceinline__ void gp_column(const double *__restrict__ tab, const double *__restrict__ rcp, int Nz,
                                          int Nt, int m, T zs, T rho2, T vd, T wd, T &ax, T &ay, T &az) {
    const int klast = m <= 1 ? Nz + 1 : Nt + 1;
    T v = vd, w = wd, vp = 0, wp = 0;   // (V, W) at degree k and k - 1 of column m
#pragma unroll 1
    for (int k = m; k <= klast; ++k) {
        if (k > m) {   // (k - m) V_km = (2k-1) z R/r^2 V_{k-1,m} - (k+m-1) (R/r)^2 V_{k-2,m}
            const T a = T(2 * k - 1) * zs, b = T(k + m - 1) * rho2, c = T(rcp[k - m]);
            const T nv = (a * v - b * vp) * c, nw = (a * w - b * wp) * c;
            vp = v; wp = w; v = nv; w = nw;
        }
        const int n = k - 1;   // degree of the coefficients that read (V, W)_km
        if (n < 2) continue;
        const double *cn = tab + (n * n - 4);
        if (m == 0) {
            if (n <= Nz) az += T(n + 1) * (T(cn[0]) * v);                 // -C_n0 = J_n, W_k0 = 0
        } else if (!kZonal && m <= n && n <= Nt) {
            az -= T(n - m + 1) * (T(cn[2 * m - 1]) * v + T(cn[2 * m]) * w);
        }
        if (m == 1) {
            if (n <= Nz) {
                const T J = T(cn[0]);
                ax += J * v;
                ay += J * w;
            }
        } else if (!kZonal && m >= 2 && n <= Nt) {                            // order m - 1 >= 1
            const T C = T(cn[2 * m - 3]), S = T(cn[2 * m - 2]);
            ax -= T(0.5) * (C * v + S * w);
            ay += T(0.5) * (S * v - C * w);
        }
        if (!kZonal && m + 1 <= n && n <= Nt) {                               // order m + 1
            const T C = T(cn[2 * m + 1]), S = T(cn[2 * m + 2]);
            const T f = T(0.5) * T((k - m) * (k - m - 1));
            ax += f * (C * v + S * w);
            ay += f * (S * v - C * w);
        }
    }
}

// Common set-up of a field evaluation: (x, y, z) R / r^2, (R / r)^2 and V_00 = R / r.
template <typename T>
__device__ __forceinline__ void gp_setup(T R, T x, T y, T z, T &xs, T &ys, T &zs, T &rho2, T &v00) {
    const T ir2 = T(1) / (x * x + y * y + z * z);
    const T q = R * ir2;
    xs = x * q; ys = y * q; zs = z * q; rho2 = R * q;
    v00 = R * sqrt(ir2);
}

template <typename T, bool kZonal>
__device__ __forceinline__ void gp_core(const double *__restrict__ tab, const double *__restrict__ rcp, int Nz, int Nt,
                                        T R, T x, T y, T z, T &ax, T &ay, T &az) {
    ax = 0; ay = 0; az = 0;
    T xs, ys, zs, rho2, vd, wd = 0;
    gp_setup(R, x, y, z, xs, ys, zs, rho2, vd);
    const int mlast = kZonal ? 1 : max(Nt + 1, 1);
#pragma unroll 1
    for (int m = 0; m <= mlast; ++m) {
        if (m > 0) {   // diagonal step: V_mm + i W_mm = (2m-1) (x + i y) R/r^2 (V + i W)_{m-1,m-1}
            const T f = T(2 * m - 1);
            const T nv = f * (xs * vd - ys * wd), nw = f * (xs * wd + ys * vd);
            vd = nv;
            wd = nw;
        }
        gp_column<T, kZonal>(tab, rcp, Nz, Nt, m, zs, rho2, vd, wd, ax, ay, az);
    }
    const T s = T(1) / (R * R);
    ax *= s; ay *= s; az *= s;
}

// Expanded coefficient table of one model for the lane-parallel evaluation: X[n][m] = (C_nm, S_nm) for
// n < kGpXN, m < kGpXM, with C_n0 = -J_n, S_n0 = 0, and zero wherever the model has no term (n < 2, n > Nz,
// m > n, and m > 0 with n > Nt). With the zeros in the table every lane runs the same instructions.
constexpr int kGpXN = EPH_GP_MAX_DEGREE + 1, kGpXM = EPH_GP_MAX_DEGREE + 3;
constexpr int kGpX = kGpXN * kGpXM * 2;
__device__ __forceinline__ void gp_expand(const double *__restrict__ tab, int Nz, int Nt, double *X, int t, int nt) {
    for (int q = t; q < kGpX; q += nt) {
        const int n = q / (kGpXM * 2), m = (q / 2) % kGpXM, sn = q & 1;
        double v = 0;
        if (n >= 2 && n <= Nz && m <= n) {
            if (m == 0) v = sn ? 0.0 : -tab[n * n - 4];
            else if (n <= Nt) v = tab[n * n - 4 + 2 * m - 1 + sn];
        }
        X[q] = v;
    }
}

// The field from an expanded table, spread over a group of G consecutive lanes (G a power of two <= 32,
// `mask` the group's lanes, q = lane index in the group): lane q walks columns q, q + G, ..., and the group
// adds the lanes' sums with a butterfly. Each lane runs its diagonal recursion and its column in one loop
// over the degree k = 0 .. Nz + 1 with selects instead of branches (the value of column m is zero below
// degree m), adding for every value V_km, W_km the three gradient terms that read it:
//   a_z -= (k-m) (C_{k-1,m} V + S_{k-1,m} W)
//   a_x -= w_B (C_{k-1,m-1} V + S_{k-1,m-1} W),  a_y += w_B (S_{k-1,m-1} V - C_{k-1,m-1} W),  w_B = 1 (m = 1), 1/2 (m > 1)
//   a_x += w_C (C_{k-1,m+1} V + S_{k-1,m+1} W),  a_y += w_C (S_{k-1,m+1} V - C_{k-1,m+1} W),  w_C = (k-m)(k-m-1)/2
// so the group finishes in about the time of one column instead of all of them in turn. Every lane of the
// group returns the field.
template <int G>
__device__ __forceinline__ v3 gp_field_lanes(const double *X, const double *rcp, int Nz, int Nt, double R, v3 r, int q,
                                             unsigned mask) {
    double ax = 0, ay = 0, az = 0;
    if (Nz >= 2) {
        double xs, ys, zs, rho2, v00;
        gp_setup(R, r.x, r.y, r.z, xs, ys, zs, rho2, v00);
        const int mlast = max(Nt + 1, 1), K = Nz + 1;
        #pragma unroll 1
        for (int m = q; m <= mlast; m += G) {
            const double md = (double)m;
            const double wB = m == 0 ? 0.0 : (m == 1 ? 1.0 : 0.5);
            const double *XA = X + m * 2, *XB = X + (m == 0 ? 0 : m - 1) * 2, *XC = X + (m + 1) * 2;
            double dv = v00, dw = 0;                 // diagonal V_kk, W_kk while k <= m
            double v = 0, w = 0, vp = 0, wp = 0;     // column m at degrees k and k - 1
            #pragma unroll 1
            for (int k = 0; k <= K; ++k) {
                const double kd = (double)k;
                const double f = 2 * kd - 1;
                const double ndv = f * (xs * dv - ys * dw), ndw = f * (xs * dw + ys * dv);
                dv = (k >= 1 && k <= m) ? ndv : dv;
                dw = (k >= 1 && k <= m) ? ndw : dw;
                const double c = rcp[k > m ? k - m : 1];
                const double a = f * zs, b = (kd + md - 1) * rho2;
                double nv = (a * v - b * vp) * c, nw = (a * w - b * wp) * c;
                nv = k == m ? dv : (k < m ? 0.0 : nv);
                nw = k == m ? dw : (k < m ? 0.0 : nw);
                vp = v; wp = w; v = nv; w = nw;
                if (k >= 1) {
                    const int row = (k - 1) * kGpXM * 2;
                    const double CA = XA[row], SA = XA[row + 1], CB = XB[row], SB = XB[row + 1];
                    const double CC = XC[row], SC = XC[row + 1];
                    const double wA = kd - md, wC = 0.5 * (kd - md) * (kd - md - 1);
                    az -= wA * (CA * v + SA * w);
                    ax += wC * (CC * v + SC * w) - wB * (CB * v + SB * w);
                    ay += wC * (SC * v - CC * w) + wB * (SB * v - CB * w);
                }
            }
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(mask, ax, o);
        ay += __shfl_xor_sync(mask, ay, o);
        az += __shfl_xor_sync(mask, az, o);
    }
    const double s = 1.0 / (R * R);
    return mk(ax * s, ay * s, az * s);
}

// The field from an expanded table on one lane, column by column (a loop over the order m), the degree
// steps of a column unrolled up to K: for every model with Nz + 1 <= K and Nt + 1 <= M (the table's zeros
// cover the terms beyond it). The recursion and gradient terms of gp_field_lanes, but a column starts at
// its diagonal value (no steps below degree m) and the terms of zero weight are skipped; every branch is
// the same on all lanes, so the lanes (one model evaluation each) never diverge.
template <int K, int M>
__device__ __forceinline__ v3 gp_field_columns(const double *X, const double *rcp, double R, v3 r) {
    double xs, ys, zs, rho2, v00;
    gp_setup(R, r.x, r.y, r.z, xs, ys, zs, rho2, v00);
    double ax = 0, ay = 0, az = 0;
    double dv = v00, dw = 0;   // diagonal V_mm, W_mm
    #pragma unroll 1
    for (int m = 0; m <= M; ++m) {
        if (m >= 1) {
            const double f = 2 * m - 1;
            const double ndv = f * (xs * dv - ys * dw), ndw = f * (xs * dw + ys * dv);
            dv = ndv;
            dw = ndw;
        }
        const double md = (double)m, wB = m == 1 ? 1.0 : 0.5;
        const double *XA = X + 2 * m, *XB = X + 2 * (m >= 1 ? m - 1 : 0), *XC = X + 2 * (m + 1);
        double v = dv, w = dw, vp = 0, wp = 0;   // column m at degrees k and k - 1
#pragma unroll
        for (int k = 1; k <= K; ++k) {
            if (k < m) continue;
            if (k > m) {
                const double a = (2 * k - 1) * zs, b = ((k - 1) + md) * rho2, c = rcp[k - m];
                const double nv = (a * v - b * vp) * c, nw = (a * w - b * wp) * c;
                vp = v; wp = w; v = nv; w = nw;
                const double wA = k - md;
                az -= wA * (XA[(k - 1) * kGpXM * 2] * v + XA[(k - 1) * kGpXM * 2 + 1] * w);
            }
            const int row = (k - 1) * kGpXM * 2;
            if (m >= 1) {
                const double CB = XB[row], SB = XB[row + 1];
                ax -= wB * (CB * v + SB * w);
                ay += wB * (SB * v - CB * w);
            }
            if (k >= m + 2) {
                const double km = k - md, wC = 0.5 * km * (km - 1);
                const double CC = XC[row], SC = XC[row + 1];
                ax += wC * (CC * v + SC * w);
                ay += wC * (SC * v - CC * w);
            }
        }
    }
    const double s = 1.0 / (R * R);
    return mk(ax * s, ay * s, az * s);
}
constexpr int kGpColK = 7, kGpColM = 5;   // models up to degree 6 and tesseral order 4
__device__ __forceinline__ bool gp_fits_columns(int Nz, int Nt) { return Nz >= 2 && Nz + 1 <= kGpColK && Nt + 1 <= kGpColM; }

// FP64 field of a geopotential model (any Nz, Nt), out of line: it sits on a cold path of the step kernel.
static __device__ __noinline__ v3 gp_field(const double *__restrict__ tab, int Nz, int Nt, double R, v3 r) {
    v3 a = mk(0, 0, 0);
    if (Nz >= 2) gp_core<double, false>(tab, GP_RCP, Nz, Nt, R, r.x, r.y, r.z, a.x, a.y, a.z);
    return a;
}

__device__ __forceinline__ float ring_fzcorr(float x, float y, int kh) {
    const int N = 32;
    x *= (float)N;
    y *= (float)N;
    int i = (int)floorf(x), j = (int)floorf(y);
    j -= kh * N;
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i >= N) i = N - 1;
    if (j >= N) j = N - 1;
    j += kh * N;
    x = __fsub_rn(x, (float)i);
    y = __fsub_rn(y, (float)j);
    const float *p = reinterpret_cast<const float *>(EPH_RING_TABLE_BITS) + 16 * (2 * N * i + j);
    float c[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) c[q] = __ldg(p + q);
    // evaluated without contraction, in the reference's association order
    auto h = [&](int a) {   // c[a] + x*(c[a+4] + x*(c[a+8] + x*c[a+12]))
        return __fadd_rn(c[a], __fmul_rn(x, __fadd_rn(c[a + 4], __fmul_rn(x, __fadd_rn(c[a + 8], __fmul_rn(x, c[a + 12]))))));
    };
    float h3 = h(3), h2 = h(2), h1 = h(1), h0 = h(0);
    return __fadd_rn(h0, __fmul_rn(y, __fadd_rn(h1, __fmul_rn(y, __fadd_rn(h2, __fmul_rn(y, h3))))));
}

template <int NC>
__device__ __forceinline__ double padesum(double x, const double (&coef)[NC][2]) {
    double resn = 0, resd = 0;
#pragma unroll
    for (int n = NC - 1; n >= 0; --n) {
        resn = x * resn + coef[n][0];
        resd = x * resd + coef[n][1];
    }
    return resn / resd;
}

// Pade coefficients of the disk field (src/physics/ring.impl:2101-2107)
__device__ __constant__ const double RING_XSERKK[5][2] = {{-4228.1846570321674587, 6387.9414439779279738}, {-13276.372802884782407, 16984.953742612298093}, {-11316.549465243054011, 8997.7319379726254196}, {-3242.2867356286923985, 403.15182320396046619}, {-704.60633921130372399, -5.7789477668119521439}};
__device__ __constant__ const double RING_XSERKM[5][2] = {{-2530.8255093002657219, 7950.8733392382639504}, {-5471.7803365810451727, 17189.101860053144376}, {-1624.0389725420726306, 7100.5562444641275465}, {1164.6058458813108946, 532.54915854738706820}, {270.03897254207263065, -5.0806023029229406554}};
__device__ __constant__ const double RING_XSER0[6][2] = {{3216.9908772759482762, 32768.000000000000000}, {-6727.1375380948220662, -93098.060290997395032}, {4534.8257724052420971, 96814.901233532309690}, {-1004.5251977686921953, -43973.540867249017404}, {17.915064837735955511, 7754.0323173314244943}, {-0.039157108395559676838, -224.00490789882410101}};
__device__ __constant__ const double RING_KSERKK[5][2] = {{-2373.3522804139070577, 1124.9866194216978637}, {-8300.7524798211745830, 17215.217000406477760}, {15279.068333441193395, 26590.060415743810476}, {-4354.4701057632348105, -9776.5071563707548874}, {-250.49346744287694398, -2385.7568792012312128}};
__device__ __constant__ const double RING_KSERKM[5][2] = {{-523.02599873176918199, 290.10526315789473684}, {-5485.2200380469245403, 5336.9790741915028535}, {-8338.1052631578947368, 15206.361445783132530}, {-2017.9378566899175650, 10515.743817374762207}, {-19.710843373493975904, 1418.8103994927076728}};
__device__ __constant__ const double RING_KSER0[6][2] = {{51471.854036415172419, 32768.000000000000000}, {-119621.18573838632696, -84345.212035111671234}, {96754.491735189724987, 78074.125512775430927}, {-31810.735585315211544, -31108.829182924968396}, {3678.1383813624327949, 4926.4461273804873303}, {-74.040670509817904983, -206.66608791871105442}};

// Geometry of a field point relative to a ring host, in the ring frame (ring.impl:2112-2118).
struct RingGeom {
    double x, y, re, re2, rz, rz2, r2;
    bool psign;
};
__device__ __forceinline__ RingGeom ring_geom(v3 r) {
    RingGeom g;
    g.psign = r.z < 0;
    if (g.psign) r.z = -r.z;
    g.x = r.x;
    g.y = r.y;
    g.re2 = r.x * r.x + r.y * r.y;
    g.re = sqrt(g.re2);
    g.rz2 = r.z * r.z;
    g.r2 = g.re2 + g.rz2;
    g.rz = r.z;
    return g;
}

// Contribution of one signed disk {GsR2, R_R, H_R} (ring.impl:2122-2190). sin and cos of
// phi = atan2(rz, re - R) are formed from the same two legs instead of from phi.
static __device__ __noinline__ v3 ring_disk_term(const double *__restrict__ disk, double host_R, const RingGeom &g) {
    const double pi = 3.1415926535897932;
    const double GsR2 = __ldg(disk), R_R = __ldg(disk + 1), H_R = __ldg(disk + 2);
    const double re = g.re, re2 = g.re2, rz = g.rz, rz2 = g.rz2, r2 = g.r2;
    double R = R_R * host_R;
    double H = H_R * host_R;
    double reR = re * R;
    double R2 = R * R, H2, fzh = 1;
    double k2dre = 4.0 / (r2 + R2 + 2 * reR);
    if (H > 0) {
        H2 = H * H;
        k2dre -= H2 * (k2dre * k2dre) * (1 - k2dre * rz2) / 48;
        fzh = (re > R ? re - R : 0);
        fzh = 4 * (rz2 + fzh * fzh);
        fzh = sqrt(fzh / (fzh + H2));
    }
    double k2 = reR * k2dre;
    k2dre *= R2 * sqrt(k2dre);
    const double dx = re - R;
    double phi = atan2(rz, dx);
    double kk = 0, lk = 0, fx;
    bool lkh = k2 >= 0.45;
    if (lkh) {
        kk = sqrt(k2);
        lk = log((1 - k2) / (8 * (1 + kk)));
        fx = (padesum(kk, RING_XSERKK) + lk * padesum(kk, RING_XSERKM)) / (k2 * k2);
    } else {
        fx = padesum(k2, RING_XSER0);
    }
    fx *= k2dre;
    double fz;
    double s, c;
    {
        const double h = sqrt(rz2 + dx * dx);
        if (h > 0) { s = rz / h; c = dx / h; }
        else { s = 0; c = 1; }   // atan2(0, 0) = 0
    }
    int kh = k2 >= .5;
    bool exphi;
    if (kh) {
        const double phimax = (pi / 2);
        exphi = c > 0;
        double ck = 1 - k2, lk2 = log(ck / 16), sk = sqrt(ck);
        double cc = exphi ? -c : c;
        double cphi = exphi ? pi - phi : phi;
        fz = cphi - (s / 8) * ((lk2 * (k2 - 5) - 2 * ck) * sk + 2 * cc * (1 + lk2) * ck);
        fz *= (double)ring_fzcorr((float)((exphi ? phi : pi - phi) * (1 / phimax)), (float)(k2 * 2), kh);
    } else {
        const double phimax = (809. / 512);
        exphi = phi > phimax;
        double cr2 = exphi ? R2 + rz2 : r2;
        double cRdr2 = (exphi ? re2 : R2) / cr2;
        fz = (pi / 8) * (4 - 3 * cRdr2) * (rz / sqrt(cr2) * cRdr2);
        fz *= (double)ring_fzcorr((float)((exphi ? pi - phi : phi) * (1 / phimax)), (float)(k2 * 2), kh);
    }
    if (exphi) {
        double ek;
        if (lkh) ek = padesum(kk, RING_KSERKK) + lk * padesum(kk, RING_KSERKM);
        else ek = padesum(k2, RING_KSER0);
        fz = pi - 2 * sqrt(1 - k2) * ek * s - fz;
    }
    double Gs = GsR2 / (host_R * host_R);
    fx *= Gs;
    fz *= Gs;
    return mk(-4 * fx * g.x, -4 * fx * g.y, -2 * fz * fzh);
}

// ring::sum: disks added in order, then the sign flip of the mirrored half-space (ring.impl:2109-2195)
static __device__ __noinline__ v3 ring_sum(const double *__restrict__ disks, int ndisk, double host_R, v3 r) {
    const RingGeom g = ring_geom(r);
    v3 ret = mk(0, 0, 0);
    for (int i = 0; i < ndisk; ++i) ret += ring_disk_term(disks + 3 * i, host_R, g);
    if (g.psign) ret.z = -ret.z;
    return ret;
}

}  // namespace eph
