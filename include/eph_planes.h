/*
 * eph_planes.h - structure-of-arrays layout of a body list, shared by every side of the C-ABI.
 *
 * A system of n bodies is exchanged as one row-major double array planes[EPH_NPLANES][n]:
 * plane p holds one scalar field for all bodies, so element (p, i) sits at planes[p*n + i].
 * Vectors take 3 consecutive planes (x, y, z); 3x3 matrices take 9 consecutive planes in the
 * reference's mat_t storage order (axis x = (xx, xy, xz), then axis y, then axis z;
 * src/math/vec_t.h:270-272, a matrix is the three column vectors x, y, z).
 * Double-double quantities (src/math/dfloat_t.h:13, `real` in src/definitions.h:6) are split
 * into a _HI and a _LO block.
 *
 * The fields are those of the reference's `class mass` (src/physics/mass.h:67-143) that the RK12
 * step reads or writes: the evolving state (mass.h:73-77), the time-variable parameters
 * (mass.h:83), the constants (mass.h:101-112), the model links (mass.h:115-117, here as indices
 * into the model tables, -1 for none) and the auxiliaries that accel() leaves behind
 * (mass.h:122-131,142-143).
 */
#ifndef EPH_PLANES_H
#define EPH_PLANES_H

enum eph_plane {
    /* evolving state, double-double (mass.h:73-75) */
    EPH_P_R_HI = 0,    EPH_P_R_LO = 3,
    EPH_P_V_HI = 6,    EPH_P_V_LO = 9,
    EPH_P_GL_HI = 12,  EPH_P_GL_LO = 15,
    EPH_P_S_HI = 18,   EPH_P_S_LO = 27,   /* surface frame, 9 planes each */
    /* evolving state, double (mass.h:77) */
    EPH_P_W = 36,                          /* angular velocity */
    /* time-variable parameters (mass.h:83) */
    EPH_P_GM = 39, EPH_P_EXJ2 = 40,
    /* constants (mass.h:101-112) */
    EPH_P_GM0 = 41, EPH_P_DGM = 42, EPH_P_DJ2 = 43, EPH_P_RADIUS = 44, EPH_P_INERTIA = 45,
    EPH_P_K2 = 46, EPH_P_K2R = 47, EPH_P_TIDE_DELAY = 48, EPH_P_TIDE_DELAY_FACTOR = 49,
    EPH_P_LUM = 50, EPH_P_RECPT = 51, EPH_P_A = 52, EPH_P_R2 = 53, EPH_P_SR2 = 54,
    EPH_P_RR2G_4C = 55,
    EPH_P_C_STATIC = 56,                   /* 9 planes */
    /* auxiliaries written by accel() (mass.h:122-131,142-143) */
    EPH_P_PHI = 65, EPH_P_BETA2 = 66,
    EPH_P_NACCEL = 67, EPH_P_DACCEL = 70, EPH_P_DTORQUE = 73, EPH_P_GACCEL = 76, EPH_P_BETA = 79,
    EPH_P_GI = 82,                         /* 9 planes */
    EPH_P_C_POTENTIAL = 91,                /* 9 planes */
    EPH_P_MIN_DISTANCE = 100, EPH_P_MAX_INFLUENCE = 101,
    /* model links (mass.h:115-117): index into the geopotential / ring tables, -1 = none */
    EPH_P_GP_INDEX = 102, EPH_P_RING_INDEX = 103,
    EPH_NPLANES = 104
};

/* Geopotential table: the reference packs degree 2..Max_N coefficients as
 * J(n)=n*n-4, C(n,m)=J(n)+2m-1, S(n,m)=J(n)+2m (src/physics/geopotential.impl:18-24). */
#define EPH_GP_MAX_DEGREE 8
#define EPH_GP_TABLE_SIZE (EPH_GP_MAX_DEGREE * (EPH_GP_MAX_DEGREE + 2) - 3) /* 77 */

/* Ring: header {GM_ratio, A, J2, GL_R2} and per-disk {GsR2, R_R, H_R} (src/physics/ring.h:8-19). */
#define EPH_RING_PARAMS 4
#define EPH_RING_MAX_DISKS 64

#endif
