// eph_system.cuh - device-side layout of one system of bodies and the RK12 step kernel's parameters.
//
// HBM layout. All per-body arrays are structure-of-arrays planes with a padded stride `ld` (n rounded
// up to a multiple of 32 bodies, so that every plane segment a CTA stages into shared memory starts
// on a 256-byte boundary and is a multiple of 16 bytes long, as the bulk-copy engine requires):
//   * public stage state, ping-pong pub[2][PUB_NPLANES][ld]: position (double-double, 6 planes),
//     velocity (double-double, 6), G*L/GM rounded to double (3), GM (1), body frame s rounded to
//     double (9, geopotential hosts) and ring frame (9, ring hosts). Written by the owning CTA at the
//     end of a stage, read by every CTA in the next one.
//   * pass-A outputs aux[AUX_NPLANES][ld]: phi/c^2, naccel/c^2 (3), beta (3), beta^2, C_potential (9).
//   * constants cst[CST_NPLANES][ld]: sR2, tide_delay_factor, R^2, luminosity, R, model indices.
//   * extended-body reactions react[n_ext][ld][2][6]: for host e and body i, -GM_i an and -GM_i (r x an)
//     of host e's geopotential (slot 0) and ring (slot 1) field at body i (written in pass A by i's
//     owner), and react_cta[n_ext][ld][6], each CTA's sum of them over its bodies (summed over the CTAs by
//     e's owner in pass B).
//   * planes[EPH_NPLANES][n]: the whole `mass` record (include/eph_planes.h), loaded at kernel start
//     and stored at kernel end by each body's owner.
// A CTA keeps the private state of the bodies it owns (start-of-step state, RK12 stage accumulators,
// auxiliaries) in shared memory for the whole launch, next to a staging tile that holds, per phase,
// the planes of every body j the pair sums read.
#pragma once
#include <stdint.h>

namespace eph {

constexpr int kThreads = 512;        // threads per CTA (16 warps; <= 128 registers per thread)
constexpr int kWarps = kThreads / 32;
constexpr int kExtWarps = 4;         // warps computing extended-body fields during the pass-A sweeps
constexpr int kOwnMax = 8;           // bodies owned by one CTA (private state lives in shared memory)
constexpr int kStages = 25;          // Feagin RK12 stages
constexpr int kMaxExt = 64;          // extended bodies (geopotential or ring) per system
constexpr int kPad = 32;             // plane stride granularity (bodies)
constexpr int kGpSmem = 12;          // geopotential models a CTA keeps (expanded) in shared memory
constexpr int kRingPar = 2;          // ring hosts whose disks are evaluated one per lane
constexpr int kRingDiskPar = 8;      // disks per ring evaluated one per lane

// public ping-pong plane offsets (within one buffer)
enum PubPlane {
    PUB_R_HI = 0, PUB_R_LO = 3, PUB_V_HI = 6, PUB_V_LO = 9, PUB_GL = 12, PUB_GM = 15,
    PUB_FRAME = 16, PUB_RFRAME = 25, PUB_NPLANES = 34
};
// pass-A output planes
enum AuxPlane { AUX_PHI = 0, AUX_NACC = 1, AUX_BETA = 4, AUX_BETA2 = 7, AUX_CPOT = 8, AUX_NPLANES = 17 };
// constant planes
enum ConstPlane { CST_SR2 = 0, CST_TDF = 1, CST_R2 = 2, CST_LUM = 3, CST_R = 4, CST_GP = 5, CST_RING = 6,
                  CST_NPLANES = 7 };

// planes staged into shared memory for the pass-A sweep (tile rows)
enum TileA { TA_R_HI = 0, TA_R_LO = 3, TA_V_HI = 6, TA_V_LO = 9, TA_GM = 12, TA_SR2 = 13, TA_TDF = 14, TA_ROWS = 15 };
// planes staged for the pass-B sweep: rows every body needs, then (from kTileBFullRows) rows only
// bodies of the full class need, staged for the full-class prefix of the tile only. Positions, GM and sR2
// sit in the rows pass A staged them in: when the whole system fits one tile they are not copied again.
enum TileB { TB_R_HI = TA_R_HI, TB_R_LO = TA_R_LO, TB_NACC = 6, TB_BETA = 9, TB_GM = TA_GM, TB_SR2 = TA_SR2,
             TB_PHI = 14, TB_BETA2 = 15, TB_GL = 16, TB_CPOT = 19, TB_R2 = 28, TB_LUM = 29, TB_ROWS = 30 };
constexpr int kTileBFullRows = TB_GL;
constexpr int kTileRows = TB_ROWS;

// Device bodies are ordered by class: the first n_full "full" bodies (any of tidal / rotational
// deformation, static harmonics, spin, luminosity, radiation receptance, geopotential or ring), then the
// point-like ones, for which the deformation, Lense-Thirring and radiation terms are exactly zero.
// Internal index k of a body maps to its position orig[k] in the caller's plane arrays.
struct SysDev {
    int n;                    // bodies
    int n_full;               // bodies of the full class (internal indices [0, n_full))
    int ld;                   // plane stride (n rounded up to kPad)
    int n_ext;                // extended bodies
    int tile;                 // bodies per shared-memory tile (multiple of kPad)
    const int *orig;          // [n] internal index -> index in `planes`
    double *pub;              // [2][PUB_NPLANES][ld]
    double *aux;              // [AUX_NPLANES][ld]
    double *cst;              // [CST_NPLANES][ld]
    double *react;            // [n_ext][ld][2][6]
    double *react_cta;        // [n_ext][ld][6]: per-CTA sums of `react` over the CTA's bodies (CTA < grid <= ld)
    double *planes;           // [EPH_NPLANES][n]
    const int *ext_body;      // [n_ext] body index of each extended body
    int n_gp;                 // geopotential models
    const int *gp_nz, *gp_nt;
    const double *gp_coef;    // [n_gp][EPH_GP_TABLE_SIZE]
    const int *ring_nd;       // ring models
    const double *ring_param; // [n_ring][4]
    const double *ring_disk;  // [n_ring][EPH_RING_MAX_DISKS][3]
    const int *own_list;      // [grid][kOwnMax], -1 padded
    unsigned int *bar;        // grid barrier: one 64-bit arrival counter (two words, 8-byte aligned), zeroed per launch
    int *status;              // device status word (0 = ok)
    unsigned long long *timers;   // optional [grid][kPhases] nanoseconds per phase (profiling), or null
    double *traj;             // optional stage records [slot][n][kTrajRec] (massless-particle integration), or null
    long long traj_base;      // slot of this launch's first stage evaluation
    long long wait_ns;        // limit of every bounded wait (grid barrier, tile copy), nanoseconds
    int stall_barrier;        // self-test only: the grid barriers wait for one arrival more than the launch has
};

constexpr long long kWaitDefaultNs = 2000000000ll;   // 2 s

// One stage record of a body (written after pass A, caller's body order): what a massless particle's
// stage evaluation reads of the massive bodies.
enum TrajField { TR_R_HI = 0, TR_R_LO = 3, TR_GM = 6, TR_PHI = 7, TR_NACC = 8, TR_BETA = 11, TR_BETA2 = 14,
                 TR_CPOT = 15, TR_R2 = 24, TR_GL = 25, TR_FRAME = 28, TR_RADIUS = 37, TR_SR2 = 38, TR_RFRAME = 39,
                 kTrajRec = 48 };

// phases of a stage evaluation, for the optional per-CTA phase timers
// (slot PH_A_COUNT counts the pass-A sweeps instead of nanoseconds)
enum Phase { PH_IO = 0, PH_RK = 1, PH_BARRIER = 2, PH_A_SWEEP = 3, PH_A_UPDATE = 4, PH_B_SWEEP = 5,
             PH_B_EXT = 6, PH_B_FINAL = 7, PH_A_COUNT = 8, kPhases = 9 };

enum Mode { MODE_INTEGRATE = 0, MODE_ACCEL = 1, MODE_DEFORM = 2 };

struct StepParams {
    int mode;
    int reset_minmax;         // integrate(): min_distance = max_influence = 0 before the steps
    int invert_min;           // integrate(): min_distance = 1/min_distance after the steps
    long long n_step;
    double dt;
    double t_eph;             // double(t_eph) of the reference (hi + lo)
};

enum Status { ST_OK = 0, ST_BARRIER_TIMEOUT = 1, ST_COPY_TIMEOUT = 2 };

}  // namespace eph
