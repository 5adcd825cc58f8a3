// eph_system.cuh - device-side layout of one system of bodies and the RK12 step kernel's parameters.
//
// HBM layout (all planes structure-of-arrays, plane p of n bodies at base + p*n):
//   * public stage state, ping-pong buffer [2]: position (double-double, 6 planes), velocity
//     (double-double, 6 planes), G*L/GM rounded to double (3 planes), GM (1 plane), body frame s
//     rounded to double (9 planes) and ring frame (9 planes). Written by the owning CTA at the end of
//     a stage, read by every CTA in the next stage.
//   * pass-A outputs: phi/c^2, naccel/c^2 (3), beta (3), beta^2, C_potential (9).
//   * per-body constants: sR2, tide_delay_factor, R2, lum, R, GM0, ... (read-only).
//   * the planes array [EPH_NPLANES][n] of include/eph_planes.h, used to load and store a whole system.
// A CTA keeps the private state of the bodies it owns (start-of-step state, RK12 stage accumulators,
// auxiliaries) in shared memory for the whole launch.
#pragma once
#include <stdint.h>

namespace eph {

constexpr int kThreads = 256;        // threads per CTA
constexpr int kOwnMax = 8;           // bodies owned by one CTA (private state lives in shared memory)
constexpr int kRegBodies = 4;        // owned bodies whose pair sums are held in registers at a time
constexpr int kStages = 25;          // Feagin RK12 stages
constexpr int kMaxExt = 64;          // extended bodies (geopotential or ring) per system

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

struct SysDev {
    int n;                    // bodies
    int n_ext;                // extended bodies
    double *pub;              // [2][PUB_NPLANES][n]
    double *aux;              // [AUX_NPLANES][n]
    double *cst;              // [CST_NPLANES][n]
    double *planes;           // [EPH_NPLANES][n]
    const int *ext_body;      // [n_ext] body index of each extended body
    const int *gp_nz, *gp_nt; // geopotential models
    const double *gp_coef;    // [n_gp][EPH_GP_TABLE_SIZE]
    const int *ring_nd;       // ring models
    const double *ring_param; // [n_ring][4]
    const double *ring_disk;  // [n_ring][EPH_RING_MAX_DISKS][3]
    const int *own_list;      // [grid][kOwnMax], -1 padded
    unsigned int *bar;        // grid barrier words {count, generation}
    int *status;              // device status word (0 = ok)
    unsigned long long *timers;   // optional [grid][kPhases] nanoseconds per phase (profiling), or null
};

// phases of a stage evaluation, for the optional per-CTA phase timers
enum Phase { PH_IO = 0, PH_RK = 1, PH_BARRIER = 2, PH_A_SWEEP = 3, PH_A_UPDATE = 4, PH_B_SWEEP = 5,
             PH_B_EXT = 6, PH_B_FINAL = 7, kPhases = 8 };

enum Mode { MODE_INTEGRATE = 0, MODE_ACCEL = 1, MODE_DEFORM = 2 };

struct StepParams {
    int mode;
    int reset_minmax;         // integrate(): min_distance = max_influence = 0 before the steps
    int invert_min;           // integrate(): min_distance = 1/min_distance after the steps
    long long n_step;
    double dt;
    double t_eph;             // double(t_eph) of the reference (hi + lo)
};

enum Status { ST_OK = 0, ST_BARRIER_TIMEOUT = 1 };

}  // namespace eph
