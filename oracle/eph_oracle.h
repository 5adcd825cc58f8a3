/*
 * eph_oracle.h - CPU restatement of the reference's RK12 step (TEST INFRASTRUCTURE ONLY).
 *
 * This is the checker the parity tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * compare the CUDA path against. It is never linked into, loaded by or called from the product
 * library. It restates, in plain C with the reference's operation order and no floating-point
 * contraction, the serial CPU branch of the reference:
 *   msystem::RungeKutta12     src/integrators/RungeKutta.impl:107-194
 *   msystem::accel (serial)   src/physics/mass.cpp:216-397 (branch :309-374)
 *   mass::deform_by           src/physics/mass.cpp:78-103
 *   force macros              src/physics/mass.impl:1-152
 *   geopotential::sum         src/physics/geopotential.impl:26-106
 *   ring::sum                 src/physics/ring.impl:2070-2195
 *   msystem::integrate        src/physics/mass.cpp:399-442
 * Its results are pinned bit-for-bit against the reference itself (tests/golden/).
 *
 * Bodies are passed in the plane layout of include/eph_planes.h.
 */
#ifndef EPH_ORACLE_H
#define EPH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_models {
    int32_t n_gp;
    const int32_t *gp_nz, *gp_nt;     /* n_gp */
    const double *gp_coef;            /* n_gp x EPH_GP_TABLE_SIZE */
    int32_t n_ring;
    const int32_t *ring_ndisk;        /* n_ring */
    const double *ring_param;         /* n_ring x 4: GM_ratio, A, J2, GL_R2 */
    const double *ring_disk;          /* n_ring x EPH_RING_MAX_DISKS x 3: GsR2, R_R, H_R */
} orc_models;

/* One acceleration evaluation, msystem::accel(-1) (serial branch). planes: [EPH_NPLANES][n], in/out. */
void orc_accel(int64_t n, double *planes, const orc_models *models);

/* msystem::deform (mass.cpp:104-110): deform_by for every body (pass A + UPDATE_HARMONICS). */
void orc_deform(int64_t n, double *planes, const orc_models *models);

/* msystem::integrate(dt, n_step, 0) without the logging: resets the per-pair maxima, runs n_step
 * RK12 steps, inverts min_distance, and advances t_eph (hi, lo) in place.
 * stage_acc (optional): receives the total acceleration gaccel+daccel+naccel after each of the
 * 25*n_step accel() calls, as [stage][3][n]. */
void orc_integrate(int64_t n, double *planes, const orc_models *models, double dt, int64_t n_step,
                   double *t_eph_hi, double *t_eph_lo, double *stage_acc);

/* As orc_integrate, also capturing the full body planes right before (stage_in) and right after
 * (stage_out) each of the 25*n_step accel() calls, as [stage][EPH_NPLANES][n]. Either may be NULL. */
void orc_integrate_stages(int64_t n, double *planes, const orc_models *models, double dt, int64_t n_step,
                          double *t_eph_hi, double *t_eph_lo, double *stage_in, double *stage_out);

/* Single evaluations of the extended-body models, for tests. */
void orc_geopotential_sum(const orc_models *models, int32_t k, double R, const double r[3], double out[3]);
void orc_ring_sum(const orc_models *models, int32_t k, double R, const double r[3], double out[3]);

#ifdef __cplusplus
}
#endif
#endif
