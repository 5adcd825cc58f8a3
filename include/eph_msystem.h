/*
 * eph_msystem.h - reference-compatible system entry points of libeph_b200.so.
 *
 * These mirror the public msystem interface of the reference for the RK12 path (src/physics/mass.h:202-358):
 * a system is loaded from the reference's config / Initial / Extra / Geopotentials / Rings files and
 * integrated with the GPU RK12 integrator. The state stays resident in device memory between calls.
 */
#ifndef EPH_MSYSTEM_H
#define EPH_MSYSTEM_H
#include <stdint.h>
#include "eph_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct eph_msystem eph_msystem;

/* msystem::load(fconfig) (src/physics/mass.h:313, src/modules/mass_loader.cpp:67-294,324-561) on CUDA
 * device `device`. Returns EPH_ERR_LOAD (with a message on stderr) when a file is missing or malformed
 * or a body fails mass::sanity (mass_loader.cpp:18-65). */
int eph_msystem_load(const char *config_path, int device, eph_msystem **out);
int eph_msystem_free(eph_msystem *ms);
/* msystem::size() (mass.h:341) */
int64_t eph_msystem_size(const eph_msystem *ms);
/* msystem::integrate(dt, n_step, USE_GPU) (mass.h:293, mass.cpp:399-442). USE_GPU=0 (the CPU
 * integrator) is not provided and returns EPH_ERR_UNSUPPORTED. */
int eph_msystem_integrate(eph_msystem *ms, double dt, int64_t n_step, int use_gpu);
/* msystem::accel(parallel_option) (mass.h:286, mass.cpp:216-221); only parallel_option > 0 (GPU). */
int eph_msystem_accel(eph_msystem *ms, int parallel_option);
/* Body state in the plane layout of eph_planes.h (operator[] of mass.h:343-354, for a whole system). */
int eph_msystem_get_planes(eph_msystem *ms, double *planes);
int eph_msystem_set_planes(eph_msystem *ms, const double *planes);
/* Ephemeris time as double-double (t_eph, mass.h:218) and the configured step (delta_t, mass.h:220). */
int eph_msystem_t_eph(const eph_msystem *ms, double *hi, double *lo);
double eph_msystem_delta_t(const eph_msystem *ms);
/* Configured integrator: 0 CPU_RK12, 1 GPU_RK12, 2 COMBINED_RK12 (mass.h:207-211). */
int eph_msystem_integrator(const eph_msystem *ms);
/* Model tables (valid while the system lives) and the 8-byte body ids (mass.h:87). */
int eph_msystem_models(const eph_msystem *ms, eph_models *out);
int eph_msystem_sids(const eph_msystem *ms, uint64_t *out);
/* The device context holding this system. */
eph_ctx *eph_msystem_ctx(eph_msystem *ms);
const char *eph_msystem_error(const eph_msystem *ms);
/* Messages below `level` are dropped (20 info, 30 warning, 40 error; default 30). */
void eph_set_log_level(int level);

#ifdef __cplusplus
}
#endif
#endif
