/*
 * eph_b200.h - C ABI of the B200 RK12 library (libeph_b200.so).
 *
 * Drop-in boundary for the reference's GPU integrator path. The reference reaches its GPU code through
 * two private msystem members defined in their own translation unit:
 *   void msystem::Cuda_RungeKutta12(fast_real dt, int_t n_step)   src/physics/mass.h:268, src/integrators/RungeKutta.cu:391-412
 *   void msystem::Cuda_accel()                                    src/physics/mass.h:270, src/integrators/RungeKutta.cu:418-438
 * called from msystem::integrate(dt, n_step, USE_GPU=1) (src/physics/mass.cpp:408-409) and
 * msystem::accel(parallel_option>0) (src/physics/mass.cpp:218-220). A replacement translation unit
 * marshals the `mass` list into the plane layout of eph_planes.h and calls the functions below
 * (ephemeris_b200/bridge/cuda_rk12_bridge.cpp is that unit). All functions return an eph_status; none
 * throws, exits or traps.
 *
 * Threading: one context per system; calls on one context are serialised by the context (the
 * reference serialises all GPU work on a global mutex, RungeKutta.cu:25,396,410). Different contexts
 * may be used from different host threads.
 */
#ifndef EPH_B200_H
#define EPH_B200_H
#include <stddef.h>
#include <stdint.h>
#include "eph_planes.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum eph_status {
    EPH_OK = 0,
    EPH_ERR_ARG = 1,          /* bad argument (null pointer, size out of range, unknown option) */
    EPH_ERR_CUDA = 2,         /* a CUDA runtime call failed; eph_last_error() has the text */
    EPH_ERR_OOM = 3,          /* device allocation failed */
    EPH_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up; the context stays usable */
    EPH_ERR_STATE = 5,        /* no system uploaded */
    EPH_ERR_LOAD = 6,         /* a config / initials file was missing or malformed */
    EPH_ERR_UNSUPPORTED = 7,  /* requested path is not provided by this library (e.g. a CPU integrator) */
    EPH_ERR_LIMIT = 8,        /* a size beyond the fixed maximum of eph_integrate_noalloc's scratch */
    EPH_ERR_STEP = 9          /* adaptive stepping gave up (step below the minimum, or too many attempts) */
} eph_status;

/* Geopotential and ring tables of a system (layouts in eph_planes.h). Model k of each kind belongs to
 * the body whose EPH_P_GP_INDEX / EPH_P_RING_INDEX plane holds k. */
typedef struct eph_models {
    int32_t n_gp;
    const int32_t *gp_nz;     /* [n_gp] maximum zonal degree (geopotential.h:7) */
    const int32_t *gp_nt;     /* [n_gp] maximum tesseral degree */
    const double *gp_coef;    /* [n_gp][EPH_GP_TABLE_SIZE] packed J/C/S coefficients (geopotential.impl:21-24) */
    int32_t n_ring;
    const int32_t *ring_ndisk;   /* [n_ring] number of signed disks (ring.h:8) */
    const double *ring_param;    /* [n_ring][4] GM_ratio, A, J2, GL_R2 (ring.h:12) */
    const double *ring_disk;     /* [n_ring][EPH_RING_MAX_DISKS][3] GsR2, R_R, H_R (ring.h:14-19) */
} eph_models;

typedef struct eph_ctx eph_ctx;

/* Create a context on CUDA device `device`. Replaces the reference's static device-memory cache
 * (RungeKutta.cu:38-47): buffers are allocated at upload and kept until the next larger upload. */
int eph_ctx_create(int device, eph_ctx **out);
int eph_ctx_destroy(eph_ctx *ctx);
/* Text of the last error on this context (never NULL). */
const char *eph_last_error(const eph_ctx *ctx);

/* Copy a system (planes [EPH_NPLANES][n] in host memory) and its models to the device
 * (cuda_rungekutta_kernel_config::load, RungeKutta.cu:77-122). */
int eph_upload_system(eph_ctx *ctx, int64_t n, const double *planes, const eph_models *models);
/* Same, with `planes` already in device memory of this context's device. */
int eph_upload_planes_device(eph_ctx *ctx, const double *d_planes);
/* Copy the whole body state back (cuda_rungekutta_kernel_config::save, RungeKutta.cu:124-133). */
int eph_download_system(eph_ctx *ctx, double *planes);
/* Device copy of the planes [EPH_NPLANES][n] (valid until the next upload of a larger system). */
int eph_device_planes(eph_ctx *ctx, double **d_planes);

/* msystem::Cuda_RungeKutta12(dt, n_step) (RungeKutta.cu:391-412): n_step Feagin RK12 steps of dt
 * starting at ephemeris time t_eph = t_eph_hi + t_eph_lo (double-double). Per-pair maxima
 * accumulate into min_distance (of 1/r) and max_influence; they are neither reset nor inverted. */
int eph_rk12(eph_ctx *ctx, double dt, int64_t n_step, double t_eph_hi, double t_eph_lo);
/* msystem::integrate(dt, n_step, USE_GPU=1) without the log lines (mass.cpp:399-442): a negative n_step
 * integrates backwards, the maxima are reset before and min_distance inverted after, and the
 * double-double t_eph advances by dt*n_step. */
int eph_integrate(eph_ctx *ctx, double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo);
/* msystem::Cuda_accel() (RungeKutta.cu:418-438): one acceleration evaluation of the uploaded state. */
int eph_accel(eph_ctx *ctx);
/* msystem::deform() (mass.cpp:104-110): tidal / rotational deformation of every body at the uploaded
 * state (potential, Newtonian acceleration, C_potential, GI), as used by the loader. */
int eph_deform(eph_ctx *ctx);

/* Self-test of the bounded waits (no counterpart in the reference, whose kernel's grid.sync cannot time
 * out): one acceleration evaluation of the uploaded system whose grid barriers wait for one arrival more
 * than the launch has, with every wait limited to wait_ns (1e5 .. 2e9 ns). Every CTA's wait runs out, the
 * kernel records the timeout and returns, and the call returns EPH_ERR_TIMEOUT; the context stays usable and
 * the next call runs normally (with the default 2 s limit). The uploaded planes are not written. */
int eph_selftest_wait_timeout(eph_ctx *ctx, int64_t wait_ns);

/* Issue this context's device work on `stream` (a cudaStream_t of the context's device; NULL restores
 * the context's own stream). Calls still return only after their work has finished. */
int eph_set_stream(eph_ctx *ctx, void *stream);

/* Launch shape: grid = CTAs (0: automatic), bodies_per_cta (0: automatic, at most EPH_MAX_BODIES_PER_CTA).
 * The reference fixes its shape in code (RungeKutta.cu:80-88); eph_autotune picks one by timing. */
#define EPH_MAX_BODIES_PER_CTA 8
int eph_set_launch(eph_ctx *ctx, int grid, int bodies_per_cta);
/* Current launch shape. */
int eph_get_launch(const eph_ctx *ctx, int *grid, int *bodies_per_cta);
/* Autotuner (the reference fixes its launch shape in code, RungeKutta.cu:80-88): times candidate launch
 * shapes (bodies per CTA, hence the grid) and ownership cost models (the weight of a delayed-tide body) of
 * the step kernel on the uploaded system, n_step RK12 steps of dt each, best of `reps` after a warm-up run,
 * every trial starting from the uploaded state; keeps the fastest through eph_set_launch /
 * eph_set_body_costs and caches it per (device, bodies, body classes), so that with use_cache a later call on
 * a system of the same key times only the cached choice. Leaves the uploaded state as it was. Returns the
 * chosen shape and the per-RK12-step times of the choice and of the built-in heuristic. */
int eph_autotune(eph_ctx *ctx, double dt, int n_step, int reps, int use_cache, int *grid, int *bodies_per_cta,
                 double *ms_per_step_tuned, double *ms_per_step_default);
/* Work estimates of the uploaded system's bodies (cost[n] > 0, caller order) that the split of bodies over
 * CTAs balances (longest processing time first); NULL restores the built-in estimate. Re-plans at once; an
 * upload keeps the override while the body count stays the same. */
int eph_set_body_costs(eph_ctx *ctx, const double *cost);
/* Bodies owned by each CTA of the current launch: bodies[grid][EPH_MAX_BODIES_PER_CTA], caller indices,
 * -1 padded (`bodies` must hold that many entries for the largest grid, i.e. the co-resident CTA count). */
int eph_get_ownership(const eph_ctx *ctx, int32_t *bodies, int *grid);
/* Kernel launches issued on this context so far. */
int64_t eph_launch_count(const eph_ctx *ctx);

/* Profiling aid: with enable != 0 every launch records, per CTA, the nanoseconds spent in each phase
 * of the step (load/store, RK combination, barrier waits, pass-A sweeps, pass-A updates, pass-B sweeps,
 * wait for the extended-body fields, finalisation) and, in the last slot, the number of pass-A sweeps.
 * eph_phase_times copies the last launch's [grid][EPH_PHASES] table (out must hold grid*EPH_PHASES values;
 * grid = CTAs of the current launch shape). */
#define EPH_PHASES 9
int eph_profile_phases(eph_ctx *ctx, int enable);
int eph_phase_times(eph_ctx *ctx, uint64_t *out, int *grid, int *phases);

/* ---- Batched ensembles (no counterpart in the reference, which integrates one msystem per call; its
 * combined integrator runs subsystems one at a time, mass_combined.cpp:286-321). Many independent systems,
 * each with its own dt, step count and ephemeris time, integrated with msystem::integrate semantics
 * (mass.cpp:399-442). Systems whose bodies are all point-like (Newtonian + 1PN only) share one persistent
 * launch, one CTA per system; any other system runs through the single-system kernel. */
/* Arithmetic modes of the batched and particle paths */
#define EPH_PREC_FP64 0
#define EPH_PREC_MIXED 1

typedef struct eph_batch eph_batch;
int eph_batch_create(int device, eph_batch **out);
int eph_batch_destroy(eph_batch *b);
const char *eph_batch_last_error(const eph_batch *b);
/* n_sys systems: system s has n_body[s] bodies, planes[s] = [EPH_NPLANES][n_body[s]] (host), models[s]
 * (NULL array or NULL entry: no geopotential / ring models). Replaces any previous batch. */
int eph_batch_upload(eph_batch *b, int32_t n_sys, const int64_t *n_body, const double *const *planes,
                     const eph_models *const *models);
/* Integrate system s by n_step[s] steps of dt[s] (negative n_step: backwards) from t_eph[s] =
 * t_eph_hi[s] + t_eph_lo[s], which advances in double-double. */
int eph_batch_integrate(eph_batch *b, const double *dt, const int64_t *n_step, double *t_eph_hi, double *t_eph_lo);
/* Copy every system's planes back into planes[s]. */
int eph_batch_download(eph_batch *b, double *const *planes);
/* Issue the batch's device work on `stream` (a cudaStream_t of its device; NULL restores its own stream).
 * Calls still return only after their work has finished. */
int eph_batch_set_stream(eph_batch *b, void *stream);
/* Arithmetic of the ensemble launch's EIH 1PN terms: EPH_PREC_FP64 (default) or EPH_PREC_MIXED (those terms in
 * FP32 from FP32 copies of the pass-A outputs, summed with a compensated FP32 sum and added into the FP64
 * totals; state, separations, the Newtonian sums, the per-pair maxima and the RK12 combination stay FP64 /
 * double-double). Applies from the next integrate; systems on the single-system path are not affected. */
int eph_batch_set_precision(eph_batch *b, int mode);
/* Systems of at least `bodies` bodies are shared by the 4 CTAs of a thread-block cluster in the ensemble
 * launch (0: the default, 96). */
int eph_batch_set_coop_min(eph_batch *b, int bodies);
/* Autotuner of the ensemble launch: times the uploaded batch's shared launch (step counts scaled by
 * step_frac, so the members keep their relative durations; best of 2 from the uploaded state, which is
 * restored) for several cluster-sharing thresholds, keeps the fastest (eph_batch_set_coop_min) and returns
 * it with the times (ms) of the choice and of the threshold in force before. */
int eph_batch_autotune(eph_batch *b, const double *dt, const int64_t *n_step, double step_frac, int *coop_min,
                       double *ms_tuned, double *ms_default);
/* Systems in the shared ensemble launch, and launches issued so far. */
int eph_batch_info(const eph_batch *b, int32_t *n_ensemble, int64_t *launches);

/* ---- Massless test particles (no counterpart in the reference, which has no massless bodies; bodies of
 * negligible GM in one msystem with the perturbers are its equivalent). The perturbers (at most 32, any
 * physics) run with msystem::integrate semantics; each particle feels every perturber's Newtonian, 1PN,
 * deformation, Lense-Thirring, geopotential and ring terms and acts on nothing. */
typedef struct eph_particles eph_particles;
int eph_particles_create(int device, eph_particles **out);
int eph_particles_destroy(eph_particles *p);
const char *eph_particles_last_error(const eph_particles *p);
/* Perturbers: planes [EPH_NPLANES][n_pert] (host) and models; particles: [12][n_part] (host) = position
 * hi (3), position lo (3), velocity hi (3), velocity lo (3) as double-double, SI units. */
int eph_particles_upload(eph_particles *p, int64_t n_pert, const double *pert_planes, const eph_models *models,
                         int64_t n_part, const double *part_state);
/* n_step steps of dt (negative n_step: backwards) from t_eph = t_eph_hi + t_eph_lo, which advances. */
int eph_particles_integrate(eph_particles *p, double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo);
/* Perturber planes and/or particle states ([12][n_part]); either pointer may be NULL. */
int eph_particles_download(eph_particles *p, double *pert_planes, double *part_state);
/* Issue the set's device work on `stream` (NULL restores its own stream); calls still return only after
 * their work has finished. */
int eph_particles_set_stream(eph_particles *p, void *stream);
/* Arithmetic of the particles' EIH 1PN terms: EPH_PREC_FP64 (default) or EPH_PREC_MIXED (those terms,
 * ~1e-8 of the Newtonian acceleration, in FP32; state, separations, Newtonian, deformation, field terms
 * and the RK12 combination stay FP64 / double-double). Applies from the next integrate. */
int eph_particles_set_precision(eph_particles *p, int mode);
/* Kernels launched so far and the summed device time of the particle kernel (CUDA events, ms). */
int eph_particles_info(const eph_particles *p, int64_t *launches, double *particle_kernel_ms);

/* ---- B-spline ephemeris fit (host; src/math/interp.h:68-150). Fits samples[mn + 1][channels], taken at
 * uniform positions 0..mn, with n + d degree-d B-splines of unit knot spacing n / mn samples:
 * coefs[n + d][channels]. Requires 1 <= d <= EPH_BSPLINE_MAX_DEGREE, n >= 1, mn + 1 >= n + d. */
#define EPH_BSPLINE_MAX_DEGREE 8
int eph_bspline_fit(int d, int64_t n, int64_t mn, int channels, const double *samples, double *coefs);
/* The same fit for n_series series on one sample grid, solved on `device` (one thread per series and
 * channel; the grid's matrix is factored once on the host): samples[n_series][mn + 1][channels] ->
 * coefs[n_series][n + d][channels] (host arrays). Bit-identical to eph_bspline_fit series by series. */
int eph_bspline_fit_batch(int device, int d, int64_t n, int64_t mn, int channels, int64_t n_series,
                          const double *samples, double *coefs);
/* c(d, k, j): B[d, x - k] = sum_j c(d,k,j) T_j(2x - 1) on x in [0, 1) (src/math/interp.h:24-30). */
double eph_bspline_cheb_coef(int d, int k, int j);

/* ---- Compressed ephemeris records (host). One record as the reference's compressor writes it
 * (ephemeris_compressor::compress_orbital_data / compress_rotational_data, src/modules/
 * ephemeris_compressor.cpp:164-530; the reader hands each one to ephemeris_compressor::interpolator,
 * ephemeris_compressor.h:74-148 and ephemeris_compressor.cpp:852-910) covering `range` seconds. Orbital
 * formats 1-4 (state vectors, Keplerian vectors, circular and raw Keplerian elements) and rotational
 * formats 5-7 (axial offset, quaternion, tidal lock); a record that is not a valid compressed record
 * returns EPH_ERR_LOAD. */
typedef struct eph_ephem eph_ephem;
int eph_ephem_open(const void *record, int64_t size, double range, eph_ephem **out);
int eph_ephem_close(eph_ephem *e);
/* Format (1-4), B-spline degree, segments, the recorded relative error and GM (0 for state vectors). */
int eph_ephem_info(const eph_ephem *e, int *format, int *degree, int64_t *segments, double *relative_error,
                   double *gm);
/* Position r[3] and velocity v[3] at time t in [0, range] (interpolator::operator(), ephemeris_compressor.cpp:
 * 1036-1053); gm may be NULL. Outside [0, range]: NaN and EPH_ERR_ARG; a rotational record:
 * EPH_ERR_UNSUPPORTED. */
int eph_ephem_state(const eph_ephem *e, double t, double *r, double *v, double *gm);
/* The same at `count` times: out[count][6] = {r, v}. Times outside [0, range] give NaN rows and EPH_ERR_ARG
 * after every other row is filled. */
int eph_ephem_states(const eph_ephem *e, int64_t count, const double *t, double *out);
/* Angular velocity w[3] and surface-frame axes x[3], z[3] at time t of a rotational record
 * (interpolator::operator()(t, rotational_state_t*), ephemeris_compressor.cpp:1017-1034); an orbital record:
 * EPH_ERR_UNSUPPORTED. A tidally locked record (format 7) needs the orbital state at the same time first
 * (EPH_ERR_STATE until one is set). */
int eph_ephem_rotation(const eph_ephem *e, double t, double *w, double *x, double *z);
/* The orbital state (position and velocity relative to the orbital centre) a tidally locked record is
 * evaluated against (interpolator::set_orbital_state, ephemeris_compressor.cpp:1010-1015). */
int eph_ephem_set_orbital_state(eph_ephem *e, const double *r, const double *v);
/* A record handle is read-only after eph_ephem_open except for eph_ephem_set_orbital_state: handles may be
 * used from several threads, one handle's orbital state from one thread at a time. */
/* The record's positions at mn + 1 uniform times over [0, range], fitted by eph_bspline_fit with degree d
 * and n segments: coefs[n + d][3], the form of the device ephemeris (eph_serve_*, eph_bspline_fit_batch). */
int eph_ephem_to_bspline(const eph_ephem *e, int d, int64_t n, int64_t mn, double *coefs);

/* ---- Ephemeris samples for a B-spline ephemeris (no counterpart in the reference's GPU path; its
 * generator records states on the host per cadence, src/modules/ephemeris_generator.cpp:128-169).
 * Integrates n_step steps of dt from t_eph (advanced, msystem::integrate's RK12) and writes the state at
 * the start and after every `stride` steps (n_step a multiple of stride):
 * out[n_step / stride + 1][n][EPH_EPHEM_CHANNELS] = position (3), velocity (3), Newtonian acceleration /
 * c^2 (3), potential / c^2 (1) of every body, in the caller's order, in SI units. */
#define EPH_EPHEM_CHANNELS 10
int eph_record_samples(eph_ctx *ctx, double dt, int64_t n_step, int64_t stride, double *t_eph_hi, double *t_eph_lo,
                       double *out);

/* ---- Serving: massless particles with adaptive RK12 against a device-resident B-spline ephemeris
 * (no counterpart in the reference). The ephemeris: n_pert bodies (GM, softening sR2 or NULL for none),
 * each fitted by eph_bspline_fit with degree `degree` on n_intervals knot intervals of `knot` seconds from
 * t0, EPH_EPHEM_CHANNELS channels: coefs[n_pert][n_intervals + degree][EPH_EPHEM_CHANNELS]. Body 0 is the
 * central body of the error measure. */
#define EPH_SERVE_MAX_PERTURBERS 1024
typedef struct eph_serve eph_serve;
int eph_serve_create(int device, int64_t n_pert, const double *gm, const double *sr2, int degree, int64_t n_intervals,
                     double t0, double knot, const double *coefs, eph_serve **out);
int eph_serve_destroy(eph_serve *s);
const char *eph_serve_last_error(const eph_serve *s);
/* Device memory the in-flight requests may hold: bytes > 0 a fixed budget; 0 (the default) admits requests
 * while the device's free memory stays above a 1 GiB reserve. The oldest queued request always launches
 * when nothing is in flight. */
int eph_serve_set_budget(eph_serve *s, int64_t bytes);
/* Record up to `cap` accepted step sizes of each later request's first block of particles (0: off). */
int eph_serve_set_step_log(eph_serve *s, int64_t cap);
/* Queue a request: part_state[12][n_part] (position hi, lo, velocity hi, lo; copied), integrated from
 * t_start to t_end (either direction, inside the ephemeris) with tolerance `tol` on the step-doubling
 * error |r_h - r_h/2| / |r - r_0| and first step h0 > 0 seconds. It launches when its memory fits. */
int eph_serve_submit(eph_serve *s, int64_t n_part, const double *part_state, double t_start, double t_end, double tol,
                     double h0, int64_t *id);
/* state: 0 queued, 1 running, 2 done. Also launches queued requests that now fit. */
int eph_serve_poll(eph_serve *s, int64_t id, int *state);
/* Wait for a launched request, copy its particles out ([12][n_part], or NULL), its accepted / rejected
 * particle-steps and (with a step log) its first block's accepted step sizes; release it. EPH_ERR_STATE if
 * it is still queued; EPH_ERR_STEP if its stepping gave up (the state is still copied out). */
int eph_serve_result(eph_serve *s, int64_t id, double *part_state, int64_t *n_accepted, int64_t *n_rejected,
                     double *step_log, int64_t *n_logged);
/* How a request runs: lanes per particle, particles per block (block b holds particles
 * [b * particles_per_block, ...)), blocks. */
int eph_serve_request_shape(eph_serve *s, int64_t id, int *lanes, int *particles_per_block, int *blocks);
/* The ephemeris on the device at time t: out[n_pert][EPH_EPHEM_CHANNELS] (host). */
int eph_serve_eval(eph_serve *s, double t, double *out);
int eph_serve_info(const eph_serve *s, int64_t *launches, int64_t *queued, int64_t *bytes_in_use);

/* ---- Force models evaluated on their own (geopotential::sum, src/physics/geopotential.h:36): the field
 * of a geopotential model coef[EPH_GP_TABLE_SIZE] (degrees 2..nz zonal, tesseral up to nt <= nz) of a body
 * of radius R at `count` body-frame positions r[count][3] (host arrays): out[count][3] = acceleration per
 * unit GM of the body, computed on `device` by the device functions the integration kernels use: lanes = 1
 * one point per thread (massless-particle kernels), lanes = 8 one point per 8 lanes (step kernel), lanes = 0
 * one point per thread as the step kernel's one-lane items (column by column for models up to degree 6
 * and order 4, else the lane evaluation on one lane). */
int eph_geopotential_field(int device, const double *coef, int nz, int nt, double R, int lanes, int64_t count,
                           const double *r, double *out);

/* Measurement aid (no counterpart in the reference): the throughput of the FP64 CUDA-core pipe that the
 * integration kernels use, measured on `device` with independent FMA chains on every SM (TFLOP/s, an FMA
 * counted as 2 flops). */
int eph_fp64_fma_rate(int device, double *tflops);

/* Limits of eph_integrate_noalloc's fixed scratch (about 3.2 MB of device memory per GPU). */
#define EPH_NOALLOC_MAX_BODIES 1024
#define EPH_NOALLOC_MAX_EXT 16     /* bodies with a geopotential or ring model */
#define EPH_NOALLOC_MAX_GP 16      /* geopotential models */
#define EPH_NOALLOC_MAX_RING 16    /* ring models */

/* No counterpart in the reference: an added entry point for callers that cannot allocate device memory
 * (a host program that owns all device memory through its own pool and forbids cudaMalloc, a plug-in with a
 * fixed per-device budget, or code that must not take cudaMalloc's implicit synchronisation mid-stream).
 * Same result as eph_upload_system + eph_integrate + eph_download_system on the same system, but the
 * caller's planes ([EPH_NPLANES][n] doubles) stay in the caller's device memory on `device` and are
 * integrated in place on `stream` (a cudaStream_t of that device, or NULL for the legacy default stream);
 * the model tables are read from host memory. The kernel's working memory is one fixed array compiled into
 * the library, which every GPU that loads the library holds until the process exits; no call allocates
 * anything, on the device or through any library. More bodies, geopotential or ring models than the
 * EPH_NOALLOC_MAX_* limits return EPH_ERR_LIMIT before any device work. The extended-body limit and the
 * planes' model indices can only be checked once the planes are on the host: each call first copies the
 * planes from the device on `stream` and waits for that copy, then returns EPH_ERR_LIMIT (too many extended
 * bodies or more co-resident CTAs than the GPU offers) or EPH_ERR_ARG (a model index out of range) before
 * any further device work. The first call on a device sets that device up (looks up the array's device
 * address, uploads the RK12 tables); make that first call before any stream capture. Every call waits on
 * `stream` for its own work. All calls share the array, and calls that overlapped on the GPU would race on
 * it: a lock inside the library serialises the calls of one process and each call returns only after its
 * work has finished. The caller's current device is restored before returning. */
int eph_integrate_noalloc(int device, void *stream, int64_t n, double *d_planes, const eph_models *models,
                          double dt, int64_t n_step, double *t_eph_hi, double *t_eph_lo);

#ifdef __cplusplus
}
#endif
#endif
