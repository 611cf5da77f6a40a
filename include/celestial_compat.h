/* celestial_compat.h - the reference engine's native C API, served by the
 * B200 engine.
 *
 * A native program written against the reference's `celestial_*` functions
 * (engine/include/celestial/interop/native_api.h) links this library instead
 * and keeps its calls.  This file declares the subset of that surface that
 * the force path covers: lifecycle, particle transfer, stepping (Verlet or
 * Yoshida4, fixed or adaptive dt, the frame accumulator), compute mode and
 * theta, energy/momentum drift, merge collisions, counts, timings, version,
 * capabilities and the last error.  Same names, arguments and return
 * conventions as the reference; one global engine, as there.
 *
 * Differences, stated once:
 *   - every compute mode runs on the GPU: the two brute-force modes (0, 2)
 *     use the FP64 direct sum in the order and rounding of the reference's
 *     CPU brute force (Engine::compute_cpu_brute_forces, coefficient
 *     m * inv^3), so CPU_BruteForce trajectories are bit-identical to the
 *     reference's (the reference's GPU brute-force kernel uses CUDA's rsqrt
 *     and FMA contraction and has no reproducible bits to match);
 *     CPU_BarnesHut (1) uses the reference-semantics walk
 *     (monopole, the reference's MAC); GPU_BarnesHut (3) the B200 group walk
 *     (monopole + quadrupole, FP32 pair forces);
 *   - collision modes: Ignore (0) and Merge (3); Elastic (1) and Inelastic (2)
 *     are refused (the last error says so) and leave the mode unchanged;
 *   - functions outside this subset (post-Newtonian terms, softening modes,
 *     GPU validation, telemetry, snapshots, JSON config, deterministic mode
 *     switches) are not provided.
 * Like the reference's, these functions share one global engine and are not
 * safe to call from several threads at once; settings made through them
 * (mode, integrator, adaptive dt, collisions) outlive shutdown and apply to
 * the next init, as the reference's global configuration does. */
#ifndef CELESTIAL_COMPAT_H
#define CELESTIAL_COMPAT_H

#include <stdint.h>

#include "nbody_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* native_api.h:8-10 */
#define CELESTIAL_API_VERSION_MAJOR 1
#define CELESTIAL_API_VERSION_MINOR 0
#define CELESTIAL_API_VERSION_PATCH 0

/* core::ErrorCode values (engine/include/celestial/core/error.hpp:9-18) */
#define CELESTIAL_OK 0
#define CELESTIAL_ERR_CUDA (-1)
#define CELESTIAL_ERR_OUT_OF_MEMORY (-2)
#define CELESTIAL_ERR_INVALID_ARGUMENT (-3)
#define CELESTIAL_ERR_DEVICE_NOT_FOUND (-5)
#define CELESTIAL_ERR_ALREADY_INITIALIZED (-7)

/* ── Lifecycle (native_api.h:28-33) ───────────────────────────────────── */
/* 0, or a negative ErrorCode; a second init without shutdown returns
 * CELESTIAL_ERR_ALREADY_INITIALIZED, as the reference does. */
NB_API int32_t celestial_init(int32_t max_particles);
NB_API void celestial_shutdown(void);

/* ── Particle transfer (native_api.h:36-56) ───────────────────────────── */
/* acc_* become the previous accelerations of the first half kick. */
NB_API void celestial_set_particles(const double* pos_x, const double* pos_y,
                                    const double* pos_z, const double* vel_x,
                                    const double* vel_y, const double* vel_z,
                                    const double* acc_x, const double* acc_y,
                                    const double* acc_z, const double* mass,
                                    const double* radius, const uint8_t* is_active,
                                    int32_t count);
/* Copy min(count, particle count) rows. */
NB_API void celestial_get_accelerations(double* out_acc_x, double* out_acc_y,
                                        double* out_acc_z, int32_t count);
NB_API void celestial_get_positions(double* out_pos_x, double* out_pos_y, double* out_pos_z,
                                    int32_t count);
NB_API void celestial_get_velocities(double* out_vel_x, double* out_vel_y, double* out_vel_z,
                                     int32_t count);

/* ── Stepping (native_api.h:58-66) ────────────────────────────────────── */
/* A step of dt 0 (forces at the current positions), as the reference. */
NB_API void celestial_compute_forces(double softening);
/* One step with the current integrator, compute mode and collision mode;
 * with adaptive dt enabled the adaptive dt is updated after it. */
NB_API void celestial_step(double dt, double softening);
/* Frame accumulator (Timestep::update, engine/src/sim/timestep.cpp:5-17):
 * steps of the init-time dt while the accumulator holds one, at most
 * max_steps_per_frame (10); each step takes the adaptive dt when enabled. */
NB_API int32_t celestial_update(double frame_time);

/* ── Configuration (native_api.h:68-84) ───────────────────────────────── */
/* 0 CPU_BruteForce, 1 CPU_BarnesHut, 2 GPU_BruteForce (default),
 * 3 GPU_BarnesHut. */
NB_API void celestial_set_compute_mode(int32_t mode);
NB_API void celestial_set_theta(double theta);
/* Stored for the next celestial_init, as the reference stores them. */
NB_API void celestial_set_dt(double dt);
NB_API void celestial_set_softening(double softening);

/* ── Integrator and adaptive dt (native_api.h:146-164) ────────────────── */
/* 0 Leapfrog_KDK (default), 1 Yoshida4. */
NB_API void celestial_set_integrator(int32_t type);
NB_API int32_t celestial_get_integrator(void);
NB_API void celestial_set_adaptive_timestep(int32_t enabled, double eta, double dt_min,
                                            double dt_max, double initial_dt);
NB_API double celestial_get_adaptive_dt(void);
NB_API int32_t celestial_is_adaptive_dt_enabled(void);

/* ── Energy and momentum drift (native_api.h:99-111, 166-169) ─────────── */
/* EnergyTracker semantics (engine/src/profile/energy_tracker.cpp:169-213):
 * the first snapshot is the reference point; PE is the exact pair sum, or
 * the tree potential above 256 bodies in the Barnes-Hut modes
 * (Engine::compute_energy_snapshot, engine/src/sim/engine.cpp:398-421). */
NB_API void celestial_compute_energy_snapshot(void);
NB_API double celestial_get_energy_drift(void);
NB_API double celestial_get_momentum_drift(void);
NB_API double celestial_get_angular_momentum_drift(void);
NB_API double celestial_get_accumulated_error(void);

/* ── Timings and counts (native_api.h:113-143, 219-225) ───────────────── */
NB_API double celestial_get_last_gpu_time_ms(void);
NB_API double celestial_get_last_tree_build_ms(void);
NB_API double celestial_get_last_tree_traverse_ms(void);
NB_API int32_t celestial_get_particle_count(void);
NB_API int32_t celestial_get_active_particle_count(void);
NB_API int32_t celestial_get_last_merge_count(void);

/* ── Collisions (native_api.h:185-218) ────────────────────────────────── */
/* CollisionMode: 0 Ignore (default), 3 Merge; 1 and 2 are refused. */
NB_API void celestial_set_collision_mode(int32_t mode);
NB_API void celestial_set_max_merges_per_frame(int32_t max_merges);
NB_API void celestial_set_max_merges_per_body(int32_t max_merges);
NB_API void celestial_set_density_preserving_merge(int32_t enabled);

/* ── Version, capabilities, errors (native_api.h:265-295) ─────────────── */
typedef struct CelestialVersion {
    int32_t major;
    int32_t minor;
    int32_t patch;
} CelestialVersion;
NB_API CelestialVersion celestial_api_version(void);
/* CelestialCapability bits (native_api.h:278-287) that this library has:
 * CUDA, BARNES_HUT, YOSHIDA4, GPU_TREE, GPU_MERGE, ADAPTIVE_DT,
 * DETERMINISTIC (results are run-to-run reproducible). */
#define CELESTIAL_CAP_CUDA (1u << 0)
#define CELESTIAL_CAP_BARNES_HUT (1u << 1)
#define CELESTIAL_CAP_YOSHIDA4 (1u << 2)
#define CELESTIAL_CAP_POST_NEWTONIAN (1u << 3)
#define CELESTIAL_CAP_GPU_TREE (1u << 4)
#define CELESTIAL_CAP_GPU_MERGE (1u << 5)
#define CELESTIAL_CAP_ADAPTIVE_DT (1u << 6)
#define CELESTIAL_CAP_DETERMINISTIC (1u << 7)
NB_API uint32_t celestial_query_capabilities(void);
/* Empty string when the last call succeeded. */
NB_API const char* celestial_get_last_error_message(void);

#ifdef __cplusplus
}
#endif

#endif /* CELESTIAL_COMPAT_H */
