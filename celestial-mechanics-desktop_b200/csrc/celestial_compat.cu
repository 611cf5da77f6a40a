// celestial_compat.cu - the reference's `celestial_*` native API on top of
// the nb_* engine (declarations and the differences in
// include/celestial_compat.h).
//
// The reference keeps one global Engine behind these functions
// (engine/src/interop/native_api.cpp:20-30); so does this file.  Every call
// maps onto the public nb_* functions: no kernel lives here.  Failures are
// recorded in the last-error string and otherwise ignored, as the reference's
// void functions swallow their exceptions (native_api.cpp:65-114).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/celestial_compat.h"

namespace {

// SimulationConfig's values that the subset uses (engine/include/celestial/
// sim/simulation_config.hpp:73-131), with the reference's defaults.
struct Config {
    double dt = 0.001;
    double softening = 1e-4;
    double theta = 0.5;
    int max_steps_per_frame = 10;
    int compute_mode = 2;  // GPU_BruteForce
    int integrator = 0;    // Leapfrog_KDK
    int collision_mode = 0;
    int max_merges_frame = 64;
    int max_merges_body = 2;
    int density_merge = 1;
    bool adaptive = false;
    double eta = 0.01, dt_min = 1e-8, dt_max = 0.01, initial_dt = 0.001;
};

struct Snapshot {
    double e = 0.0, px = 0.0, py = 0.0, pz = 0.0, lx = 0.0, ly = 0.0, lz = 0.0;
};

nb_engine* g_h = nullptr;
int g_capacity = 0;
Config g_config;  // what the next celestial_init uses (celestial_set_dt / _softening)
Config g_run;     // the running engine's settings
double g_adaptive_dt = 0.001;  // AdaptiveTimestep::current_dt_
double g_accumulator = 0.0;    // Timestep::accumulator
bool g_has_initial = false;
Snapshot g_initial, g_current;
double g_accumulated_error = 0.0;
char g_err[512] = {0};

void set_error(const char* msg) {
    std::snprintf(g_err, sizeof(g_err), "%s", msg ? msg : "");
}

// A failed nb_* call: keep its message.
bool failed(int32_t r, const char* what) {
    if (r == NB_OK) return false;
    const char* m = g_h ? nb_last_error(g_h) : "";
    std::snprintf(g_err, sizeof(g_err), "%s failed (%d): %s", what, r, m ? m : "");
    return true;
}

int32_t to_error_code(int32_t r) {
    switch (r) {
        case NB_OK: return CELESTIAL_OK;
        case NB_ERR_NO_DEVICE: return CELESTIAL_ERR_DEVICE_NOT_FOUND;
        case NB_ERR_INVALID_ARG: return CELESTIAL_ERR_INVALID_ARGUMENT;
        case NB_ERR_CAPACITY: return CELESTIAL_ERR_OUT_OF_MEMORY;
        case NB_ERR_CUDA: return CELESTIAL_ERR_CUDA;
        default: return -100;
    }
}

int mode_flags(const Config& c) {
    int f = 0;
    switch (c.compute_mode) {
        // the reference's CPU brute-force arithmetic and order
        // (Engine::compute_cpu_brute_forces, engine.cpp:649-674)
        case 0: case 2: f = NB_MODE_DIRECT_FP64 | NB_FLAG_ORDER_SIMD; break;
        case 1: f = NB_MODE_BARNES_HUT_REF; break;
        default: f = NB_MODE_BARNES_HUT; break;
    }
    if (c.integrator == 1) f |= NB_FLAG_YOSHIDA4;
    if (c.collision_mode == 3) f |= NB_FLAG_COLLISIONS;
    return f;
}

void apply_params(const Config& c) {
    nb_set_param_f64(g_h, NB_PARAM_THETA, c.theta);
    nb_set_param_i32(g_h, NB_PARAM_MAX_MERGES_FRAME, c.max_merges_frame);
    nb_set_param_i32(g_h, NB_PARAM_MAX_MERGES_BODY, c.max_merges_body);
    nb_set_param_i32(g_h, NB_PARAM_DENSITY_MERGE, c.density_merge);
}

// Engine::step (engine/src/sim/engine.cpp:200-300): one step, then the
// adaptive dt from the new accelerations (AdaptiveTimestep::update,
// engine/src/sim/adaptive_timestep.cpp:12-23).
void step_once(double dt, double softening) {
    if (failed(nb_step(g_h, 1, dt, softening, mode_flags(g_run)), "nb_step")) return;
    if (g_run.adaptive) {
        double a_max = 0.0;
        if (failed(nb_max_acceleration(g_h, &a_max), "nb_max_acceleration")) return;
        if (a_max <= 0.0 || softening <= 0.0) {
            g_adaptive_dt = g_run.dt_max;
        } else {
            const double dt_new = g_run.eta * std::sqrt(softening / a_max);
            g_adaptive_dt = std::clamp(dt_new, g_run.dt_min, g_run.dt_max);
        }
    }
    set_error(nullptr);
}

// One field triple of the device state (positions, velocities or
// accelerations) straight into the caller's arrays: nb_get_state skips the
// NULL outputs, so only these three arrays of n rows cross PCIe.
void copy_out(int which, double* a, double* b, double* c, int32_t count) {
    if (!g_h || !a || !b || !c || count <= 0) return;
    int32_t n = 0, na = 0;
    if (failed(nb_get_body_count(g_h, &n, &na), "nb_get_body_count")) return;
    if (count < n) {
        // the caller's arrays hold fewer rows than the state: stage through
        // host scratch of n rows and copy the first `count`
        std::vector<double> t[3];
        for (auto& v : t) v.resize((size_t)n);
        double* o[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr};
        for (int k = 0; k < 3; k++) o[3 * which + k] = t[k].data();
        if (failed(nb_get_state(g_h, nullptr, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7],
                                o[8], nullptr, nullptr, nullptr, nullptr),
                   "nb_get_state"))
            return;
        std::memcpy(a, t[0].data(), (size_t)count * sizeof(double));
        std::memcpy(b, t[1].data(), (size_t)count * sizeof(double));
        std::memcpy(c, t[2].data(), (size_t)count * sizeof(double));
    } else {
        double* o[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr};
        o[3 * which] = a;
        o[3 * which + 1] = b;
        o[3 * which + 2] = c;
        if (failed(nb_get_state(g_h, nullptr, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7],
                                o[8], nullptr, nullptr, nullptr, nullptr),
                   "nb_get_state"))
            return;
    }
    set_error(nullptr);
}

}  // namespace

extern "C" {

NB_API int32_t celestial_init(int32_t max_particles) {
    if (g_h) {
        set_error("Engine already initialized");
        return CELESTIAL_ERR_ALREADY_INITIALIZED;
    }
    nb_engine* h = nullptr;
    const int32_t r = nb_create(max_particles, 0, &h);
    if (r != NB_OK) {
        std::snprintf(g_err, sizeof(g_err), "nb_create failed (%d)", r);
        return to_error_code(r);
    }
    g_h = h;
    g_capacity = max_particles;
    g_run = g_config;
    g_adaptive_dt = g_run.initial_dt;
    g_accumulator = 0.0;
    g_has_initial = false;
    g_accumulated_error = 0.0;
    apply_params(g_run);
    set_error(nullptr);
    return CELESTIAL_OK;
}

NB_API void celestial_shutdown(void) {
    if (g_h) nb_destroy(g_h);
    g_h = nullptr;
    g_capacity = 0;
}

NB_API void celestial_set_particles(const double* pos_x, const double* pos_y,
                                    const double* pos_z, const double* vel_x,
                                    const double* vel_y, const double* vel_z,
                                    const double* acc_x, const double* acc_y,
                                    const double* acc_z, const double* mass,
                                    const double* radius, const uint8_t* is_active,
                                    int32_t count) {
    if (!g_h) return;
    const int32_t r = nb_set_state(g_h, count, pos_x, pos_y, pos_z, vel_x, vel_y, vel_z, mass,
                                   radius, nullptr, is_active, nullptr, acc_x, acc_y, acc_z);
    if (failed(r, "nb_set_state")) return;
    // a new scene restarts the energy tracker (Engine::set_particles calls
    // energy_tracker_.reset(), engine/src/sim/engine.cpp:195): drifts and the
    // accumulated error are measured from the next snapshot of this scene
    g_has_initial = false;
    g_initial = Snapshot{};
    g_current = Snapshot{};
    g_accumulated_error = 0.0;
    set_error(nullptr);
}

NB_API void celestial_get_accelerations(double* out_acc_x, double* out_acc_y,
                                        double* out_acc_z, int32_t count) {
    copy_out(2, out_acc_x, out_acc_y, out_acc_z, count);
}

NB_API void celestial_get_positions(double* out_pos_x, double* out_pos_y, double* out_pos_z,
                                    int32_t count) {
    copy_out(0, out_pos_x, out_pos_y, out_pos_z, count);
}

NB_API void celestial_get_velocities(double* out_vel_x, double* out_vel_y, double* out_vel_z,
                                     int32_t count) {
    copy_out(1, out_vel_x, out_vel_y, out_vel_z, count);
}

NB_API void celestial_compute_forces(double softening) {
    if (g_h) step_once(0.0, softening);
}

NB_API void celestial_step(double dt, double softening) {
    if (g_h) step_once(dt, softening);
}

NB_API int32_t celestial_update(double frame_time) {
    if (!g_h) return 0;
    double effective = g_run.adaptive ? g_adaptive_dt : g_run.dt;
    g_accumulator += frame_time;
    int steps = 0;
    while (g_accumulator >= g_run.dt && steps < g_run.max_steps_per_frame) {
        g_accumulator -= g_run.dt;
        steps++;
    }
    for (int i = 0; i < steps; i++) {
        step_once(effective, g_run.softening);
        if (g_run.adaptive) effective = g_adaptive_dt;
    }
    return steps;
}

NB_API void celestial_set_compute_mode(int32_t mode) {
    if (!g_h) return;
    if (mode < 0 || mode > 3) {
        set_error("compute mode must be 0..3");
        return;
    }
    g_run.compute_mode = g_config.compute_mode = mode;
}

NB_API void celestial_set_theta(double theta) {
    if (!g_h) return;
    if (failed(nb_set_param_f64(g_h, NB_PARAM_THETA, theta), "set theta")) return;
    g_run.theta = g_config.theta = theta;
}

NB_API void celestial_set_dt(double dt) {
    if (g_h) g_config.dt = dt;
}

NB_API void celestial_set_softening(double softening) {
    if (g_h) g_config.softening = softening;
}

NB_API void celestial_set_integrator(int32_t type) {
    if (!g_h) return;
    g_run.integrator = g_config.integrator = type == 1 ? 1 : 0;
}

NB_API int32_t celestial_get_integrator(void) { return g_h ? g_run.integrator : 0; }

NB_API void celestial_set_adaptive_timestep(int32_t enabled, double eta, double dt_min,
                                            double dt_max, double initial_dt) {
    if (!g_h) return;
    g_run.adaptive = enabled != 0;
    g_run.eta = eta;
    g_run.dt_min = dt_min;
    g_run.dt_max = dt_max;
    g_run.initial_dt = initial_dt;
    g_adaptive_dt = initial_dt;  // AdaptiveTimestep::configure
    g_config.adaptive = g_run.adaptive;
    g_config.eta = eta;
    g_config.dt_min = dt_min;
    g_config.dt_max = dt_max;
    g_config.initial_dt = initial_dt;
}

NB_API double celestial_get_adaptive_dt(void) { return g_h ? g_adaptive_dt : 0.0; }

NB_API int32_t celestial_is_adaptive_dt_enabled(void) { return g_h && g_run.adaptive ? 1 : 0; }

NB_API void celestial_compute_energy_snapshot(void) {
    if (!g_h) return;
    int32_t n = 0, na = 0;
    nb_get_body_count(g_h, &n, &na);
    const bool tree = n > 256 && (g_run.compute_mode == 1 || g_run.compute_mode == 3);
    double out[13];
    if (failed(nb_diagnostics(g_h, g_run.softening, tree ? 1 : 0, out), "nb_diagnostics")) return;
    Snapshot s;
    s.e = out[2];
    s.px = out[3]; s.py = out[4]; s.pz = out[5];
    s.lx = out[6]; s.ly = out[7]; s.lz = out[8];
    if (!g_has_initial) {
        g_initial = s;
        g_has_initial = true;
    }
    g_current = s;
    g_accumulated_error += std::abs(celestial_get_energy_drift());
    set_error(nullptr);
}

NB_API double celestial_get_energy_drift(void) {
    if (!g_h || !g_has_initial || g_initial.e == 0.0) return 0.0;
    return (g_current.e - g_initial.e) / std::abs(g_initial.e);
}

NB_API double celestial_get_momentum_drift(void) {
    if (!g_h || !g_has_initial) return 0.0;
    const double dx = g_current.px - g_initial.px, dy = g_current.py - g_initial.py,
                 dz = g_current.pz - g_initial.pz;
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

NB_API double celestial_get_angular_momentum_drift(void) {
    if (!g_h || !g_has_initial) return 0.0;
    const double dx = g_current.lx - g_initial.lx, dy = g_current.ly - g_initial.ly,
                 dz = g_current.lz - g_initial.lz;
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

NB_API double celestial_get_accumulated_error(void) { return g_h ? g_accumulated_error : 0.0; }

NB_API double celestial_get_last_gpu_time_ms(void) {
    double t[NB_T_COUNT] = {0};
    if (!g_h || nb_get_timings(g_h, t, NB_T_COUNT) != NB_OK) return 0.0;
    return t[NB_T_TOTAL];
}

NB_API double celestial_get_last_tree_build_ms(void) {
    double t[NB_T_COUNT] = {0};
    if (!g_h || nb_get_timings(g_h, t, NB_T_COUNT) != NB_OK) return 0.0;
    return t[NB_T_BUILD];
}

NB_API double celestial_get_last_tree_traverse_ms(void) {
    double t[NB_T_COUNT] = {0};
    if (!g_h || nb_get_timings(g_h, t, NB_T_COUNT) != NB_OK) return 0.0;
    return t[NB_T_TRAVERSAL];
}

NB_API int32_t celestial_get_particle_count(void) {
    int32_t n = 0, na = 0;
    if (!g_h || nb_get_body_count(g_h, &n, &na) != NB_OK) return 0;
    return n;
}

NB_API int32_t celestial_get_active_particle_count(void) {
    int32_t n = 0, na = 0;
    if (!g_h || nb_get_body_count(g_h, &n, &na) != NB_OK) return 0;
    return na;
}

NB_API int32_t celestial_get_last_merge_count(void) {
    int64_t c[NB_C_COUNT] = {0};
    if (!g_h || nb_get_counters(g_h, c, NB_C_COUNT) != NB_OK) return 0;
    return (int32_t)c[NB_C_MERGES];
}

NB_API void celestial_set_collision_mode(int32_t mode) {
    if (!g_h) return;
    if (mode != 0 && mode != 3) {
        set_error("collision mode not supported: only Ignore (0) and Merge (3)");
        return;
    }
    g_run.collision_mode = g_config.collision_mode = mode;
    set_error(nullptr);
}

NB_API void celestial_set_max_merges_per_frame(int32_t max_merges) {
    if (!g_h) return;
    if (!failed(nb_set_param_i32(g_h, NB_PARAM_MAX_MERGES_FRAME, max_merges), "set max merges"))
        g_run.max_merges_frame = g_config.max_merges_frame = max_merges;
}

NB_API void celestial_set_max_merges_per_body(int32_t max_merges) {
    if (!g_h) return;
    if (!failed(nb_set_param_i32(g_h, NB_PARAM_MAX_MERGES_BODY, max_merges), "set max merges"))
        g_run.max_merges_body = g_config.max_merges_body = max_merges;
}

NB_API void celestial_set_density_preserving_merge(int32_t enabled) {
    if (!g_h) return;
    const int v = enabled != 0;
    if (!failed(nb_set_param_i32(g_h, NB_PARAM_DENSITY_MERGE, v), "set density merge"))
        g_run.density_merge = g_config.density_merge = v;
}

NB_API CelestialVersion celestial_api_version(void) {
    CelestialVersion v;
    v.major = CELESTIAL_API_VERSION_MAJOR;
    v.minor = CELESTIAL_API_VERSION_MINOR;
    v.patch = CELESTIAL_API_VERSION_PATCH;
    return v;
}

NB_API uint32_t celestial_query_capabilities(void) {
    return CELESTIAL_CAP_CUDA | CELESTIAL_CAP_BARNES_HUT | CELESTIAL_CAP_YOSHIDA4 |
           CELESTIAL_CAP_GPU_TREE | CELESTIAL_CAP_GPU_MERGE | CELESTIAL_CAP_ADAPTIVE_DT |
           CELESTIAL_CAP_DETERMINISTIC;
}

NB_API const char* celestial_get_last_error_message(void) { return g_err; }

}  // extern "C"
