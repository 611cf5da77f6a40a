// ref_engine.cpp - extern "C" wrappers over the reference's own simulation
// Engine (engine/src/sim/engine.cpp) and EnergyTracker
// (engine/src/profile/energy_tracker.cpp), compiled in place by
// oracle/Makefile into oracle/_ref/libcelestial_ref.so.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle's FP64 direct sum, Verlet and
// Yoshida4 steps, adaptive time step and energy restatements, and the
// celestial_* compatibility layer, to the reference's running CPU code.
//
// The reference's host code is compiled with g++, so CELESTIAL_HAS_CUDA is 0
// (engine/include/celestial/core/platform.hpp:31-42) and the Engine's GPU
// members are compiled out.  The reference ships its device context and its
// asynchronous GPU pipeline only as .cu sources written for a CUDA build; a
// host-only build has no definition of them.  This file supplies the two
// pieces a host-only link needs:
//   * cuda::DeviceContext reporting "no CUDA device", so Engine::init
//     (engine.cpp:64-98) takes its CPU paths: dc.has_cuda() is false and
//     no GPU subsystem is initialised;
//   * sim::AsyncPipeline members that throw if ever called; only the GPU
//     brute-force path calls them, and it is never selected here.
#include <celestial/cuda/device_context.hpp>
#include <celestial/profile/energy_tracker.hpp>
#include <celestial/sim/async_pipeline.hpp>
#include <celestial/sim/engine.hpp>

#include <cstdint>
#include <vector>

using namespace celestial;

namespace celestial::cuda {

DeviceContext& DeviceContext::instance() {
    static DeviceContext ctx;
    return ctx;
}

DeviceContext::~DeviceContext() = default;

void DeviceContext::init() {
    initialized_ = true;
    has_cuda_ = false;
}

void DeviceContext::shutdown() { initialized_ = false; }

}  // namespace celestial::cuda

namespace celestial::sim {

namespace {
[[noreturn]] void no_gpu_pipeline() {
    throw core::CelestialException(core::ErrorCode::CudaError,
                                   "host-only reference build: no GPU pipeline");
}
}  // namespace

void AsyncPipeline::init(i32) { no_gpu_pipeline(); }
void AsyncPipeline::destroy() {}
void AsyncPipeline::submit_step(const physics::ParticleSystem&, double, double, bool) {
    no_gpu_pipeline();
}
void AsyncPipeline::retrieve_results(physics::ParticleSystem&) { no_gpu_pipeline(); }

}  // namespace celestial::sim

namespace {

struct EngineRun {
    sim::Engine eng;
    int32_t n = 0;
};

// Engine::init with the settings the harness exposes; everything else keeps
// SimulationConfig's defaults (engine/include/celestial/sim/simulation_config.hpp).
void init_engine(sim::Engine& eng, int32_t n, int32_t compute_mode, int32_t integrator,
                 double theta, double dt, double eps, int32_t adaptive, double eta,
                 double dt_min, double dt_max, double initial_dt) {
    sim::SimulationConfig cfg;
    cfg.max_particles = n > 16 ? n : 16;
    cfg.compute_mode = static_cast<sim::SimulationConfig::ComputeMode>(compute_mode);
    cfg.integrator = integrator == 1 ? sim::IntegratorType::Yoshida4
                                     : sim::IntegratorType::Leapfrog_KDK;
    cfg.theta = theta;
    cfg.dt = dt;
    cfg.softening = eps;
    cfg.adaptive_dt.enabled = adaptive != 0;
    cfg.adaptive_dt.eta = eta;
    cfg.adaptive_dt.dt_min = dt_min;
    cfg.adaptive_dt.dt_max = dt_max;
    cfg.adaptive_dt.initial_dt = initial_dt;
    eng.init(cfg);
    if (adaptive) {
        sim::AdaptiveTimestepConfig a = cfg.adaptive_dt;
        eng.set_adaptive_timestep(a);
    }
}

void read_back(const sim::Engine& eng, int32_t n, double* px, double* py, double* pz,
               double* vx, double* vy, double* vz, double* ax, double* ay, double* az) {
    eng.get_positions(px, py, pz, n);
    eng.get_velocities(vx, vy, vz, n);
    eng.get_accelerations(ax, ay, az, n);
}

}  // namespace

extern "C" {

// Engine::set_particles + `steps` x Engine::step(dt, eps) (engine.cpp:162-311)
// in compute mode 0 (CPU_BruteForce) or 1 (CPU_BarnesHut), integrator 0
// (Leapfrog_KDK) or 1 (Yoshida4).  The state arrays are read as the initial
// state (acc doubles as old_acc, as set_particles copies it) and receive
// the final one.  Returns 0, or -1 when the reference threw.
int32_t ref_engine_steps(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                         double* vz, double* ax, double* ay, double* az, const double* m,
                         const double* radius, const uint8_t* active, int32_t compute_mode,
                         int32_t integrator, double theta, double dt, double eps,
                         int32_t steps) {
    try {
        EngineRun r;
        init_engine(r.eng, n, compute_mode, integrator, theta, dt, eps, 0, 0.01, 1e-8, 0.01,
                    0.001);
        std::vector<double> rad(radius ? radius : px, (radius ? radius : px) + n);
        if (!radius) rad.assign((size_t)n, 0.0);
        r.eng.set_particles(px, py, pz, vx, vy, vz, ax, ay, az, m, rad.data(), active, n);
        for (int32_t s = 0; s < steps; s++) r.eng.step(dt, eps);
        read_back(r.eng, n, px, py, pz, vx, vy, vz, ax, ay, az);
        r.eng.shutdown();
        return 0;
    } catch (...) {
        return -1;
    }
}

// `frames` x Engine::update(frame_time) (engine.cpp:313-327: the fixed-step
// accumulator, with the adaptive time step when `adaptive`), CPU_BruteForce
// or CPU_BarnesHut.  steps_out[f] receives the steps frame f took and
// dt_out (may be NULL) the adaptive dt after the last frame.  Returns 0 or -1.
int32_t ref_engine_update(int32_t n, double* px, double* py, double* pz, double* vx,
                          double* vy, double* vz, double* ax, double* ay, double* az,
                          const double* m, const uint8_t* active, int32_t compute_mode,
                          int32_t integrator, double theta, double dt, double eps,
                          int32_t adaptive, double eta, double dt_min, double dt_max,
                          double initial_dt, double frame_time, int32_t frames,
                          int32_t* steps_out, double* dt_out) {
    try {
        EngineRun r;
        init_engine(r.eng, n, compute_mode, integrator, theta, dt, eps, adaptive, eta, dt_min,
                    dt_max, initial_dt);
        std::vector<double> rad((size_t)n, 0.0);
        r.eng.set_particles(px, py, pz, vx, vy, vz, ax, ay, az, m, rad.data(), active, n);
        for (int32_t f = 0; f < frames; f++) {
            const int k = r.eng.update(frame_time);
            if (steps_out) steps_out[f] = k;
        }
        if (dt_out) *dt_out = r.eng.current_adaptive_dt();
        read_back(r.eng, n, px, py, pz, vx, vy, vz, ax, ay, az);
        r.eng.shutdown();
        return 0;
    } catch (...) {
        return -1;
    }
}

// EnergyTracker::compute (engine/src/profile/energy_tracker.cpp:8-90).
// out13: KE, PE, E, Px, Py, Pz, Lx, Ly, Lz, COMx, COMy, COMz, M.
void ref_energy_tracker(int32_t n, const double* px, const double* py, const double* pz,
                        const double* vx, const double* vy, const double* vz, const double* m,
                        const uint8_t* active, double eps, double* out13) {
    profile::EnergyTracker tracker;
    const profile::EnergyTracker::Snapshot s =
        tracker.compute(px, py, pz, vx, vy, vz, m, active, n, eps);
    double M = 0.0;
    for (int32_t i = 0; i < n; i++)
        if (active[i]) M += m[i];
    const double o[13] = {s.kinetic_energy, s.potential_energy, s.total_energy, s.momentum_x,
                          s.momentum_y,     s.momentum_z,       s.angular_momentum_x,
                          s.angular_momentum_y, s.angular_momentum_z, s.com_x, s.com_y,
                          s.com_z, M};
    for (int k = 0; k < 13; k++) out13[k] = o[k];
}

}  // extern "C"
