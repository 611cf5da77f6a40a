// ref_harness.cpp - extern "C" wrappers over the reference engine's own CPU
// code, compiled in place from the reference sources by oracle/Makefile into
// oracle/_ref/libcelestial_ref.so.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle restatement (nbody_oracle.c) to
// the reference itself and serves as the "reference" CPU baseline.  Nothing
// in the engine links it.
//
// Wrapped reference code:
//   OctreeBuilder::build        engine/src/physics/octree_builder.cpp:8-47
//   BarnesHutSolver::compute_forces  engine/src/physics/barnes_hut_solver.cpp:11-85
//   ParticleSystem::compact     engine/src/physics/particle_system.cpp:156-183
//   CollisionResolver::resolve  engine/src/physics/collision_resolver.cpp:20-100
//   morton_from_unit            engine/include/celestial/cuda/morton.hpp:29-35
#include <cuda_runtime.h>  // cudaStream_t in morton.hpp's launch declarations only

#include <celestial/cuda/morton.hpp>
#include <celestial/job/job_system.hpp>
#include <celestial/physics/barnes_hut_solver.hpp>
#include <celestial/physics/collision_resolver.hpp>
#include <celestial/physics/density_model.hpp>
#include <celestial/physics/octree_builder.hpp>
#include <celestial/physics/octree_pool.hpp>
#include <celestial/physics/particle_system.hpp>

#include <cstdint>
#include <cstring>
#include <vector>

using namespace celestial;

namespace {

void load_particles(physics::ParticleSystem& ps, int32_t n, const double* px, const double* py,
                    const double* pz, const double* m, const uint8_t* active) {
    ps.allocate(n > 0 ? n : 1);
    ps.set_count(n);
    for (int32_t i = 0; i < n; i++) {
        ps.pos_x[i] = px[i];
        ps.pos_y[i] = py[i];
        ps.pos_z[i] = pz[i];
        ps.mass[i] = m ? m[i] : 1.0;
        ps.is_active[i] = active[i];
        ps.is_collidable[i] = 1;
    }
}

void ensure_jobs(int32_t threads) {
    auto& js = job::JobSystem::instance();
    if (!js.is_initialized()) js.init(threads > 0 ? threads : -1);
}

}  // namespace

extern "C" {

uint64_t ref_morton_from_unit(double ux, double uy, double uz) {
    return cuda::morton_from_unit(ux, uy, uz);
}

// Returns the node count, or -1 when cap is too small.  Node order is the
// reference pool's allocation order; root is node 0.
int32_t ref_octree_build(int32_t n, const double* px, const double* py, const double* pz,
                         const double* m, const uint8_t* active, double min_node_size,
                         int32_t cap, double* center4, double* mass, double* com3,
                         int32_t* children8, int32_t* body, uint8_t* is_leaf) {
    physics::ParticleSystem ps;
    load_particles(ps, n, px, py, pz, m, active);
    physics::OctreePool pool;
    physics::OctreeBuilder builder;
    builder.min_node_size = min_node_size;
    int32_t root = builder.build(pool, ps);
    if (root < 0) return 0;
    int32_t count = pool.count();
    if (count > cap) return -1;
    for (int32_t k = 0; k < count; k++) {
        const physics::OctreeNode& nd = pool[k];
        center4[4 * k + 0] = nd.center_x;
        center4[4 * k + 1] = nd.center_y;
        center4[4 * k + 2] = nd.center_z;
        center4[4 * k + 3] = nd.half_size;
        mass[k] = nd.total_mass;
        com3[3 * k + 0] = nd.com_x;
        com3[3 * k + 1] = nd.com_y;
        com3[3 * k + 2] = nd.com_z;
        for (int o = 0; o < 8; o++) children8[8 * k + o] = nd.children[o];
        body[k] = nd.body_index;
        is_leaf[k] = nd.is_leaf;
    }
    return count;
}

// BarnesHutSolver::compute_forces (monopole, theta clamped to >= 0.2).
// Returns the traversal time in ms as measured by the solver itself.
double ref_bh_forces(int32_t n, const double* px, const double* py, const double* pz,
                     const double* m, const uint8_t* active, double eps, double theta,
                     int32_t parallel, int32_t threads, double* ax, double* ay, double* az,
                     double* build_ms) {
    physics::ParticleSystem ps;
    load_particles(ps, n, px, py, pz, m, active);
    physics::BarnesHutSolver bh;
    bh.theta = theta;
    bh.use_parallel = parallel != 0;
    if (bh.use_parallel) ensure_jobs(threads);
    bh.compute_forces(ps, eps);
    std::memcpy(ax, ps.acc_x, sizeof(double) * n);
    std::memcpy(ay, ps.acc_y, sizeof(double) * n);
    std::memcpy(az, ps.acc_z, sizeof(double) * n);
    if (build_ms) *build_ms = bh.last_build_time_ms;
    return bh.last_traversal_time_ms;
}

// ParticleSystem::compact on (pos, vel, mass, active).  Arrays are rewritten
// in place; returns the new count.
int32_t ref_compact(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                    double* vz, double* m, uint8_t* active) {
    physics::ParticleSystem ps;
    load_particles(ps, n, px, py, pz, m, active);
    for (int32_t i = 0; i < n; i++) {
        ps.vel_x[i] = vx[i];
        ps.vel_y[i] = vy[i];
        ps.vel_z[i] = vz[i];
    }
    int32_t c = ps.compact();
    for (int32_t i = 0; i < c; i++) {
        px[i] = ps.pos_x[i]; py[i] = ps.pos_y[i]; pz[i] = ps.pos_z[i];
        vx[i] = ps.vel_x[i]; vy[i] = ps.vel_y[i]; vz[i] = ps.vel_z[i];
        m[i] = ps.mass[i];
        active[i] = ps.is_active[i];
    }
    return c;
}

// CollisionResolver::resolve in Merge mode over the given pairs.
int32_t ref_resolve_merges(int32_t n, double* px, double* py, double* pz, double* vx,
                           double* vy, double* vz, double* m, double* radius, double* density,
                           uint8_t* active, int32_t n_pairs, const int32_t* lo,
                           const int32_t* hi, int32_t max_per_frame, int32_t max_per_body,
                           int32_t density_merge, double min_radius) {
    physics::ParticleSystem ps;
    load_particles(ps, n, px, py, pz, m, active);
    for (int32_t i = 0; i < n; i++) {
        ps.vel_x[i] = vx[i]; ps.vel_y[i] = vy[i]; ps.vel_z[i] = vz[i];
        ps.radius[i] = radius[i];
        ps.density[i] = density ? density[i] : 0.0;
    }
    physics::CollisionResolverConfig cfg;
    cfg.mode = physics::CollisionMode::Merge;
    cfg.max_merges_per_frame = max_per_frame;
    cfg.max_merges_per_body = max_per_body;
    cfg.density_preserving_merge = density_merge != 0;
    physics::DensityModel dm;
    physics::DensityConfig dcfg;
    dcfg.min_radius = min_radius;
    dm.configure(dcfg);
    physics::CollisionResolver res;
    res.configure(cfg);
    res.set_density_model(&dm);
    std::vector<physics::CollisionPair> pairs;
    pairs.reserve(n_pairs);
    for (int32_t k = 0; k < n_pairs; k++) pairs.push_back({lo[k], hi[k], 0.0});
    res.resolve(ps, pairs);
    for (int32_t i = 0; i < n; i++) {
        px[i] = ps.pos_x[i]; py[i] = ps.pos_y[i]; pz[i] = ps.pos_z[i];
        vx[i] = ps.vel_x[i]; vy[i] = ps.vel_y[i]; vz[i] = ps.vel_z[i];
        m[i] = ps.mass[i];
        radius[i] = ps.radius[i];
        if (density) density[i] = ps.density[i];
        active[i] = ps.is_active[i];
    }
    return res.last_merge_count();
}

}  // extern "C"
