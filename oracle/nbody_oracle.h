/*
 * nbody_oracle.h - CPU restatement of the reference's force-path arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * engine: tests, the smoke check and the CPU-baseline leg of the benchmark
 * call it.  The engine never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the reference project root).
 */
#ifndef NBODY_ORACLE_H
#define NBODY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Direct sum, CpuParallelBackend.ComputeForces + GravityKernel. */
void or_direct_forces(int32_t n, const double* px, const double* py, const double* pz,
                      const double* m, const double* radius, const uint8_t* active,
                      double eps, int32_t shell, double* ax, double* ay, double* az,
                      int32_t threads);
/* Same arithmetic for a list of target bodies only (ForceErrorAnalyzer samples). */
void or_direct_forces_targets(int32_t n, const double* px, const double* py, const double* pz,
                              const double* m, const double* radius, const uint8_t* active,
                              double eps, int32_t shell, int32_t n_t, const int32_t* targets,
                              double* ax, double* ay, double* az, int32_t threads);
/* Bounding box of active bodies (BarnesHutBackend.cs:150-170) -> min3,max3. */
void or_bbox(int32_t n, const double* px, const double* py, const double* pz,
             const uint8_t* active, double* out6);
/* Root cube from the bounding box (octree_builder.cpp:29-35, gpu_tree.cu:163-167). */
void or_cube_from_bbox(const double* bbox6, double* cube4);
/* Morton keys, morton_code_kernel semantics (morton_kernel.cu:11-76, morton.hpp:13-35). */
void or_morton_aabb(int32_t n, const double* px, const double* py, const double* pz,
                    const uint8_t* active, const double* bbox6, uint64_t* keys, int32_t* idx);
/* Octree-aligned keys in a cube: q = floor((p - (c - h)) / (2h) * 2^21). */
void or_morton_cube(int32_t n, const double* px, const double* py, const double* pz,
                    const uint8_t* active, const double* cube4, uint64_t* keys, int32_t* idx);
uint64_t or_expand_bits_21(uint64_t v);
/* Stable LSD sort of (key, value) by key (the intended semantics of
 * launch_radix_sort, morton_kernel.cu:185-230). */
void or_stable_sort(int32_t n, uint64_t* keys, int32_t* values);

/* Point-region octree by insertion (octree_builder.cpp:8-135,
 * octree_node.hpp:53-67).  Node arrays of capacity `cap`; returns the node
 * count or -1 when cap is too small.  children is 8 per node. */
int32_t or_octree_build(int32_t n, const double* px, const double* py, const double* pz,
                        const double* m, const uint8_t* active, double min_node_size,
                        int32_t cap, double* center4, double* mass, double* com3,
                        int32_t* children8, int32_t* body, uint8_t* is_leaf);
/* Barnes-Hut walk over that octree (barnes_hut_solver.cpp:11-30,230-286;
 * theta clamped to >= 0.2), plus the shell theorem at leaves when `shell`
 * (BarnesHutBackend.cs:392-459). */
void or_bh_forces(int32_t n, const double* px, const double* py, const double* pz,
                  const double* radius, const uint8_t* active, double eps, double theta,
                  int32_t shell, const double* center4, const double* mass, const double* com3,
                  const int32_t* children8, const int32_t* body, const uint8_t* is_leaf,
                  double* ax, double* ay, double* az, int32_t threads);

/* Compaction destination rows (compact_kernel.cu:31-40 mask + exclusive scan). */
int32_t or_compact_indices(int32_t n, const uint8_t* active, const double* mass, int32_t* dest);

/* All overlapping pairs (lo, hi), lo < hi, sorted (collision_kernel.cu:40-52
 * overlap test; CollisionResolver::sort_pairs order).  Returns the count
 * (pairs beyond max_pairs are counted, not written). */
int32_t or_broad_phase_parallel(int32_t n, const double* px, const double* py, const double* pz,
                                const double* radius, const uint8_t* active,
                                const uint8_t* collidable, int32_t max_pairs, int32_t* lo,
                                int32_t* hi, int32_t threads);
int32_t or_broad_phase(int32_t n, const double* px, const double* py, const double* pz,
                       const double* radius, const uint8_t* active, const uint8_t* collidable,
                       int32_t max_pairs, int32_t* lo, int32_t* hi);
/* Sequential merge of sorted pairs (collision_resolver.cpp:20-100,190-250;
 * density_model.cpp).  Returns merges performed. */
int32_t or_resolve_merges(int32_t n, double* px, double* py, double* pz, double* vx,
                          double* vy, double* vz, double* m, double* radius, double* density,
                          uint8_t* active, int32_t n_pairs, const int32_t* lo, const int32_t* hi,
                          int32_t max_per_frame, int32_t max_per_body, int32_t density_merge,
                          double min_radius);

/* Velocity Verlet with direct-sum forces (SoAVerletIntegrator.cs:48-116). */
/* Direct sums in the other reference backends' orders (see nbody_oracle.c):
 * order 0 CpuParallelBackend, 1 SimdSingleThreadBackend (= the native
 * engine's CPU brute force), 2 CpuSingleThreadBackend. */
void or_direct_forces_simd(int32_t n, const double* px, const double* py, const double* pz,
                           const double* m, const double* radius, const uint8_t* active,
                           double eps, int32_t shell, double* ax, double* ay, double* az,
                           int32_t threads);
void or_direct_forces_pairwise(int32_t n, const double* px, const double* py, const double* pz,
                               const double* m, const double* radius, const uint8_t* active,
                               double eps, int32_t shell, double* ax, double* ay, double* az);
void or_direct_forces_order(int32_t n, const double* px, const double* py, const double* pz,
                            const double* m, const double* radius, const uint8_t* active,
                            double eps, int32_t shell, int32_t order, double* ax, double* ay,
                            double* az, int32_t threads);
void or_verlet_direct_order(int32_t n, double* px, double* py, double* pz, double* vx,
                            double* vy, double* vz, double* ax, double* ay, double* az,
                            const double* m, const uint8_t* active, double eps, double dt,
                            int32_t steps, int32_t order, int32_t threads);
void or_yoshida_direct_order(int32_t n, double* px, double* py, double* pz, double* vx,
                             double* vy, double* vz, double* ax, double* ay, double* az,
                             const double* m, const uint8_t* active, double eps, double dt,
                             int32_t steps, int32_t order, int32_t threads);
void or_energy_tracker(int32_t n, const double* px, const double* py, const double* pz,
                       const double* vx, const double* vy, const double* vz, const double* m,
                       const uint8_t* active, double eps, double* o);
void or_verlet_direct(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                      double* vz, double* ax, double* ay, double* az, const double* m,
                      const uint8_t* active, double eps, double dt, int32_t steps,
                      int32_t threads);
/* Yoshida4 steps: three Verlet sub-steps of w1 dt, w0 dt, w1 dt
 * (engine/src/sim/engine.cpp:685-746,1057-1066; yoshida.hpp:19-24). */
void or_yoshida_direct(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                       double* vz, double* ax, double* ay, double* az, const double* m,
                       const uint8_t* active, double eps, double dt, int32_t steps,
                       int32_t threads);
/* The adaptive dt after a step (adaptive_timestep.cpp:12-17, engine.cpp:491-501). */
double or_adaptive_dt(int32_t n, const double* ax, const double* ay, const double* az,
                      const uint8_t* active, double eps, double eta, double dt_min,
                      double dt_max);
/* KE, PE, E, P[3], L[3], COM[3], M (EnergyCalculator.cs:16-78,
 * NewtonianGravity.cs:68-77). */
void or_energy(int32_t n, const double* px, const double* py, const double* pz,
               const double* vx, const double* vy, const double* vz, const double* m,
               const uint8_t* active, double eps, double* out13, int32_t threads);
/* ForceErrorAnalyzer.CompareForces per-body relative error statistics
 * (ForceErrorAnalyzer.cs:100-134) -> mean, max, rms; returns count. */
int32_t or_force_error(int32_t n, const double* ax, const double* ay, const double* az,
                       const double* rx, const double* ry, const double* rz,
                       const uint8_t* active, double* out3);

#ifdef __cplusplus
}
#endif
#endif
