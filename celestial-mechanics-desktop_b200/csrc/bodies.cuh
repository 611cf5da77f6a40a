// bodies.cuh - per-body kernels: Verlet kicks, bounding box, Morton keys,
// gathers into Morton order.
#pragma once
#include "common.cuh"

namespace nb {

// Device structure-of-arrays, the BodySoA fields of the force path
// (src/CelestialMechanics.Physics/SoA/BodySoA.cs:39-175), rows in the
// caller's order (compaction keeps the order).
struct State {
    double *px, *py, *pz, *vx, *vy, *vz, *ax, *ay, *az;
    double *mass, *radius, *density;
    uint8_t *active, *collidable;
    int32_t* ids;  // original body index of each row
};

// Every launcher's optional `dn` is a device row count that replaces n when
// smaller (the grid stays sized for n): a captured step whose rows shrink
// after each compaction reads its current row count there.
// bbox_ord: 6 order-mapped words (min xyz, max xyz), reset to (~0, 0)
// before the kernel.  n_active: active count (reset to 0).
void launch_kick_drift_bbox(cudaStream_t st, int n, State s, bool kick, double dt,
                            unsigned long long* bbox_ord, int* n_active, int* err,
                            const int* dn = nullptr);
void launch_kick(cudaStream_t st, int n, State s, double dt, const int* dn = nullptr);
// Cube (cx, cy, cz, half) from the bbox words (gpu_tree.cu:163-167), or a
// given cube when `given` is non-null.
void launch_cube(cudaStream_t st, const unsigned long long* bbox_ord, const double* given,
                 double* cube);
// Octree-aligned keys in the cube + all 8 digit histograms (hist zeroed).
// Optionally, by row: rows = (x, y, z, m) and amag = |acc| (the previous
// step's acceleration), for launch_gather.
void launch_keys_cube(cudaStream_t st, int n, const State& s, const double* cube,
                      uint64_t* keys, uint32_t* vals, uint32_t* hist, double4* rows = nullptr,
                      float* amag = nullptr, const int* dn = nullptr);
// Reference keys: per-axis AABB, scale 2^21-1 (morton_kernel.cu:11-76).
void launch_keys_aabb(cudaStream_t st, int n, const State& s,
                      const unsigned long long* bbox_ord, uint64_t* keys, uint32_t* vals);
// Gather the first n sorted rows: sbody = (x, y, z, m), srad = radius,
// samag = |acc| (optional; the previous step's acceleration).  With `rows`
// (and `amag` for samag) from launch_keys_cube, each body's record is read
// whole instead of field by field.
void launch_gather(cudaStream_t st, int n, const State& s, const uint32_t* sidx,
                   double4* sbody, float* srad, float* samag = nullptr,
                   const double4* rows = nullptr, const float* amag = nullptr,
                   const int* dn = nullptr);
// Zero acc of all rows (inactive rows keep 0).
void launch_zero_acc(cudaStream_t st, int n, State s, const int* dn = nullptr);

}  // namespace nb
