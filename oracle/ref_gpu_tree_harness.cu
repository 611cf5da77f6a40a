// ref_gpu_tree_harness.cu - the reference's GPU Barnes-Hut force path,
// GpuTreeSolver::compute_forces (engine/src/cuda/gpu_tree.cu:112-193: bbox
// reduction, Morton codes, its radix sort, the single-thread tree insertion of
// :269-464, the per-body FP64 traversal of :508-597), timed on the B200 as
// the reference GPU baseline of the 2^20-body Barnes-Hut workload.
//
// BASELINE INFRASTRUCTURE ONLY: nothing in the engine links it.
//
// gpu_tree.cu does not link on its own: it declares five energy reductions
// `extern` inside an anonymous namespace (gpu_tree.cu:1195-1237), which no
// other translation unit can define.  This file includes gpu_tree.cu
// unchanged (its path comes from the build recipe as GPU_TREE_SRC) and defines
// those five in the same translation unit.  They belong to
// GpuTreeSolver::compute_gpu_energy, which the force path never calls; here
// they throw, so a call would fail loudly instead of returning numbers.
#include GPU_TREE_SRC

#include <vector>

namespace celestial::cuda {
namespace {

[[noreturn]] void energy_not_built() {
    throw core::CelestialException(core::ErrorCode::InvalidArgument,
                                   "reference energy reductions are not part of this harness",
                                   __FILE__, __LINE__);
}

void gpu_reduce_kinetic_energy(const double*, const double*, const double*, const double*,
                               const uint8_t*, int32_t, double*, double&, cudaStream_t) {
    energy_not_built();
}
void gpu_reduce_momentum(const double*, const double*, const double*, const double*,
                         const uint8_t*, int32_t, double*, double*, double*, double&, double&,
                         double&, cudaStream_t) {
    energy_not_built();
}
void gpu_reduce_angular_momentum(const double*, const double*, const double*, const double*,
                                 const double*, const double*, const double*, const uint8_t*,
                                 int32_t, double*, double*, double*, double&, double&, double&,
                                 cudaStream_t) {
    energy_not_built();
}
void gpu_reduce_com(const double*, const double*, const double*, const double*, const uint8_t*,
                    int32_t, double*, double*, double*, double*, double&, double&, double&,
                    double&, cudaStream_t) {
    energy_not_built();
}
void launch_gpu_potential_energy(const double*, const double*, const double*, const double*,
                                 const uint8_t*, int32_t, const double*, const double*,
                                 const double*, const double*, const double*, const int32_t*,
                                 const int32_t*, const uint8_t*, double, double, double*, double*,
                                 double&, cudaStream_t) {
    energy_not_built();
}

}  // namespace
}  // namespace celestial::cuda

extern "C" {

// GpuTreeSolver::compute_forces on the current device for n bodies at rest
// (velocities and radii 0): one untimed evaluation, then `reps` timed ones
// (CUDA events around each, on the solver's stream); accelerations of the
// last one, and the solver's own build / traversal split of the last one
// (host clock, as the reference records it).  Returns 0, or -1 on a CUDA
// error or a reference exception.
int32_t ref_gpu_tree(int32_t n, const double* px, const double* py, const double* pz,
                     const double* mass, const uint8_t* active, double eps, double theta,
                     int32_t reps, double* ax, double* ay, double* az, double* ms_per_eval,
                     double* build_ms, double* traverse_ms) {
    using celestial::cuda::GpuTreeSolver;
    using celestial::memory::GpuPool;
    try {
        cudaStream_t st = nullptr;
        if (cudaStreamCreate(&st) != cudaSuccess) return -1;
        int32_t rc = 0;
        {
            GpuPool pool;
            pool.init(n);
            std::vector<double> zero((size_t)n, 0.0);
            const double* z = zero.data();
            pool.upload_all(px, py, pz, z, z, z, z, z, z, z, z, z, mass, z, active, n, st);
            pool.set_count(n);
            GpuTreeSolver solver;
            solver.theta = theta;
            solver.init(n);
            solver.compute_forces(pool, n, eps, st);
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            double total = 0.0;
            for (int32_t r = 0; r < reps; r++) {
                cudaEventRecord(e0, st);
                solver.compute_forces(pool, n, eps, st);
                cudaEventRecord(e1, st);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                total += ms;
            }
            *ms_per_eval = reps > 0 ? total / reps : 0.0;
            *build_ms = solver.last_sort_time_ms + solver.last_build_time_ms;
            *traverse_ms = solver.last_traverse_time_ms;
            std::vector<double> vx((size_t)n), vy((size_t)n), vz((size_t)n);
            pool.download_state(zero.data(), vx.data(), vy.data(), vx.data(), vy.data(),
                                vz.data(), ax, ay, az, n, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            solver.destroy();
            pool.destroy();
        }
        cudaStreamDestroy(st);
        return rc;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
