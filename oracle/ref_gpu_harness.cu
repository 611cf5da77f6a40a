// ref_gpu_harness.cu - extern "C" wrappers over two of the reference's own
// CUDA kernels, compiled in place for sm_100a by oracle/Makefile into
// oracle/_ref/libcelestial_ref_gpu.so:
//   launch_gravity_kernel  engine/src/cuda/gravity_kernel.cu:20-95, 278-295
//                          (tiled FP64 all-pairs gravity, 256-thread tiles)
//   launch_radix_sort      engine/src/cuda/morton_kernel.cu:87-230
//                          (16 passes of 4 bits over (u64 key, i32 value))
//
// BASELINE AND TEST INFRASTRUCTURE ONLY: the reference's GPU path timed on
// the same B200 as the engine, and the record of what its radix sort does
// with a given input.  Nothing in the engine links it.  Device buffers are
// allocated here per call (this is not a hot path).
#include <cuda_runtime.h>

#include <celestial/cuda/morton.hpp>

#include <cstdint>

namespace celestial::cuda {
// defined in engine/src/cuda/gravity_kernel.cu (declared by its callers)
void launch_gravity_kernel(double* d_pos_x, double* d_pos_y, double* d_pos_z, double* d_mass,
                           uint8_t* d_is_active, double* d_acc_x, double* d_acc_y,
                           double* d_acc_z, int32_t n, double softening, cudaStream_t stream);
}  // namespace celestial::cuda

namespace {

struct Buffers {
    void* p[16] = {};
    int k = 0;
    template <typename T>
    T* alloc(size_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
        p[k++] = q;
        return (T*)q;
    }
    ~Buffers() {
        for (int i = 0; i < k; i++) cudaFree(p[i]);
    }
};

}  // namespace

extern "C" {

// The reference's FP64 gravity kernel on the current device: `reps` timed
// launches after one warm-up, CUDA events; accelerations of the last launch.
// Returns 0, or -1 on a CUDA error or a reference exception.
int32_t ref_gpu_gravity(int32_t n, const double* px, const double* py, const double* pz,
                        const double* mass, const uint8_t* active, double eps, int32_t reps,
                        double* ax, double* ay, double* az, double* ms_per_launch) {
    try {
        Buffers b;
        double *dx = b.alloc<double>(n), *dy = b.alloc<double>(n), *dz = b.alloc<double>(n);
        double *dm = b.alloc<double>(n), *ox = b.alloc<double>(n), *oy = b.alloc<double>(n);
        double* oz = b.alloc<double>(n);
        uint8_t* da = b.alloc<uint8_t>(n);
        if (!dx || !dy || !dz || !dm || !ox || !oy || !oz || !da) return -1;
        const size_t d = sizeof(double) * (size_t)n;
        cudaMemcpy(dx, px, d, cudaMemcpyHostToDevice);
        cudaMemcpy(dy, py, d, cudaMemcpyHostToDevice);
        cudaMemcpy(dz, pz, d, cudaMemcpyHostToDevice);
        cudaMemcpy(dm, mass, d, cudaMemcpyHostToDevice);
        cudaMemcpy(da, active, (size_t)n, cudaMemcpyHostToDevice);
        cudaMemset(ox, 0, d);
        cudaMemset(oy, 0, d);
        cudaMemset(oz, 0, d);
        celestial::cuda::launch_gravity_kernel(dx, dy, dz, dm, da, ox, oy, oz, n, eps, nullptr);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        for (int r = 0; r < reps; r++)
            celestial::cuda::launch_gravity_kernel(dx, dy, dz, dm, da, ox, oy, oz, n, eps, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_per_launch) *ms_per_launch = reps > 0 ? ms / reps : 0.0;
        cudaMemcpy(ax, ox, d, cudaMemcpyDeviceToHost);
        cudaMemcpy(ay, oy, d, cudaMemcpyDeviceToHost);
        cudaMemcpy(az, oz, d, cudaMemcpyDeviceToHost);
        return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

// The reference's radix sort of (key, value) pairs in place, timed once
// (CUDA events).  Returns 0, or -1 on a CUDA error or a reference exception.
int32_t ref_gpu_radix_sort(int32_t n, uint64_t* keys, int32_t* values, double* ms) {
    try {
        Buffers b;
        uint64_t *k0 = b.alloc<uint64_t>(n), *k1 = b.alloc<uint64_t>(n);
        int32_t *v0 = b.alloc<int32_t>(n), *v1 = b.alloc<int32_t>(n);
        int32_t* hist = b.alloc<int32_t>(celestial::cuda::radix_sort_histogram_bytes(n) / 4 + 1);
        int32_t* offs = b.alloc<int32_t>(celestial::cuda::radix_sort_offset_bytes() / 4 + 1);
        if (!k0 || !k1 || !v0 || !v1 || !hist || !offs) return -1;
        cudaMemcpy(k0, keys, sizeof(uint64_t) * (size_t)n, cudaMemcpyHostToDevice);
        cudaMemcpy(v0, values, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        celestial::cuda::launch_radix_sort(k0, v0, n, k1, v1, hist, offs, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
        cudaMemcpy(keys, k0, sizeof(uint64_t) * (size_t)n, cudaMemcpyDeviceToHost);
        cudaMemcpy(values, v0, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost);
        return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
