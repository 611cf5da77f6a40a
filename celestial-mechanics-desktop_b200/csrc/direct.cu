// direct.cu - softened O(n^2) direct sums.
//
// k_direct_fp64_pairs restates CpuParallelBackend.ComputeForces
// (src/CelestialMechanics.Physics/Solvers/CpuParallelBackend.cs:99-142) with
// GravityKernel.AccelerationCoeffFromSource (GravityKernel.cs:9-33): every
// FP64 operation rounded exactly as the C# code rounds it (no FMA
// contraction) and every target's terms summed in source-row order, so its
// output is bit-identical to that backend's.  It also
// replaces the reference GPU gravity_kernel (engine/src/cuda/gravity_kernel.cu:
// 20-95), which loads inactive sources with their real mass.
//
// k_direct_fp32 is the throughput kernel: Morton-sorted targets, j-tiles of
// bodies staged in shared memory as FP32 coordinates differenced in FP64
// against the block's reference body, two targets per thread so every
// broadcast shared-memory read feeds two pair evaluations, and a Kahan fold
// of each tile's FP32 partial sum.
#include "direct.cuh"

namespace nb {

constexpr int kD32Threads = 256;
constexpr int kD32Per = 2;  // targets per thread
constexpr int kD32Tile = kD32Threads;

__device__ __forceinline__ void kahan32(float& s, float& c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Targets and sources are the n sorted bodies (all active).  Block b handles
// targets [b*512, b*512+512); its reference point is its first body.  The
// self pair has dx = dy = dz = 0 and contributes 0 when eps > 0; GUARD (used
// when eps == 0) zeroes 1/r at r = 0 instead of evaluating 0 * inf.
template <bool SHELL, bool GUARD>
__global__ void __launch_bounds__(kD32Threads)
k_direct_fp32(int n, const double4* __restrict__ sbody, const float* __restrict__ srad,
              const uint32_t* __restrict__ sidx, float eps2, double* __restrict__ ax,
              double* __restrict__ ay, double* __restrict__ az,
              unsigned long long* __restrict__ counter) {
    __shared__ float4 sj[kD32Tile];
    __shared__ float2 ss[kD32Tile];
    const int t0 = blockIdx.x * (kD32Threads * kD32Per);
    const double4 ref = sbody[t0];
    float bx[kD32Per], by[kD32Per], bz[kD32Per];
    float sx[kD32Per], sy[kD32Per], sz[kD32Per], cx[kD32Per], cy[kD32Per], cz[kD32Per];
#pragma unroll
    for (int u = 0; u < kD32Per; u++) {
        const int i = t0 + u * kD32Threads + threadIdx.x;
        const double4 b = sbody[i < n ? i : n - 1];
        bx[u] = (float)(b.x - ref.x);
        by[u] = (float)(b.y - ref.y);
        bz[u] = (float)(b.z - ref.z);
        sx[u] = sy[u] = sz[u] = cx[u] = cy[u] = cz[u] = 0.f;
    }
    for (int base = 0; base < n; base += kD32Tile) {
        const int j = base + threadIdx.x;
        if (j < n) {
            const double4 q = sbody[j];
            sj[threadIdx.x] = make_float4((float)(q.x - ref.x), (float)(q.y - ref.y),
                                          (float)(q.z - ref.z), (float)q.w);
            if (SHELL) {
                const float R = srad[j];
                const float id = rsqrtf(R * R + eps2);
                ss[threadIdx.x] = make_float2(R > 0.f ? R * R : 0.f, (float)q.w * id * id * id);
            }
        } else {
            sj[threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (SHELL) ss[threadIdx.x] = make_float2(0.f, 0.f);
        }
        __syncthreads();
        const int cnt = min(kD32Tile, n - base);
        float tx[kD32Per], ty[kD32Per], tz[kD32Per];
#pragma unroll
        for (int u = 0; u < kD32Per; u++) tx[u] = ty[u] = tz[u] = 0.f;
#pragma unroll 8
        for (int k = 0; k < cnt; k++) {
            const float4 q = sj[k];
            float2 sh;
            if (SHELL) sh = ss[k];
#pragma unroll
            for (int u = 0; u < kD32Per; u++) {
                const float dx = bx[u] - q.x, dy = by[u] - q.y, dz = bz[u] - q.z;
                const float raw = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const float r2 = raw + eps2;
                const float inv = (GUARD && !(r2 > 0.f)) ? 0.f : rsqrtf(r2);
                float f = q.w * (inv * inv * inv);
                if (SHELL && raw < sh.x) f = sh.y;
                tx[u] = fmaf(-f, dx, tx[u]);
                ty[u] = fmaf(-f, dy, ty[u]);
                tz[u] = fmaf(-f, dz, tz[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kD32Per; u++) {
            kahan32(sx[u], cx[u], tx[u]);
            kahan32(sy[u], cy[u], ty[u]);
            kahan32(sz[u], cz[u], tz[u]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kD32Per; u++) {
        const int i = t0 + u * kD32Threads + threadIdx.x;
        if (i < n) {
            const uint32_t row = sidx[i];
            ax[row] = (double)sx[u] - (double)cx[u];
            ay[row] = (double)sy[u] - (double)cy[u];
            az[row] = (double)sz[u] - (double)cz[u];
        }
    }
    if (threadIdx.x == 0 && counter) {
        const int nt = min(kD32Threads * kD32Per, n - t0);
        atomicAdd(counter, (unsigned long long)nt * (unsigned long long)n);
    }
}

// The arithmetic is split in two phases so that the costly per-pair part
// (sqrt, division) runs on every thread of the block: for a tile of kPTj
// sources, 256 threads compute the kPTi x kPTj pair terms c*dx, c*dy, c*dz
// (each rounded exactly as above) into shared memory; then 3 x kPTi threads
// subtract them in source order, one (target, component) chain per thread.
// The sequence of roundings of every target's sum is unchanged, so the
// result is bit-identical to CpuParallelBackend's.
constexpr int kPTi = 8;     // targets per block
constexpr int kPTj = 128;   // sources per tile
constexpr int kPThreads = 256;

template <bool SHELL>
__global__ void __launch_bounds__(kPThreads)
k_direct_fp64_pairs(int n, const double* __restrict__ px, const double* __restrict__ py,
                    const double* __restrict__ pz, const double* __restrict__ m,
                    const double* __restrict__ rad, const uint8_t* __restrict__ act,
                    double eps2, double* __restrict__ ax, double* __restrict__ ay,
                    double* __restrict__ az) {
    __shared__ double s_t[3][kPTi][kPTj + 1];  // pair terms (padded against bank conflicts)
    __shared__ uint8_t s_ok[kPTi][kPTj];        // term is added (active source, not self)
    __shared__ double s_i[kPTi][3];
    __shared__ uint8_t s_iact[kPTi];
    const int i0 = blockIdx.x * kPTi;
    if (threadIdx.x < kPTi) {
        const int i = i0 + threadIdx.x;
        const bool me = i < n && act[i];
        s_iact[threadIdx.x] = me;
        s_i[threadIdx.x][0] = me ? px[i] : 0.0;
        s_i[threadIdx.x][1] = me ? py[i] : 0.0;
        s_i[threadIdx.x][2] = me ? pz[i] : 0.0;
    }
    __syncthreads();
    // accumulator thread: (target, component)
    const int acc_t = threadIdx.x / 3, acc_c = threadIdx.x % 3;
    const bool accum = threadIdx.x < 3 * kPTi;
    double sum = 0.0;
    for (int base = 0; base < n; base += kPTj) {
        for (int p = threadIdx.x; p < kPTi * kPTj; p += kPThreads) {
            const int ti = p / kPTj, tj = p % kPTj;
            const int i = i0 + ti, j = base + tj;
            bool ok = j < n && s_iact[ti] && j != i && act[j];
            double tx = 0.0, ty = 0.0, tz = 0.0;
            if (ok) {
                const double dx = __dsub_rn(s_i[ti][0], px[j]);
                const double dy = __dsub_rn(s_i[ti][1], py[j]);
                const double dz = __dsub_rn(s_i[ti][2], pz[j]);
                const double raw = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                             __dmul_rn(dz, dz));
                const double mj = m[j];
                double c;
                const double R = SHELL ? rad[j] : 0.0;
                if (!SHELL || R <= 0.0) {
                    const double inv = 1.0 / sqrt(__dadd_rn(raw, eps2));
                    c = __dmul_rn(__dmul_rn(__dmul_rn(mj, inv), inv), inv);
                } else if (sqrt(raw) < R) {
                    const double den = __dadd_rn(__dmul_rn(R, R), eps2);
                    const double ids = 1.0 / sqrt(den);
                    c = __dmul_rn(mj, ids) / den;
                } else {
                    const double inv = 1.0 / sqrt(__dadd_rn(raw, eps2));
                    c = __dmul_rn(__dmul_rn(__dmul_rn(mj, inv), inv), inv);
                }
                tx = __dmul_rn(c, dx);
                ty = __dmul_rn(c, dy);
                tz = __dmul_rn(c, dz);
            }
            s_t[0][ti][tj] = tx;
            s_t[1][ti][tj] = ty;
            s_t[2][ti][tj] = tz;
            s_ok[ti][tj] = ok;
        }
        __syncthreads();
        if (accum) {
            const int cnt = min(kPTj, n - base);
            for (int tj = 0; tj < cnt; tj++)
                if (s_ok[acc_t][tj]) sum = __dsub_rn(sum, s_t[acc_c][acc_t][tj]);
        }
        __syncthreads();
    }
    if (accum) {
        const int i = i0 + acc_t;
        if (i < n) (acc_c == 0 ? ax : acc_c == 1 ? ay : az)[i] = sum;
    }
}

void direct_fp64(cudaStream_t st, int n, const double* px, const double* py, const double* pz,
                 const double* m, const double* rad, const uint8_t* act, double eps, bool shell,
                 double* ax, double* ay, double* az) {
    if (n <= 0) return;
    const double eps2 = eps * eps;
    const int g = ceil_div(n, kPTi);
    if (shell) k_direct_fp64_pairs<true><<<g, kPThreads, 0, st>>>(n, px, py, pz, m, rad, act, eps2, ax, ay, az);
    else k_direct_fp64_pairs<false><<<g, kPThreads, 0, st>>>(n, px, py, pz, m, rad, act, eps2, ax, ay, az);
}

void direct_fp32(cudaStream_t st, int n, const double4* sbody, const float* srad,
                 const uint32_t* sidx, double eps, bool shell, double* ax, double* ay,
                 double* az, unsigned long long* counter) {
    if (n <= 0) return;
    const float eps2 = (float)(eps * eps);
    const int g = ceil_div(n, kD32Threads * kD32Per);
    if (eps2 > 0.f) {
        if (shell) k_direct_fp32<true, false><<<g, kD32Threads, 0, st>>>(n, sbody, srad, sidx, eps2, ax, ay, az, counter);
        else k_direct_fp32<false, false><<<g, kD32Threads, 0, st>>>(n, sbody, srad, sidx, eps2, ax, ay, az, counter);
    } else {
        if (shell) k_direct_fp32<true, true><<<g, kD32Threads, 0, st>>>(n, sbody, srad, sidx, eps2, ax, ay, az, counter);
        else k_direct_fp32<false, true><<<g, kD32Threads, 0, st>>>(n, sbody, srad, sidx, eps2, ax, ay, az, counter);
    }
}

}  // namespace nb
