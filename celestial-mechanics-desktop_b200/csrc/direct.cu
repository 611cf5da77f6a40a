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
// k_direct_fp32 is the throughput kernel: Morton-sorted targets in tiles of
// 256 x kD32Per, sources in chunks, one persistent launch over a work queue
// of (target tile, source chunk) items so the grid ends evenly; j-tiles of
// 1024 sources arrive raw by cp.async into one of two shared-memory buffers
// while the previous tile is evaluated, and are converted to FP32
// coordinates differenced in FP64 against the target tile's centre of mass;
// kD32Per targets per thread so every broadcast shared-memory read feeds
// several pair evaluations; a Kahan fold of each j-tile's FP32 partial sum.  The chunk partials are written in FP64
// and k_direct_reduce adds them in chunk order, so the result does not depend
// on scheduling.
#include <algorithm>

#include "direct.cuh"

namespace nb {

#ifndef NB_D32_THREADS
#define NB_D32_THREADS 256
#endif
constexpr int kD32Threads = NB_D32_THREADS;
#ifndef NB_D32_PER
#define NB_D32_PER 10
#endif
// targets per thread (even: packed in pairs).  10 keeps five independent
// packed chains per source in flight at 240 registers (one block of 8 warps
// per SM); measured against 4 (2 blocks per SM), 6 and 8 it feeds the FMA
// pipe best.
constexpr int kD32Per = NB_D32_PER;
static_assert(kD32Per % 2 == 0, "targets are packed two per f32x2 register");
// Sources staged per thread per j-tile: 4 (1024-source tiles) measured
// 70.95 % of FP32 peak against 70.4 % for 1 and 69.9 % for the register
// prefetch of one source per thread it replaces.
#ifndef NB_D32_STAGE
#define NB_D32_STAGE 4
#endif
constexpr int kD32Stage = NB_D32_STAGE;              // sources staged per thread per j-tile
constexpr int kD32Tile = kD32Threads * kD32Stage;    // sources per j-tile
// dynamic shared memory: two raw FP64 source buffers (cp.async double
// buffering), their radii, and the converted FP32 tile
constexpr size_t kD32Smem = 2 * kD32Tile * sizeof(double4) + 2 * kD32Tile * sizeof(float) +
                            2 * kD32Tile * sizeof(float4) + kD32Tile * sizeof(float2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
constexpr int kD32MinChunk = 4096;    // sources per chunk at least
#ifndef NB_D32_UNROLL
#define NB_D32_UNROLL 8
#endif
constexpr int kD32Unroll = NB_D32_UNROLL;  // source loop unroll

__device__ __forceinline__ void kahan32(float& s, float& c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Targets and sources are the n sorted bodies (all active).  Item it covers
// target tile it / chunks and source chunk it % chunks; its partial sums go
// to part[(chunk * 3 + axis) * n + target].  The self pair has
// dx = dy = dz = 0 and contributes 0 when eps > 0; GUARD (used when
// eps == 0) zeroes 1/r at r = 0 instead of evaluating 0 * inf.
template <bool SHELL, bool GUARD>
__global__ void __launch_bounds__(kD32Threads)
k_direct_fp32(int n, const double4* __restrict__ sbody, const float* __restrict__ srad,
              float eps2, int n_items, int chunks, int chunk_len, unsigned* __restrict__ ctr,
              double* __restrict__ part, unsigned long long* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char s_d32[];
    double4* raw = (double4*)s_d32;                       // [2][kD32Tile]
    float* rawR = (float*)(raw + 2 * kD32Tile);           // [2][kD32Tile]
    float4* sj = (float4*)(rawR + 2 * kD32Tile);
    float4* sj2 = sj + kD32Tile;
    float2* ss = (float2*)(sj2 + kD32Tile);
    __shared__ double s_box[4][kD32Threads / 32];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(ctr, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has the item before thread 0 fetches the next
        if (it >= n_items) break;
        const int tile = it / chunks, chunk = it - tile * chunks;
        const int t0 = tile * (kD32Threads * kD32Per);
        const int j0 = chunk * chunk_len, j1 = min(n, j0 + chunk_len);
        // reference point: the target tile's centre of mass (the FP32
        // coordinates are most precise where the mass is)
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // m, m x, m y, m z
#pragma unroll
        for (int u = 0; u < kD32Per; u++) {
            const int i = t0 + u * kD32Threads + threadIdx.x;
            if (i < n) {
                const double4 b = sbody[i];
                acc[0] += b.w;
                acc[1] += b.w * b.x;
                acc[2] += b.w * b.y;
                acc[3] += b.w * b.z;
            }
        }
        for (int k = 0; k < 4; k++)
            for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xFFFFFFFFu, acc[k], o);
        if ((threadIdx.x & 31) == 0)
            for (int k = 0; k < 4; k++) s_box[k][threadIdx.x >> 5] = acc[k];
        __syncthreads();
        double4 ref;
        {
            double m = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
            for (int w = 0; w < kD32Threads / 32; w++) {
                m += s_box[0][w];
                mx += s_box[1][w];
                my += s_box[2][w];
                mz += s_box[3][w];
            }
            ref = m > 0.0 ? make_double4(mx / m, my / m, mz / m, 0.0) : sbody[t0];
        }
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
        // the next j-tile's raw sources arrive by cp.async while the current
        // one is evaluated (two raw buffers)
        auto issue = [&](int b0, int buf) {
#pragma unroll
            for (int u = 0; u < kD32Stage; u++) {
                const int k = u * kD32Threads + threadIdx.x;
                if (b0 + k < j1) {
                    double4* dst = raw + buf * kD32Tile + k;
                    cp_async16(dst, &sbody[b0 + k]);
                    cp_async16((char*)dst + 16, (const char*)&sbody[b0 + k] + 16);
                    if (SHELL) cp_async4(rawR + buf * kD32Tile + k, &srad[b0 + k]);
                }
            }
            cp_async_commit();
        };
        issue(j0, 0);
        int buf = 0;
        for (int base = j0; base < j1; base += kD32Tile, buf ^= 1) {
            if (base + kD32Tile < j1) {
                issue(base + kD32Tile, buf ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();  // every thread's copies of this tile have landed
#pragma unroll
            for (int u = 0; u < kD32Stage; u++) {
                const int k = u * kD32Threads + threadIdx.x;
                const int j = base + k;
                float4 q4 = make_float4(0.f, 0.f, 0.f, 0.f);
                float R = 0.f;
                if (j < j1) {
                    const double4 qn = raw[buf * kD32Tile + k];
                    q4 = make_float4((float)(qn.x - ref.x), (float)(qn.y - ref.y),
                                     (float)(qn.z - ref.z), (float)qn.w);
                    if (SHELL) R = rawR[buf * kD32Tile + k];
                }
                if constexpr (SHELL) {
                    sj[k] = q4;
                    const float id = rsqrtf(R * R + eps2);
                    ss[k] = j < j1 ? make_float2(R > 0.f ? R * R : 0.f, q4.w * id * id * id)
                                   : make_float2(0.f, 0.f);
                } else {
                    // each source duplicated into both halves of the packed pairs
                    sj[k] = make_float4(q4.x, q4.x, q4.y, q4.y);
                    sj2[k] = make_float4(q4.z, q4.z, q4.w, q4.w);
                }
            }
            __syncthreads();
            const int cnt = min(kD32Tile, j1 - base);
            float tx[kD32Per], ty[kD32Per], tz[kD32Per];
#pragma unroll
            for (int u = 0; u < kD32Per; u++) tx[u] = ty[u] = tz[u] = 0.f;
            if constexpr (SHELL) {
#pragma unroll 4
                for (int k = 0; k < cnt; k++) {
                    const float4 q = sj[k];
                    const float2 sh = ss[k];
#pragma unroll
                    for (int u = 0; u < kD32Per; u++) {
                        const float dx = bx[u] - q.x, dy = by[u] - q.y, dz = bz[u] - q.z;
                        const float raw = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float r2 = raw + eps2;
                        const float inv = (GUARD && !(r2 > 0.f)) ? 0.f : rsqrt_ftz(r2);
                        float f = q.w * (inv * inv * inv);
                        if (raw < sh.x) f = sh.y;
                        tx[u] = fmaf(-f, dx, tx[u]);
                        ty[u] = fmaf(-f, dy, ty[u]);
                        tz[u] = fmaf(-f, dz, tz[u]);
                    }
                }
            } else {
                // two targets per packed instruction; d = q - b, so each half
                // rounds exactly as fmaf(-f, b - q, t) and fmaf(b - q, b - q, .)
                constexpr int P = kD32Per / 2;
                f32x2 BX[P], BY[P], BZ[P], AX[P], AY[P], AZ[P];
#pragma unroll
                for (int p = 0; p < P; p++) {
                    BX[p] = pk2(bx[2 * p], bx[2 * p + 1]);
                    BY[p] = pk2(by[2 * p], by[2 * p + 1]);
                    BZ[p] = pk2(bz[2 * p], bz[2 * p + 1]);
                    AX[p] = AY[p] = AZ[p] = 0ull;
                }
                const f32x2 E2 = pk2(eps2, eps2);
#pragma unroll kD32Unroll
                for (int k = 0; k < cnt; k++) {
                    const float4 qa = sj[k], qb = sj2[k];
                    const f32x2 qx = pk2(qa.x, qa.y), qy = pk2(qa.z, qa.w);
                    const f32x2 qz = pk2(qb.x, qb.y), qm = pk2(qb.z, qb.w);
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        const f32x2 dx = sub2(qx, BX[p]), dy = sub2(qy, BY[p]), dz = sub2(qz, BZ[p]);
                        const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
                        float ra, rb;
                        upk2(r2, ra, rb);
                        float ia = rsqrt_ftz(ra), ib = rsqrt_ftz(rb);
                        if (GUARD) {
                            ia = ra > 0.f ? ia : 0.f;
                            ib = rb > 0.f ? ib : 0.f;
                        }
                        const f32x2 inv = pk2(ia, ib);
                        const f32x2 f = mul2(mul2(mul2(inv, inv), inv), qm);
                        AX[p] = fma2(f, dx, AX[p]);
                        AY[p] = fma2(f, dy, AY[p]);
                        AZ[p] = fma2(f, dz, AZ[p]);
                    }
                }
#pragma unroll
                for (int p = 0; p < P; p++) {
                    upk2(AX[p], tx[2 * p], tx[2 * p + 1]);
                    upk2(AY[p], ty[2 * p], ty[2 * p + 1]);
                    upk2(AZ[p], tz[2 * p], tz[2 * p + 1]);
                }
            }
#pragma unroll
            for (int u = 0; u < kD32Per; u++) {
                kahan32(sx[u], cx[u], tx[u]);
                kahan32(sy[u], cy[u], ty[u]);
                kahan32(sz[u], cz[u], tz[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kD32Per; u++) {
            const int i = t0 + u * kD32Threads + threadIdx.x;
            if (i < n) {
                part[(size_t)(chunk * 3 + 0) * n + i] = (double)sx[u] - (double)cx[u];
                part[(size_t)(chunk * 3 + 1) * n + i] = (double)sy[u] - (double)cy[u];
                part[(size_t)(chunk * 3 + 2) * n + i] = (double)sz[u] - (double)cz[u];
            }
        }
        if (threadIdx.x == 0 && counter) {
            const int nt = min(kD32Threads * kD32Per, n - t0);
            atomicAdd(counter, (unsigned long long)nt * (unsigned long long)(j1 - j0));
        }
    }
}

// Sum of the chunk partials in chunk order, written by body row.
__global__ void k_direct_reduce(int n, int chunks, const double* __restrict__ part,
                                const uint32_t* __restrict__ sidx, double* __restrict__ ax,
                                double* __restrict__ ay, double* __restrict__ az) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < chunks; c++)
        for (int k = 0; k < 3; k++) s[k] += part[(size_t)(c * 3 + k) * n + i];
    const uint32_t row = sidx[i];
    ax[row] = s[0];
    ay[row] = s[1];
    az[row] = s[2];
}

// The arithmetic is split in two phases so that the costly per-pair part
// (sqrt, division) runs on every thread of the block: for a tile of kPTj
// sources, 256 threads compute the kPTi x kPTj pair terms c*dx, c*dy, c*dz
// (each rounded exactly as above) into shared memory; then 3 x kPTi threads
// subtract them in source order, one (target, component) chain per thread.
// The sequence of roundings of every target's sum is unchanged, so the
// result is bit-identical to CpuParallelBackend's.
//
// ORDER selects the rounding and summation order of another CPU backend of
// the desktop app (without the shell theorem; with it every backend runs
// CpuParallelBackend's arithmetic):
//   kOrderParallel  CpuParallelBackend: c = ((m*inv)*inv)*inv, one running sum;
//   kOrderSimd      SimdSingleThreadBackend (SimdSingleThreadBackend.cs:43-165)
//                   and the native engine's CPU brute force (engine/src/sim/
//                   engine.cpp:649-674): c = m*((inv*inv)*inv), sources in
//                   row order (the vector lanes are summed in lane order);
//   kOrderPairwise  CpuSingleThreadBackend's Newton's-third-law loop
//                   (CpuSingleThreadBackend.cs:50-159): the same c, and a
//                   body's sum is (its running sum over lower rows, which the
//                   loop adds into ax[j] as +c*(x_lower - x_j), i.e. minus
//                   the term) + (its running sum over higher rows).
constexpr int kPTi = 8;     // targets per block
constexpr int kPTj = 128;   // sources per tile
constexpr int kPThreads = 256;

template <bool SHELL, int ORDER>
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
    constexpr bool kSplit = !SHELL && ORDER == kOrderPairwise;
    double sum = 0.0;
    double hi = 0.0;  // kSplit: the sum over higher rows (sum holds the lower rows')
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
                if (!SHELL && ORDER != kOrderParallel) {
                    const double inv = 1.0 / sqrt(__dadd_rn(raw, eps2));
                    c = __dmul_rn(mj, __dmul_rn(__dmul_rn(inv, inv), inv));
                } else if (!SHELL || R <= 0.0) {
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
            if (kSplit) {
                const int split = i0 + acc_t - base;  // first tj with j > i
                for (int tj = 0; tj < cnt; tj++) {
                    if (!s_ok[acc_t][tj]) continue;
                    if (tj < split) sum = __dsub_rn(sum, s_t[acc_c][acc_t][tj]);
                    else hi = __dsub_rn(hi, s_t[acc_c][acc_t][tj]);
                }
            } else {
                for (int tj = 0; tj < cnt; tj++)
                    if (s_ok[acc_t][tj]) sum = __dsub_rn(sum, s_t[acc_c][acc_t][tj]);
            }
        }
        __syncthreads();
    }
    if (accum) {
        const int i = i0 + acc_t;
        if (kSplit) sum = __dadd_rn(sum, hi);
        if (i < n) (acc_c == 0 ? ax : acc_c == 1 ? ay : az)[i] = sum;
    }
}

void direct_fp64(cudaStream_t st, int n, const double* px, const double* py, const double* pz,
                 const double* m, const double* rad, const uint8_t* act, double eps, bool shell,
                 int order, double* ax, double* ay, double* az) {
    if (n <= 0) return;
    const double eps2 = eps * eps;
    const int g = ceil_div(n, kPTi);
    if (shell)
        k_direct_fp64_pairs<true, kOrderParallel><<<g, kPThreads, 0, st>>>(
            n, px, py, pz, m, rad, act, eps2, ax, ay, az);
    else if (order == kOrderSimd)
        k_direct_fp64_pairs<false, kOrderSimd><<<g, kPThreads, 0, st>>>(
            n, px, py, pz, m, rad, act, eps2, ax, ay, az);
    else if (order == kOrderPairwise)
        k_direct_fp64_pairs<false, kOrderPairwise><<<g, kPThreads, 0, st>>>(
            n, px, py, pz, m, rad, act, eps2, ax, ay, az);
    else
        k_direct_fp64_pairs<false, kOrderParallel><<<g, kPThreads, 0, st>>>(
            n, px, py, pz, m, rad, act, eps2, ax, ay, az);
}

void direct_fp32(cudaStream_t st, int n, const double4* sbody, const float* srad,
                 const uint32_t* sidx, double eps, bool shell, double* ax, double* ay,
                 double* az, unsigned long long* counter, void* scratch, size_t scratch_bytes,
                 unsigned* ctr, int sms) {
    if (n <= 0) return;
    const float eps2 = (float)(eps * eps);
    using K = void (*)(int, const double4*, const float*, float, int, int, int, unsigned*,
                       double*, unsigned long long*);
    const K k = eps2 > 0.f ? (shell ? k_direct_fp32<true, false> : k_direct_fp32<false, false>)
                           : (shell ? k_direct_fp32<true, true> : k_direct_fp32<false, true>);
    cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kD32Smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kD32Threads, kD32Smem);
    const int resident = sms * (per_sm > 0 ? per_sm : 1);
    const int tiles = ceil_div(n, kD32Threads * kD32Per);
    // Chunks per tile: at least 4 waves of items where the scratch and the
    // kD32MinChunk floor allow, and among those the count whose last wave is
    // fullest (every item costs the same, so a part-filled last wave idles
    // the rest of the GPU: 3 chunks of 1024 tiles on 296 resident blocks
    // leave 62 % of the 11th wave empty, 2 or 4 chunks about 8 %).
    const long long cmax = std::max<long long>(
        1, std::min<long long>(std::max(1, ceil_div(n, kD32MinChunk)),
                               (long long)(scratch_bytes / (sizeof(double) * 3 * (size_t)n))));
    const long long cmin = std::min<long long>(cmax, std::max(1, ceil_div(4LL * resident, tiles)));
    auto fill = [&](long long c) {
        const long long nc = ceil_div(n, ceil_div(n, (int)c));  // chunks actually formed
        const long long it = (long long)tiles * nc;
        return (double)it / (double)(((it + resident - 1) / resident) * resident);
    };
    double best = 0.0;
    for (long long c = cmin; c <= cmax; c++) best = std::max(best, fill(c));
    long long chunks = cmin;  // the fewest chunks within 0.5 % of the best fill
    while (chunks < cmax && fill(chunks) < best - 0.005) chunks++;
    const int chunk_len = ceil_div(n, (int)chunks);
    const int nchunks = ceil_div(n, chunk_len);
    const int items = tiles * nchunks;
    cudaMemsetAsync(ctr, 0, sizeof(unsigned), st);
    k<<<std::min(items, resident), kD32Threads, kD32Smem, st>>>(n, sbody, srad, eps2, items, nchunks,
                                                         chunk_len, ctr, (double*)scratch,
                                                         counter);
    k_direct_reduce<<<ceil_div(n, 256), 256, 0, st>>>(n, nchunks, (const double*)scratch, sidx,
                                                      ax, ay, az);
}

}  // namespace nb
