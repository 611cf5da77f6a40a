// bodies.cu - per-body kernels of the step.
#include "bodies.cuh"

#include <algorithm>

namespace nb {

// Half kick + drift of SoAVerletIntegrator.Step phases 1-2
// (SoAVerletIntegrator.cs:70-88) fused with the bounding box of the active
// bodies (BarnesHutBackend.cs:150-170; replaces reduction_kernel.cu:68-132 +
// the host finish of gpu_tree.cu:207-259, so no host sync).  FP64, explicit
// round-to-nearest operations: v += (dt/2) a, x += dt v, exactly as the
// reference rounds them.
__global__ void k_kick_drift_bbox(int n, State s, int kick, double dt,
                                  unsigned long long* bbox_ord, int* n_active, int* err,
                                  const int* dn) {
    __shared__ double sh[6][8];
    __shared__ int sa[8];
    n = dev_rows(n, dn);
    const double half = 0.5 * dt;
    double lo[3] = {1.0e308 * 10, 1.0e308 * 10, 1.0e308 * 10};
    double hi[3] = {-lo[0], -lo[0], -lo[0]};
    int act = 0;
    // a grid-stride loop over a few resident waves of blocks: each block adds
    // its box and count to the 7 global words once (one block per 256 rows
    // made those same-address atomics, not memory, bound the pass at 8M rows)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!s.active[i]) continue;
        double x = s.px[i], y = s.py[i], z = s.pz[i];
        if (kick) {
            double vx = __dadd_rn(s.vx[i], __dmul_rn(half, s.ax[i]));
            double vy = __dadd_rn(s.vy[i], __dmul_rn(half, s.ay[i]));
            double vz = __dadd_rn(s.vz[i], __dmul_rn(half, s.az[i]));
            x = __dadd_rn(x, __dmul_rn(dt, vx));
            y = __dadd_rn(y, __dmul_rn(dt, vy));
            z = __dadd_rn(z, __dmul_rn(dt, vz));
            s.vx[i] = vx; s.vy[i] = vy; s.vz[i] = vz;
            s.px[i] = x; s.py[i] = y; s.pz[i] = z;
        }
        if (!isfinite(x) || !isfinite(y) || !isfinite(z) || !isfinite(s.mass[i]))
            dev_flag(err, kErrNonFinite);
        lo[0] = fmin(lo[0], x); hi[0] = fmax(hi[0], x);
        lo[1] = fmin(lo[1], y); hi[1] = fmax(hi[1], y);
        lo[2] = fmin(lo[2], z); hi[2] = fmax(hi[2], z);
        act++;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        lo[k] = warp_min(lo[k]);
        hi[k] = warp_max(hi[k]);
    }
    act = warp_sum(act);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            sh[k][warp] = lo[k];
            sh[3 + k][warp] = hi[k];
        }
        sa[warp] = act;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        double v = sh[k][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = (k < 3) ? fmin(v, sh[k][w]) : fmax(v, sh[k][w]);
        if (k < 3 ? (v < 1.0e308) : (v > -1.0e308)) {
            unsigned long long o = dbl_to_ord(v);
            if (k < 3) atomicMin(&bbox_ord[k], o);
            else atomicMax(&bbox_ord[k], o);
        }
    }
    if (threadIdx.x == 6) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sa[w];
        if (t) atomicAdd(n_active, t);
    }
}

// Phases 4-5 (SoAVerletIntegrator.cs:95-116): v += (dt/2) a for active rows;
// the acceleration buffer itself is the next step's "old" acceleration.
__global__ void k_kick(int n, State s, double dt, const int* dn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dev_rows(n, dn) || !s.active[i]) return;
    const double half = 0.5 * dt;
    s.vx[i] = __dadd_rn(s.vx[i], __dmul_rn(half, s.ax[i]));
    s.vy[i] = __dadd_rn(s.vy[i], __dmul_rn(half, s.ay[i]));
    s.vz[i] = __dadd_rn(s.vz[i], __dmul_rn(half, s.az[i]));
}

__global__ void k_cube(const unsigned long long* bbox_ord, const double* given, double* cube) {
    if (threadIdx.x != 0) return;
    if (given) {
        for (int k = 0; k < 4; k++) cube[k] = given[k];
        return;
    }
    double mn[3], mx[3];
    for (int k = 0; k < 3; k++) {
        mn[k] = ord_to_dbl(bbox_ord[k]);
        mx[k] = ord_to_dbl(bbox_ord[3 + k]);
    }
    // gpu_tree.cu:163-167 / octree_builder.cpp:29-35
    double cx = __dmul_rn(__dadd_rn(mn[0], mx[0]), 0.5);
    double cy = __dmul_rn(__dadd_rn(mn[1], mx[1]), 0.5);
    double cz = __dmul_rn(__dadd_rn(mn[2], mx[2]), 0.5);
    double e = fmax(fmax(__dsub_rn(mx[0], mn[0]), __dsub_rn(mx[1], mn[1])), __dsub_rn(mx[2], mn[2]));
    double h = fmax(__dmul_rn(e, 0.5), 1e-10);
    h = __dmul_rn(h, 1.001);
    cube[0] = cx; cube[1] = cy; cube[2] = cz; cube[3] = h;
}

__device__ __forceinline__ uint64_t quant_cube(double p, double lo, double inv2h) {
    double u = __dmul_rn(__dsub_rn(p, lo), inv2h);
    u = fmax(0.0, fmin(1.0, u));
    uint64_t q = (uint64_t)__dmul_rn(u, 2097152.0);
    return q > 2097151ull ? 2097151ull : q;
}

constexpr int kKeyThreads = 256;
constexpr int kKeyItems = 8;  // keys per thread: one block's histograms cover 2048 keys

// Cube-mode keys of kKeyItems keys per thread, plus the digit histograms of
// all 8 sort passes; a block folds its 2048 keys into shared bins and adds
// the non-zero bins to the global counts (fewer global atomics per key).
// With `rows`, every row's (x, y, z, m) is also written there in row order,
// and with `amag` its |a| (the acceleration buffer still holds the previous
// step's), so the gather after the sort reads one 32-byte record and one
// word per body instead of seven scattered 8-byte fields.
__global__ void __launch_bounds__(kKeyThreads)
k_keys_cube(int n, State s, const double* __restrict__ cube, uint64_t* __restrict__ keys,
            uint32_t* __restrict__ vals, uint32_t* __restrict__ hist, double4* __restrict__ rows,
            float* __restrict__ amag, const int* dn) {
    __shared__ uint32_t sh[8][256];
    n = dev_rows(n, dn);
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    const double h = cube[3];
    const double inv2h = 1.0 / __dmul_rn(2.0, h);
    const double lx = __dsub_rn(cube[0], h), ly = __dsub_rn(cube[1], h), lz = __dsub_rn(cube[2], h);
    for (int k = 0; k < kKeyItems; k++) {
        const int i = (blockIdx.x * kKeyItems + k) * kKeyThreads + threadIdx.x;
        uint64_t key = kInactiveKey;
        if (i < n) {
            const double x = s.px[i], y = s.py[i], z = s.pz[i];
            if (s.active[i])
                key = (spread21(quant_cube(x, lx, inv2h)) << 2) |
                      (spread21(quant_cube(y, ly, inv2h)) << 1) | spread21(quant_cube(z, lz, inv2h));
            keys[i] = key;
            vals[i] = (uint32_t)i;
            if (rows) rows[i] = make_double4(x, y, z, s.mass[i]);
            if (amag) {
                const double ax = s.ax[i], ay = s.ay[i], az = s.az[i];
                amag[i] = (float)sqrt(ax * ax + ay * ay + az * az);
            }
        }
        // plain shared atomics: measured faster than warp-aggregating the
        // digits with match_any (whose issue cost exceeds the serialisation
        // of the few same-bin lanes of a clustered system's high digits)
        if (i < n) {
#pragma unroll
            for (int p = 0; p < 8; p++) atomicAdd(&sh[p][(uint32_t)(key >> (8 * p)) & 0xFF], 1u);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) {
        uint32_t v = (&sh[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

// morton_code_kernel semantics (morton_kernel.cu:11-45 with the inverse
// ranges of launch_morton_codes, :57-64) and morton_from_unit
// (morton.hpp:29-35).
__global__ void k_keys_aabb(int n, State s, const unsigned long long* __restrict__ bbox_ord,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vals[i] = (uint32_t)i;
    if (!s.active[i]) {
        keys[i] = kInactiveKey;
        return;
    }
    double mn[3], r[3], inv[3];
    for (int k = 0; k < 3; k++) {
        mn[k] = ord_to_dbl(bbox_ord[k]);
        r[k] = __dsub_rn(ord_to_dbl(bbox_ord[3 + k]), mn[k]);
        inv[k] = (r[k] > 1e-30) ? 1.0 / r[k] : 0.0;
    }
    const double p[3] = {s.px[i], s.py[i], s.pz[i]};
    uint64_t q[3];
    for (int k = 0; k < 3; k++) {
        double u = __dmul_rn(__dsub_rn(p[k], mn[k]), inv[k]);
        u = fmax(0.0, fmin(1.0, u));
        q[k] = (uint64_t)__dmul_rn(u, 2097151.0);
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
}

__global__ void k_gather(int n, State s, const uint32_t* __restrict__ sidx,
                         double4* __restrict__ sbody, float* __restrict__ srad,
                         float* __restrict__ samag, const double4* __restrict__ rows,
                         const float* __restrict__ amag, const int* dn) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= dev_rows(n, dn)) return;
    const uint32_t i = sidx[k];
    if (rows) {
        sbody[k] = rows[i];
        if (srad) srad[k] = s.radius ? (float)s.radius[i] : 0.f;
        if (samag) samag[k] = amag[i];
        return;
    }
    sbody[k] = make_double4(s.px[i], s.py[i], s.pz[i], s.mass[i]);
    if (srad) srad[k] = s.radius ? (float)s.radius[i] : 0.f;
    if (samag) {  // |a| of the previous step (acceleration buffer before it is overwritten)
        const double ax = s.ax[i], ay = s.ay[i], az = s.az[i];
        samag[k] = (float)sqrt(ax * ax + ay * ay + az * az);
    }
}

__global__ void k_zero_acc(int n, State s, const int* dn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dev_rows(n, dn)) return;
    s.ax[i] = 0.0;
    s.ay[i] = 0.0;
    s.az[i] = 0.0;
}

void launch_kick_drift_bbox(cudaStream_t st, int n, State s, bool kick, double dt,
                            unsigned long long* bbox_ord, int* n_active, int* err,
                            const int* dn) {
    cudaMemsetAsync(bbox_ord, 0xFF, 3 * sizeof(unsigned long long), st);
    cudaMemsetAsync(bbox_ord + 3, 0, 3 * sizeof(unsigned long long), st);
    cudaMemsetAsync(n_active, 0, sizeof(int), st);
    if (n <= 0) return;
    k_kick_drift_bbox<<<std::min(ceil_div(n, 256), kSMs * 8), 256, 0, st>>>(
        n, s, kick ? 1 : 0, dt, bbox_ord, n_active, err, dn);
}

void launch_kick(cudaStream_t st, int n, State s, double dt, const int* dn) {
    if (n > 0) k_kick<<<ceil_div(n, 256), 256, 0, st>>>(n, s, dt, dn);
}

void launch_cube(cudaStream_t st, const unsigned long long* bbox_ord, const double* given,
                 double* cube) {
    k_cube<<<1, 32, 0, st>>>(bbox_ord, given, cube);
}

void launch_keys_cube(cudaStream_t st, int n, const State& s, const double* cube,
                      uint64_t* keys, uint32_t* vals, uint32_t* hist, double4* rows,
                      float* amag, const int* dn) {
    cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, st);
    if (n > 0)
        k_keys_cube<<<ceil_div(n, kKeyThreads * kKeyItems), kKeyThreads, 0, st>>>(
            n, s, cube, keys, vals, hist, rows, amag, dn);
}

void launch_keys_aabb(cudaStream_t st, int n, const State& s,
                      const unsigned long long* bbox_ord, uint64_t* keys, uint32_t* vals) {
    if (n > 0) k_keys_aabb<<<ceil_div(n, 256), 256, 0, st>>>(n, s, bbox_ord, keys, vals);
}

void launch_gather(cudaStream_t st, int n, const State& s, const uint32_t* sidx,
                   double4* sbody, float* srad, float* samag, const double4* rows,
                   const float* amag, const int* dn) {
    if (n > 0)
        k_gather<<<ceil_div(n, 256), 256, 0, st>>>(n, s, sidx, sbody, srad, samag, rows, amag,
                                                   dn);
}

void launch_zero_acc(cudaStream_t st, int n, State s, const int* dn) {
    if (n > 0) k_zero_acc<<<ceil_div(n, 256), 256, 0, st>>>(n, s, dn);
}

}  // namespace nb
