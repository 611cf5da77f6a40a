// diag.cu - FP64 energy / momentum diagnostics and the force-error audit.
//
// Replaces the reference's block reductions that finish on the host
// (engine/src/cuda/reduction_kernel.cu:138-290, gpu_reduction.cu:13-40,
// 345-560) with two-level device reductions in a fixed order, so results are
// deterministic run to run; definitions follow EnergyCalculator
// (src/CelestialMechanics.Physics/Validation/EnergyCalculator.cs:16-78) and
// NewtonianGravity.ComputePotentialEnergy (Forces/NewtonianGravity.cs:68-77).
#include "diag.cuh"

#include <algorithm>

namespace nb {

constexpr int kDiagThreads = 256;
constexpr int kDiagVals = 12;  // KE, Px, Py, Pz, Lx, Ly, Lz, Mx, My, Mz, M, PE

// Block partial sums of the per-body terms (fixed shuffle-tree order).
__global__ void __launch_bounds__(kDiagThreads)
k_diag_partials(int n, State s, const double* __restrict__ pe_terms, double* __restrict__ part) {
    __shared__ double sh[kDiagVals][kDiagThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[kDiagVals];
#pragma unroll
    for (int k = 0; k < kDiagVals; k++) v[k] = 0.0;
    if (i < n && s.active[i]) {
        const double m = s.mass[i];
        const double vx = s.vx[i], vy = s.vy[i], vz = s.vz[i];
        const double x = s.px[i], y = s.py[i], z = s.pz[i];
        v[0] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
        const double mvx = vx * m, mvy = vy * m, mvz = vz * m;
        v[1] = mvx; v[2] = mvy; v[3] = mvz;
        v[4] = y * mvz - z * mvy;
        v[5] = z * mvx - x * mvz;
        v[6] = x * mvy - y * mvx;
        v[7] = m * x; v[8] = m * y; v[9] = m * z;
        v[10] = m;
        v[11] = pe_terms ? pe_terms[i] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kDiagVals; k++) v[k] = warp_sum(v[k]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < kDiagVals; k++) sh[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x < kDiagVals) {
        double t = 0.0;
        for (int w = 0; w < kDiagThreads / 32; w++) t += sh[threadIdx.x][w];
        part[(size_t)blockIdx.x * kDiagVals + threadIdx.x] = t;
    }
}

__global__ void k_diag_final(int nblocks, const double* __restrict__ part, double* __restrict__ out) {
    // thread k sums column k over the blocks in block order
    if (threadIdx.x >= kDiagVals) return;
    double t = 0.0;
    for (int b = 0; b < nblocks; b++) t += part[(size_t)b * kDiagVals + threadIdx.x];
    out[threadIdx.x] = t;
}

// Exact pair potential: row i holds sum_{j>i, active} -m_i m_j / sqrt(r^2+eps^2).
__global__ void k_pe_rows(int n, State s, double eps2, double* __restrict__ rows) {
    __shared__ double4 sj[128];
    __shared__ uint8_t sa[128];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool me = i < n && s.active[i];
    const double xi = me ? s.px[i] : 0, yi = me ? s.py[i] : 0, zi = me ? s.pz[i] : 0;
    const double mi = me ? s.mass[i] : 0;
    double acc = 0.0;
    const int start = blockIdx.x * blockDim.x;
    for (int base = start; base < n; base += 128) {
        const int j = base + threadIdx.x;
        sj[threadIdx.x] = (j < n) ? make_double4(s.px[j], s.py[j], s.pz[j], s.mass[j]) : make_double4(0, 0, 0, 0);
        sa[threadIdx.x] = (j < n) ? s.active[j] : 0;
        __syncthreads();
        if (me) {
            const int cnt = min(128, n - base);
            for (int k = 0; k < cnt; k++) {
                if (base + k <= i || !sa[k]) continue;
                const double4 q = sj[k];
                const double rx = q.x - xi, ry = q.y - yi, rz = q.z - zi;
                const double d2 = rx * rx + ry * ry + rz * rz + eps2;
                acc += -1.0 * mi * q.w / sqrt(d2);
            }
        }
        __syncthreads();
    }
    if (i < n) rows[i] = acc;
}

// 1/2 m_i phi_i terms from the tree potential.
__global__ void k_pe_from_phi(int n, State s, const double* __restrict__ phi, double* __restrict__ rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rows[i] = s.active[i] ? 0.5 * s.mass[i] * phi[i] : 0.0;
}

void diagnostics(cudaStream_t st, int n, const State& s, double eps, int pe_mode,
                 const double* phi, double* rows, double* part, double* out12) {
    const int nb = ceil_div(n > 0 ? n : 1, kDiagThreads);
    if (pe_mode == 0) {
        if (n > 0) k_pe_rows<<<ceil_div(n, 128), 128, 0, st>>>(n, s, eps * eps, rows);
    } else {
        if (n > 0) k_pe_from_phi<<<ceil_div(n, 256), 256, 0, st>>>(n, s, phi, rows);
    }
    if (n > 0) k_diag_partials<<<nb, kDiagThreads, 0, st>>>(n, s, rows, part);
    k_diag_final<<<1, 32, 0, st>>>(n > 0 ? nb : 0, part, out12);
}

size_t diag_partial_bytes(int capacity) {
    return sizeof(double) * kDiagVals * (size_t)ceil_div(capacity > 0 ? capacity : 1, kDiagThreads);
}

// FP64 direct sum for target rows (ForceErrorAnalyzer's exact reference:
// the softened Newtonian pair term of CpuSingleThreadBackend, evaluated in
// FP64 with FMA contraction and the 1/sqrt below, so it agrees with the CPU
// sum to a few FP64 ulps per pair, not bit for bit).  Block (tile, chunk) sums
// kTgtTile targets over one chunk of the sources: each source is loaded once
// per tile rather than once per target, and the chunks give enough blocks
// for a few hundred targets.  The block's threads split the chunk, the
// block reduces in a fixed shuffle-tree order, and the chunk partials are
// summed in chunk order, so the result is deterministic.
constexpr int kTgtTile = 8;

// 1/sqrt(x) in FP64 from the FP32 hardware estimate (relative error below
// 2^-22) and one third-order Householder step, y <- y (1 + e/2 + 3e^2/8)
// with e = 1 - x y^2, which cubes the relative error (below 2^-64, so the
// result is within FP64 rounding).  x outside [1e-36, 1e36] (beyond the
// FP32 normal range after conversion) takes the library routine.
__device__ __forceinline__ double rsqrt_f64(double x) {
    if (!(x >= 1e-36 && x <= 1e36)) return rsqrt(x);
    const double y = (double)rsqrt_ftz((float)x);
    const double e = fma(-x, y * y, 1.0);
    return fma(y * e, fma(e, 0.375, 0.5), y);
}
constexpr int kTgtThreads = 256;
constexpr int kTgtUnroll = 4;
constexpr int kTgtMinChunk = 16384;

__global__ void __launch_bounds__(kTgtThreads)
k_direct_targets(int n, State s, double eps2, const int32_t* __restrict__ targets, int nt,
                 int chunk, double* __restrict__ out) {
    __shared__ double sh[3 * kTgtTile][kTgtThreads / 32];
    const int t0 = blockIdx.x * kTgtTile;
    int id[kTgtTile];
    double xi[kTgtTile], yi[kTgtTile], zi[kTgtTile], ax[kTgtTile], ay[kTgtTile], az[kTgtTile];
#pragma unroll
    for (int k = 0; k < kTgtTile; k++) {
        id[k] = t0 + k < nt ? targets[t0 + k] : -1;
        const int i = id[k] < 0 ? 0 : id[k];
        xi[k] = s.px[i];
        yi[k] = s.py[i];
        zi[k] = s.pz[i];
        ax[k] = ay[k] = az[k] = 0.0;
    }
    auto pull = [&](int j, double xj, double yj, double zj, double mj) {
#pragma unroll
        for (int k = 0; k < kTgtTile; k++) {
            if (j == id[k]) continue;
            const double dx = xi[k] - xj, dy = yi[k] - yj, dz = zi[k] - zj;
            const double inv = rsqrt_f64(fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2))));
            const double c = mj * inv * inv * inv;
            ax[k] -= c * dx;
            ay[k] -= c * dy;
            az[k] -= c * dz;
        }
    };
    const int j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
    int j = j0 + threadIdx.x;
    // kTgtUnroll sources per round, all their words loaded before any use
    // (one memory latency per round); sources in the same order as one by one
    for (; j + (kTgtUnroll - 1) * kTgtThreads < j1; j += kTgtUnroll * kTgtThreads) {
        double xs[kTgtUnroll], ys[kTgtUnroll], zs[kTgtUnroll], ms[kTgtUnroll];
        uint8_t as[kTgtUnroll];
#pragma unroll
        for (int u = 0; u < kTgtUnroll; u++) {
            const int jj = j + u * kTgtThreads;
            xs[u] = s.px[jj];
            ys[u] = s.py[jj];
            zs[u] = s.pz[jj];
            ms[u] = s.mass[jj];
            as[u] = s.active[jj];
        }
#pragma unroll
        for (int u = 0; u < kTgtUnroll; u++)
            if (as[u]) pull(j + u * kTgtThreads, xs[u], ys[u], zs[u], ms[u]);
    }
    for (; j < j1; j += kTgtThreads)
        if (s.active[j]) pull(j, s.px[j], s.py[j], s.pz[j], s.mass[j]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kTgtTile; k++) {
        const double vx = warp_sum(ax[k]), vy = warp_sum(ay[k]), vz = warp_sum(az[k]);
        if (lane == 0) {
            sh[3 * k][warp] = vx;
            sh[3 * k + 1][warp] = vy;
            sh[3 * k + 2][warp] = vz;
        }
    }
    __syncthreads();
    if (threadIdx.x < 3 * kTgtTile && t0 + threadIdx.x / 3 < nt) {
        double t = 0;
        for (int w = 0; w < kTgtThreads / 32; w++) t += sh[threadIdx.x][w];
        out[((size_t)blockIdx.y * nt + t0) * 3 + threadIdx.x] = t;
    }
}

// Largest |a|^2 over the active rows, a2 = ax*ax + ay*ay + az*az rounded as
// Engine::compute_max_acceleration's CPU loop rounds it (engine/src/sim/
// engine.cpp:491-501), which also skips NaN.  a2 >= 0, so its bit pattern
// orders like an unsigned integer and atomicMax on the bits is exact.
__global__ void k_max_acc2(int n, State s, unsigned long long* __restrict__ out) {
    unsigned long long m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!s.active[i]) continue;
        const double a2 = __dadd_rn(__dadd_rn(__dmul_rn(s.ax[i], s.ax[i]), __dmul_rn(s.ay[i], s.ay[i])),
                                    __dmul_rn(s.az[i], s.az[i]));
        if (!(a2 > 0.0)) continue;
        const unsigned long long b = (unsigned long long)__double_as_longlong(a2);
        m = b > m ? b : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xFFFFFFFFu, m, o);
        m = v > m ? v : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

void max_acc2(cudaStream_t st, int n, const State& s, unsigned long long* out, int sms) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (n > 0) k_max_acc2<<<std::min(ceil_div(n, 256), sms * 4), 256, 0, st>>>(n, s, out);
}

// ---- the learned MAC's in-run audit ------------------------------------------
//
// Direct-sum accelerations of sampled targets from the force evaluation's
// Morton-sorted FP64 copy of the active bodies (sbody).  Sources come in tiles
// of 256 consecutive sorted bodies, which sit close together: every tile is
// differenced in FP64 against its first body, rounded to FP32, and each
// target's FP64 position is differenced against the same point once per
// tile, so a pair's FP32 separation carries a relative error of a few FP32
// ulps of the separation itself (not of the system's extent).  The pair terms
// are packed FP32 (two targets per instruction, FTZ rsqrt), each tile's FP32
// partial sum is added to an FP64 accumulator, and the chunk partials are
// summed in chunk order: deterministic, and within ~1e-6 relative of the FP64
// direct sum, three orders of magnitude below the audit's error bound.
constexpr int kAudThreads = 256;
constexpr int kAudPer = 4;                          // targets per thread, packed in pairs
constexpr int kAudTargets = kAudThreads * kAudPer;  // targets per block
constexpr int kAudTile = kAudThreads;               // sources per shared-memory tile
constexpr int kAudMinChunk = 2048;

__global__ void __launch_bounds__(kAudThreads)
k_audit_targets(int ns, const double4* __restrict__ sbody, float eps2, const State s,
                const int32_t* __restrict__ targets, int nt, int chunk,
                double* __restrict__ part) {
    __shared__ float4 sj[kAudTile];
    __shared__ float4 sj2[kAudTile];
    constexpr int P = kAudPer / 2;
    const int t0 = blockIdx.x * kAudTargets;
    double px[kAudPer], py[kAudPer], pz[kAudPer], ax[kAudPer], ay[kAudPer], az[kAudPer];
#pragma unroll
    for (int u = 0; u < kAudPer; u++) {
        const int k = t0 + u * kAudThreads + threadIdx.x;
        const int i = targets[k < nt ? k : nt - 1];
        px[u] = s.px[i];
        py[u] = s.py[i];
        pz[u] = s.pz[i];
        ax[u] = ay[u] = az[u] = 0.0;
    }
    const f32x2 E2 = pk2(eps2, eps2);
    const int j0 = blockIdx.y * chunk, j1 = min(ns, j0 + chunk);
    for (int base = j0; base < j1; base += kAudTile) {
        const double4 r0 = sbody[base];  // the tile's reference point
        const int j = base + threadIdx.x;
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);  // past the end: massless
        if (j < j1) {
            const double4 b = sbody[j];
            q = make_float4((float)(b.x - r0.x), (float)(b.y - r0.y), (float)(b.z - r0.z),
                            (float)b.w);
        }
        __syncthreads();  // the previous tile is consumed
        sj[threadIdx.x] = make_float4(q.x, q.x, q.y, q.y);
        sj2[threadIdx.x] = make_float4(q.z, q.z, q.w, q.w);
        __syncthreads();
        f32x2 BX[P], BY[P], BZ[P], AX[P], AY[P], AZ[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            BX[p] = pk2((float)(px[2 * p] - r0.x), (float)(px[2 * p + 1] - r0.x));
            BY[p] = pk2((float)(py[2 * p] - r0.y), (float)(py[2 * p + 1] - r0.y));
            BZ[p] = pk2((float)(pz[2 * p] - r0.z), (float)(pz[2 * p + 1] - r0.z));
            AX[p] = AY[p] = AZ[p] = 0ull;
        }
        const int cnt = min(kAudTile, j1 - base);
#pragma unroll 8
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
                const f32x2 inv = pk2(rsqrt_ftz(ra), rsqrt_ftz(rb));
                const f32x2 f = mul2(mul2(mul2(inv, inv), inv), qm);
                AX[p] = fma2(f, dx, AX[p]);
                AY[p] = fma2(f, dy, AY[p]);
                AZ[p] = fma2(f, dz, AZ[p]);
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++) {
            float lo, hi;
            upk2(AX[p], lo, hi);
            ax[2 * p] += lo;
            ax[2 * p + 1] += hi;
            upk2(AY[p], lo, hi);
            ay[2 * p] += lo;
            ay[2 * p + 1] += hi;
            upk2(AZ[p], lo, hi);
            az[2 * p] += lo;
            az[2 * p + 1] += hi;
        }
    }
#pragma unroll
    for (int u = 0; u < kAudPer; u++) {
        const int k = t0 + u * kAudThreads + threadIdx.x;
        if (k >= nt) continue;
        double* o = part + ((size_t)blockIdx.y * nt + k) * 3;
        o[0] = ax[u];
        o[1] = ay[u];
        o[2] = az[u];
    }
}

// out3[v] = sum over chunks c of part[c][v], in chunk order.
__global__ void k_direct_targets_reduce(int nv, int chunks, const double* __restrict__ part,
                                        double* __restrict__ out3) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    double t = 0;
    for (int c = 0; c < chunks; c++) t += part[(size_t)c * nv + v];
    out3[v] = t;
}

namespace {
// Chunks per tile: about 8 blocks per SM in all, at least kTgtMinChunk
// sources per chunk.
int targets_chunks(int n, int nt, int sms) {
    const int tiles = ceil_div(nt, kTgtTile);
    const int want = ceil_div(sms * 8, tiles);
    return std::max(1, std::min(want, ceil_div(n, kTgtMinChunk)));
}
}  // namespace

size_t direct_targets_scratch_bytes(int sms) {
    // chunks > 1 only when tiles < 8 sms, and then chunks * nt < 2 * 8 sms * kTgtTile
    return sizeof(double) * 3 * (size_t)(16 * sms * kTgtTile);
}

void direct_targets(cudaStream_t st, int n, const State& s, double eps, int nt,
                    const int32_t* targets, double* out3, double* scratch, int sms) {
    if (nt <= 0 || n <= 0) {
        if (nt > 0) cudaMemsetAsync(out3, 0, sizeof(double) * 3 * (size_t)nt, st);
        return;
    }
    const int chunks = targets_chunks(n, nt, sms);
    const int chunk = ceil_div(ceil_div(n, chunks), kTgtThreads) * kTgtThreads;
    const int used = ceil_div(n, chunk);
    const dim3 grid(ceil_div(nt, kTgtTile), used);
    if (used == 1) {
        k_direct_targets<<<grid, kTgtThreads, 0, st>>>(n, s, eps * eps, targets, nt, chunk, out3);
        return;
    }
    k_direct_targets<<<grid, kTgtThreads, 0, st>>>(n, s, eps * eps, targets, nt, chunk, scratch);
    k_direct_targets_reduce<<<ceil_div(3 * nt, 256), 256, 0, st>>>(3 * nt, used, scratch, out3);
}

size_t audit_targets_scratch_bytes(int sms) {
    return sizeof(double) * 3 * (size_t)(2 * sms + 1) * kAudTargets;
}

bool audit_targets(cudaStream_t st, int ns, const double4* sbody, const State& s, double eps,
                   int nt, const int32_t* targets, double* out3, double* scratch, int sms) {
    if (nt <= 0 || ns <= 0 || !(eps > 0.0)) return false;
    const int tiles = ceil_div(nt, kAudTargets);
    // about two blocks per SM in all, at least kAudMinChunk sources per chunk,
    // and no more chunk partials than the scratch holds
    const size_t cap = (size_t)(2 * sms + 1) * kAudTargets;
    int chunks = std::max(1, std::min(ceil_div(2 * sms, tiles), ceil_div(ns, kAudMinChunk)));
    if ((size_t)chunks * (size_t)nt > cap) chunks = (int)(cap / (size_t)nt);
    if (chunks < 1) return false;
    const int chunk = ceil_div(ceil_div(ns, chunks), kAudTile) * kAudTile;
    const int used = ceil_div(ns, chunk);
    k_audit_targets<<<dim3(tiles, used), kAudThreads, 0, st>>>(ns, sbody, (float)(eps * eps), s,
                                                                targets, nt, chunk, scratch);
    k_direct_targets_reduce<<<ceil_div(3 * nt, 256), 256, 0, st>>>(3 * nt, used, scratch, out3);
    return true;
}

}  // namespace nb
