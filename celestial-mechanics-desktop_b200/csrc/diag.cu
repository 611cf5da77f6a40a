// diag.cu - FP64 energy / momentum diagnostics and the force-error audit.
//
// Replaces the reference's block reductions that finish on the host
// (engine/src/cuda/reduction_kernel.cu:138-290, gpu_reduction.cu:13-40,
// 345-560) with two-level device reductions in a fixed order, so results are
// deterministic run to run; definitions follow EnergyCalculator
// (src/CelestialMechanics.Physics/Validation/EnergyCalculator.cs:16-78) and
// NewtonianGravity.ComputePotentialEnergy (Forces/NewtonianGravity.cs:68-77).
#include "diag.cuh"

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

// FP64 direct sum for target rows (ForceErrorAnalyzer's exact reference,
// CpuSingleThreadBackend arithmetic per pair): one block per target, sources
// split over the block's threads, fixed-order block reduction.
__global__ void k_direct_targets(int n, State s, double eps2, const int32_t* __restrict__ targets,
                                 double* __restrict__ out3) {
    __shared__ double sh[3][8];
    const int i = targets[blockIdx.x];
    const double xi = s.px[i], yi = s.py[i], zi = s.pz[i];
    double ax = 0, ay = 0, az = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        if (j == i || !s.active[j]) continue;
        const double dx = xi - s.px[j], dy = yi - s.py[j], dz = zi - s.pz[j];
        const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + eps2);
        const double c = s.mass[j] * inv * inv * inv;
        ax -= c * dx;
        ay -= c * dy;
        az -= c * dz;
    }
    ax = warp_sum(ax);
    ay = warp_sum(ay);
    az = warp_sum(az);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = ax;
        sh[1][warp] = ay;
        sh[2][warp] = az;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[threadIdx.x][w];
        out3[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
    }
}

void direct_targets(cudaStream_t st, int n, const State& s, double eps, int nt,
                    const int32_t* targets, double* out3) {
    if (nt > 0) k_direct_targets<<<nt, 256, 0, st>>>(n, s, eps * eps, targets, out3);
}

}  // namespace nb
