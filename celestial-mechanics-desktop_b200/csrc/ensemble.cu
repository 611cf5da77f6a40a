// ensemble.cu - many independent systems of uneven size, one CUDA-graph
// launch per step.
//
// No reference counterpart: the reference steps one system per
// NBodySolver.Step (src/CelestialMechanics.Physics/Solvers/NBodySolver.cs:
// 290-391) and one ComputeForces per system.  Here all systems live packed in
// one device structure-of-arrays and one Verlet step of all of them is a
// captured graph with two branches:
//   * direct branch (systems of at most ds_max_n bodies): one persistent
//     kernel over a work queue of (system, target tile) items, largest
//     systems first; each item stages its system's sources through shared
//     memory and evaluates FP32 pair forces on coordinates differenced in
//     FP64 against the system's centre of mass, with a compensated sum per
//     tile.
//     Tile shape (threads x targets per thread) is picked by nb_ens_autotune.
//   * tree branch (larger systems): one Morton sort and one tree over all of
//     them, keys = system index (12 bits, four octree levels) | a 17-bit per
//     axis Morton code in the system's own cube; the octree below level 4 is
//     then per system, multipoles take each system's cell sizes, and the
//     persistent group walk starts every group at its own system's root.
// Kick-drift and the closing kick are single launches over all bodies.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "bodies.cuh"
#include "sort.cuh"
#include "tree.cuh"
#include "walk.cuh"
#include "../../include/nbody_b200.h"

namespace nb {
namespace {

struct EnsScal {
    unsigned long long bbox_ord[6];
    int n_active;
    unsigned group_ctr;
    int n_groups;
    unsigned ds_ctr;
    int err[kErrCount];
    unsigned long long counters[4];
};

// ---- direct branch ---------------------------------------------------------

struct EnsDirect {
    const double *px, *py, *pz, *m;
    double *ax, *ay, *az;
    const int* off;        // system offsets (internal order)
    const double4* ref;    // per system: centre of mass (reference point), mass
    const int2* items;     // (system, tile)
    int n_items;
    unsigned* ctr;         // work-queue counter (zeroed per launch)
    float eps2;
};

__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

template <int TPB, int TPT, bool GUARD>
__global__ void __launch_bounds__(TPB) k_ens_direct(EnsDirect a) {
    __shared__ float4 sj[TPB];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(a.ctr, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has the item before thread 0 fetches the next
        if (it >= a.n_items) break;
        const int2 w = a.items[it];
        const int b0 = a.off[w.x], ns = a.off[w.x + 1] - b0;
        const double4 c = a.ref[w.x];
        const double cx = c.x, cy = c.y, cz = c.z;
        float xi[TPT], yi[TPT], zi[TPT];
        float fx[TPT], fy[TPT], fz[TPT], kx[TPT], ky[TPT], kz[TPT];
#pragma unroll
        for (int k = 0; k < TPT; k++) {
            const int t = w.y * TPB * TPT + k * TPB + threadIdx.x;
            const bool v = t < ns;
            xi[k] = v ? (float)(a.px[b0 + t] - cx) : 0.f;
            yi[k] = v ? (float)(a.py[b0 + t] - cy) : 0.f;
            zi[k] = v ? (float)(a.pz[b0 + t] - cz) : 0.f;
            fx[k] = fy[k] = fz[k] = kx[k] = ky[k] = kz[k] = 0.f;
        }
        for (int j0 = 0; j0 < ns; j0 += TPB) {
            const int j = j0 + threadIdx.x;
            sj[threadIdx.x] = j < ns ? make_float4((float)(a.px[b0 + j] - cx),
                                                   (float)(a.py[b0 + j] - cy),
                                                   (float)(a.pz[b0 + j] - cz), (float)a.m[b0 + j])
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
            __syncthreads();
            const int jn = min(TPB, ns - j0);
            float tx[TPT], ty[TPT], tz[TPT];
#pragma unroll
            for (int k = 0; k < TPT; k++) tx[k] = ty[k] = tz[k] = 0.f;
#pragma unroll 4
            for (int jj = 0; jj < jn; jj++) {
                const float4 q = sj[jj];
#pragma unroll
                for (int k = 0; k < TPT; k++) {
                    const float dx = q.x - xi[k], dy = q.y - yi[k], dz = q.z - zi[k];
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, a.eps2)));
                    float inv = rsqrt_ftz(r2);
                    if (GUARD) inv = r2 > 0.f ? inv : 0.f;
                    const float s = q.w * inv * inv * inv;
                    tx[k] = fmaf(dx, s, tx[k]);
                    ty[k] = fmaf(dy, s, ty[k]);
                    tz[k] = fmaf(dz, s, tz[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < TPT; k++) {
                kahan_add(fx[k], kx[k], tx[k]);
                kahan_add(fy[k], ky[k], ty[k]);
                kahan_add(fz[k], kz[k], tz[k]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int k = 0; k < TPT; k++) {
            const int t = w.y * TPB * TPT + k * TPB + threadIdx.x;
            if (t < ns) {
                a.ax[b0 + t] = (double)fx[k];
                a.ay[b0 + t] = (double)fy[k];
                a.az[b0 + t] = (double)fz[k];
            }
        }
    }
}

// Tile shapes the autotuner chooses from: threads per block x targets per thread.
struct DirectShape {
    int tpb, tpt;
};
constexpr DirectShape kShapes[] = {{64, 1}, {64, 2}, {64, 4}, {128, 1}, {128, 2},
                                   {128, 4}, {256, 1}, {256, 2}, {256, 4}};
constexpr int kNumShapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));

using DirectKernel = void (*)(EnsDirect);

template <int TPB, int TPT>
DirectKernel pick2(bool guard) {
    return guard ? k_ens_direct<TPB, TPT, true> : k_ens_direct<TPB, TPT, false>;
}

DirectKernel pick_direct(int shape, bool guard) {
    switch (shape) {
        case 0: return pick2<64, 1>(guard);
        case 1: return pick2<64, 2>(guard);
        case 2: return pick2<64, 4>(guard);
        case 3: return pick2<128, 1>(guard);
        case 4: return pick2<128, 2>(guard);
        case 5: return pick2<128, 4>(guard);
        case 6: return pick2<256, 1>(guard);
        case 7: return pick2<256, 2>(guard);
        default: return pick2<256, 4>(guard);
    }
}

// ---- tree branch -----------------------------------------------------------

// One block per system: bounding box -> cube (cx, cy, cz, half) with the
// single-system rule (max extent / 2, floor 1e-10, x 1.001), half x 16, and
// the centre of mass (the bounding-box centre for a massless system).  Sums
// are reduced in a fixed order, so the result does not depend on timing.
__global__ void k_ens_cubes(const int* __restrict__ off, State s, double4* __restrict__ cubes,
                            double* __restrict__ half16, double4* __restrict__ com) {
    __shared__ double red[10][32];
    const int sys = blockIdx.x;
    const int b0 = off[sys], b1 = off[sys + 1];
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    double sm[4] = {0.0, 0.0, 0.0, 0.0};  // m, m x, m y, m z
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double p[3] = {s.px[i], s.py[i], s.pz[i]};
        const double m = s.mass[i];
        for (int k = 0; k < 3; k++) {
            mn[k] = fmin(mn[k], p[k]);
            mx[k] = fmax(mx[k], p[k]);
            sm[1 + k] += m * p[k];
        }
        sm[0] += m;
    }
    for (int k = 0; k < 3; k++) {
        mn[k] = warp_min(mn[k]);
        mx[k] = warp_max(mx[k]);
    }
    for (int k = 0; k < 4; k++)
        for (int o = 16; o > 0; o >>= 1) sm[k] += __shfl_xor_sync(0xFFFFFFFFu, sm[k], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        for (int k = 0; k < 3; k++) {
            red[k][wid] = mn[k];
            red[3 + k][wid] = mx[k];
        }
        for (int k = 0; k < 4; k++) red[6 + k][wid] = sm[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; w++) {
            for (int k = 0; k < 3; k++) {
                red[k][0] = fmin(red[k][0], red[k][w]);
                red[3 + k][0] = fmax(red[3 + k][0], red[3 + k][w]);
            }
            for (int k = 0; k < 4; k++) red[6 + k][0] += red[6 + k][w];
        }
        const double cx = __dmul_rn(__dadd_rn(red[0][0], red[3][0]), 0.5);
        const double cy = __dmul_rn(__dadd_rn(red[1][0], red[4][0]), 0.5);
        const double cz = __dmul_rn(__dadd_rn(red[2][0], red[5][0]), 0.5);
        const double e = fmax(fmax(__dsub_rn(red[3][0], red[0][0]), __dsub_rn(red[4][0], red[1][0])),
                              __dsub_rn(red[5][0], red[2][0]));
        double h = fmax(__dmul_rn(e, 0.5), 1e-10);
        h = __dmul_rn(h, 1.001);
        cubes[sys] = make_double4(cx, cy, cz, h);
        half16[sys] = h * 16.0;
        const double M = red[6][0];
        com[sys] = M > 0.0 ? make_double4(red[7][0] / M, red[8][0] / M, red[9][0] / M, M)
                           : make_double4(cx, cy, cz, 0.0);
    }
}

__device__ __forceinline__ uint64_t quant17(double p, double lo, double inv2h) {
    double u = __dmul_rn(__dsub_rn(p, lo), inv2h);
    u = fmax(0.0, fmin(1.0, u));
    const uint64_t q = (uint64_t)__dmul_rn(u, 131072.0);
    return q > 131071ull ? 131071ull : q;
}

// Keys (system | 17-bit Morton in the system's cube) and the 8 digit
// histograms of the radix sort (hist zeroed before); kEnsKeyItems keys per
// thread, so a block's shared bins cover 2048 keys before the global adds.
constexpr int kEnsKeyItems = 8;
__global__ void k_ens_keys(int n, State s, const int* __restrict__ sys_of,
                           const double4* __restrict__ cubes, uint64_t* __restrict__ keys,
                           uint32_t* __restrict__ vals, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[8][256];
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    for (int k = 0; k < kEnsKeyItems; k++) {
        const int i = (blockIdx.x * kEnsKeyItems + k) * blockDim.x + threadIdx.x;
        uint64_t key = 0;
        if (i < n) {
            const int sys = sys_of[i];
            const double4 c = cubes[sys];
            const double inv2h = 1.0 / __dmul_rn(2.0, c.w);
            const double lx = __dsub_rn(c.x, c.w), ly = __dsub_rn(c.y, c.w), lz = __dsub_rn(c.z, c.w);
            key = ((uint64_t)sys << kEnsSysShift) |
                  (spread21(quant17(s.px[i], lx, inv2h)) << 2) |
                  (spread21(quant17(s.py[i], ly, inv2h)) << 1) | spread21(quant17(s.pz[i], lz, inv2h));
            keys[i] = key;
            vals[i] = (uint32_t)i;
        }
#pragma unroll
        for (int p = 0; p < 8; p++) {
            const uint32_t d = (uint32_t)(key >> (8 * p)) & 0xFF;
            const bool live = i < n;
            const unsigned lm = __ballot_sync(0xFFFFFFFFu, live);
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, live ? d : 0x100u) & lm;
            if (live && (peers & lanemask_lt()) == 0) atomicAdd(&sh[p][d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) {
        const uint32_t v = (&sh[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

// The root of system s is the shallowest walk-tree node whose body range is
// exactly the system's sorted range (the common key prefix of a system is at
// least its 12 system bits, so that node holds no other system's bodies).
__global__ void k_ens_roots(TreeBufs t, const uint64_t* __restrict__ skeys,
                            const int* __restrict__ off, unsigned long long* __restrict__ best) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= *t.n_nodes) return;
    const int4 lk = t.link[w];
    if (lk.w <= 0) return;
    const int sys = (int)(skeys[lk.z] >> kEnsSysShift);
    if (lk.z == off[sys] && lk.w == off[sys + 1] - off[sys])
        atomicMin(&best[sys], ((unsigned long long)t.level[w] << 32) | (unsigned)w);
}

__global__ void k_ens_roots_unpack(int nsys, const unsigned long long* __restrict__ best,
                                   int* __restrict__ root, int* err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const unsigned long long b = best[s];
    if (b == ~0ull) {
        dev_flag(err, kErrCapacity);
        root[s] = 0;
    } else {
        root[s] = (int)(b & 0xFFFFFFFFull);
    }
}

// ---- audits ----------------------------------------------------------------

// FP64 direct sum of target rows against their own system: one warp per
// (system, target); writes |a - a_ref|^2 and |a_ref|^2.
__global__ void k_ens_audit(const int2* __restrict__ items, int n_items, const int* __restrict__ off,
                            const double* __restrict__ px, const double* __restrict__ py,
                            const double* __restrict__ pz, const double* __restrict__ m,
                            const double* __restrict__ ax, const double* __restrict__ ay,
                            const double* __restrict__ az, double eps2, double2* __restrict__ out) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= n_items) return;
    const int2 it = items[wid];  // system, body (absolute row)
    const int b0 = off[it.x], b1 = off[it.x + 1], i = it.y;
    const double xi = px[i], yi = py[i], zi = pz[i];
    double sx = 0, sy = 0, sz = 0;
    for (int j = b0 + lane; j < b1; j += 32) {
        if (j == i) continue;
        const double dx = px[j] - xi, dy = py[j] - yi, dz = pz[j] - zi;
        const double r2 = dx * dx + dy * dy + dz * dz + eps2;
        if (!(r2 > 0.0)) continue;
        const double inv = 1.0 / sqrt(r2);
        const double s = m[j] * inv * inv * inv;
        sx += dx * s;
        sy += dy * s;
        sz += dz * s;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xFFFFFFFFu, sx, o);
        sy += __shfl_xor_sync(0xFFFFFFFFu, sy, o);
        sz += __shfl_xor_sync(0xFFFFFFFFu, sz, o);
    }
    if (lane == 0) {
        const double ex = ax[i] - sx, ey = ay[i] - sy, ez = az[i] - sz;
        out[wid] = make_double2(ex * ex + ey * ey + ez * ez, sx * sx + sy * sy + sz * sz);
    }
}

// Per body: kinetic energy and half its softened potential energy inside its
// own system (FP64, one warp per body).
__global__ void k_ens_energy(int n, const int* __restrict__ sys_of_all, const int* __restrict__ off,
                             const double* __restrict__ px, const double* __restrict__ py,
                             const double* __restrict__ pz, const double* __restrict__ vx,
                             const double* __restrict__ vy, const double* __restrict__ vz,
                             const double* __restrict__ m, double eps2, double2* __restrict__ out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= n) return;
    const int sys = sys_of_all[i];
    const int b0 = off[sys], b1 = off[sys + 1];
    const double xi = px[i], yi = py[i], zi = pz[i];
    double pe = 0;
    for (int j = b0 + lane; j < b1; j += 32) {
        if (j == i) continue;
        const double dx = px[j] - xi, dy = py[j] - yi, dz = pz[j] - zi;
        pe += m[j] / sqrt(dx * dx + dy * dy + dz * dz + eps2);
    }
    for (int o = 16; o > 0; o >>= 1) pe += __shfl_xor_sync(0xFFFFFFFFu, pe, o);
    if (lane == 0) {
        const double v2 = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
        out[i] = make_double2(0.5 * m[i] * v2, -0.5 * m[i] * pe);
    }
}

__global__ void k_permute(int n, const int* __restrict__ perm, const double* __restrict__ src,
                          double* __restrict__ dst, int scatter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (scatter) dst[perm[i]] = src[i];
    else dst[i] = src[perm[i]];
}

}  // namespace
}  // namespace nb

struct nb_ensemble {
    int device = 0, sms = 148;
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    char err_msg[512] = {0};
    std::vector<void*> allocs;
    // systems: caller order -> internal order (direct systems first)
    int nsys = 0, nds = 0, nbh = 0;        // systems
    int n = 0, n_ds = 0, n_bh = 0;        // bodies
    std::vector<int> sizes;               // caller order
    std::vector<int> order;               // internal position -> caller system
    std::vector<int> caller_off;          // caller-order offsets
    std::vector<int> off;                 // internal offsets
    int ds_max_n = 2048;
    double theta = 0.5;
    int leaf_cap = 8;
    int walk_shape = 0;                   // tree branch: walk block shape (0: 8 warps, 1: 4)
    int group_span = 0;                   // tree branch: walk-group span (0: sibling packing)
    int group_bodies = 32;                // tree branch: bodies per walk group (64 with span >= 64)
    int shape = 4;                        // direct tile shape (128 x 2 until tuned)
    int shape_blocks[nb::kNumShapes] = {0};  // resident blocks per SM of each shape
    // device
    nb::State s{}, sbh{};
    int *d_off = nullptr, *d_off_bh = nullptr, *d_sys_of_bh = nullptr, *d_sys_of = nullptr;
    int* d_perm = nullptr;                // internal row -> caller row
    double* d_stage = nullptr;
    double4* d_cubes = nullptr;           // per system (internal order)
    double* d_half16 = nullptr;
    double4* d_com = nullptr;
    int* d_root = nullptr;
    unsigned long long* d_root_best = nullptr;
    int2* d_items = nullptr;
    int n_items = 0, items_cap = 0;
    uint64_t *keys0 = nullptr, *keys1 = nullptr;
    uint32_t *vals0 = nullptr, *vals1 = nullptr;
    void* sort_ws = nullptr;
    double4* sbody = nullptr;
    void* tree_mem = nullptr;
    nb::TreeBufs tree{};
    int* front = nullptr;
    int2* groups = nullptr;
    nb::WalkConfig wcfg{};
    nb::EnsScal* scal = nullptr;
    // state
    bool has_state = false, has_acc = false;
    // graph of one step
    cudaGraphExec_t graph = nullptr;
    double g_dt = 0, g_eps = -1, g_theta = -1;
    int g_shape = -1, g_walk = -1, g_span = -1, g_bodies = -1;
    // counters of the last evaluation
    long long ds_pairs = 0;
    long long bh_cell = 0, bh_body = 0;
    long long graph_launches = 0;
    float last_ms = 0.f;
};

namespace {

using nb::EnsScal;

int efail(nb_ensemble* h, int code, const char* fmt, ...) {
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err_msg, sizeof(h->err_msg), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define NE_CUDA(h, call)                                                                 \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return efail((h), NB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int ealloc(nb_ensemble* h, T** p, size_t count) {
    const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
        return efail(h, NB_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    h->allocs.push_back(q);
    *p = (T*)q;
    return NB_OK;
}

int ens_check(nb_ensemble* h) {
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st2);
    if (e != cudaSuccess) return efail(h, NB_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return efail(h, NB_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    int err[nb::kErrCount];
    e = cudaMemcpy(err, h->scal->err, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return efail(h, NB_ERR_CUDA, "error word: %s", cudaGetErrorString(e));
    cudaMemsetAsync(h->scal->err, 0, sizeof(err), h->st);
    if (err[nb::kErrNonFinite]) return efail(h, NB_ERR_NONFINITE, "non-finite position or mass");
    if (err[nb::kErrTimeout]) return efail(h, NB_ERR_TIMEOUT, "a bounded device wait expired");
    if (err[nb::kErrOverflow]) return efail(h, NB_ERR_STACK_OVERFLOW, "tree-walk frontier overflow");
    if (err[nb::kErrCapacity]) return efail(h, NB_ERR_CAPACITY, "a system root was not found");
    return NB_OK;
}

// Work items of the direct branch for a tile shape: (system, tile), systems
// with more bodies first so the longest items start first.
int build_items(nb_ensemble* h, int shape) {
    const int tile = nb::kShapes[shape].tpb * nb::kShapes[shape].tpt;
    std::vector<int> sysv(h->nds);
    std::iota(sysv.begin(), sysv.end(), 0);
    std::stable_sort(sysv.begin(), sysv.end(), [&](int a, int b) {
        return (h->off[a + 1] - h->off[a]) > (h->off[b + 1] - h->off[b]);
    });
    std::vector<int2> items;
    for (int k : sysv) {
        const int ns = h->off[k + 1] - h->off[k];
        for (int t = 0; t * tile < ns; t++) items.push_back(make_int2(k, t));
    }
    h->n_items = (int)items.size();
    if (h->n_items > h->items_cap) return efail(h, NB_ERR_CAPACITY, "direct work items");
    if (h->n_items)
        NE_CUDA(h, cudaMemcpyAsync(h->d_items, items.data(), sizeof(int2) * items.size(),
                                   cudaMemcpyHostToDevice, h->st));
    NE_CUDA(h, cudaStreamSynchronize(h->st));
    return NB_OK;
}

void launch_direct(nb_ensemble* h, cudaStream_t st, double eps) {
    if (h->n_items <= 0) return;
    cudaMemsetAsync(&h->scal->ds_ctr, 0, sizeof(unsigned), st);
    nb::EnsDirect a;
    a.px = h->s.px;
    a.py = h->s.py;
    a.pz = h->s.pz;
    a.m = h->s.mass;
    a.ax = h->s.ax;
    a.ay = h->s.ay;
    a.az = h->s.az;
    a.off = h->d_off;
    a.ref = h->d_com;
    a.items = h->d_items;
    a.n_items = h->n_items;
    a.ctr = &h->scal->ds_ctr;
    a.eps2 = (float)(eps * eps);
    const int grid = std::min(h->n_items, h->sms * std::max(1, h->shape_blocks[h->shape]));
    nb::pick_direct(h->shape, !(eps > 0.0))<<<grid, nb::kShapes[h->shape].tpb, 0, st>>>(a);
}

// Per-system cubes and centres of mass of the current positions.
void launch_cubes(nb_ensemble* h) {
    nb::k_ens_cubes<<<h->nsys, 256, 0, h->st>>>(h->d_off, h->s, h->d_cubes, h->d_half16,
                                                h->d_com);
}

// The tree branch: keys, sort, tree and walk of all tree systems on `st`.
void launch_tree(nb_ensemble* h, cudaStream_t st, double eps) {
    EnsScal* sc = h->scal;
    if (h->n_bh > 0) {
        const int n = h->n_bh;
        const double4* cubes = h->d_cubes + h->nds;  // tree systems follow the direct ones
        const double* half16 = h->d_half16 + h->nds;
        uint32_t* hist = (uint32_t*)h->sort_ws;
        cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, st);
        nb::k_ens_keys<<<nb::ceil_div(n, 256 * nb::kEnsKeyItems), 256, 0, st>>>(
            n, h->sbh, h->d_sys_of_bh, cubes, h->keys0, h->vals0, hist);
        nb::sort_pairs(st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, true, sc->err,
                       h->sms);
        nb::launch_gather(st, n, h->sbh, h->vals0, h->sbody, nullptr, nullptr);
        nb::tree_build(st, h->tree, n, h->keys0, h->sbody, nullptr, half16, h->leaf_cap, sc->err,
                       half16);
        cudaMemsetAsync(h->d_root_best, 0xFF, sizeof(unsigned long long) * h->nbh, st);
        nb::k_ens_roots<<<nb::ceil_div(2 * (long long)n, 256), 256, 0, st>>>(h->tree, h->keys0,
                                                                            h->d_off_bh,
                                                                            h->d_root_best);
        nb::k_ens_roots_unpack<<<nb::ceil_div(h->nbh, 128), 128, 0, st>>>(h->nbh, h->d_root_best,
                                                                         h->d_root, sc->err);
        nb::WalkArgs a{};
        a.n = n;
        a.sbody = h->sbody;
        a.skeys = h->keys0;
        a.sidx = h->vals0;
        a.t = h->tree;
        a.theta2 = h->theta * h->theta;
        a.eps2 = eps * eps;
        a.ax = h->sbh.ax;
        a.ay = h->sbh.ay;
        a.az = h->sbh.az;
        a.front = h->front;
        a.group_ctr = &sc->group_ctr;
        a.groups = h->groups;
        a.n_groups = &sc->n_groups;
        a.pack = 2.25;
        a.group_span = h->group_span;
        a.group_size = h->group_bodies;
        a.counters = sc->counters;
        a.err = sc->err;
        a.sys_root = h->d_root;
        nb::walk_group(st, h->wcfg, a, true, false, false, 0, h->walk_shape);
    }
}

// Forces at the current positions: the direct branch on the second stream,
// the tree branch on the first; the first stream waits for both.
void enqueue_forces(nb_ensemble* h, double eps) {
    EnsScal* sc = h->scal;
    launch_cubes(h);
    cudaEventRecord(h->ev_fork, h->st);
    cudaStreamWaitEvent(h->st2, h->ev_fork, 0);
    launch_direct(h, h->st2, eps);
    cudaEventRecord(h->ev_join, h->st2);
    cudaMemsetAsync(sc->counters, 0, sizeof(sc->counters), h->st);
    launch_tree(h, h->st, eps);
    cudaStreamWaitEvent(h->st, h->ev_join, 0);
}

// Walk-group spans the tree autotuner tries (0: sibling packing).  Choices
// 0..7 are walk shape k / 4 with span kEnsSpans[k % 4] and 32-body groups;
// choices 8..10 are shape 0 with span kEnsSpans[k - 7] and 64-body groups.
constexpr int kEnsSpans[4] = {0, 256, 512, 1024};
struct EnsTreeChoice {
    int shape, span, bodies;
};
static EnsTreeChoice ens_tree_choice(int k) {
    if (k < 8) return {k / 4, kEnsSpans[k % 4], 32};
    return {0, kEnsSpans[k - 7], 64};
}

// A span cell must lie inside one system: with span below the smallest tree
// system's body count, a walk-tree node holding at most `span` bodies can
// contain neither a whole system nor parts of two.
int smallest_tree_system(const nb_ensemble* h) {
    int m = 1 << 30;
    for (int k = h->nds; k < h->nsys; k++) m = std::min(m, h->off[k + 1] - h->off[k]);
    return m;
}
static_assert(NB_ENS_TREE_CHOICES == 11, "two walk shapes x four spans, and three spans of 64-body groups");

void collect(nb_ensemble* h) {
    unsigned long long c[4] = {0, 0, 0, 0};
    if (cudaMemcpy(c, h->scal->counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
        h->bh_cell = (long long)c[0];
        h->bh_body = (long long)c[1];
    }
}

int ens_graph(nb_ensemble* h, double dt, double eps) {
    if (h->graph && h->g_dt == dt && h->g_eps == eps && h->g_theta == h->theta &&
        h->g_shape == h->shape && h->g_walk == h->walk_shape && h->g_span == h->group_span &&
        h->g_bodies == h->group_bodies)
        return NB_OK;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    NE_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    EnsScal* sc = h->scal;
    nb::launch_kick_drift_bbox(h->st, h->n, h->s, true, dt, sc->bbox_ord, &sc->n_active, sc->err);
    enqueue_forces(h, eps);
    nb::launch_kick(h->st, h->n, h->s, dt);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return efail(h, NB_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        h->graph = nullptr;
        return efail(h, NB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    }
    h->g_dt = dt;
    h->g_eps = eps;
    h->g_theta = h->theta;
    h->g_shape = h->shape;
    h->g_walk = h->walk_shape;
    h->g_span = h->group_span;
    h->g_bodies = h->group_bodies;
    return NB_OK;
}

int ens_arrays(nb_ensemble* h, nb::State& s) {
    int r;
    double** d[] = {&s.px, &s.py, &s.pz, &s.vx, &s.vy, &s.vz, &s.ax, &s.ay, &s.az, &s.mass};
    for (double** p : d)
        if ((r = ealloc(h, p, (size_t)h->n))) return r;
    return ealloc(h, &s.active, (size_t)h->n);
}

}  // namespace

extern "C" {

NB_API int32_t nb_ens_create(int32_t n_systems, const int32_t* sizes, int32_t ds_max_n,
                             int32_t device, nb_ensemble** out) {
    if (!out) return NB_ERR_INVALID_ARG;
    *out = nullptr;
    if (n_systems <= 0 || !sizes || ds_max_n < 0) return NB_ERR_INVALID_ARG;
    long long total = 0;
    int ntree = 0;
    for (int i = 0; i < n_systems; i++) {
        if (sizes[i] <= 0) return NB_ERR_INVALID_ARG;
        total += sizes[i];
        if (sizes[i] > ds_max_n) ntree++;
    }
    if (total > (1ll << 30)) return NB_ERR_CAPACITY;
    if (ntree > (1 << nb::kEnsSysBits)) return NB_ERR_CAPACITY;  // system field of the keys
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return NB_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return NB_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return NB_ERR_NO_DEVICE;
    if (prop.major != 10) return NB_ERR_NO_DEVICE;  // built for sm_100a only
    nb_ensemble* h = new (std::nothrow) nb_ensemble();
    if (!h) return NB_ERR_CAPACITY;
    h->device = device;
    h->sms = prop.multiProcessorCount;
    h->nsys = n_systems;
    h->ds_max_n = ds_max_n;
    h->sizes.assign(sizes, sizes + n_systems);
    h->caller_off.assign(n_systems + 1, 0);
    for (int i = 0; i < n_systems; i++) h->caller_off[i + 1] = h->caller_off[i] + sizes[i];
    for (int i = 0; i < n_systems; i++)
        if (sizes[i] <= ds_max_n) h->order.push_back(i);
    h->nds = (int)h->order.size();
    for (int i = 0; i < n_systems; i++)
        if (sizes[i] > ds_max_n) h->order.push_back(i);
    h->nbh = n_systems - h->nds;
    h->off.assign(n_systems + 1, 0);
    for (int k = 0; k < n_systems; k++) h->off[k + 1] = h->off[k] + sizes[h->order[k]];
    h->n = h->off[n_systems];
    h->n_ds = h->off[h->nds];
    h->n_bh = h->n - h->n_ds;
    int r = NB_OK;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return NB_ERR_CUDA;
    }
    nb::sort_init();
    nb::walk_init(h->sms, h->wcfg);
    for (int k = 0; k < nb::kNumShapes; k++) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, nb::pick_direct(k, false),
                                                      nb::kShapes[k].tpb, 0);
        h->shape_blocks[k] = b;
    }
    const size_t n = (size_t)h->n, nbhb = (size_t)std::max(h->n_bh, 1);
    do {
        if ((r = ens_arrays(h, h->s))) break;
        h->sbh = h->s;
        double** v[] = {&h->sbh.px, &h->sbh.py, &h->sbh.pz, &h->sbh.vx, &h->sbh.vy, &h->sbh.vz,
                        &h->sbh.ax, &h->sbh.ay, &h->sbh.az, &h->sbh.mass};
        for (double** p : v) *p += h->n_ds;
        h->sbh.active += h->n_ds;
        if ((r = ealloc(h, &h->d_off, (size_t)n_systems + 1))) break;
        if ((r = ealloc(h, &h->d_off_bh, (size_t)h->nbh + 1))) break;
        if ((r = ealloc(h, &h->d_sys_of, n)) || (r = ealloc(h, &h->d_sys_of_bh, nbhb))) break;
        if ((r = ealloc(h, &h->d_perm, n)) || (r = ealloc(h, &h->d_stage, n))) break;
        if ((r = ealloc(h, &h->d_cubes, (size_t)n_systems)) ||
            (r = ealloc(h, &h->d_half16, (size_t)n_systems)) ||
            (r = ealloc(h, &h->d_com, (size_t)n_systems)) ||
            (r = ealloc(h, &h->d_root, (size_t)std::max(h->nbh, 1))) ||
            (r = ealloc(h, &h->d_root_best, (size_t)std::max(h->nbh, 1))))
            break;
        // enough items for the smallest tile
        h->items_cap = 0;
        for (int k = 0; k < h->nds; k++) h->items_cap += (sizes[h->order[k]] + 63) / 64;
        if ((r = ealloc(h, &h->d_items, (size_t)std::max(h->items_cap, 1)))) break;
        if (h->n_bh > 0) {
            const int cap = h->n_bh;
            if ((r = ealloc(h, &h->keys0, nbhb)) || (r = ealloc(h, &h->keys1, nbhb)) ||
                (r = ealloc(h, &h->vals0, nbhb)) || (r = ealloc(h, &h->vals1, nbhb)))
                break;
            if ((r = ealloc(h, (char**)&h->sort_ws, nb::sort_workspace_bytes(cap)))) break;
            if ((r = ealloc(h, &h->sbody, nbhb))) break;
            if ((r = ealloc(h, (char**)&h->tree_mem, nb::tree_bytes(cap)))) break;
            nb::tree_carve(h->tree, h->tree_mem, cap);
            if ((r = ealloc(h, (char**)&h->front, nb::walk_front_bytes(h->wcfg)))) break;
            if ((r = ealloc(h, &h->groups, nbhb))) break;
        }
        if ((r = ealloc(h, &h->scal, 1))) break;
        if (cudaMemset(h->scal, 0, sizeof(EnsScal)) != cudaSuccess) { r = NB_ERR_CUDA; break; }
        if (cudaMemset(h->s.active, 1, n) != cudaSuccess) { r = NB_ERR_CUDA; break; }
        // host-built maps
        std::vector<int> sys_of(n), perm(n), off_bh(h->nbh + 1), sys_of_bh(nbhb, 0);
        for (int k = 0; k < n_systems; k++)
            for (int i = h->off[k]; i < h->off[k + 1]; i++) {
                sys_of[i] = k;
                perm[i] = h->caller_off[h->order[k]] + (i - h->off[k]);
            }
        for (int k = 0; k <= h->nbh; k++) off_bh[k] = h->off[h->nds + k] - h->n_ds;
        for (int k = 0; k < h->nbh; k++)
            for (int i = off_bh[k]; i < off_bh[k + 1]; i++) sys_of_bh[i] = k;
        if (cudaMemcpy(h->d_off, h->off.data(), sizeof(int) * (n_systems + 1),
                       cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_off_bh, off_bh.data(), sizeof(int) * (h->nbh + 1),
                       cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_sys_of, sys_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(h->d_perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            cudaMemcpy(h->d_sys_of_bh, sys_of_bh.data(), sizeof(int) * nbhb,
                       cudaMemcpyHostToDevice) != cudaSuccess) {
            r = NB_ERR_CUDA;
            break;
        }
        for (cudaEvent_t* e : {&h->ev_fork, &h->ev_join})
            if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) r = NB_ERR_CUDA;
        for (cudaEvent_t* e : {&h->ev_t0, &h->ev_t1})
            if (cudaEventCreate(e) != cudaSuccess) r = NB_ERR_CUDA;
        if (r) break;
        for (int k = 0; k < h->nds; k++)
            h->ds_pairs += (long long)h->sizes[h->order[k]] * (h->sizes[h->order[k]] - 1);
        r = build_items(h, h->shape);
    } while (0);
    if (r != NB_OK) {
        nb_ens_destroy(h);
        return r;
    }
    *out = h;
    return NB_OK;
}

NB_API int32_t nb_ens_destroy(nb_ensemble* h) {
    if (!h) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->st2) cudaStreamSynchronize(h->st2);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    for (void* p : h->allocs) cudaFree(p);
    for (cudaEvent_t e : {h->ev_fork, h->ev_join, h->ev_t0, h->ev_t1})
        if (e) cudaEventDestroy(e);
    if (h->st2) cudaStreamDestroy(h->st2);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return NB_OK;
}

NB_API const char* nb_ens_last_error(const nb_ensemble* h) { return h ? h->err_msg : "null handle"; }

NB_API int32_t nb_ens_info(const nb_ensemble* h, int64_t* out, int32_t n) {
    if (!h || !out) return NB_ERR_INVALID_ARG;
    const int64_t v[] = {h->nsys, h->nds, h->nbh, h->n, h->n_ds, h->n_bh};
    for (int i = 0; i < n && i < (int)(sizeof(v) / sizeof(v[0])); i++) out[i] = v[i];
    return NB_OK;
}

NB_API int32_t nb_ens_set_param_f64(nb_ensemble* h, int32_t p, double v) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (p == NB_PARAM_THETA) {
        if (!(v >= 0.0)) return efail(h, NB_ERR_INVALID_ARG, "theta must be >= 0");
        h->theta = v;
        return NB_OK;
    }
    return efail(h, NB_ERR_INVALID_ARG, "unknown f64 parameter %d", p);
}

NB_API int32_t nb_ens_set_param_i32(nb_ensemble* h, int32_t p, int32_t v) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (p == NB_PARAM_LEAF_CAPACITY) {
        if (v < 1 || v > 32) return efail(h, NB_ERR_INVALID_ARG, "leaf capacity must be 1..32");
        h->leaf_cap = v;
        if (h->graph) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
        }
        return NB_OK;
    }
    if (p == NB_PARAM_GROUP_SPAN) {
        if (v != 0 && (v < 32 || v > 1024))
            return efail(h, NB_ERR_INVALID_ARG, "group span must be 0 or 32..1024");
        if (v != 0 && v >= smallest_tree_system(h))
            return efail(h, NB_ERR_INVALID_ARG,
                         "group span must be below the smallest tree system's body count");
        h->group_span = v;
        return NB_OK;
    }
    if (p == NB_PARAM_GROUP_BODIES) {
        if (v != 32 && v != 64) return efail(h, NB_ERR_INVALID_ARG, "group size must be 32 or 64");
        h->group_bodies = v;
        return NB_OK;
    }
    if (p == NB_PARAM_ENS_WALK_SHAPE) {
        if (v < 0 || v > 1) return efail(h, NB_ERR_INVALID_ARG, "walk shape must be 0 or 1");
        h->walk_shape = v;
        return NB_OK;
    }
    if (p == NB_PARAM_ENS_DIRECT_SHAPE) {
        if (v < 0 || v >= nb::kNumShapes)
            return efail(h, NB_ERR_INVALID_ARG, "shape must be 0..%d", nb::kNumShapes - 1);
        cudaSetDevice(h->device);
        h->shape = v;
        return build_items(h, v);
    }
    return efail(h, NB_ERR_INVALID_ARG, "unknown i32 parameter %d", p);
}

NB_API int32_t nb_ens_set_state(nb_ensemble* h, const double* px, const double* py,
                                const double* pz, const double* vx, const double* vy,
                                const double* vz, const double* mass) {
    if (!h || !px || !py || !pz || !vx || !vy || !vz || !mass) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    const double* src[] = {px, py, pz, vx, vy, vz, mass};
    double* dst[] = {h->s.px, h->s.py, h->s.pz, h->s.vx, h->s.vy, h->s.vz, h->s.mass};
    for (int k = 0; k < 7; k++) {
        for (size_t i = 0; i < (size_t)h->n; i++)
            if (!std::isfinite(src[k][i])) return efail(h, NB_ERR_NONFINITE, "non-finite input");
        NE_CUDA(h, cudaMemcpyAsync(h->d_stage, src[k], sizeof(double) * h->n,
                                   cudaMemcpyHostToDevice, h->st));
        nb::k_permute<<<nb::ceil_div(h->n, 256), 256, 0, h->st>>>(h->n, h->d_perm, h->d_stage,
                                                                 dst[k], 0);
    }
    NE_CUDA(h, cudaMemsetAsync(h->s.ax, 0, sizeof(double) * h->n, h->st));
    NE_CUDA(h, cudaMemsetAsync(h->s.ay, 0, sizeof(double) * h->n, h->st));
    NE_CUDA(h, cudaMemsetAsync(h->s.az, 0, sizeof(double) * h->n, h->st));
    h->has_state = true;
    h->has_acc = false;
    return ens_check(h);
}

NB_API int32_t nb_ens_get_state(nb_ensemble* h, double* px, double* py, double* pz, double* vx,
                                double* vy, double* vz, double* ax, double* ay, double* az) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    cudaSetDevice(h->device);
    double* dst[] = {px, py, pz, vx, vy, vz, ax, ay, az};
    const double* src[] = {h->s.px, h->s.py, h->s.pz, h->s.vx, h->s.vy, h->s.vz,
                           h->s.ax, h->s.ay, h->s.az};
    for (int k = 0; k < 9; k++) {
        if (!dst[k]) continue;
        nb::k_permute<<<nb::ceil_div(h->n, 256), 256, 0, h->st>>>(h->n, h->d_perm, src[k],
                                                                 h->d_stage, 1);
        NE_CUDA(h, cudaMemcpyAsync(dst[k], h->d_stage, sizeof(double) * h->n,
                                   cudaMemcpyDeviceToHost, h->st));
        NE_CUDA(h, cudaStreamSynchronize(h->st));
    }
    return ens_check(h);
}

NB_API int32_t nb_ens_compute_forces(nb_ensemble* h, double softening) {
    if (!h || !(softening >= 0.0)) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    cudaSetDevice(h->device);
    cudaEventRecord(h->ev_t0, h->st);
    enqueue_forces(h, softening);
    cudaEventRecord(h->ev_t1, h->st);
    int r = ens_check(h);
    if (r) return r;
    cudaEventElapsedTime(&h->last_ms, h->ev_t0, h->ev_t1);
    collect(h);
    h->has_acc = true;
    return NB_OK;
}

NB_API int32_t nb_ens_step(nb_ensemble* h, int32_t n_steps, double dt, double softening) {
    if (!h || n_steps < 0 || !(softening >= 0.0) || !std::isfinite(dt)) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    if (n_steps == 0) return NB_OK;
    cudaSetDevice(h->device);
    int r;
    if (!h->has_acc && (r = nb_ens_compute_forces(h, softening))) return r;
    if ((r = ens_graph(h, dt, softening))) return r;
    cudaEventRecord(h->ev_t0, h->st);
    for (int k = 0; k < n_steps; k++) NE_CUDA(h, cudaGraphLaunch(h->graph, h->st));
    cudaEventRecord(h->ev_t1, h->st);
    if ((r = ens_check(h))) return r;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
    h->last_ms = ms / n_steps;
    h->graph_launches += n_steps;
    collect(h);
    return NB_OK;
}

NB_API int32_t nb_ens_autotune(nb_ensemble* h, double softening, int32_t* shape,
                               double* ms_per_shape) {
    if (!h || !(softening >= 0.0)) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    cudaSetDevice(h->device);
    int best = h->shape;
    float best_ms = 1e30f;
    launch_cubes(h);  // reference points of the direct systems
    for (int k = 0; k < nb::kNumShapes; k++) {
        if (ms_per_shape) ms_per_shape[k] = -1.0;
        if (h->shape_blocks[k] <= 0) continue;
        h->shape = k;
        int r = build_items(h, k);
        if (r) return r;
        launch_direct(h, h->st, softening);  // warm-up
        float t = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            cudaEventRecord(h->ev_t0, h->st);
            launch_direct(h, h->st, softening);
            cudaEventRecord(h->ev_t1, h->st);
            if ((r = ens_check(h))) return r;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
            t = std::min(t, ms);
        }
        if (ms_per_shape) ms_per_shape[k] = t;
        if (t < best_ms) {
            best_ms = t;
            best = k;
        }
    }
    h->shape = best;
    if (shape) *shape = best;
    return build_items(h, best);
}

NB_API int32_t nb_ens_autotune_tree(nb_ensemble* h, double softening, int32_t* choice,
                                    double* ms_per_choice) {
    if (!h || !(softening >= 0.0)) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    cudaSetDevice(h->device);
    int best = 0;
    float best_ms = 1e30f;
    if (h->n_bh > 0) {
        launch_cubes(h);  // the tree systems' cubes of the current positions
        const int smallest = smallest_tree_system(h);
        for (int k = 0; k < NB_ENS_TREE_CHOICES; k++) {
            if (ms_per_choice) ms_per_choice[k] = -1.0;
            const EnsTreeChoice c = ens_tree_choice(k);
            if (c.span >= smallest) continue;  // could cross systems
            h->walk_shape = c.shape;
            h->group_span = c.span;
            h->group_bodies = c.bodies;
            launch_tree(h, h->st, softening);  // warm-up
            float t = 1e30f;
            for (int rep = 0; rep < 3; rep++) {
                cudaEventRecord(h->ev_t0, h->st);
                launch_tree(h, h->st, softening);
                cudaEventRecord(h->ev_t1, h->st);
                const int r = ens_check(h);
                if (r) return r;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1);
                t = std::min(t, ms);
            }
            if (ms_per_choice) ms_per_choice[k] = t;
            if (t < best_ms) {
                best_ms = t;
                best = k;
            }
        }
    } else if (ms_per_choice) {
        for (int k = 0; k < NB_ENS_TREE_CHOICES; k++) ms_per_choice[k] = -1.0;
    }
    const EnsTreeChoice c = ens_tree_choice(best);
    h->walk_shape = c.shape;
    h->group_span = c.span;
    h->group_bodies = c.bodies;
    if (choice) *choice = best;
    // the accelerations of the tree systems come from the chosen configuration
    if (h->n_bh > 0) {
        launch_tree(h, h->st, softening);
        return ens_check(h);
    }
    return NB_OK;
}

NB_API int32_t nb_ens_force_error(nb_ensemble* h, int32_t samples, uint64_t seed,
                                  double softening, double* rms, double* max_err) {
    if (!h || samples <= 0 || !rms || !(softening >= 0.0)) return NB_ERR_INVALID_ARG;
    if (!h->has_acc) return efail(h, NB_ERR_STATE, "no force evaluation yet");
    cudaSetDevice(h->device);
    std::vector<int2> items;
    std::vector<int> item_sys;  // caller system of each item
    for (int k = 0; k < h->nsys; k++) {
        const int ns = h->off[k + 1] - h->off[k];
        const int m = std::min(ns, samples);
        for (int q = 0; q < m; q++) {
            const int t = (int)((seed % (uint64_t)ns + (uint64_t)q * ns / m) % (uint64_t)ns);
            items.push_back(make_int2(k, h->off[k] + t));
            item_sys.push_back(h->order[k]);
        }
    }
    int2* d_it = nullptr;
    double2* d_out = nullptr;
    NE_CUDA(h, cudaMalloc(&d_it, sizeof(int2) * items.size()));
    if (cudaMalloc(&d_out, sizeof(double2) * items.size()) != cudaSuccess) {
        cudaFree(d_it);
        return efail(h, NB_ERR_CUDA, "force error: out of device memory");
    }
    std::vector<double2> res(items.size());
    cudaMemcpyAsync(d_it, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, h->st);
    const int ni = (int)items.size();
    nb::k_ens_audit<<<nb::ceil_div((long long)ni * 32, 256), 256, 0, h->st>>>(
        d_it, ni, h->d_off, h->s.px, h->s.py, h->s.pz, h->s.mass, h->s.ax, h->s.ay, h->s.az,
        softening * softening, d_out);
    cudaMemcpyAsync(res.data(), d_out, sizeof(double2) * items.size(), cudaMemcpyDeviceToHost, h->st);
    int r = ens_check(h);
    cudaFree(d_it);
    cudaFree(d_out);
    if (r) return r;
    std::vector<double> s2(h->nsys, 0.0), mx(h->nsys, 0.0);
    std::vector<int> cnt(h->nsys, 0);
    for (size_t i = 0; i < items.size(); i++) {
        if (!(res[i].y > 1e-60)) continue;
        const double e = std::sqrt(res[i].x / res[i].y);
        const int c = item_sys[i];
        s2[c] += e * e;
        mx[c] = std::max(mx[c], e);
        cnt[c]++;
    }
    for (int c = 0; c < h->nsys; c++) {
        rms[c] = cnt[c] ? std::sqrt(s2[c] / cnt[c]) : 0.0;
        if (max_err) max_err[c] = mx[c];
    }
    return NB_OK;
}

NB_API int32_t nb_ens_energy(nb_ensemble* h, double softening, double* energy, double* kinetic,
                             double* potential) {
    if (!h || !energy || !(softening >= 0.0)) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return efail(h, NB_ERR_STATE, "no state set");
    cudaSetDevice(h->device);
    double2* d_out = nullptr;
    NE_CUDA(h, cudaMalloc(&d_out, sizeof(double2) * h->n));
    std::vector<double2> res(h->n);
    nb::k_ens_energy<<<nb::ceil_div((long long)h->n * 32, 256), 256, 0, h->st>>>(
        h->n, h->d_sys_of, h->d_off, h->s.px, h->s.py, h->s.pz, h->s.vx, h->s.vy, h->s.vz,
        h->s.mass, softening * softening, d_out);
    cudaMemcpyAsync(res.data(), d_out, sizeof(double2) * h->n, cudaMemcpyDeviceToHost, h->st);
    const int r = ens_check(h);
    cudaFree(d_out);
    if (r) return r;
    for (int k = 0; k < h->nsys; k++) {
        double ke = 0, pe = 0;
        for (int i = h->off[k]; i < h->off[k + 1]; i++) {
            ke += res[i].x;
            pe += res[i].y;
        }
        const int c = h->order[k];
        energy[c] = ke + pe;
        if (kinetic) kinetic[c] = ke;
        if (potential) potential[c] = pe;
    }
    return NB_OK;
}

NB_API int32_t nb_ens_get_counters(const nb_ensemble* h, int64_t* out, int32_t n) {
    if (!h || !out) return NB_ERR_INVALID_ARG;
    const int64_t v[] = {h->ds_pairs, h->bh_cell, h->bh_body, h->graph_launches, h->n_items,
                         h->shape, h->walk_shape, h->group_span};
    for (int i = 0; i < n && i < (int)(sizeof(v) / sizeof(v[0])); i++) out[i] = v[i];
    return NB_OK;
}

NB_API int32_t nb_ens_get_timings(const nb_ensemble* h, double* ms_per_step) {
    if (!h || !ms_per_step) return NB_ERR_INVALID_ARG;
    *ms_per_step = h->last_ms;
    return NB_OK;
}

}  // extern "C"
