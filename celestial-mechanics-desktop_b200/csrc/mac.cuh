// mac.cuh - the learned multipole acceptance criterion (MAC): features of a
// (walk group, cell) pair and the warp-wide BF16 tensor-core MLP 8-64-64-1
// that predicts log2 of the cell's monopole+quadrupole force error relative
// to the group's smallest acceleration.  No reference counterpart: it
// replaces the geometric acceptance test (engine/src/cuda/gpu_tree.cu:567-569,
// src/CelestialMechanics.Physics/Solvers/BarnesHutBackend.cs:431-447) inside
// a band of opening angles.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace nb {

constexpr int kMacIn = 8, kMacHid = 64;
// FP32 master parameters, in this order.
constexpr int kMacW1 = 0;                         // [8][64]   (in, out)
constexpr int kMacB1 = kMacW1 + kMacIn * kMacHid;  // [64]
constexpr int kMacW2 = kMacB1 + kMacHid;           // [64][64]  (in, out)
constexpr int kMacB2 = kMacW2 + kMacHid * kMacHid; // [64]
constexpr int kMacW3 = kMacB2 + kMacHid;           // [64]
constexpr int kMacB3 = kMacW3 + kMacHid;           // [1]
constexpr int kMacParams = kMacB3 + 1;             // 4801

// Device image used by the kernels: weights as BF16 mma B-fragments
// (m16n8k16, lane-ordered so each lane reads one uint2), biases and the last
// layer in FP32, the feature / target normalisation, and the linear screen
// (y ~ lin_w . x_norm + lin_b, fitted to the network's own output; the walk
// asks the network only where the screen lies within lin_margin of the
// budget).
struct __align__(16) MacDev {
    uint2 w1f[8][32];      // layer 1: n-tile x lane (K padded 8 -> 16)
    uint2 w2f[4][8][32];   // layer 2: k-tile x n-tile x lane
    float b1[kMacHid], b2[kMacHid], w3[kMacHid], b3;
    float mean[kMacIn], inv_std[kMacIn];
    float y_mean, y_std;
    float lin_w[kMacIn], lin_b, lin_margin;
    // the screen on raw features (normalisation folded in):
    // y ~ scr_w . f + scr_b
    float scr_w[kMacIn], scr_b;
};
// 8-byte loads (mac_ldf2 / mac_ld2) are used on these members only
static_assert(offsetof(MacDev, w1f) % 8 == 0 && offsetof(MacDev, w2f) % 8 == 0 &&
                  offsetof(MacDev, b1) % 8 == 0 && offsetof(MacDev, b2) % 8 == 0 &&
                  offsetof(MacDev, w3) % 8 == 0,
              "8-byte aligned network members");
// host-visible screen block: lin_w[8], lin_b, lin_margin (normalised units)
constexpr int kMacScreen = kMacIn + 2;

// Harvest record: raw features and what the target kernel needs.
struct MacRecord {
    float f[kMacIn];
    int node;       // walk-tree node
    int body;       // sorted index of the group body nearest the node's COM
    float a_min;    // smallest |a| of the group's bodies (previous step)
    float pad;
};

__device__ __forceinline__ float mac_log2(float x) { return __log2f(fmaxf(x, 1e-30f)); }

// The 8 features of a (group, cell) pair; d2: squared distance from the
// cell's COM to the group's box (> 0), h: cell half-size, qn2: squared
// Frobenius norm of the traceless quadrupole.
__device__ __forceinline__ void mac_features(float f[kMacIn], float d2, float h, float mass,
                                             float qn2, int count, float r_grp, int nvalid,
                                             float a_min, float a_max, float eps) {
    const float d = sqrtf(d2);
    const float s = 2.f * h;
    f[0] = mac_log2(s / d);                                   // size over distance
    f[1] = mac_log2(sqrtf(qn2) / (mass * s * s) + 1e-6f);     // quadrupole over mass size^2
    f[2] = fminf(fmaxf(mac_log2(mass / (d2 * fmaxf(a_min, 1e-30f))), -60.f), 60.f);
    f[3] = mac_log2(r_grp / d + 1e-6f);                       // group extent over distance
    f[4] = mac_log2((float)count);
    f[5] = mac_log2((float)nvalid);
    f[6] = mac_log2(d / fmaxf(eps, 1e-30f));
    f[7] = fminf(mac_log2(a_max / fmaxf(a_min, 1e-30f)), 60.f);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b.x), "r"(b.y));
}

// Global loads of the network image that the compiler may not hoist out of
// the caller's loops (the walk would otherwise keep the 40 weight fragments
// in registers for the whole traversal and spill).
__device__ __forceinline__ uint2 mac_ld2(const uint2* p) {
    uint2 v;
    asm volatile("ld.global.nc.v2.u32 {%0,%1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float2 mac_ldf2(const float* p) {
    float2 v;
    asm volatile("ld.global.nc.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float mac_ldf(const float* p) {
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

// Warp-wide MLP on up to 32 rows staged in xs (row-major, 8 BF16 per row =
// 4 uint32).  rows: number of valid rows (<= 16 uses one m-tile).  Writes the
// normalised prediction of each row to ys[row].  w: the image in global
// memory.  All 32 lanes must call it.
__device__ __forceinline__ void mac_mlp_warp(const MacDev* w, const uint32_t* xs, float* ys,
                                             int rows) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mtiles = rows > 16 ? 2 : 1;
    for (int mt = 0; mt < mtiles; mt++) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        // layer 1 A fragment: columns 2t, 2t+1 of the 8 features; 8..15 are 0
        const uint32_t a0 = xs[r0 * 4 + t], a1 = xs[r1 * 4 + t];
        uint32_t h1[4][4];  // layer-2 A fragments (k-tiles of 16 hidden units)
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int nt = 2 * kt + half;
                const float2 bb = mac_ldf2(&w->b1[nt * 8 + 2 * t]);
                float c[4] = {bb.x, bb.y, bb.x, bb.y};
                mma_bf16(c, a0, a1, 0u, 0u, mac_ld2(&w->w1f[nt][lane]));
                h1[kt][2 * half + 0] = pack_bf16(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
                h1[kt][2 * half + 1] = pack_bf16(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
            }
        }
        float y0 = 0.f, y1 = 0.f;
#pragma unroll 2
        for (int nt = 0; nt < 8; nt++) {
            const float2 bb = mac_ldf2(&w->b2[nt * 8 + 2 * t]);
            float c[4] = {bb.x, bb.y, bb.x, bb.y};
#pragma unroll
            for (int kt = 0; kt < 4; kt++)
                mma_bf16(c, h1[kt][0], h1[kt][1], h1[kt][2], h1[kt][3], mac_ld2(&w->w2f[kt][nt][lane]));
            const float2 ww = mac_ldf2(&w->w3[nt * 8 + 2 * t]);
            y0 = fmaf(fmaxf(c[0], 0.f), ww.x, fmaf(fmaxf(c[1], 0.f), ww.y, y0));
            y1 = fmaf(fmaxf(c[2], 0.f), ww.x, fmaf(fmaxf(c[3], 0.f), ww.y, y1));
        }
        y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 1);
        y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 2);
        y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 1);
        y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 2);
        if (t == 0) {
            const float b3 = mac_ldf(&w->b3);
            ys[r0] = y0 + b3;
            ys[r1] = y1 + b3;
        }
    }
    __syncwarp();
}

}  // namespace nb
