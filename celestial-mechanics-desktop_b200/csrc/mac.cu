// mac.cu - training data, training and the device image of the learned MAC.
//
// * k_mac_targets: for every harvested (group, cell) record, the exact FP64
//   force of the cell's bodies on the group body nearest the cell's centre of
//   mass against the monopole+quadrupole approximation the walk uses; the
//   target is log2(|difference| / smallest |a| of the group).  One warp per
//   record splits the cell's bodies.
// * k_mac_train: forward and backward of the 8-64-64-1 network on 16-row
//   tiles per warp with BF16 mma.sync tensor-core tiles (FP32 accumulate) for
//   every product: X W1, H1 W2, the activation gradient G2 W2^T, and the
//   weight gradients H1^T G2 and X^T G1.  Block partial gradients go to shared
//   memory, then once per block to the global FP32 gradient.
// * k_mac_adam: Adam on the FP32 master parameters; k_mac_image rebuilds the
//   BF16 fragment image (MacDev) the walk and the training kernel read.
#include "mac.cuh"
#include "mac_train.cuh"
#include "sort.cuh"
#include "tree.cuh"

namespace nb {

// ---- targets ---------------------------------------------------------------

__global__ void k_mac_targets(int nrec, const MacRecord* __restrict__ rec,
                              const double4* __restrict__ sbody, TreeBufs t, double eps2,
                              float* __restrict__ X, float* __restrict__ Y, int* __restrict__ n_out,
                              int out_off, int out_cap) {
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= nrec) return;
    const MacRecord R = rec[r];
    const double4 b = sbody[R.body];
    const int4 lk = t.link[R.node];
    double ex = 0, ey = 0, ez = 0;
    for (int j = lk.z + lane; j < lk.z + lk.w; j += 32) {
        if (j == R.body) continue;
        const double4 p = sbody[j];
        const double dx = p.x - b.x, dy = p.y - b.y, dz = p.z - b.z;
        const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + eps2);
        const double f = p.w * inv * inv * inv;
        ex += f * dx;
        ey += f * dy;
        ez += f * dz;
    }
    ex = warp_sum(ex);
    ey = warp_sum(ey);
    ez = warp_sum(ez);
    if (lane != 0) return;
    // the walk's approximation, in FP64: d = body - COM
    const double4 cm = t.com[R.node];
    const float4 q0 = t.q0[R.node];
    const double qxx = q0.x, qyy = q0.y, qxy = q0.z, qxz = q0.w, qyz = t.q1[R.node].x;
    const double qzz = -(qxx + qyy);
    const double dx = b.x - cm.x, dy = b.y - cm.y, dz = b.z - cm.z;
    const double r2 = dx * dx + dy * dy + dz * dz + eps2;
    const double inv = 1.0 / sqrt(r2);
    const double inv2 = inv * inv, inv3 = inv * inv2, inv5 = inv3 * inv2;
    const double qx = qxx * dx + qxy * dy + qxz * dz;
    const double qy = qxy * dx + qyy * dy + qyz * dz;
    const double qz = qxz * dx + qyz * dy + qzz * dz;
    const double rqr = dx * qx + dy * qy + dz * qz;
    const double f = -cm.w * inv3 - 2.5 * rqr * inv5 * inv2;
    const double ax = f * dx + qx * inv5, ay = f * dy + qy * inv5, az = f * dz + qz * inv5;
    const double err = sqrt((ax - ex) * (ax - ex) + (ay - ey) * (ay - ey) + (az - ez) * (az - ez));
    (void)n_out;
    const int slot = r;  // records come sorted, usable ones first (mac_sort_records)
    if (out_off + slot >= out_cap) return;
    for (int k = 0; k < kMacIn; k++) X[(size_t)(out_off + slot) * kMacIn + k] = R.f[k];
    Y[out_off + slot] = (float)log2(err / (double)R.a_min + 1e-30);
}

// Harvest records in a fixed order: key = (no |a| estimate) << 63 | body << 32
// | node, so the training set does not depend on the order in which warps
// appended records; usable records (a_min > 0) are counted into *n_valid.
__global__ void k_mac_rec_keys(int nrec, const MacRecord* __restrict__ rec,
                               uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                               int* __restrict__ n_valid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrec) return;
    const MacRecord R = rec[i];
    const bool ok = R.a_min > 0.f;
    keys[i] = ((uint64_t)(ok ? 0 : 1) << 63) | ((uint64_t)(uint32_t)R.body << 32) |
              (uint64_t)(uint32_t)R.node;
    vals[i] = (uint32_t)i;
    if (ok) atomicAdd(n_valid, 1);
}

__global__ void k_mac_rec_gather(int nrec, const MacRecord* __restrict__ rec,
                                 const uint32_t* __restrict__ order, MacRecord* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrec) out[i] = rec[order[i]];
}

void mac_sort_records(cudaStream_t st, int nrec, const MacRecord* rec, MacRecord* sorted,
                      uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, void* ws,
                      int* n_valid, int* err, int sms) {
    cudaMemsetAsync(n_valid, 0, sizeof(int), st);
    if (nrec <= 0) return;
    k_mac_rec_keys<<<ceil_div(nrec, 256), 256, 0, st>>>(nrec, rec, k0, v0, n_valid);
    sort_pairs(st, nrec, k0, v0, k1, v1, ws, false, err, sms);
    k_mac_rec_gather<<<ceil_div(nrec, 256), 256, 0, st>>>(nrec, rec, v0, sorted);
}

void mac_targets(cudaStream_t st, int nrec, const MacRecord* rec, const double4* sbody,
                 const TreeBufs& t, double eps, float* X, float* Y, int* n_out, int out_off,
                 int out_cap) {
    if (nrec <= 0) return;
    k_mac_targets<<<ceil_div((long long)nrec * 32, 256), 256, 0, st>>>(
        nrec, rec, sbody, t, eps * eps, X, Y, n_out, out_off, out_cap);
}

// ---- device image ------------------------------------------------------------

__global__ void k_mac_image(const float* __restrict__ P, const float* __restrict__ norm,
                            MacDev* __restrict__ w) {
    const int tid = threadIdx.x;
    // lane-ordered B fragments: lane = 4 * g + t holds (k = 2t, 2t+1 | 2t+8, 2t+9; n = g)
    for (int e = tid; e < 8 * 32; e += blockDim.x) {
        const int nt = e / 32, lane = e % 32, g = lane >> 2, t4 = lane & 3;
        const int n = nt * 8 + g;
        auto W1 = [&](int k) { return k < kMacIn ? P[kMacW1 + k * kMacHid + n] : 0.f; };
        w->w1f[nt][lane] = make_uint2(pack_bf16(W1(2 * t4), W1(2 * t4 + 1)),
                                      pack_bf16(W1(2 * t4 + 8), W1(2 * t4 + 9)));
    }
    for (int e = tid; e < 4 * 8 * 32; e += blockDim.x) {
        const int kt = e / 256, nt = (e / 32) % 8, lane = e % 32, g = lane >> 2, t4 = lane & 3;
        const int n = nt * 8 + g, k0 = kt * 16 + 2 * t4;
        auto W2 = [&](int k) { return P[kMacW2 + k * kMacHid + n]; };    // W2[k][n]
        w->w2f[kt][nt][lane] = make_uint2(pack_bf16(W2(k0), W2(k0 + 1)), pack_bf16(W2(k0 + 8), W2(k0 + 9)));
    }
    for (int e = tid; e < kMacHid; e += blockDim.x) {
        w->b1[e] = P[kMacB1 + e];
        w->b2[e] = P[kMacB2 + e];
        w->w3[e] = P[kMacW3 + e];
    }
    if (tid == 0) w->b3 = P[kMacB3];
    if (tid < kMacIn) {
        w->mean[tid] = norm[tid];
        w->inv_std[tid] = 1.f / norm[kMacIn + tid];
    }
    if (tid == 0) {
        w->y_mean = norm[2 * kMacIn];
        w->y_std = norm[2 * kMacIn + 1];
    }
}

void mac_image(cudaStream_t st, const float* P, const float* norm, MacDev* w) {
    k_mac_image<<<1, 256, 0, st>>>(P, norm, w);
}

// ---- training --------------------------------------------------------------

// Gradient accumulator of one training block, laid out like the parameter
// vector plus the loss; the blocks' accumulators are summed in a fixed order
// (k_mac_grad_reduce), so a gradient is bitwise reproducible.
constexpr int kAccLoss = kMacParams;
constexpr int kAccFloats = (kMacParams + 1 + 3) / 4 * 4;

// grad = the blocks' partials summed in block order; the loss is added to
// *loss (it accumulates over the batches of an epoch).
__global__ void k_mac_grad_reduce(int nblocks, const float* __restrict__ part,
                                  float* __restrict__ grad, float* __restrict__ loss) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e > kMacParams) return;
    float sum = 0.f;
#pragma unroll 8
    for (int b = 0; b < nblocks; b++) sum += part[(size_t)b * kAccFloats + e];
    if (e < kMacParams) grad[e] = sum;
    else *loss += sum;
}

__global__ void k_mac_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ m,
                           float* __restrict__ v, int n, float lr, float b1, float b2,
                           float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = G[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

size_t mac_grad_partial_bytes(int sms) { return sizeof(float) * (size_t)kAccFloats * sms * 4; }

void mac_grad(cudaStream_t st, const float* X, const float* Y, const int* order, int row0,
              int nrows, const float* P, const MacDev* w, float* grad, float* loss, int sms,
              float* part, int* err) {
    if (nrows <= 0) {
        cudaMemsetAsync(grad, 0, sizeof(float) * kMacParams, st);
        return;
    }
    // tcgen05: one CTA per SM (its shared memory admits one), tiles of 128 rows
    cudaFuncSetAttribute((const void*)k_mac_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mac_train_tc_smem());
    const int tiles = (nrows + 127) / 128;
    const int blocks = min(tiles, sms);
    k_mac_train_tc<<<blocks, 128, mac_train_tc_smem(), st>>>(
        X, Y, order, row0, nrows, P, w, 1.f / (float)nrows, part, kAccFloats, kAccLoss, err);
    k_mac_grad_reduce<<<ceil_div(kMacParams + 1, 256), 256, 0, st>>>(blocks, part, grad, loss);
}

void mac_adam(cudaStream_t st, float* P, const float* G, float* m, float* v, int step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_mac_adam<<<ceil_div(kMacParams, 256), 256, 0, st>>>(P, G, m, v, kMacParams, lr, b1, b2, c1,
                                                            c2, 1e-8f);
}

// ---- per-node screen terms (learned walk) --------------------------------------

// For every walk-tree node: the part of the linear screen that depends on the
// cell only, scr_w0 log2(2h) + scr_w1 f1 + scr_w4 log2(count) (f0 = log2 2h
// - log2 d and f1, f4 as in mac_features), and log2 of its mass.
__global__ void k_mac_node_terms(TreeBufs t, const MacDev* __restrict__ w,
                                 float2* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *t.n_nodes) return;
    const float mass = (float)t.com[i].w;
    const float4 q = t.q0[i];
    const float4 q1 = t.q1[i];
    const float s = 2.f * q1.y;
    const float qyz = q1.x, qzz = -(q.x + q.y);
    const float qn2 = q.x * q.x + q.y * q.y + qzz * qzz + 2.f * (q.z * q.z + q.w * q.w + qyz * qyz);
    const float f1 = mac_log2(sqrtf(qn2) / (mass * s * s) + 1e-6f);
    const float cn = w->scr_w[0] * mac_log2(s) + w->scr_w[1] * f1 +
                     w->scr_w[4] * mac_log2((float)t.link[i].w);
    out[i] = make_float2(cn, mac_log2(mass));
}

void mac_node_terms(cudaStream_t st, const TreeBufs& t, int n, const MacDev* w, float2* out) {
    if (n > 0) k_mac_node_terms<<<ceil_div(2LL * n, 256), 256, 0, st>>>(t, w, out);
}

// ---- prediction (the walk's inference routine on given feature rows) -------

__global__ void k_mac_predict(const float* __restrict__ X, int n, const MacDev* __restrict__ w,
                              float* __restrict__ out) {
    __shared__ uint32_t xs[4][32 * 4];
    __shared__ float ys[4][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = (blockIdx.x * 4 + warp) * 32;
    const int r = r0 + lane;
    float f[kMacIn];
    for (int k = 0; k < kMacIn; k++)
        f[k] = r < n ? (X[(size_t)r * kMacIn + k] - w->mean[k]) * w->inv_std[k] : 0.f;
    for (int k = 0; k < kMacIn; k += 2) xs[warp][lane * 4 + k / 2] = pack_bf16(f[k], f[k + 1]);
    __syncwarp();
    mac_mlp_warp(w, xs[warp], ys[warp], 32);
    if (r < n) out[r] = ys[warp][lane] * w->y_std + w->y_mean;
}

void mac_predict(cudaStream_t st, const float* X, int n, const MacDev* w, float* out) {
    if (n > 0) k_mac_predict<<<ceil_div(n, 128), 128, 0, st>>>(X, n, w, out);
}

}  // namespace nb
