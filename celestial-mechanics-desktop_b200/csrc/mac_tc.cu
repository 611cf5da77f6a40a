// mac_tc.cu - the learned MAC's training step on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory).
//
// One CTA of 128 threads per SM walks the batch in tiles of 128 rows; row r
// of a tile is TMEM lane r and thread r.  The threads stage every operand in
// shared memory as BF16 in the canonical no-swizzle K-major layout (core
// matrices of 8 rows x 16 bytes; element (row, k) of an operand with K
// columns at (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// SBO = K / 8 * 128 bytes), and one thread issues the MMAs (M = 128, BF16 x
// BF16 -> FP32 in TMEM, K = 16 per instruction):
//
//   z1  = X  W1          (N 64, K 16: the 8 features padded to 16)
//   z2  = H1 W2          (N 64, K 64)       H1 = bf16(relu(z1 + b1))
//   dH1 = G2 W2^T        (N 64, K 64)       G2 = bf16(dy w3 [z2 + b2 > 0])
//   dW2 += H1^T G2       (M 64 used of 128, N 64, K = the tile's 128 rows)
//   dW1^T += G1^T X      (M 64 used, N 16, K 128)  G1 = bf16(dH1 [h1 > 0])
//
// z1, z2 and dH1 share 64 TMEM columns (each is read back with tcgen05.ld
// before the next MMA overwrites it); dW2 and dW1^T accumulate over the CTA's
// tiles in their own columns.  BF16 rounding happens at exactly the points of
// the warp-level kernel and the numpy oracle (normalised inputs, W1, W2, h1,
// g2, g1); the output layer, the loss, dy and the bias / w3 gradients are
// FP32 on the CUDA cores.  Row sums run in a fixed order (a column sum over
// a shared-memory transpose) and the tensor-core accumulation order is fixed
// by the static tile assignment, so a gradient is bitwise reproducible.
// Every wait on an MMA completion is bounded: on expiry the kernel records
// NB_ERR_TIMEOUT, stops issuing, waits (bounded) for what it issued, frees
// its tensor memory and returns.
#include "mac.cuh"
#include "mac_train.cuh"

namespace nb {

namespace {

constexpr int kTcRows = 128;     // rows per tile: TMEM lanes, threads
constexpr int kTcCols = 256;     // TMEM columns allocated per CTA
constexpr int kColZ = 0;         // z1, z2, dH1 (64 columns)
constexpr int kColDW2 = 64;      // dW2 accumulator (rows 0..63)
constexpr int kColDW1 = 128;     // dW1^T accumulator (rows 0..63, 16 columns)
constexpr uint32_t kTcSpin = 1u << 22;

// shared-memory operands (bytes from the 1024-aligned base)
__host__ __device__ constexpr uint32_t tile_bytes(int rows, int k) { return (uint32_t)rows * k * 2; }
constexpr uint32_t kOffX = 0;                                    // 128 x 16: A of z1
constexpr uint32_t kOffXT = kOffX + tile_bytes(128, 16);         // 16 x 128: B of dW1^T
constexpr uint32_t kOffW1 = kOffXT + tile_bytes(16, 128);        // 64 x 16 (n = j, k = f)
constexpr uint32_t kOffW2T = kOffW1 + tile_bytes(64, 16);        // 64 x 64 (n = j, k = i)
constexpr uint32_t kOffW2 = kOffW2T + tile_bytes(64, 64);        // 64 x 64 (n = i, k = j)
constexpr uint32_t kOffH1 = kOffW2 + tile_bytes(64, 64);         // 128 x 64: A of z2
constexpr uint32_t kOffH1T = kOffH1 + tile_bytes(128, 64);       // 128 x 128: A of dW2
constexpr uint32_t kOffG2 = kOffH1T + tile_bytes(128, 128);      // 128 x 64: A of dH1
constexpr uint32_t kOffG2T = kOffG2 + tile_bytes(128, 64);       // 64 x 128: B of dW2
constexpr uint32_t kOffG1T = kOffG2T + tile_bytes(64, 128);      // 128 x 128: A of dW1^T
constexpr uint32_t kOffRed = kOffG1T + tile_bytes(128, 128);     // 128 x 65 floats
constexpr uint32_t kOffAcc = kOffRed + 128 * 65 * 4;             // 64 x 3 + 2 floats
constexpr uint32_t kOffBar = kOffAcc + (3 * 64 + 8) * 4;         // mbarrier (8 bytes)
constexpr uint32_t kOffTmem = kOffBar + 8;                       // TMEM base address
constexpr uint32_t kTcSmem = kOffTmem + 8 + 1024;                // + alignment slack
static_assert(kOffH1T % 1024 == 0 && kOffG1T % 1024 == 0 && kOffBar % 8 == 0,
              "operand alignment");
static_assert(kTcSmem <= 227 * 1024, "one CTA's shared memory");

// Byte offset of element (row, k) in a K-major operand with K columns.
__device__ __forceinline__ uint32_t kmaj(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor of a K-major no-swizzle operand whose
// K = 16 slice starts at `addr` (shared window): leading byte offset 128
// (the two 8-column core matrices of the slice), stride byte offset K / 8 *
// 128 (the next 8 rows), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int K) {
    const uint64_t sbo = (uint64_t)(K / 8 * 128);
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((128u >> 4) & 0x3FFFu) << 16) |
           (((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D FP32, A and B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       bool accumulate) {
    // all output lanes enabled (disable-output-lane mask of zeros)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate), "r"(0u)
        : "memory");
}

// D (+)= A B^T over K in slices of 16: A rows x K at a_addr, B N x K at b_addr.
__device__ __forceinline__ void tc_gemm(uint32_t d_tmem, uint32_t a_addr, int a_K, uint32_t b_addr,
                                        int b_K, int K, uint32_t idesc, bool accumulate) {
    for (int k = 0; k < K / 16; k++)
        tc_mma(d_tmem, smem_desc(a_addr + 256u * k, a_K), smem_desc(b_addr + 256u * k, b_K), idesc,
               accumulate || k > 0);
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait for the barrier's phase; true when it completed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (uint32_t i = 0; i < kTcSpin; i++)
        if (mbar_try(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the tensor cores
__device__ __forceinline__ void fence_smem_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Fixed-order column sums of a 128 x 64 block of per-row values: each
// thread writes its row, then thread j < 64 adds column j over the rows in
// order into acc[j].  All threads call it.
__device__ __forceinline__ void col_sums(float* red, const float (&row)[64], float* acc) {
    const int t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < 64; j++) red[t * 65 + j] = row[j];
    __syncthreads();
    if (t < 64) {
        float s = 0.f;
        for (int r = 0; r < kTcRows; r++) s += red[r * 65 + t];
        acc[t] += s;
    }
    __syncthreads();
}

}  // namespace

// rows order[row0 .. row0 + nrows) of the batch; part: this CTA's partial
// gradient (kAccFloats floats per block, the loss at kAccLoss).
__global__ void __launch_bounds__(kTcRows, 1)
k_mac_train_tc(const float* __restrict__ X, const float* __restrict__ Y,
               const int* __restrict__ order, int row0, int nrows, const float* __restrict__ P,
               const MacDev* __restrict__ w, float inv_batch, float* __restrict__ part,
               int acc_floats, int loss_index, int* err) {
    extern __shared__ unsigned char s_raw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)s_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const int t = threadIdx.x, warp = t >> 5;
    float* red = (float*)(sm + kOffRed);
    float* acc = (float*)(sm + kOffAcc);  // dw3[64], db2[64], db1[64], db3, loss
    const uint32_t bar = sbase + kOffBar;
    uint32_t* tmem_slot = (uint32_t*)(sm + kOffTmem);

    // zero the operands' padding (rows 64..127 of H1^T and G1^T, features
    // 8..15) and the accumulators; load the weights as BF16
    for (int e = t; e < (int)(tile_bytes(128, 128) / 4); e += kTcRows) {
        ((uint32_t*)(sm + kOffH1T))[e] = 0u;
        ((uint32_t*)(sm + kOffG1T))[e] = 0u;
    }
    for (int e = t; e < (int)(tile_bytes(128, 16) / 4); e += kTcRows) {
        ((uint32_t*)(sm + kOffX))[e] = 0u;
        ((uint32_t*)(sm + kOffXT))[e] = 0u;
    }
    for (int e = t; e < 3 * 64 + 8; e += kTcRows) acc[e] = 0.f;
    for (int e = t; e < 64 * 16; e += kTcRows) {  // W1^T: (n = j, k = f), f >= 8 zero
        const int j = e / 16, f = e % 16;
        st_bf16(sm, kOffW1 + kmaj(j, f, 16), f < kMacIn ? P[kMacW1 + f * kMacHid + j] : 0.f);
    }
    for (int e = t; e < 64 * 64; e += kTcRows) {
        const int a = e / 64, b = e % 64;
        const float v = P[kMacW2 + a * kMacHid + b];  // W2[i = a][j = b]
        st_bf16(sm, kOffW2T + kmaj(b, a, 64), v);      // (n = j, k = i)
        st_bf16(sm, kOffW2 + kmaj(a, b, 64), v);       // (n = i, k = j)
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         sbase + kOffTmem),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes
    const float b3 = w->b3, y_mean = w->y_mean, y_std = w->y_std;

    uint32_t phase = 0;
    bool failed = false;
    int issued = 0;  // commits that may still be in flight
    // one MMA group: wait for its commit (bounded), uniformly over the CTA;
    // on expiry the phase and `issued` stay as they are for the final wait
    auto sync_mma = [&]() -> bool {
        const bool ok = mbar_wait(bar, phase);
        const bool bad = __syncthreads_or(!ok);
        if (bad) return false;
        phase ^= 1u;
        issued = 0;
        fence_after();
        return true;
    };
    const int tiles = (nrows + kTcRows - 1) / kTcRows;
    int it = 0;  // tiles done by this CTA
    for (int tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x, it++) {
        const int r = tile * kTcRows + t;
        const bool valid = r < nrows;
        const int row = valid ? order[row0 + r] : 0;
        // 1. normalised features (BF16) as X and X^T
        for (int f = 0; f < kMacIn; f++) {
            const float v = valid ? (X[(size_t)row * kMacIn + f] - w->mean[f]) * w->inv_std[f] : 0.f;
            st_bf16(sm, kOffX + kmaj(t, f, 16), v);
            st_bf16(sm, kOffXT + kmaj(f, t, 128), v);
        }
        fence_smem_async();
        __syncthreads();
        if (t == 0) {
            fence_after();
            tc_gemm(tmem + kColZ, sbase + kOffX, 16, sbase + kOffW1, 16, 16, idesc_bf16(128, 64),
                    false);
            tc_commit(bar);
        }
        issued = 1;
        if (!sync_mma()) { failed = true; break; }
        // 2. h1 = relu(z1 + b1) as H1 and H1^T
        {
            float z[32];
            for (int half = 0; half < 2; half++) {
                tmem_ld32(lane_addr + kColZ + 32 * half, z);
#pragma unroll
                for (int c = 0; c < 32; c++) {
                    const int i = 32 * half + c;
                    const __nv_bfloat16 hb = __float2bfloat16_rn(fmaxf(z[c] + w->b1[i], 0.f));
                    *reinterpret_cast<__nv_bfloat16*>(sm + kOffH1 + kmaj(t, i, 64)) = hb;
                    *reinterpret_cast<__nv_bfloat16*>(sm + kOffH1T + kmaj(i, t, 128)) = hb;
                }
            }
        }
        fence_before();
        fence_smem_async();
        __syncthreads();
        if (t == 0) {
            fence_after();
            tc_gemm(tmem + kColZ, sbase + kOffH1, 64, sbase + kOffW2T, 64, 64, idesc_bf16(128, 64),
                    false);
            tc_commit(bar);
        }
        issued = 1;
        if (!sync_mma()) { failed = true; break; }
        // 3. output, loss, dy; g2 = dy w3 [z2 + b2 > 0] as G2 and G2^T
        {
            float g[64];
            float a2[64];
            float z[32];
            for (int half = 0; half < 2; half++) {
                tmem_ld32(lane_addr + kColZ + 32 * half, z);
#pragma unroll
                for (int c = 0; c < 32; c++) a2[32 * half + c] = z[c] + w->b2[32 * half + c];
            }
            float y = 0.f;
#pragma unroll
            for (int j = 0; j < 64; j++) y = fmaf(fmaxf(a2[j], 0.f), w->w3[j], y);
            y += b3;
            float d = 0.f, lsq = 0.f;
            if (valid) {
                const float tg = (Y[row] - y_mean) / y_std;
                d = 2.f * (y - tg) * inv_batch;
                lsq = (y - tg) * (y - tg);
            }
            float row_w3[64];
#pragma unroll
            for (int j = 0; j < 64; j++) {
                g[j] = a2[j] > 0.f ? d * w->w3[j] : 0.f;
                row_w3[j] = fmaxf(a2[j], 0.f) * d;
                const __nv_bfloat16 gb = __float2bfloat16_rn(g[j]);
                *reinterpret_cast<__nv_bfloat16*>(sm + kOffG2 + kmaj(t, j, 64)) = gb;
                *reinterpret_cast<__nv_bfloat16*>(sm + kOffG2T + kmaj(j, t, 128)) = gb;
            }
            col_sums(red, row_w3, acc);        // dw3
            col_sums(red, g, acc + 64);        // db2
            // db3 and the loss: fixed-order sums over the rows
            red[t * 65] = d;
            red[t * 65 + 1] = lsq;
            __syncthreads();
            if (t == 0) {
                float sd = 0.f, sl = 0.f;
                for (int q = 0; q < kTcRows; q++) {
                    sd += red[q * 65];
                    sl += red[q * 65 + 1];
                }
                acc[192] += sd;
                acc[193] += sl;
            }
        }
        fence_before();
        fence_smem_async();
        __syncthreads();
        if (t == 0) {
            fence_after();
            tc_gemm(tmem + kColZ, sbase + kOffG2, 64, sbase + kOffW2, 64, 64, idesc_bf16(128, 64),
                    false);
            tc_gemm(tmem + kColDW2, sbase + kOffH1T, 128, sbase + kOffG2T, 128, 128,
                    idesc_bf16(128, 64), it > 0);
            tc_commit(bar);
        }
        issued = 1;
        if (!sync_mma()) { failed = true; break; }
        // 4. g1 = dH1 [h1 > 0] as G1^T; db1
        {
            float z[32];
            float g1[64];
            for (int half = 0; half < 2; half++) {
                tmem_ld32(lane_addr + kColZ + 32 * half, z);
#pragma unroll
                for (int c = 0; c < 32; c++) {
                    const int i = 32 * half + c;
                    const float hi = __bfloat162float(
                        *reinterpret_cast<const __nv_bfloat16*>(sm + kOffH1 + kmaj(t, i, 64)));
                    g1[i] = hi > 0.f ? z[c] : 0.f;
                    st_bf16(sm, kOffG1T + kmaj(i, t, 128), g1[i]);
                }
            }
            col_sums(red, g1, acc + 128);
        }
        fence_before();
        fence_smem_async();
        __syncthreads();
        if (t == 0) {
            fence_after();
            tc_gemm(tmem + kColDW1, sbase + kOffG1T, 128, sbase + kOffXT, 128, 128,
                    idesc_bf16(128, 16), it > 0);
            tc_commit(bar);
        }
        issued = 1;
        // the next tile rewrites X, H1, G2 and G1^T: wait for every reader
        if (!sync_mma()) { failed = true; break; }
    }
    if (failed) {
        if (t == 0) dev_flag(err, kErrTimeout);
        // what was issued may still complete: wait once more (bounded)
        if (issued) mbar_wait(bar, phase);
    } else if (it > 0) {
        // 5. the accumulated dW2 (rows i < 64) and dW1^T (rows j < 64)
        float* pb = part + (size_t)blockIdx.x * acc_floats;
        if (t < 64) {
            float z[32];
            for (int half = 0; half < 2; half++) {
                tmem_ld32(lane_addr + kColDW2 + 32 * half, z);
#pragma unroll
                for (int c = 0; c < 32; c++) pb[kMacW2 + t * kMacHid + 32 * half + c] = z[c];
            }
            tmem_ld32(lane_addr + kColDW1, z);
#pragma unroll
            for (int f = 0; f < kMacIn; f++) pb[kMacW1 + f * kMacHid + t] = z[f];
            pb[kMacW3 + t] = acc[t];
            pb[kMacB2 + t] = acc[64 + t];
            pb[kMacB1 + t] = acc[128 + t];
        }
        if (t == 0) {
            pb[kMacB3] = acc[192];
            pb[loss_index] = acc[193];
        }
    } else {
        // a CTA without a tile contributes zero
        float* pb = part + (size_t)blockIdx.x * acc_floats;
        for (int e = t; e < acc_floats; e += kTcRows) pb[e] = 0.f;
    }
    fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcCols)
                     : "memory");
}

size_t mac_train_tc_smem() { return kTcSmem; }

}  // namespace nb
