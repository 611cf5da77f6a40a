// sort.cu - stable LSD radix sort of (uint64 key, uint32 value) pairs.
//
// Replaces the reference's launch_radix_sort (engine/src/cuda/morton_kernel.cu:
// 87-230: 16 passes of 4 bits, a <<<1,16>>> serial prefix over all blocks and
// an unstable shared-memory atomicAdd scatter) with a one-sweep design:
//   * one histogram kernel computes the digit counts of all 8 passes at once
//     (fused into the Morton kernel on the tree path);
//   * each 8-bit pass is a single kernel: tiles of 4096, 2048 or 1024 keys
//     (by n) are ranked stably with warp ballots and staged in digit order
//     in shared memory, the per-digit tile offsets are chained across tiles
//     by decoupled look-back, and keys are written out digit-run by
//     digit-run from the staging copy.
// Every look-back spin is bounded (kSpinLimit); on expiry the kernel records
// NB_ERR_TIMEOUT in the device error word and the result is discarded.
#include "sort.cuh"

namespace nb {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
// Keys per thread: 16, 8 or 4 (tiles of 4096, 2048 or 1024 keys).  Fewer,
// larger tiles shorten the look-back chain, which bounds a pass while the
// keys sit in L2: 2048-key tiles from 2 x 256 keys per SM up to 8 x 256,
// 4096-key tiles above.  Measured per 8-pass sort (Plummer Morton keys):
// 262,145 keys 0.113 / 0.097 / 0.110 ms with 1024 / 2048 / 4096-key tiles;
// 2^20 keys 0.197 / 0.164 ms with 2048 / 4096; 2^23 keys 0.913 / 0.701 ms.
constexpr int kSortMinItems = 4;
constexpr int kSortMinTile = kSortThreads * kSortMinItems;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPre = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;
// Look-back words read per round trip: 8 and 32 measured the same (0.163
// and 0.165 ms per 2^20-key sort): past 8 the words a round trip brings are
// not what limits the chain.
#ifndef NB_SORT_LOOK
#define NB_SORT_LOOK 8
#endif
constexpr int kLookBatch = NB_SORT_LOOK;

template <int ITEMS>
const void* k_sort_pass_ptr();

void sort_init() {
    cudaFuncSetAttribute(k_sort_pass_ptr<16>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         16 * kSortThreads * 16);
    cudaFuncSetAttribute(k_sort_pass_ptr<8>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         8 * kSortThreads * 16);
    cudaFuncSetAttribute(k_sort_pass_ptr<4>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         4 * kSortThreads * 16);
}

// histograms, tile counters, and look-back words for the smallest tile
size_t sort_workspace_bytes(int capacity) {
    size_t tiles = (size_t)ceil_div(capacity > 0 ? capacity : 1, kSortMinTile);
    return sizeof(uint32_t) * (8 * 256 + 8 + 8 * tiles * 256);
}

// Digit histograms of all 8 passes (used when the keys were not produced by a
// kernel that already counted them).
__global__ void k_sort_histogram(int n, const uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ hist, const int* dn) {
    __shared__ uint32_t sh[8][256];
    n = dev_rows(n, dn);
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
#pragma unroll
        for (int p = 0; p < 8; p++) atomicAdd(&sh[p][(k >> (8 * p)) & 0xFF], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) {
        uint32_t v = (&sh[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
    return *(const volatile uint32_t*)p;
}

// Exclusive scans of two values per thread over the block's 256 threads (one
// digit each): warp shuffles, then the 8 warp totals through shared memory.
__device__ __forceinline__ void block_excl_scan2(uint32_t a, uint32_t b, uint32_t (*s_tot)[kSortWarps],
                                                 uint32_t& ea, uint32_t& eb) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = a, y = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t tx = __shfl_up_sync(0xFFFFFFFFu, x, o);
        const uint32_t ty = __shfl_up_sync(0xFFFFFFFFu, y, o);
        if (lane >= o) { x += tx; y += ty; }
    }
    if (lane == 31) { s_tot[0][warp] = x; s_tot[1][warp] = y; }
    __syncthreads();
    uint32_t pa = 0, pb = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++)
        if (w < warp) { pa += s_tot[0][w]; pb += s_tot[1][w]; }
    ea = pa + x - a;
    eb = pb + y - b;
}

// One stable 8-bit pass over tiles of ITEMS x 256 keys.  hist: the 256
// global counts of this digit; look: tiles x 256 look-back words (zeroed);
// tile_ctr: dynamic tile index.  Order of work: rank, publish the tile's
// digit counts, stage the tile in digit order in shared memory, and only then
// look back, so the predecessors' prefixes have had the staging time to
// arrive; the values never occupy registers (cp.async straight to shared
// memory), which keeps the kernel at 80 registers, 3 blocks per SM.
template <int ITEMS>
__global__ void __launch_bounds__(kSortThreads, 3)
k_sort_pass(int n, int shift, const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
            uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
            const uint32_t* __restrict__ hist, uint32_t* look, uint32_t* tile_ctr, int* err,
            const int* dn) {
    constexpr int kSortItems = ITEMS;
    constexpr int kSortTile = kSortThreads * ITEMS;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    uint64_t* s_keys = (uint64_t*)s_dyn;                    // tile-sorted keys
    uint32_t* s_vals = (uint32_t*)(s_dyn + 8 * kSortTile);  // tile-sorted values
    uint32_t* s_vin = s_vals + kSortTile;                   // values in load order
    __shared__ uint16_t s_wcnt[kSortWarps][256];  // per-warp digit counts, then offsets
    __shared__ uint32_t s_tile_excl[256];          // exclusive scan of tile counts over digits
    __shared__ uint32_t s_glob[256];               // global write base of each digit
    __shared__ uint32_t s_tot[2][kSortWarps];
    __shared__ int s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = (int)atomicAdd(tile_ctr, 1u);
    for (int t = tid; t < kSortWarps * 256; t += kSortThreads) (&s_wcnt[0][0])[t] = 0;
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * kSortTile;
    n = dev_rows(n, dn);
    // tiles past a device count that shrank: nothing to sort, and no later
    // tile looks back at them
    if (base >= n && tile > 0) return;
    const int valid = min(kSortTile, n - base);

    // Load: warp w owns the contiguous segment [base + 32 ITEMS w, + 32 ITEMS),
    // item k of lane l is element 32k + l of it, so (warp, k, lane) order is
    // index order and the ranking below is stable.  Values travel to shared
    // memory by cp.async (no registers held) in the same order.
    uint64_t key[kSortItems];
    uint32_t rk[kSortItems / 2];
    const int seg = base + warp * (32 * kSortItems);
    const int lseg = warp * (32 * kSortItems);
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        const int i = seg + k * 32 + lane;
        if (i < n) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(s_vin + lseg + k * 32 + lane);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(vin + i));
        }
    }
    asm volatile("cp.async.commit_group;");
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        int i = seg + k * 32 + lane;
        key[k] = (i < n) ? kin[i] : ~0ull;
    }
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        uint32_t d = (uint32_t)(key[k] >> shift) & 0xFF;
        unsigned peers = 0xFFFFFFFFu;
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        uint32_t before = s_wcnt[warp][d];
        const uint32_t r = before + __popc(peers & lanemask_lt());
        if (k & 1) rk[k >> 1] |= r << 16;
        else rk[k >> 1] = r;
        __syncwarp();
        if ((peers & lanemask_lt()) == 0) s_wcnt[warp][d] = (uint16_t)(before + __popc(peers));
        __syncwarp();
    }
    __syncthreads();

    // Thread t owns digit t: warp prefix, tile count.
    const int d = tid;
    uint32_t tile_cnt = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        uint32_t c = s_wcnt[w][d];
        s_wcnt[w][d] = (uint16_t)tile_cnt;
        tile_cnt += c;
    }
    uint32_t tail = (uint32_t)(kSortTile - valid);
    uint32_t real_cnt = (d == 255) ? tile_cnt - tail : tile_cnt;

    uint32_t* my = look + (size_t)tile * 256;
    if (tile == 0) atomicExch(&my[d], kFlagPre | real_cnt);
    else atomicExch(&my[d], kFlagAgg | real_cnt);

    uint32_t excl = 0;
    auto look_back = [&]() {
        if (tile > 0) {
            int j = tile - 1;
            uint32_t spins = 0;
            for (;;) {
                uint32_t v[kLookBatch];
#pragma unroll
                for (int q = 0; q < kLookBatch; q++)
                    v[q] = (j - q >= 0) ? ld_volatile(look + (size_t)(j - q) * 256 + d) : 0u;
                int used = 0;
                bool done = false;
#pragma unroll
                for (int q = 0; q < kLookBatch; q++) {
                    const uint32_t f = v[q] & ~kValMask;
                    if (f == 0) break;
                    excl += v[q] & kValMask;
                    used = q + 1;
                    if (f == kFlagPre || j - q == 0) {
                        done = true;
                        break;
                    }
                }
                if (done) break;
                j -= used;
                if (used == 0 && ++spins > kSpinLimit) {
                    dev_flag(err, kErrTimeout);
                    break;
                }
            }
            __threadfence();
            atomicExch(&my[d], kFlagPre | (excl + real_cnt));
        }
    };
    uint32_t tex, gex;
    block_excl_scan2(tile_cnt, hist[d], s_tot, tex, gex);
    s_tile_excl[d] = tex;
    asm volatile("cp.async.wait_all;");
    __syncthreads();
    // Stage in shared memory in tile-sorted order.
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        uint32_t dg = (uint32_t)(key[k] >> shift) & 0xFF;
        const uint32_t r = (k & 1) ? (rk[k >> 1] >> 16) : (rk[k >> 1] & 0xFFFFu);
        uint32_t pos = s_tile_excl[dg] + s_wcnt[warp][dg] + r;
        s_keys[pos] = key[k];
        s_vals[pos] = s_vin[lseg + k * 32 + lane];
    }
    look_back();
    s_glob[d] = gex + excl - tex;
    __syncthreads();
    for (int s = tid; s < valid; s += kSortThreads) {
        uint64_t k = s_keys[s];
        uint32_t dg = (uint32_t)(k >> shift) & 0xFF;
        uint32_t g = s_glob[dg] + (uint32_t)s;
        kout[g] = k;
        vout[g] = s_vals[s];
    }
}

template <int ITEMS>
const void* k_sort_pass_ptr() {
    return (const void*)k_sort_pass<ITEMS>;
}

// Sort n pairs.  Data starts in (k0, v0); the result ends in (k0, v0) (8
// passes, even count).  ws: sort_workspace_bytes(capacity) bytes.  When
// `hist_ready` the 8x256 histograms at the head of ws are already filled (by
// the fused Morton kernel); otherwise they are computed here.  Returns the
// first failing status among this call's own memsets and launches (the
// launches go through cudaLaunchKernelEx, whose return value belongs to that
// launch alone, so an error left pending by earlier unrelated work is
// neither reported nor cleared here).
cudaError_t sort_pairs(cudaStream_t st, int n, uint64_t* k0, uint32_t* v0, uint64_t* k1,
                       uint32_t* v1, void* ws, bool hist_ready, int* err, int sms, const int* dn) {
    if (n <= 1) return cudaSuccess;
    uint32_t* hist = (uint32_t*)ws;
    uint32_t* ctr = hist + 8 * 256;
    uint32_t* look = ctr + 8;
#ifdef NB_SORT_ITEMS
    const int items = NB_SORT_ITEMS;
#else
    const int items = n > sms * 8 * kSortThreads   ? 16
                      : n > sms * 2 * kSortThreads ? 8
                                                   : 4;
#endif
    const int tiles = ceil_div(n, items * kSortThreads);
    cudaError_t e;
    cudaLaunchConfig_t cfg = {};
    cfg.stream = st;
    if (!hist_ready) {
        if ((e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, st)) != cudaSuccess) return e;
        cfg.gridDim = dim3(min(ceil_div(n, 256 * 8), sms * 8));
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = 0;
        if ((e = cudaLaunchKernelEx(&cfg, k_sort_histogram, n, (const uint64_t*)k0, hist, dn)) !=
            cudaSuccess)
            return e;
    }
    if ((e = cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * (8 + (size_t)8 * tiles * 256), st)) !=
        cudaSuccess)
        return e;
    uint64_t* ks = k0;
    uint32_t* vs = v0;
    uint64_t* kd = k1;
    uint32_t* vd = v1;
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(kSortThreads);
    cfg.dynamicSmemBytes = (size_t)items * kSortThreads * 16;
    using Pass = void (*)(int, int, const uint64_t*, const uint32_t*, uint64_t*, uint32_t*,
                          const uint32_t*, uint32_t*, uint32_t*, int*, const int*);
    const Pass pass = items == 16 ? k_sort_pass<16> : items == 8 ? k_sort_pass<8> : k_sort_pass<4>;
    for (int p = 0; p < 8; p++) {
        if ((e = cudaLaunchKernelEx(&cfg, pass, n, 8 * p, (const uint64_t*)ks,
                                    (const uint32_t*)vs, kd, vd, (const uint32_t*)(hist + 256 * p),
                                    look + (size_t)p * tiles * 256, ctr + p, err, dn)) !=
            cudaSuccess)
            return e;
        uint64_t* tk = ks; ks = kd; kd = tk;
        uint32_t* tv = vs; vs = vd; vd = tv;
    }
    return cudaSuccess;
}

}  // namespace nb
