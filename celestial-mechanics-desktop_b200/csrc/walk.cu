// walk.cu - Barnes-Hut force walks over the walk tree.
//
// k_walk_group replaces tree_traverse_kernel (engine/src/cuda/gpu_tree.cu:
// 508-597: one thread per body, FP64, a 128-entry local stack that silently
// drops children on overflow) with a warp-cooperative walk in the style of
// Bedorf, Gaburov & Portegies Zwart 2012 (Bonsai):
//   * a warp owns a group of 32 consecutive Morton-sorted bodies and walks
//     the tree once for all of them with a warp-shared stack, testing 32
//     candidate nodes per round (one per lane);
//   * the opening test is the reference's geometric MAC, 4h^2 < theta^2 d^2
//     (gpu_tree.cu:567-569), with d the distance from the cell's centre of
//     mass to the group's bounding box, so it is at least as strict as the
//     per-body test for every body of the group;
//   * accepted cells and the bodies of opened leaves are appended (ballot /
//     warp scan) to shared-memory interaction lists that the 32 lanes then
//     evaluate against their own body: broadcast reads, FP32 FMA chains;
//   * coordinates are differenced in FP64 against the group centre once per
//     list entry and per body, then the pair math is FP32 with monopole +
//     traceless quadrupole; every list flush is summed in FP32 and folded
//     into a compensated (Kahan) accumulator;
//   * stack overflow is reported (NB_ERR_STACK_OVERFLOW), never dropped
//     silently.
#include "walk.cuh"

#include <algorithm>

namespace nb {

constexpr int kWalkWarps = 8;
constexpr int kWalkThreads = kWalkWarps * 32;
// Interaction-list capacities per warp (entries before a flush).  128 / 128
// measured within 1 % of 96 / 96 and 64 / 64 on both walks: a smaller list
// gives L1 more of the shared-memory carve-out but flushes more often.
#ifndef NB_WALK_CELL_CAP
#define NB_WALK_CELL_CAP 128
#endif
#ifndef NB_WALK_PART_CAP
#define NB_WALK_PART_CAP 128
#endif
constexpr int kCellCap = NB_WALK_CELL_CAP;
constexpr int kPartCap = NB_WALK_PART_CAP;
// a round appends up to 64 cells (its own 32 and a mid-round network call's
// 32, room made at its start) and bodies 32 at a time
static_assert(kCellCap >= 64 && kPartCap >= 32, "interaction-list capacities");
// per-warp shared memory, in floats
constexpr int kWarpFloats = kCellCap * 10 + kPartCap * 4 + kPartCap * 2 + kPartCap;
constexpr int kWalkSmem = kWalkWarps * kWarpFloats * 4;
constexpr int kMaxWalkRounds = 1 << 22;
constexpr int kMacGeometric = 0, kMacHarvest = 1, kMacLearned = 2;
// Block shape of the learned walk: warps per block and blocks per SM it is
// compiled for (its registers, not shared memory, bound the occupancy).
// 5 x 4 = 20 warps per SM at 96 registers (a few spilled) measured 1.7 %
// faster than 8 x 2 = 16 warps at 128 registers; 6 x 3 and 8 x 3 slower.
#ifndef NB_WALK_MAC_BLOCKS
#define NB_WALK_MAC_BLOCKS 4
#endif
#ifndef NB_WALK_MAC_WARPS
#define NB_WALK_MAC_WARPS 5
#endif
constexpr int kMacWarps = NB_WALK_MAC_WARPS;
// learned variant: + per warp 32 staged rows (4 words), 32 outputs and 32
// pending node ids
constexpr int kMacWarpWords = 32 * 4 + 32 + 32;
constexpr int kWalkSmemMac = kMacWarps * (kWarpFloats + kMacWarpWords) * 4;
static_assert(NB_WALK_MAC_BLOCKS * (kWalkSmemMac + 1024) <= 228 * 1024, "learned walk blocks per SM");
static_assert(kMacWarps <= kWalkWarps, "the stacks are sized for the geometric block shape");

// Non-binding prefetch of the line holding *p into L1 (no register).
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ void kahan(float& s, float& c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

// GUARD (softening 0 only): 1/r is taken as 0 at r = 0, so a body's own entry
// in its particle list adds 0 instead of 0 * inf.  With softening > 0 the
// own entry has r^2 = eps^2 and dx = dy = dz = 0, which adds exactly 0.
// MAC selects the acceptance test: kMacGeometric (4h^2 < theta^2 d^2);
// kMacHarvest (geometric at theta, and every candidate of a sampled group
// with theta <= 2h/d < theta_hi is recorded for training); kMacLearned
// (geometric below theta, open at or above theta_hi, the network decides in
// between).
// SHAPE (geometric walk only) selects the block shape: 0 = 8 warps x 3
// blocks per SM, 1 = 4 warps x 6 blocks per SM (the same warps per SM in
// smaller blocks; the ensembles' autotuner picks one).
constexpr int kWalkWarpsSmall = 4;
// GS = 64 (groups of up to 64 bodies, two per lane): more work per warp and
// more live registers, so fewer and larger-register warps per SM.
#ifndef NB_WALK64_WARPS
#define NB_WALK64_WARPS 8
#endif
#ifndef NB_WALK64_BLOCKS
#define NB_WALK64_BLOCKS 2
#endif
#ifndef NB_WALK64_MAC_WARPS
#define NB_WALK64_MAC_WARPS 4
#endif
#ifndef NB_WALK64_MAC_BLOCKS
#define NB_WALK64_MAC_BLOCKS 4
#endif
constexpr int kMacWarps64 = NB_WALK64_MAC_WARPS;
constexpr int kWalkSmemMac64 = kMacWarps64 * (kWarpFloats + kMacWarpWords) * 4;
constexpr int kWalkSmem64 = NB_WALK64_WARPS * kWarpFloats * 4;
static_assert(NB_WALK64_MAC_BLOCKS * (kWalkSmemMac64 + 1024) <= 228 * 1024, "learned walk blocks");
static_assert(kMacWarps64 <= kWalkWarps && NB_WALK64_WARPS <= kWalkWarps,
              "the stacks are sized for the geometric block shape");
template <int MAC, int SHAPE, int GS = 32>
struct WalkShape {
    static constexpr int warps =
        GS == 64 ? (MAC == kMacLearned ? kMacWarps64 : NB_WALK64_WARPS)
                 : (MAC == kMacLearned ? kMacWarps : (SHAPE == 1 ? kWalkWarpsSmall : kWalkWarps));
    static constexpr int min_blocks =
        GS == 64 ? (MAC == kMacLearned ? NB_WALK64_MAC_BLOCKS : NB_WALK64_BLOCKS)
                 : (MAC == kMacLearned ? NB_WALK_MAC_BLOCKS : (SHAPE == 1 ? 6 : 3));
};

// ---- interaction-list evaluation ---------------------------------------------
//
// Lists live in shared memory pair-blocked: field f of entry e at
// [(e / 2) * W + 2 f + e % 2] (cells W = 20: rel x, y, z, -mass, Qxx, Qyy,
// Qzz, Qxy, Qxz, Qyz; bodies W = 8: rel x, y, z, -mass), so one 16-byte load
// gives two fields of two entries as a register pair for the packed f32x2
// arithmetic.  The list loops are out-of-line functions (NB_WALK_NOINLINE):
// the learned walk reaches them from three places and inlining every copy
// cost it instruction-cache misses.
#ifdef NB_WALK_NOINLINE
#define NB_WALK_EVAL __device__ __noinline__
#else
#define NB_WALK_EVAL __device__ __forceinline__
#endif

__device__ __forceinline__ float fold2(f32x2 T) {
    float a0, a1;
    upk2(T, a0, a1);
    return a0 + a1;
}

// Terms of cell entries 2m, 2m+1 (the block at blk) on one body.
template <bool QUAD>
__device__ __forceinline__ void cell_pair_terms(const float* blk_f, float eps2, f32x2 BX, f32x2 BY,
                                                f32x2 BZ, f32x2& TX, f32x2& TY, f32x2& TZ) {
    const float4* blk = (const float4*)blk_f;
    const f32x2 E2 = pk2(eps2, eps2), M25 = pk2(-2.5f, -2.5f);
    const float4 v0 = blk[0], v1 = blk[1];
    const f32x2 dx = sub2(BX, pk2(v0.x, v0.y));
    const f32x2 dy = sub2(BY, pk2(v0.z, v0.w));
    const f32x2 dz = sub2(BZ, pk2(v1.x, v1.y));
    const f32x2 nm = pk2(v1.z, v1.w);  // -mass
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
    float ra, rb;
    upk2(r2, ra, rb);
    const f32x2 inv = pk2(rsqrt_ftz(ra), rsqrt_ftz(rb));
    const f32x2 inv2 = mul2(inv, inv);
    const f32x2 inv3 = mul2(inv, inv2);
    if constexpr (QUAD) {
        const float4 v2 = blk[2], v3 = blk[3], v4 = blk[4];
        const f32x2 qxx = pk2(v2.x, v2.y), qyy = pk2(v2.z, v2.w);
        const f32x2 qzz = pk2(v3.x, v3.y), qxy = pk2(v3.z, v3.w);
        const f32x2 qxz = pk2(v4.x, v4.y), qyz = pk2(v4.z, v4.w);
        const f32x2 qx = fma2(qxx, dx, fma2(qxy, dy, mul2(qxz, dz)));
        const f32x2 qy = fma2(qxy, dx, fma2(qyy, dy, mul2(qyz, dz)));
        const f32x2 qz = fma2(qxz, dx, fma2(qyz, dy, mul2(qzz, dz)));
        const f32x2 rqr = fma2(dx, qx, fma2(dy, qy, mul2(dz, qz)));
        const f32x2 inv5 = mul2(inv3, inv2);
        // a = -M r / r^3 + Q r / r^5 - (5/2) (r.Q.r) r / r^7
        const f32x2 f = fma2(mul2(M25, rqr), mul2(inv5, inv2), mul2(nm, inv3));
        TX = fma2(f, dx, fma2(qx, inv5, TX));
        TY = fma2(f, dy, fma2(qy, inv5, TY));
        TZ = fma2(f, dz, fma2(qz, inv5, TZ));
    } else {
        const f32x2 f = mul2(nm, inv3);
        TX = fma2(f, dx, TX);
        TY = fma2(f, dy, TY);
        TZ = fma2(f, dz, TZ);
    }
}

// Terms of body entries 2m, 2m+1 (the block at blk) on one body.  GUARD
// (softening 0 only): 1/r is taken as 0 at r = 0.
template <bool GUARD>
__device__ __forceinline__ void body_pair_terms(const float* blk_f, float eps2, f32x2 BX, f32x2 BY,
                                                f32x2 BZ, f32x2& TX, f32x2& TY, f32x2& TZ) {
    const float4* blk = (const float4*)blk_f;
    const f32x2 E2 = pk2(eps2, eps2);
    const float4 v0 = blk[0], v1 = blk[1];
    const f32x2 dx = sub2(BX, pk2(v0.x, v0.y));
    const f32x2 dy = sub2(BY, pk2(v0.z, v0.w));
    const f32x2 dz = sub2(BZ, pk2(v1.x, v1.y));
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
    float ra, rb;
    upk2(r2, ra, rb);
    const float ia = (GUARD && !(ra > 0.f)) ? 0.f : rsqrt_ftz(ra);
    const float ib = (GUARD && !(rb > 0.f)) ? 0.f : rsqrt_ftz(rb);
    const f32x2 inv = pk2(ia, ib);
    // -(m / r^3); the term is -(m/r^3) (b - p), as fmaf(-f, dx, t)
    const f32x2 f = mul2(pk2(v1.z, v1.w), mul2(mul2(inv, inv), inv));
    TX = fma2(f, dx, TX);
    TY = fma2(f, dy, TY);
    TZ = fma2(f, dz, TZ);
}

// A cell list's terms on one body: pair blocks rep, rep + nrep, ... < npair.
template <bool QUAD>
NB_WALK_EVAL float3 cells_one(const float* cbuf, int npair, int rep, int nrep, float bx, float by,
                              float bz, float eps2) {
    const f32x2 BX = pk2(bx, bx), BY = pk2(by, by), BZ = pk2(bz, bz);
    f32x2 TX = 0ull, TY = 0ull, TZ = 0ull;
#pragma unroll 2
    for (int m = rep; m < npair; m += nrep)
        cell_pair_terms<QUAD>(cbuf + m * 20, eps2, BX, BY, BZ, TX, TY, TZ);
    return make_float3(fold2(TX), fold2(TY), fold2(TZ));
}

// A cell list's terms on both bodies of a two-body lane, each pair block
// read once for the two.
template <bool QUAD>
NB_WALK_EVAL void cells_two(const float* cbuf, int npair, float bx, float by, float bz, float cx,
                            float cy, float cz, float eps2, float3& a, float3& b) {
    const f32x2 BX = pk2(bx, bx), BY = pk2(by, by), BZ = pk2(bz, bz);
    const f32x2 CX = pk2(cx, cx), CY = pk2(cy, cy), CZ = pk2(cz, cz);
    f32x2 TX = 0ull, TY = 0ull, TZ = 0ull, UX = 0ull, UY = 0ull, UZ = 0ull;
    for (int m = 0; m < npair; m++) {
        cell_pair_terms<QUAD>(cbuf + m * 20, eps2, BX, BY, BZ, TX, TY, TZ);
        cell_pair_terms<QUAD>(cbuf + m * 20, eps2, CX, CY, CZ, UX, UY, UZ);
    }
    a = make_float3(fold2(TX), fold2(TY), fold2(TZ));
    b = make_float3(fold2(UX), fold2(UY), fold2(UZ));
}

template <bool GUARD>
NB_WALK_EVAL float3 parts_one(const float* pbuf, int npair, int rep, int nrep, float bx, float by,
                              float bz, float eps2) {
    const f32x2 BX = pk2(bx, bx), BY = pk2(by, by), BZ = pk2(bz, bz);
    f32x2 TX = 0ull, TY = 0ull, TZ = 0ull;
#pragma unroll 4
    for (int m = rep; m < npair; m += nrep)
        body_pair_terms<GUARD>(pbuf + m * 8, eps2, BX, BY, BZ, TX, TY, TZ);
    return make_float3(fold2(TX), fold2(TY), fold2(TZ));
}

template <bool GUARD>
NB_WALK_EVAL void parts_two(const float* pbuf, int npair, float bx, float by, float bz, float cx,
                            float cy, float cz, float eps2, float3& a, float3& b) {
    const f32x2 BX = pk2(bx, bx), BY = pk2(by, by), BZ = pk2(bz, bz);
    const f32x2 CX = pk2(cx, cx), CY = pk2(cy, cy), CZ = pk2(cz, cz);
    f32x2 TX = 0ull, TY = 0ull, TZ = 0ull, UX = 0ull, UY = 0ull, UZ = 0ull;
#pragma unroll 2
    for (int m = 0; m < npair; m++) {
        body_pair_terms<GUARD>(pbuf + m * 8, eps2, BX, BY, BZ, TX, TY, TZ);
        body_pair_terms<GUARD>(pbuf + m * 8, eps2, CX, CY, CZ, UX, UY, UZ);
    }
    a = make_float3(fold2(TX), fold2(TY), fold2(TZ));
    b = make_float3(fold2(UX), fold2(UY), fold2(UZ));
}

template <bool QUAD, bool SHELL, bool POT, bool GUARD, int MAC, int SHAPE = 0, int GS = 32>
__global__ void __launch_bounds__(WalkShape<MAC, SHAPE, GS>::warps * 32,
                                  WalkShape<MAC, SHAPE, GS>::min_blocks)
k_walk_group(WalkArgs a) {
    constexpr int WARPS = WalkShape<MAC, SHAPE, GS>::warps;
    // two-body lanes evaluate each list block for both bodies in one pass
    // (one shared-memory read of the block for the two; each body's terms
    // are summed in the same order as in a pass per body).  The harvest walk
    // keeps a pass per body.  The learned walk fits the fused passes only
    // because no list is flushed inside a round (see the loop below): with
    // flushes there it spilled 76-92 bytes and ran 2.22 -> 3.07 ms at 2^20
    constexpr bool FUSE2 = MAC != kMacHarvest;
    extern __shared__ __align__(16) float s_walk[];
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* base = s_walk + warp * kWarpFloats;
    // Interaction lists in a pair-blocked layout: field f of entry e sits at
    // [(e / 2) * W + 2 f + e % 2], so one 16-byte load returns two fields of
    // entries 2m and 2m+1 as register pairs for the packed f32x2 arithmetic.
    // cells (W = 20): rel x, y, z, -mass, Qxx, Qyy, Qzz, Qxy, Qxz, Qyz
    // bodies (W = 8): rel x, y, z, -mass
    float* cbuf = base;
    float* pbuf = base + kCellCap * 10;
    float2* p1 = (float2*)(pbuf + kPartCap * 4);     // R^2, m / (R^2 + eps^2)^1.5
    int* p2 = (int*)(p1 + kPartCap);                 // sorted index
    int* fa = a.front + (size_t)(blockIdx.x * WARPS + warp) * a.front_cap;
    const float eps2 = (float)a.eps2;
    const float theta2 = (float)a.theta2;
    const int ngroups = *a.n_groups;
    unsigned long long cnt_cell = 0, cnt_body = 0, cnt_mlp = 0;
    // learned MAC: the network is read through L1 from global memory (11 KB,
    // shared by every block of the SM), rows are staged per warp in shared
    const MacDev* __restrict__ wmac = a.mac;
    uint32_t* xs = nullptr;
    float* ys = nullptr;
    int* pend = nullptr;
    if (MAC == kMacLearned) {
        xs = (uint32_t*)(s_walk + WARPS * kWarpFloats) + warp * kMacWarpWords;
        ys = (float*)(xs + 32 * 4);
        pend = (int*)(ys + 32);
    }

    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(a.group_ctr, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        const int2 grp = a.groups[g];  // body_first, body_count (<= 64)
        const int nvalid = grp.y;
        // A group of 33..64 bodies gives every lane two: body `lane` (A) and
        // body `32 + lane` (B, when present); the warp walks once for both and
        // evaluates each interaction list for A and then for B.
        const bool two = GS == 64 && nvalid > 32;
        // A group of nvalid <= 16 bodies is replicated over the warp: lane
        // (rep, slot) holds body `slot` and evaluates every nrep-th list entry
        // starting at `rep`; the replicas' sums are combined at the end.
        const int lw = (nvalid <= 1) ? 0 : two ? 5 : 32 - __clz(nvalid - 1);  // log2(width)
        const int slot = lane & ((1 << lw) - 1);
        const int rep = lane >> lw, nrep = 32 >> lw;
        const int s = grp.x + slot;
        const bool valid = slot < nvalid;
        const int s2 = s + 32;
        const bool valid2 = two && 32 + lane < nvalid;
        const double4 b = a.sbody[valid ? s : grp.x];
        const double4 b2 = valid2 ? a.sbody[s2] : b;
        const double mnx = warp_min(fmin(b.x, b2.x)), mny = warp_min(fmin(b.y, b2.y));
        const double mnz = warp_min(fmin(b.z, b2.z));
        const double mxx = warp_max(fmax(b.x, b2.x)), mxy = warp_max(fmax(b.y, b2.y));
        const double mxz = warp_max(fmax(b.z, b2.z));
        const double gcx = 0.5 * (mnx + mxx), gcy = 0.5 * (mny + mxy), gcz = 0.5 * (mnz + mxz);
        // half extents, rounded outwards so the FP32 box contains every body
        const float ghx = (float)(0.5 * (mxx - mnx)) * 1.000001f + 1e-30f;
        const float ghy = (float)(0.5 * (mxy - mny)) * 1.000001f + 1e-30f;
        const float ghz = (float)(0.5 * (mxz - mnz)) * 1.000001f + 1e-30f;
        const float bx = (float)(b.x - gcx), by = (float)(b.y - gcy), bz = (float)(b.z - gcz);
        const float bx2 = (float)(b2.x - gcx), by2 = (float)(b2.y - gcy), bz2 = (float)(b2.z - gcz);
        // smallest / largest |a| of the group's bodies (previous step), and
        // whether this group's candidates are recorded (harvest)
        float a_min = 0.f, a_max = 0.f, r_grp = 0.f;
        float scr_g = 0.f, scr_w0 = 0.f, scr_w2 = 0.f, scr_w3 = 0.f, scr_mg = 0.f, scr_la = 0.f;
        bool sampled = false;
        if (MAC != kMacGeometric) {
            const float am = a.samag[valid ? s : grp.x];
            const float am2 = valid2 ? a.samag[s2] : am;
            a_min = fminf(am, am2);
            a_max = fmaxf(am, am2);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a_min = fminf(a_min, __shfl_xor_sync(FULL, a_min, o));
                a_max = fmaxf(a_max, __shfl_xor_sync(FULL, a_max, o));
            }
            r_grp = fmaxf(ghx, fmaxf(ghy, ghz));
            if (MAC == kMacLearned) {
                // screen terms that depend on the group only, with the budget
                // moved to this side: y - budget = scr_g + node term
                // + scr_w0 log2 d^2 + scr_w2 f2 + scr_w3 f3
                const float f5 = mac_log2((float)nvalid);
                const float f7 = fminf(mac_log2(a_max / fmaxf(a_min, 1e-30f)), 60.f);
                const float w6 = mac_ldf(&wmac->scr_w[6]);
                scr_g = mac_ldf(&wmac->scr_b) + mac_ldf(&wmac->scr_w[5]) * f5 +
                        mac_ldf(&wmac->scr_w[7]) * f7 -
                        w6 * mac_log2(fmaxf(sqrtf(eps2), 1e-30f)) - a.mac_budget;
                scr_w0 = 0.5f * (w6 - mac_ldf(&wmac->scr_w[0]));
                scr_w2 = mac_ldf(&wmac->scr_w[2]);
                scr_w3 = mac_ldf(&wmac->scr_w[3]);
                scr_mg = mac_ldf(&wmac->lin_margin);
                scr_la = mac_log2(fmaxf(a_min, 1e-30f));
            }
            if (MAC == kMacHarvest) {
                unsigned hsh = (unsigned)grp.x * 2654435761u ^ (unsigned)a.mac_seed;
                hsh ^= hsh >> 15;
                hsh *= 2246822519u;
                hsh ^= hsh >> 13;
                sampled = (hsh & 0xFFFFu) < a.mac_sample;
            }
        }

        float sax = 0.f, say = 0.f, saz = 0.f, cax = 0.f, cay = 0.f, caz = 0.f;
        float spot = 0.f, cpot = 0.f;
        // body B's accumulators (groups of more than 32 bodies)
        float sbx = 0.f, sby = 0.f, sbz = 0.f, cbx = 0.f, cby = 0.f, cbz = 0.f;
        float spot2 = 0.f, cpot2 = 0.f;
        int nc = 0, np = 0;
        unsigned long long grp_entries = 0;  // list entries of this group (load-balance record)

        // The cell list's terms on the body at (bx, by, bz) (group-centred).
        // Both bodies of a two-body lane in one pass over the cell list: each
        // pair block is read from shared memory once for the two.
        auto eval_cells2 = [&](float& tx, float& ty, float& tz, float& ux, float& uy, float& uz) {
            float3 a3, b3;
            cells_two<QUAD>(cbuf, (nc + 1) >> 1, bx, by, bz, bx2, by2, bz2, eps2, a3, b3);
            tx = a3.x; ty = a3.y; tz = a3.z;
            ux = b3.x; uy = b3.y; uz = b3.z;
        };
        auto eval_cells = [&](float bx, float by, float bz, float& tx, float& ty, float& tz,
                              float& tp) {
            tx = ty = tz = tp = 0.f;
            if constexpr (!POT) {
                const float3 t3 = cells_one<QUAD>(cbuf, (nc + 1) >> 1, rep, nrep, bx, by, bz, eps2);
                tx = t3.x;
                ty = t3.y;
                tz = t3.z;
            } else {
#pragma unroll 4
                for (int j = rep; j < nc; j += nrep) {
                    const float* e = cbuf + (j >> 1) * 20 + (j & 1);
                    const float ax_ = e[0], ay_ = e[2], az_ = e[4], am = -e[6];
                    const float dx = bx - ax_, dy = by - ay_, dz = bz - az_;
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
                    const float inv = rsqrt_ftz(r2);
                    const float inv2 = inv * inv;
                    const float inv3 = inv * inv2;
                    if (QUAD) {
                        const float qxx = e[8], qyy = e[10], qzz = e[12], qxy = e[14];
                        const float qxz = e[16], qyz = e[18];
                        const float qx = fmaf(qxx, dx, fmaf(qxy, dy, qxz * dz));
                        const float qy = fmaf(qxy, dx, fmaf(qyy, dy, qyz * dz));
                        const float qz = fmaf(qxz, dx, fmaf(qyz, dy, qzz * dz));
                        const float rqr = fmaf(dx, qx, fmaf(dy, qy, dz * qz));
                        const float inv5 = inv3 * inv2;
                        const float f = fmaf(-2.5f * rqr, inv5 * inv2, -am * inv3);
                        tx = fmaf(f, dx, fmaf(qx, inv5, tx));
                        ty = fmaf(f, dy, fmaf(qy, inv5, ty));
                        tz = fmaf(f, dz, fmaf(qz, inv5, tz));
                        tp = fmaf(-0.5f * rqr, inv5, fmaf(-am, inv, tp));
                    } else {
                        const float f = -am * inv3;
                        tx = fmaf(f, dx, tx);
                        ty = fmaf(f, dy, ty);
                        tz = fmaf(f, dz, tz);
                        tp = fmaf(-am, inv, tp);
                    }
                }
            }
        };
        auto flush_cells = [&]() {
            if constexpr (!POT) {
                // an odd count is padded with a massless, quadrupole-free entry
                // far away, whose terms are exactly zero
                if (nc & 1) {
                    if (lane < 10) cbuf[(nc >> 1) * 20 + lane * 2 + 1] = lane < 3 ? 1e15f : 0.f;
                    __syncwarp();
                }
            }
            float tx, ty, tz, tp;
            if (!POT && FUSE2 && two) {
                float ux, uy, uz;
                eval_cells2(tx, ty, tz, ux, uy, uz);
                kahan(sbx, cbx, ux);
                kahan(sby, cby, uy);
                kahan(sbz, cbz, uz);
            } else {
                eval_cells(bx, by, bz, tx, ty, tz, tp);
                if (two) {
                    float ux, uy, uz, up;
                    eval_cells(bx2, by2, bz2, ux, uy, uz, up);
                    kahan(sbx, cbx, ux);
                    kahan(sby, cby, uy);
                    kahan(sbz, cbz, uz);
                    if (POT) kahan(spot2, cpot2, up);
                }
            }
            kahan(sax, cax, tx);
            kahan(say, cay, ty);
            kahan(saz, caz, tz);
            if (POT) kahan(spot, cpot, tp);
            cnt_cell += (unsigned long long)nc * nvalid;
            grp_entries += nc;
            nc = 0;
            __syncwarp();
        };
        auto eval_parts2 = [&](float& tx, float& ty, float& tz, float& ux, float& uy, float& uz) {
            float3 a3, b3;
            parts_two<GUARD>(pbuf, (np + 1) >> 1, bx, by, bz, bx2, by2, bz2, eps2, a3, b3);
            tx = a3.x; ty = a3.y; tz = a3.z;
            ux = b3.x; uy = b3.y; uz = b3.z;
        };
        // The body list's terms on body `self` at (bx, by, bz).
        auto eval_parts = [&](float bx, float by, float bz, int self, float& tx, float& ty,
                              float& tz, float& tp) {
            tx = ty = tz = tp = 0.f;
            if constexpr (!SHELL && !POT) {
                const float3 t3 = parts_one<GUARD>(pbuf, (np + 1) >> 1, rep, nrep, bx, by, bz, eps2);
                tx = t3.x;
                ty = t3.y;
                tz = t3.z;
            } else {
#pragma unroll 4
                for (int j = rep; j < np; j += nrep) {
                    const float* e = pbuf + (j >> 1) * 8 + (j & 1);
                    const float px_ = e[0], py_ = e[2], pz_ = e[4], pm = -e[6];
                    const float dx = bx - px_, dy = by - py_, dz = bz - pz_;
                    const float raw = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    const float r2 = raw + eps2;
                    const float inv = (GUARD && !(r2 > 0.f)) ? 0.f : rsqrt_ftz(r2);
                    float f = pm * (inv * inv * inv);
                    if (SHELL) {
                        const float2 S = p1[j];
                        if (raw < S.x) f = S.y;
                    }
                    tx = fmaf(-f, dx, tx);
                    ty = fmaf(-f, dy, ty);
                    tz = fmaf(-f, dz, tz);
                    if (POT) {
                        if (p2[j] != self) tp = fmaf(-pm, inv, tp);
                    }
                }
            }
        };
        auto flush_parts = [&]() {
            if constexpr (!SHELL && !POT) {
                if (np & 1) {  // pad: a massless body far away
                    if (lane < 4) pbuf[(np >> 1) * 8 + lane * 2 + 1] = lane < 3 ? 1e15f : 0.f;
                    __syncwarp();
                }
            }
            float tx, ty, tz, tp;
            if (!SHELL && !POT && FUSE2 && two) {
                float ux, uy, uz;
                eval_parts2(tx, ty, tz, ux, uy, uz);
                kahan(sbx, cbx, ux);
                kahan(sby, cby, uy);
                kahan(sbz, cbz, uz);
            } else {
                eval_parts(bx, by, bz, s, tx, ty, tz, tp);
                if (two) {
                    float ux, uy, uz, up;
                    eval_parts(bx2, by2, bz2, s2, ux, uy, uz, up);
                    kahan(sbx, cbx, ux);
                    kahan(sby, cby, uy);
                    kahan(sbz, cbz, uz);
                    if (POT) kahan(spot2, cpot2, up);
                }
            }
            kahan(sax, cax, tx);
            kahan(say, cay, ty);
            kahan(saz, caz, tz);
            if (POT) kahan(spot, cpot, tp);
            cnt_body += (unsigned long long)np * nvalid;
            grp_entries += np;
            np = 0;
            __syncwarp();
        };

        // Warp-shared LIFO stack of nodes still to test: 32 are popped per
        // round (one per lane), children of opened nodes are pushed on top.
        int* stk = fa;
        int sp = 1;
        // batched systems: the walk starts at the group's own system root
        if (lane == 0) stk[0] = a.sys_root ? a.sys_root[a.skeys[grp.x] >> kEnsSysShift] : 0;
        __syncwarp();
        // One candidate node per lane, decided: accepted cells -> cell list,
        // children of opened nodes -> stack, bodies of leaves -> particle list.
        auto emit = [&](int node, bool take_cell, bool is_leaf, bool open, int4 lk, float rx,
                        float ry, float rz, float mass, float4 nq0, float nqyz) {
            // 1. accepted cells -> cell list
            const unsigned mcell = __ballot_sync(FULL, take_cell);
            if (mcell) {
                const int k = __popc(mcell);  // room was made at the round's start
                if (take_cell) {
                    const int cs = nc + __popc(mcell & lanemask_lt());
                    float* e = cbuf + (cs >> 1) * 20 + (cs & 1);
                    e[0] = rx;
                    e[2] = ry;
                    e[4] = rz;
                    e[6] = -mass;
                    if (QUAD) {
                        // Qxx, Qyy, Qxy, Qxz: preloaded by the geometric test
                        const float4 q = MAC == kMacGeometric ? nq0 : a.t.q0[node];
                        e[8] = q.x;
                        e[10] = q.y;
                        e[12] = -(q.x + q.y);
                        e[14] = q.z;
                        e[16] = q.w;
                        e[18] = MAC == kMacGeometric ? nqyz : a.t.q1[node].x;
                    }
                }
                nc += k;
                __syncwarp();
            }
            // 2. children of opened nodes -> pushed on the stack
            const int nch = open ? lk.y : 0;
            const int inc = warp_incl_scan(nch);
            const int tot = __shfl_sync(FULL, inc, 31);
            if (tot > 0) {
                if (sp + tot > a.front_cap) {
                    if (lane == 0) dev_flag(a.err, kErrOverflow);
                } else {
                    for (int k = 0; k < nch; k++) stk[sp + inc - nch + k] = lk.x + k;
                    sp += tot;
                }
                __syncwarp();
            }
            // 3. bodies of leaves that were not accepted -> particle list
            const int cb = is_leaf ? lk.w : 0;
            const int incl = warp_incl_scan(cb);
            const int T = __shfl_sync(FULL, incl, 31);
            for (int t0 = 0; t0 < T; t0 += 32) {
                if (np + 32 > kPartCap) flush_parts();
                const int t = t0 + lane;
                int pos = 0;  // first lane whose inclusive count exceeds t
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int v = __shfl_sync(FULL, incl, pos + step - 1);
                    if (v <= t) pos += step;
                }
                const int ofirst = __shfl_sync(FULL, lk.z, pos);
                const int oexcl = __shfl_sync(FULL, incl - cb, pos);
                const int take = min(32, T - t0);
                if (lane < take) {
                    const int bi = ofirst + (t - oexcl);
                    const double4 q = a.sbody[bi];
                    float* e = pbuf + ((np + lane) >> 1) * 8 + ((np + lane) & 1);
                    e[0] = (float)(q.x - gcx);
                    e[2] = (float)(q.y - gcy);
                    e[4] = (float)(q.z - gcz);
                    e[6] = -(float)q.w;
                    if (SHELL) {
                        const float R = a.srad[bi];
                        const float R2 = R * R;
                        const float id = rsqrtf(R2 + eps2);
                        p1[np + lane] = make_float2(R > 0.f ? R2 : 0.f, (float)q.w * id * id * id);
                    }
                    if (POT) p2[np + lane] = bi;
                }
                np += take;
                __syncwarp();
            }
        };
        // Learned MAC: candidates the screen leaves undecided wait in the
        // pending list (node ids in pend, normalised features in xs); the
        // network decides a full list, or whatever is pending when the stack
        // runs dry, in one call, and the decisions are emitted then.
        int npend = 0;
        auto flush_pending = [&]() {
            __syncwarp();
            mac_mlp_warp(wmac, xs, ys, npend);
            cnt_mlp += npend;
            const bool mine = lane < npend;
            const int pn = mine ? pend[lane] : -1;
            int4 plk = make_int4(0, 0, 0, 0);
            float prx = 0.f, pry = 0.f, prz = 0.f, pm = 0.f;
            bool tc = false, lf = false, op = false;
            if (mine) {
                plk = a.t.link[pn];
                const double4 cm = a.t.com[pn];
                prx = (float)(cm.x - gcx);
                pry = (float)(cm.y - gcy);
                prz = (float)(cm.z - gcz);
                pm = (float)cm.w;
                tc = ys[lane] < a.mac_budget;
                if (!tc) {
                    if (plk.y == 0) lf = true;
                    else op = true;
                }
            }
            npend = 0;
            __syncwarp();
            emit(pn, tc, lf, op, plk, prx, pry, prz, pm, make_float4(0.f, 0.f, 0.f, 0.f), 0.f);
        };
        int rounds = 0;
        while (sp > 0 || (MAC == kMacLearned && npend > 0)) {
            if (++rounds > kMaxWalkRounds) {
                if (lane == 0) dev_flag(a.err, kErrOverflow);
                break;
            }
            // room for the cells this round appends: up to 32 from its own
            // nodes and, in the learned walk, up to 32 more decided by a
            // mid-round network call.  Flushing here rather than inside the
            // append keeps the round's node words out of the flush's live
            // registers (both walks 2.8 % faster at 2^20; it is what lets the
            // learned walk fuse its two-body passes without spilling)
            if (nc > kCellCap - (MAC == kMacLearned ? 64 : 32)) flush_cells();
            if (MAC == kMacLearned && sp == 0) {
                flush_pending();
                continue;
            }
            {
                const int take = min(32, sp);
                const int node = (lane < take) ? stk[sp - take + lane] : -1;
                sp -= take;
                __syncwarp();  // every lane holds its node before the pushes below
                bool take_cell = false, is_leaf = false, open = false, in_band = false;
                int4 lk = make_int4(0, 0, 0, 0);
                float rx = 0.f, ry = 0.f, rz = 0.f, mass = 0.f, half = 0.f, d2 = 0.f;
                float4 nq0 = make_float4(0.f, 0.f, 0.f, 0.f);
                float nqyz = 0.f;
                bool live = false;
                if (node >= 0) {
                    // geometric test: every word of the node the test and the
                    // cell list need, loaded together (one memory latency per
                    // round); the learned variant, short of registers, loads
                    // the quadrupole only for accepted cells
#ifndef NB_WALK_NO_PREFETCH
                    if (MAC == kMacLearned) {
                        // the words this round may read after the test (the
                        // per-node screen term, the quadrupole of an accepted
                        // or undecided cell) start their trip to L1 now, beside
                        // the node words, instead of one memory latency later
                        prefetch_l1(&a.t.q0[node]);
                        prefetch_l1(&a.t.q1[node]);
                        prefetch_l1(&a.mac_node[node]);
                    }
#endif
                    lk = a.t.link[node];
                    const double4 cm = a.t.com[node];
                    float4 nq1 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (MAC == kMacGeometric) {
                        nq1 = a.t.q1[node];
                        if (QUAD) nq0 = a.t.q0[node];
                        nqyz = nq1.x;
                    }
                    if (cm.w > 0.0) {
                        live = true;
                        half = MAC == kMacGeometric ? nq1.y : a.t.q1[node].y;
                        rx = (float)(cm.x - gcx);
                        ry = (float)(cm.y - gcy);
                        rz = (float)(cm.z - gcz);
                        mass = (float)cm.w;
                        const float dx = fmaxf(fabsf(rx) - ghx, 0.f);
                        const float dy = fmaxf(fabsf(ry) - ghy, 0.f);
                        const float dz = fmaxf(fabsf(rz) - ghz, 0.f);
                        d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float s2 = 4.f * half * half;
                        take_cell = d2 > 0.f && s2 < theta2 * d2;
                        if (MAC != kMacGeometric)
                            in_band = d2 > 0.f && !take_cell && s2 < a.mac_theta_hi2 * d2;
                    }
                }
                if (MAC == kMacLearned) {
                    // In the band a cell of one body is exact and taken; a
                    // linear screen fitted to the network decides the clear
                    // cases; the network decides the rest.
                    bool unsure = false;
                    if (in_band && lk.w == 1) {
                        take_cell = true;
                    } else if (in_band) {
                        // the screen from its per-node and per-group parts:
                        // only the distance-dependent features are formed here
                        const float2 nt = a.mac_node[node];
                        const float l2d2 = mac_log2(d2);
                        const float f2 = fminf(fmaxf(nt.y - l2d2 - scr_la, -60.f), 60.f);
                        const float f3 = mac_log2(fmaf(r_grp, rsqrt_ftz(d2), 1e-6f));
                        const float yl = scr_g + nt.x + fmaf(scr_w0, l2d2, fmaf(scr_w2, f2, scr_w3 * f3));
                        if (yl < -scr_mg) take_cell = true;
                        else if (yl <= scr_mg) unsure = true;
                    }
                    const unsigned hard = __ballot_sync(FULL, unsure);
                    if (hard) {
                        const int nh = __popc(hard);
                        if (npend + nh > 32) flush_pending();
                        const int rank = npend + __popc(hard & lanemask_lt());
                        if (unsure) {
                            float f[kMacIn];
                            const float4 q = a.t.q0[node];
                            const float qyz = a.t.q1[node].x, qzz = -(q.x + q.y);
                            const float qn2 = q.x * q.x + q.y * q.y + qzz * qzz +
                                              2.f * (q.z * q.z + q.w * q.w + qyz * qyz);
                            mac_features(f, d2, half, mass, qn2, lk.w, r_grp, nvalid, a_min,
                                         a_max, sqrtf(eps2));
#pragma unroll
                            for (int k = 0; k < kMacIn; k += 2)
                                xs[rank * 4 + k / 2] = pack_bf16(
                                    (f[k] - mac_ldf(&wmac->mean[k])) * mac_ldf(&wmac->inv_std[k]),
                                    (f[k + 1] - mac_ldf(&wmac->mean[k + 1])) *
                                        mac_ldf(&wmac->inv_std[k + 1]));
                            pend[rank] = node;
                            live = false;  // decided when the pending list is flushed
                        }
                        npend += nh;
                        __syncwarp();
                    }
                }
                if (MAC == kMacHarvest && sampled && in_band) {
                    // record the pair: features and the group body nearest the COM
                    float f[kMacIn];
                    const float4 q = a.t.q0[node];
                    const float qyz = a.t.q1[node].x, qzz = -(q.x + q.y);
                    const float qn2 = q.x * q.x + q.y * q.y + qzz * qzz +
                                      2.f * (q.z * q.z + q.w * q.w + qyz * qyz);
                    mac_features(f, d2, half, mass, qn2, lk.w, r_grp, nvalid, a_min, a_max,
                                 sqrtf(eps2));
                    const double4 cm = a.t.com[node];
                    int best = grp.x;
                    double bd = 1e300;
                    for (int j = grp.x; j < grp.x + nvalid; j++) {
                        const double4 p = a.sbody[j];
                        const double ex = p.x - cm.x, ey = p.y - cm.y, ez = p.z - cm.z;
                        const double dd = ex * ex + ey * ey + ez * ez;
                        if (dd < bd) { bd = dd; best = j; }
                    }
                    const int slot_r = atomicAdd(a.n_records, 1);
                    if (slot_r < a.record_cap) {
                        MacRecord r;
                        for (int k = 0; k < kMacIn; k++) r.f[k] = f[k];
                        r.node = node;
                        r.body = best;
                        r.a_min = a_min;
                        r.pad = 0.f;
                        a.records[slot_r] = r;
                    }
                }
                if (live && !take_cell) {
                    if (lk.y == 0) is_leaf = true;
                    else open = true;
                }
                emit(node, take_cell, is_leaf, open, lk, rx, ry, rz, mass, nq0, nqyz);
            }
        }
        if (nc) flush_cells();
        if (np) flush_parts();
        if (lane == 0 && a.counters) atomicMax(&a.counters[2], grp_entries);
        // combine the replicas of each body (lanes equal modulo the width)
        double fx = (double)sax - (double)cax, fy = (double)say - (double)cay;
        double fz = (double)saz - (double)caz, fp = (double)spot - (double)cpot;
        for (int o = 1 << lw; o < 32; o <<= 1) {
            fx += __shfl_xor_sync(FULL, fx, o);
            fy += __shfl_xor_sync(FULL, fy, o);
            fz += __shfl_xor_sync(FULL, fz, o);
            if (POT) fp += __shfl_xor_sync(FULL, fp, o);
        }
        if (valid && rep == 0) {
            const uint32_t row = a.sidx[s];
            a.ax[row] = fx;
            a.ay[row] = fy;
            a.az[row] = fz;
            if (POT) a.pot[row] = fp;
        }
        if (valid2) {
            const uint32_t row = a.sidx[s2];
            a.ax[row] = (double)sbx - (double)cbx;
            a.ay[row] = (double)sby - (double)cby;
            a.az[row] = (double)sbz - (double)cbz;
            if (POT) a.pot[row] = (double)spot2 - (double)cpot2;
        }
    }
    if (lane == 0 && a.counters) {
        atomicAdd(&a.counters[0], cnt_cell);
        atomicAdd(&a.counters[1], cnt_body);
        if (MAC == kMacLearned) atomicAdd(&a.counters[3], cnt_mlp);
    }
}

// Per-body FP64 walk with the reference's semantics: MAC 4h^2 < theta^2 d^2
// with d to the cell's centre of mass (barnes_hut_solver.cpp:269-283),
// monopole only, leaves direct, self skipped, mass-0 nodes skipped, children
// visited in the reference's octant order x + 2y + 4z (octree_node.hpp:53-59).
// Arithmetic order follows compute_force_on_body (barnes_hut_solver.cpp:
// 230-286) without FMA contraction; leaves use GravityKernel's shell theorem
// when `shell` (BarnesHutBackend.cs:410-424).
__device__ __forceinline__ double mono_factor(double m, double d2, double eps2) {
    double inv = 1.0 / sqrt(__dadd_rn(d2, eps2));
    double inv3 = __dmul_rn(__dmul_rn(inv, inv), inv);
    return __dmul_rn(m, inv3);
}

template <bool SHELL>
__global__ void k_walk_reference(WalkArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    const double4 b = a.sbody[s];
    double ax = 0.0, ay = 0.0, az = 0.0;
    int stack[176];
    int sp = 0;
    stack[sp++] = 0;
    int visits = 0;  // every node is visited at most once per body
    while (sp > 0) {
        if (++visits > 2 * a.n + 64) {
            dev_flag(a.err, kErrOverflow);
            break;
        }
        const int k = stack[--sp];
        const double4 cm = a.t.com[k];
        if (cm.w == 0.0) continue;
        const int4 lk = a.t.link[k];
        const double dx = __dsub_rn(b.x, cm.x), dy = __dsub_rn(b.y, cm.y), dz = __dsub_rn(b.z, cm.z);
        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if (lk.y == 0) {
            for (int j = lk.z; j < lk.z + lk.w; j++) {
                if (j == s) continue;
                double ex = dx, ey = dy, ez = dz, e2 = d2, m = cm.w;
                if (lk.w > 1) {  // a level-21 bucket of coincident keys: body by body
                    const double4 q = a.sbody[j];
                    ex = __dsub_rn(b.x, q.x); ey = __dsub_rn(b.y, q.y); ez = __dsub_rn(b.z, q.z);
                    e2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
                    m = q.w;
                }
                double f;
                if (SHELL) {
                    const double R = (double)a.srad[j];
                    if (R > 0.0 && sqrt(e2) < R) {
                        const double den = __dadd_rn(__dmul_rn(R, R), a.eps2);
                        const double ids = 1.0 / sqrt(den);
                        f = __dmul_rn(m, ids) / den;
                    } else {
                        const double inv = 1.0 / sqrt(__dadd_rn(e2, a.eps2));
                        f = __dmul_rn(__dmul_rn(__dmul_rn(m, inv), inv), inv);
                    }
                } else {
                    f = mono_factor(m, e2, a.eps2);
                }
                ax = __dsub_rn(ax, __dmul_rn(f, ex));
                ay = __dsub_rn(ay, __dmul_rn(f, ey));
                az = __dsub_rn(az, __dmul_rn(f, ez));
            }
            continue;
        }
        const double h = (double)a.t.q1[k].y;
        const double s2 = __dmul_rn(__dmul_rn(4.0, h), h);
        if (d2 > 0.0 && s2 < __dmul_rn(a.theta2, d2)) {
            const double f = mono_factor(cm.w, d2, a.eps2);
            ax = __dsub_rn(ax, __dmul_rn(f, dx));
            ay = __dsub_rn(ay, __dmul_rn(f, dy));
            az = __dsub_rn(az, __dmul_rn(f, dz));
            continue;
        }
        // children: push in decreasing reference octant so octant 0 pops first
        const int lev = a.t.level[k] + 1;  // subdivision level of this cell
        const int shift = 63 - 3 * lev;
        int oct_child[8];
#pragma unroll
        for (int o = 0; o < 8; o++) oct_child[o] = -1;
        for (int c = lk.x; c < lk.x + lk.y; c++) {
            const uint64_t key = a.skeys[a.t.link[c].z];
            const int dg = (int)((key >> shift) & 7);  // Morton digit x<<2 | y<<1 | z
            const int oct = ((dg >> 2) & 1) | (dg & 2) | ((dg & 1) << 2);
            oct_child[oct] = c;
        }
        for (int o = 7; o >= 0; o--) {
            if (oct_child[o] < 0) continue;
            if (sp < 176) stack[sp++] = oct_child[o];
            else dev_flag(a.err, kErrOverflow);
        }
    }
    const uint32_t row = a.sidx[s];
    a.ax[row] = ax;
    a.ay[row] = ay;
    a.az[row] = az;
}

// Group order in the list does not matter: every group's walk and sums are
// independent of the others, so results are deterministic.
// One thread per node holding more than 32 bodies: its children with at
// most 32 bodies are consecutive in body order, and runs of them are packed
// greedily into groups of at most 32 bodies (siblings share the parent's
// cell, so a packed group stays compact); a level-21 bucket of more than 32
// equal keys is cut into slices of 32.  pack = 0 keeps one child per group.
struct Box {
    double lo[3], hi[3];
    __device__ void empty() {
        for (int a = 0; a < 3; a++) { lo[a] = 1e300; hi[a] = -1e300; }
    }
    __device__ void add(const Box& b) {
        for (int a = 0; a < 3; a++) { lo[a] = fmin(lo[a], b.lo[a]); hi[a] = fmax(hi[a], b.hi[a]); }
    }
    __device__ double ext() const {  // largest half extent
        return 0.5 * fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    }
};

// Sibling runs are packed only while the packed box stays within `pack`
// times the larger part's box, and only while it does not reach into the
// body box of a sibling of more than 32 bodies outside the run: siblings
// that sit far apart in a sparse cell would otherwise make one group whose
// box encloses a dense sibling (at the top levels, the whole core), and whose
// opening test then walks the tree down to every body.  (Measured at N=1M: factor 2-2.5 raises
// lane fill from 0.30 to 0.57-0.71.)
__device__ __forceinline__ Box node_box(const TreeBufs& t, int c) {
    const float4 l = t.blo[c], h = t.bhi[c];
    Box b;
    b.lo[0] = l.x; b.lo[1] = l.y; b.lo[2] = l.z;
    b.hi[0] = h.x; b.hi[1] = h.y; b.hi[2] = h.z;
    return b;
}

__device__ __forceinline__ bool boxes_meet(const Box& a, const Box& b) {
    for (int k = 0; k < 3; k++)
        if (a.hi[k] < b.lo[k] || b.hi[k] < a.lo[k]) return false;
    return true;
}

__global__ void k_find_groups(TreeBufs t, int2* __restrict__ groups, int* __restrict__ n_groups,
                              double pack) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= *t.n_nodes) return;
    const int4 lk = t.link[w];
    if (lk.w <= 32) {
        if (w == 0) groups[atomicAdd(n_groups, 1)] = make_int2(lk.z, lk.w);  // small root
        return;  // otherwise its parent packs it
    }
    if (lk.y == 0) {
        for (int off = 0; off < lk.w; off += 32)
            groups[atomicAdd(n_groups, 1)] = make_int2(lk.z + off, min(32, lk.w - off));
        return;
    }
    int run_first = 0, run_cnt = 0, run_c0 = 0;
    Box run;
    run.empty();
    for (int c = lk.x; c < lk.x + lk.y; c++) {
        const int4 cl = t.link[c];
        if (cl.w > 32) {  // handled by its own thread
            if (run_cnt) groups[atomicAdd(n_groups, 1)] = make_int2(run_first, run_cnt);
            run_cnt = 0;
            continue;
        }
        const Box cb = node_box(t, c);
        bool merge = false;
        if (pack > 0.0 && run_cnt > 0 && run_cnt + cl.w <= 32) {
            Box m = run;
            m.add(cb);
            merge = m.ext() <= pack * fmax(run.ext(), cb.ext());
            for (int k = lk.x; merge && k < lk.x + lk.y; k++)
                if ((k < run_c0 || k > c) && t.link[k].w > 32 && boxes_meet(m, node_box(t, k)))
                    merge = false;
        }
        if (merge) {
            run_cnt += cl.w;
            run.add(cb);
        } else {
            if (run_cnt) groups[atomicAdd(n_groups, 1)] = make_int2(run_first, run_cnt);
            run_first = cl.z;
            run_cnt = cl.w;
            run_c0 = c;
            run = cb;
        }
    }
    if (run_cnt) groups[atomicAdd(n_groups, 1)] = make_int2(run_first, run_cnt);
}

// Span grouping: the walk-tree nodes holding at most `span` bodies whose
// parent holds more ("span cells"; the root when it holds at most span, and
// leaf buckets of coincident keys that hold more) are cut into runs of `size`
// (32 or 64) consecutive sorted bodies, the last run taking the rest.  Every
// warp lane then holds a body (or two), while a group's box stays inside its
// span cell, which holds at most `span` bodies: a group can never enclose a
// dense region it does not belong to.
__global__ void k_find_groups_span(TreeBufs t, int2* __restrict__ groups,
                                   int* __restrict__ n_groups, int span, int size) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= *t.n_nodes) return;
    const int4 lk = t.link[w];
    if (lk.w > span && lk.y != 0) return;  // an internal node above the span cells
    const int pw = t.parent_walk[w];
    if (pw >= 0 && t.link[pw].w <= span) return;  // inside a span cell: its ancestor cuts it
    for (int off = 0; off < lk.w; off += size)
        groups[atomicAdd(n_groups, 1)] = make_int2(lk.z + off, min(size, lk.w - off));
}

void find_groups(cudaStream_t st, const TreeBufs& t, const double4* sbody, int n, int2* groups,
                 int* n_groups, double pack, int span, int size) {
    cudaMemsetAsync(n_groups, 0, sizeof(int), st);
    if (n <= 0) return;
    if (span >= 32)
        k_find_groups_span<<<ceil_div(2 * n, 256), 256, 0, st>>>(t, groups, n_groups, span,
                                                                 size == 64 ? 64 : 32);
    else
        k_find_groups<<<ceil_div(2 * n, 256), 256, 0, st>>>(t, groups, n_groups, pack);
}

using WalkKernel = void (*)(WalkArgs);

// The instantiated variants: (quad) x {plain, shell, potential} x (guard).
static WalkKernel pick_walk(bool quad, bool shell, bool pot, bool guard) {
#define NB_WALK_PICK(Q, S, P)                                            \
    return guard ? k_walk_group<Q, S, P, true, kMacGeometric>                \
                 : k_walk_group<Q, S, P, false, kMacGeometric>
    if (pot) {
        if (quad) NB_WALK_PICK(true, false, true);
        NB_WALK_PICK(false, false, true);
    }
    if (shell) {
        if (quad) NB_WALK_PICK(true, true, false);
        NB_WALK_PICK(false, true, false);
    }
    if (quad) NB_WALK_PICK(true, false, false);
    NB_WALK_PICK(false, false, false);
#undef NB_WALK_PICK
}

void walk_init(int sms, WalkConfig& cfg) {
    for (int v = 0; v < 16; v++) {
        const bool pot = v & 4, shell = (v & 2) && !pot;
        cudaFuncSetAttribute((const void*)pick_walk(v & 1, shell, pot, v & 8),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kWalkSmem);
    }
    cudaFuncSetAttribute((const void*)k_walk_group<true, false, false, false, kMacHarvest>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kWalkSmem);
    cudaFuncSetAttribute((const void*)k_walk_group<true, false, false, false, kMacLearned>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kWalkSmemMac);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_walk_group<true, false, false, false, kMacGeometric>, kWalkThreads, kWalkSmem);
    if (per_sm < 1) per_sm = 1;
    cfg.blocks = sms * per_sm;
    // the small-block shape of the quadrupole walk (ensembles)
    for (int g = 0; g < 2; g++)
        cudaFuncSetAttribute(g ? (const void*)k_walk_group<true, false, false, true, kMacGeometric, 1>
                               : (const void*)k_walk_group<true, false, false, false, kMacGeometric, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kWalkWarpsSmall * kWarpFloats * 4);
    int per_sm_small = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm_small, k_walk_group<true, false, false, false, kMacGeometric, 1>,
        kWalkWarpsSmall * 32, kWalkWarpsSmall * kWarpFloats * 4);
    if (per_sm_small < 1) per_sm_small = 1;
    int per_sm_mac = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm_mac, k_walk_group<true, false, false, false, kMacLearned>, kMacWarps * 32,
        kWalkSmemMac);
    if (per_sm_mac < 1) per_sm_mac = 1;
    // as many resident blocks as fit, within the stacks sized for the
    // geometric grid (cfg.blocks x kWalkWarps warps)
    cfg.blocks_mac = sms * per_sm_mac;
    if (cfg.blocks_mac * kMacWarps > cfg.blocks * kWalkWarps)
        cfg.blocks_mac = cfg.blocks * kWalkWarps / kMacWarps;
    cfg.blocks_small = sms * per_sm_small;
    if (cfg.blocks_small * kWalkWarpsSmall > cfg.blocks * kWalkWarps)
        cfg.blocks_small = cfg.blocks * kWalkWarps / kWalkWarpsSmall;
    // the 64-body-group variants
    const void* g64[4] = {(const void*)k_walk_group<true, false, false, false, kMacGeometric, 0, 64>,
                          (const void*)k_walk_group<true, false, false, true, kMacGeometric, 0, 64>,
                          (const void*)k_walk_group<true, false, false, false, kMacHarvest, 0, 64>,
                          (const void*)k_walk_group<true, false, false, false, kMacLearned, 0, 64>};
    for (int k = 0; k < 4; k++)
        cudaFuncSetAttribute(g64[k], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             k == 3 ? kWalkSmemMac64 : kWalkSmem64);
    int per_sm64 = 0, per_sm_mac64 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm64, k_walk_group<true, false, false, false, kMacGeometric, 0, 64>,
        NB_WALK64_WARPS * 32, kWalkSmem64);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm_mac64, k_walk_group<true, false, false, false, kMacLearned, 0, 64>,
        kMacWarps64 * 32, kWalkSmemMac64);
    cfg.blocks64 = sms * std::max(per_sm64, 1);
    if (cfg.blocks64 * NB_WALK64_WARPS > cfg.blocks * kWalkWarps)
        cfg.blocks64 = cfg.blocks * kWalkWarps / NB_WALK64_WARPS;
    cfg.blocks_mac64 = sms * std::max(per_sm_mac64, 1);
    if (cfg.blocks_mac64 * kMacWarps64 > cfg.blocks * kWalkWarps)
        cfg.blocks_mac64 = cfg.blocks * kWalkWarps / kMacWarps64;
    cfg.front_cap = 16384;
}

size_t walk_front_bytes(const WalkConfig& cfg) {
    return (size_t)cfg.blocks * kWalkWarps * cfg.front_cap * sizeof(int);
}

void walk_group(cudaStream_t st, const WalkConfig& cfg, WalkArgs a, bool quad, bool shell,
                bool pot, int mac, int shape) {
    if (a.n <= 0) return;
    a.front_cap = cfg.front_cap;
    // groups of up to 64 bodies: span groups of span >= 64, for the
    // quadrupole walks without the shell theorem or potentials
    const bool g64 = a.group_size == 64 && a.group_span >= 64 && quad && !shell && !pot &&
                     (mac != kMacGeometric || shape == 0);
    find_groups(st, a.t, a.sbody, a.n, a.groups, a.n_groups, a.pack, a.group_span,
                g64 ? 64 : 32);
    cudaMemsetAsync(a.group_ctr, 0, sizeof(unsigned), st);
    if (g64) {
        if (mac == kMacHarvest)
            k_walk_group<true, false, false, false, kMacHarvest, 0, 64>
                <<<cfg.blocks64, NB_WALK64_WARPS * 32, kWalkSmem64, st>>>(a);
        else if (mac == kMacLearned)
            k_walk_group<true, false, false, false, kMacLearned, 0, 64>
                <<<cfg.blocks_mac64, kMacWarps64 * 32, kWalkSmemMac64, st>>>(a);
        else if (a.eps2 > 0.0)
            k_walk_group<true, false, false, false, kMacGeometric, 0, 64>
                <<<cfg.blocks64, NB_WALK64_WARPS * 32, kWalkSmem64, st>>>(a);
        else
            k_walk_group<true, false, false, true, kMacGeometric, 0, 64>
                <<<cfg.blocks64, NB_WALK64_WARPS * 32, kWalkSmem64, st>>>(a);
        return;
    }
    if (mac == kMacHarvest) {
        k_walk_group<true, false, false, false, kMacHarvest>
            <<<cfg.blocks, kWalkThreads, kWalkSmem, st>>>(a);
        return;
    }
    if (mac == kMacLearned) {
        k_walk_group<true, false, false, false, kMacLearned>
            <<<cfg.blocks_mac, kMacWarps * 32, kWalkSmemMac, st>>>(a);
        return;
    }
    if (shape == 1 && quad && !shell && !pot) {
        const WalkKernel k = a.eps2 > 0.0
                                 ? k_walk_group<true, false, false, false, kMacGeometric, 1>
                                 : k_walk_group<true, false, false, true, kMacGeometric, 1>;
        k<<<cfg.blocks_small, kWalkWarpsSmall * 32, kWalkWarpsSmall * kWarpFloats * 4, st>>>(a);
        return;
    }
    const WalkKernel k = pick_walk(quad, shell, pot, !(a.eps2 > 0.0));
    k<<<cfg.blocks, kWalkThreads, kWalkSmem, st>>>(a);
}

void walk_reference(cudaStream_t st, WalkArgs a, bool shell) {
    if (a.n <= 0) return;
    if (shell) k_walk_reference<true><<<ceil_div(a.n, 128), 128, 0, st>>>(a);
    else k_walk_reference<false><<<ceil_div(a.n, 128), 128, 0, st>>>(a);
}

}  // namespace nb
