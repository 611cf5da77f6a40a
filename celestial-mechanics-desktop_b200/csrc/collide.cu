// collide.cu - collision broad phase, deterministic merges, compaction.
//
// Broad phase: replaces broad_phase_collision_kernel (engine/src/cuda/
// collision_kernel.cu:16-64), which only compares each body with the next 31
// in Morton order and so misses pairs, with a query of the octree: a warp
// descends, for a group of up to 32 consecutive sorted bodies, into every
// cell whose box, grown by the largest radius inside it, meets the group's
// spheres; at the leaves each body gets the reference's exact FP64 test
// |xi - xj|^2 < (ri + rj)^2 (collision_kernel.cu:40-52).  Each pair
// is emitted once (by its lower row) as the key lo << 32 | hi and the keys
// are radix-sorted, which is CollisionResolver::sort_pairs' order
// (engine/src/physics/collision_resolver.cpp:8-18).
//
// Merge: the reference GPU kernel (resolve_merges_kernel.cu:43-194) resolves
// pairs under try-locks, so which pairs merge depends on thread timing.  Here
// the pairs are decided in parallel in conflict-free rounds (k_merge_rounds)
// that reproduce the CPU resolver's sequential semantics
// (collision_resolver.cpp:20-100, 190-250) bit for bit: deterministic and
// identical to the CPU reference.
//
// Compaction: replaces the ~35-launch scan/scatter of compact_kernel.cu:
// 191-407 (with a host scan above 262,144 bodies) by two kernels: warp ballot
// / popc ranks with a decoupled look-back across 4096-row tiles give every
// row its destination, then one thread per row moves every state field.
// Mask is_active && mass > 0 (compact_kernel.cu:39); row order is preserved.
#include <climits>

#include "collide.cuh"
#include "sort.cuh"
#include "walk.cuh"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace nb {

constexpr int kCompThreads = 256;
constexpr int kCompItems = 16;
constexpr int kCompTile = kCompThreads * kCompItems;
constexpr uint32_t kCFlagAgg = 1u << 30;
constexpr uint32_t kCFlagPre = 2u << 30;
constexpr uint32_t kCValMask = (1u << 30) - 1;

int collide_alloc(CollideBufs& b, int capacity, const std::function<int(void**, size_t)>& alloc) {
    b.capacity = capacity;
    b.pair_cap = capacity / 4 > 4096 ? capacity / 4 : 4096;
    int r;
    if ((r = alloc((void**)&b.pair_keys, sizeof(uint64_t) * b.pair_cap))) return r;
    if ((r = alloc((void**)&b.pair_vals, sizeof(uint32_t) * b.pair_cap))) return r;
    if ((r = alloc((void**)&b.pair_keys_alt, sizeof(uint64_t) * b.pair_cap))) return r;
    if ((r = alloc((void**)&b.pair_vals_alt, sizeof(uint32_t) * b.pair_cap))) return r;
    if ((r = alloc((void**)&b.pair_sort_ws, sort_workspace_bytes(b.pair_cap)))) return r;
    if ((r = alloc((void**)&b.merge_count, sizeof(int) * (size_t)capacity))) return r;
    if ((r = alloc((void**)&b.owner, sizeof(int) * (size_t)capacity))) return r;
    const size_t tiles = (size_t)ceil_div(capacity, kCompTile) + 1;
    if ((r = alloc((void**)&b.look, sizeof(uint32_t) * tiles))) return r;
    return alloc((void**)&b.tile_ctr, sizeof(uint32_t) * 4);
}

// ---- broad phase ----------------------------------------------------------

// Warp-cooperative broad phase: one warp per walk group of up to 32
// consecutive sorted bodies.  The warp walks the tree once for the group's
// box, the union of its collidable bodies' spheres (x +- r) widened by a pad
// of 1e-9 of the cube's half-size, as the nodes' body boxes are: a node is
// accepted when the gap between the group box and its padded body box is
// within the node's largest radius (1 + 1e-9).  The ball of every body lies inside the group box, so every
// node a body's own query accepts is accepted here; accepted leaves are
// collected, and each lane runs the exact FP64 test of its body against their
// bodies (higher rows only), so the pair set is the per-body query's.
constexpr int kBpWarps = 8;
constexpr int kBpStack = 1024;   // nodes pending per warp
constexpr int kBpLeaves = 64;    // candidate leaves per evaluation

__global__ void __launch_bounds__(kBpWarps * 32)
k_broad_phase_groups(State s, const uint32_t* __restrict__ sidx, TreeBufs t,
                     const double* __restrict__ cube, const int2* __restrict__ groups,
                     const int* __restrict__ n_groups, unsigned* group_ctr,
                     uint64_t* __restrict__ pairs, int cap, int* __restrict__ count, int* err) {
    __shared__ int s_stack[kBpWarps][kBpStack];
    __shared__ int2 s_leaf[kBpWarps][kBpLeaves];
    __shared__ double s_cand[kBpWarps][4][32];  // staged candidates: x, y, z, radius
    __shared__ uint32_t s_crow[kBpWarps][32];
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int* stk = s_stack[warp];
    int2* lv = s_leaf[warp];
    double* cx = s_cand[warp][0];
    double* cy = s_cand[warp][1];
    double* cz = s_cand[warp][2];
    double* crad = s_cand[warp][3];
    uint32_t* cr = s_crow[warp];
    const double pad = 1e-9 * cube[3];
    const int ng = *n_groups;
    const int nnodes = *t.n_nodes;
    for (;;) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(group_ctr, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ng) break;
        const int2 grp = groups[g];
        const bool valid = lane < grp.y;
        const uint32_t row = valid ? sidx[grp.x + lane] : 0u;
        const bool mine = valid && s.collidable[row];
        const double x = mine ? s.px[row] : 0.0, y = mine ? s.py[row] : 0.0;
        const double z = mine ? s.pz[row] : 0.0, r = mine ? s.radius[row] : 0.0;
        if (!__any_sync(FULL, mine)) continue;
        const double glo[3] = {warp_min(mine ? x - r : 1e300) - pad,
                               warp_min(mine ? y - r : 1e300) - pad,
                               warp_min(mine ? z - r : 1e300) - pad};
        const double ghi[3] = {warp_max(mine ? x + r : -1e300) + pad,
                               warp_max(mine ? y + r : -1e300) + pad,
                               warp_max(mine ? z + r : -1e300) + pad};
        // The exact test of this lane's body against the bodies of the
        // collected leaves: the leaves' bodies are flattened 32 at a time,
        // each lane loads one candidate into the warp's staging slots (32
        // independent loads per round trip), then every lane tests its body
        // against the staged candidates (broadcast shared-memory reads).  The
        // test rounds as the all-pairs loop does, without FMA contraction.
        int nl = 0;
        auto evaluate = [&]() {
            __syncwarp();
            for (int b0 = 0; b0 < nl; b0 += 32) {
                const int2 L = (b0 + lane < nl) ? lv[b0 + lane] : make_int2(0, 0);
                const int incl = warp_incl_scan(L.y);
                const int T = __shfl_sync(FULL, incl, 31);
                for (int t0 = 0; t0 < T; t0 += 32) {
                    const int tt = t0 + lane;
                    int pos = 0;  // first lane whose inclusive count exceeds tt
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int v = __shfl_sync(FULL, incl, pos + step - 1);
                        if (v <= tt) pos += step;
                    }
                    const int first = __shfl_sync(FULL, L.x, pos);
                    const int excl = __shfl_sync(FULL, incl - L.y, pos);
                    const int take = min(32, T - t0);
                    if (lane < take) {
                        const uint32_t rj = sidx[first + (tt - excl)];
                        // a body that is not collidable gets row 0, which no
                        // lane's row is below: never tested
                        cr[lane] = s.collidable[rj] ? rj : 0u;
                        cx[lane] = s.px[rj];
                        cy[lane] = s.py[rj];
                        cz[lane] = s.pz[rj];
                        crad[lane] = s.radius[rj];
                    }
                    __syncwarp();
                    if (mine) {
                        for (int k = 0; k < take; k++) {
                            const uint32_t rj = cr[k];
                            if (rj <= row) continue;
                            const double dx = x - cx[k], dy = y - cy[k], dz = z - cz[k];
                            const double dd = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                                        __dmul_rn(dz, dz));
                            const double sr = r + crad[k];
                            if (dd < __dmul_rn(sr, sr)) {
                                const int slot = atomicAdd(count, 1);
                                if (slot < cap) pairs[slot] = ((uint64_t)row << 32) | rj;
                                else dev_flag(err, kErrCapacity);
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            nl = 0;
            __syncwarp();
        };
        int sp = 1;
        if (lane == 0) stk[0] = 0;
        __syncwarp();
        int visited = 0;
        while (sp > 0) {
            if (visited > nnodes) {  // each node is taken at most once per group
                if (lane == 0) dev_flag(err, kErrOverflow);
                break;
            }
            const int take = min(32, sp);
            const int node = lane < take ? stk[sp - take + lane] : -1;
            sp -= take;
            visited += take;
            __syncwarp();
            bool accept = false;
            int4 lk = make_int4(0, 0, 0, 0);
            if (node >= 0) {
                // the node's body box (FP32, rounded outwards, so it holds
                // every body of the node) and its largest radius: the words
                // arrive together, and the box is tighter than the cell's
                lk = t.link[node];
                const float reach = t.q1[node].z;
                const float4 bl = t.blo[node], bh = t.bhi[node];
                const double b0[3] = {(double)bl.x - pad, (double)bl.y - pad, (double)bl.z - pad};
                const double b1[3] = {(double)bh.x + pad, (double)bh.y + pad, (double)bh.z + pad};
                double d2 = 0.0;
                for (int a = 0; a < 3; a++) {
                    const double e = ghi[a] < b0[a] ? b0[a] - ghi[a]
                                                    : (glo[a] > b1[a] ? glo[a] - b1[a] : 0.0);
                    d2 += e * e;
                }
                const double rr = (double)reach;
                accept = d2 <= rr * rr * (1.0 + 1e-9);
            }
            // accepted leaves -> candidates
            const bool is_leaf = accept && lk.y == 0;
            const unsigned ml = __ballot_sync(FULL, is_leaf);
            if (ml) {
                if (nl + __popc(ml) > kBpLeaves) evaluate();
                if (is_leaf) lv[nl + __popc(ml & lanemask_lt())] = make_int2(lk.z, lk.w);
                nl += __popc(ml);
                __syncwarp();
            }
            // children of accepted internal nodes -> stack
            const int nch = (accept && lk.y > 0) ? lk.y : 0;
            const int inc = warp_incl_scan(nch);
            const int tot = __shfl_sync(FULL, inc, 31);
            if (tot > 0) {
                if (sp + tot > kBpStack) {
                    if (lane == 0) dev_flag(err, kErrOverflow);
                } else {
                    for (int k = 0; k < nch; k++) stk[sp + inc - nch + k] = lk.x + k;
                    sp += tot;
                }
                __syncwarp();
            }
        }
        if (nl) evaluate();
    }
}

__global__ void k_iota(int n, uint32_t* v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

int broad_phase(cudaStream_t st, CollideBufs& b, CollideArgs& a, bool build_tree, int* np) {
    *np = 0;
    if (a.n <= 0) return NB_OK;
    if (!a.reuse_tree) {
        if (build_tree) {
            launch_kick_drift_bbox(st, a.n, a.s, false, 0.0, a.bbox_ord, a.n_active_dev, a.err);
            launch_cube(st, a.bbox_ord, nullptr, a.cube);
        }
        launch_keys_cube(st, a.n, a.s, a.cube, a.keys0, a.vals0, (uint32_t*)a.sort_ws);
        sort_pairs(st, a.n, a.keys0, a.vals0, a.keys1, a.vals1, a.sort_ws, true, a.err, a.sms);
        launch_gather(st, a.n_active, a.s, a.vals0, a.sbody, a.srad);
        tree_build(st, a.tree, a.n_active, a.keys0, a.sbody, a.srad, a.cube, a.leaf_cap, a.err);
    }
    cudaMemsetAsync(a.n_pairs, 0, sizeof(int), st);
    if (a.n_active > 0) {
        // walk groups of the tree (sibling packing), one warp each
        find_groups(st, a.tree, a.sbody, a.n_active, a.groups, a.n_groups, 2.25, 0);
        cudaMemsetAsync(a.group_ctr, 0, sizeof(unsigned), st);
        k_broad_phase_groups<<<a.sms * 4, kBpWarps * 32, 0, st>>>(
            a.s, a.vals0, a.tree, a.cube, a.groups, a.n_groups, a.group_ctr,
            b.pair_keys, b.pair_cap, a.n_pairs, a.err);
    }
    int cnt = 0;
    if (cudaMemcpyAsync(&cnt, a.n_pairs, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return NB_ERR_CUDA;
    const int w = cnt < b.pair_cap ? cnt : b.pair_cap;
    if (w > 1) {
        k_iota<<<ceil_div(w, 256), 256, 0, st>>>(w, b.pair_vals);
        sort_pairs(st, w, b.pair_keys, b.pair_vals, b.pair_keys_alt, b.pair_vals_alt,
                   b.pair_sort_ws, false, a.err, a.sms);
    }
    *np = cnt;
    return NB_OK;
}

// ---- merge --------------------------------------------------------------

__device__ double dm_density(double mass, double radius, double min_radius) {
    const double r = (radius > min_radius) ? radius : min_radius;
    const double volume = __dmul_rn(__dmul_rn(__dmul_rn((4.0 / 3.0) * M_PI, r), r), r);
    if (volume < 1e-30) return 0.0;
    return mass / volume;
}

__device__ double dm_radius(double mass, double density, double min_radius) {
    if (density < 1e-30 || mass < 1e-30) return min_radius;
    const double r = cbrt(__dmul_rn(3.0, mass) / __dmul_rn(4.0 * M_PI, density));
    return (r > min_radius) ? r : min_radius;
}

__device__ __forceinline__ double wavg(double ma, double a, double mb, double b, double M) {
    return __dadd_rn(__dmul_rn(ma, a), __dmul_rn(mb, b)) / M;
}

// CollisionResolver::resolve in Merge mode (collision_resolver.cpp:20-100)
// with resolve_merge (:190-250) and DensityModel (density_model.cpp:10-22):
// pairs in sorted order; a pair is skipped when either body is inactive,
// when max_frame merges happened before it, or when either body already took
// part in max_body merges; otherwise the heavier body (the first on a tie)
// takes the pair's mass, momentum-weighted velocity, mass-weighted position
// and density-preserving radius, and the other becomes inactive.
// The same resolver semantics with the pairs decided in parallel, bit for
// bit the sequential loop's result.  One block takes the sorted pairs in
// windows of kMergeThreads (one pair per thread) and resolves each window in
// rounds.  In a round a pending pair is ready when it is the lowest pending
// pair touching each of its two bodies (the `owner` words, reset for the
// pending pairs' bodies and lowered by atomicMin): no earlier pending pair
// can change its bodies' flags, counts, masses or positions any more, and the
// ready pairs of a round touch disjoint bodies.  The per-frame cap depends on
// the merges of all earlier pairs: with E merges among the resolved earlier
// pairs and U earlier pairs still pending, the merge count at this pair lies
// in [E, E + U]; the pair waits while that range straddles the cap.  The
// lowest pending pair is always ready with U = 0, so every round resolves at
// least one pair; after max_frame merges every later pair is a skip.
constexpr int kMergeThreads = 1024;

__device__ __forceinline__ void merge_pair(State& s, int a, int b, int density_merge,
                                           double min_radius, int* counts) {
    const double ma = s.mass[a], mb = s.mass[b];
    const double M = __dadd_rn(ma, mb);
    if (!(M < 1e-30)) {
        const double vx = wavg(ma, s.vx[a], mb, s.vx[b], M);
        const double vy = wavg(ma, s.vy[a], mb, s.vy[b], M);
        const double vz = wavg(ma, s.vz[a], mb, s.vz[b], M);
        const double x = wavg(ma, s.px[a], mb, s.px[b], M);
        const double y = wavg(ma, s.py[a], mb, s.py[b], M);
        const double z = wavg(ma, s.pz[a], mb, s.pz[b], M);
        const int sv = (ma >= mb) ? a : b;
        const int vc = (ma >= mb) ? b : a;
        double rm;
        if (density_merge) {
            double sd = s.density[sv];
            if (sd < 1e-30) sd = dm_density(s.mass[sv], s.radius[sv], min_radius);
            rm = dm_radius(M, sd, min_radius);
        } else {
            const double ra = s.radius[a], rb = s.radius[b];
            rm = cbrt(__dadd_rn(__dmul_rn(__dmul_rn(ra, ra), ra), __dmul_rn(__dmul_rn(rb, rb), rb)));
        }
        s.px[sv] = x; s.py[sv] = y; s.pz[sv] = z;
        s.vx[sv] = vx; s.vy[sv] = vy; s.vz[sv] = vz;
        s.mass[sv] = M;
        s.radius[sv] = rm;
        s.density[sv] = dm_density(M, rm, min_radius);
        s.active[vc] = 0;
    }
    const int surv = (s.mass[a] > 0 && s.active[a]) ? a : b;
    counts[surv]++;
}

// Exclusive count of `flag` over the threads before this one in the block,
// and the block's total.  All threads call it.
__device__ __forceinline__ int block_excl_count(bool flag, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, flag);
    __syncthreads();  // s_warp may still be read by the previous call
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < kMergeThreads / 32; w++) {
        const int c = s_warp[w];
        if (w < warp) off += c;
        tot += c;
    }
    *total = tot;
    return off + __popc(m & lanemask_lt());
}

// Ascending sort of the w pair keys (distinct) by the merge block itself,
// so that the pair count never has to reach the host: up to kBitonicMax keys
// a bitonic network in shared memory, above that a stable LSD radix sort of
// 8 passes over the block in global memory (alt as the other buffer; the
// result ends in keys).  The large case needs more than kBitonicMax pairs in
// one step, over 100 times the disk workload's usual count.
constexpr int kBitonicMax = 2048;

__device__ void block_sort_pairs(uint64_t* keys, uint64_t* alt, int w) {
    __shared__ uint64_t s_b[kBitonicMax];
    __shared__ uint16_t s_wc[kMergeThreads / 32][256];  // per-warp digit counts, then offsets
    __shared__ uint32_t s_base[256], s_tot[256];
    const int t = threadIdx.x, warp = t >> 5;
    if (w <= 1) return;
    if (w <= kBitonicMax) {
        int n2 = 2;
        while (n2 < w) n2 <<= 1;
        for (int i = t; i < n2; i += kMergeThreads) s_b[i] = i < w ? keys[i] : ~0ull;
        __syncthreads();
        for (int k = 2; k <= n2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = t; i < n2; i += kMergeThreads) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const uint64_t a = s_b[i], b = s_b[ixj];
                        if ((a > b) == ((i & k) == 0)) {
                            s_b[i] = b;
                            s_b[ixj] = a;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = t; i < w; i += kMergeThreads) keys[i] = s_b[i];
        __syncthreads();
        return;
    }
    uint64_t* src = keys;
    uint64_t* dst = alt;
    for (int p = 0; p < 8; p++) {
        const int shift = 8 * p;
        if (t < 256) s_tot[t] = 0;
        __syncthreads();
        for (int i = t; i < w; i += kMergeThreads) atomicAdd(&s_tot[(src[i] >> shift) & 0xFF], 1u);
        __syncthreads();
        if (t == 0) {
            uint32_t run = 0;
            for (int d = 0; d < 256; d++) {
                s_base[d] = run;
                run += s_tot[d];
            }
        }
        __syncthreads();
        for (int c = 0; c < w; c += kMergeThreads) {
            const int i = c + t;
            const bool valid = i < w;
            const uint64_t key = valid ? src[i] : 0ull;
            const uint32_t d = (uint32_t)(key >> shift) & 0xFF;
            for (int x = t; x < (kMergeThreads / 32) * 256; x += kMergeThreads) (&s_wc[0][0])[x] = 0;
            __syncthreads();
            unsigned peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const unsigned bal = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
                peers &= ((d >> b) & 1u) ? bal : ~bal;
            }
            const int rank = __popc(peers & lanemask_lt());
            if (valid && rank == 0) s_wc[warp][d] = (uint16_t)__popc(peers);
            __syncthreads();
            if (t < 256) {
                uint32_t run = 0;
                for (int x = 0; x < kMergeThreads / 32; x++) {
                    const uint32_t v = s_wc[x][t];
                    s_wc[x][t] = (uint16_t)run;
                    run += v;
                }
                s_tot[t] = run;
            }
            __syncthreads();
            if (valid) dst[s_base[d] + s_wc[warp][d] + rank] = key;
            __syncthreads();
            if (t < 256) s_base[t] += s_tot[t];
            __syncthreads();
        }
        uint64_t* tmp = src;
        src = dst;
        dst = tmp;
    }
}

// np_dev: with it the pair count is read on the device (the broad phase's
// count, capped at np), the pairs are still unsorted and the block sorts them
// first (pairs_alt: its second buffer); without it np pairs are sorted.
__global__ void __launch_bounds__(kMergeThreads)
k_merge_rounds(State s, uint64_t* __restrict__ pairs, uint64_t* __restrict__ pairs_alt, int np,
               const int* np_dev, int max_frame, int max_body, int density_merge,
               double min_radius, int* __restrict__ counts, int* __restrict__ owner,
               int* __restrict__ n_merges, int* err) {
    __shared__ int s_warp[kMergeThreads / 32];
    const int t = threadIdx.x;
    if (np_dev) {
        np = min(*np_dev, np);
        block_sort_pairs(pairs, pairs_alt, np);
    }
    int merged = 0;  // merges of the finished windows (the same in every thread)
    for (int base = 0; base < np && merged < max_frame; base += kMergeThreads) {
        const int k = base + t;
        bool pending = k < np;
        bool event = false;  // this pair merged (or counted as a merge)
        int a = 0, b = 0;
        if (pending) {
            const uint64_t pk = pairs[k];
            a = (int)(pk >> 32);
            b = (int)(pk & 0xFFFFFFFFu);
        }
        int left = 0;
        block_excl_count(pending, s_warp, &left);
        for (int round = 0; left > 0; round++) {
            if (round > kMergeThreads) {  // cannot happen: a round resolves >= 1 pair
                if (t == 0) dev_flag(err, kErrTimeout);
                break;
            }
            if (pending) {
                owner[a] = INT_MAX;
                owner[b] = INT_MAX;
            }
            __syncthreads();
            if (pending) {
                atomicMin(&owner[a], k);
                atomicMin(&owner[b], k);
            }
            __syncthreads();
            const bool ready = pending && owner[a] == k && owner[b] == k;
            int tot_unused = 0;
            const int pend_before = block_excl_count(pending, s_warp, &tot_unused);
            const int ev_before = block_excl_count(event, s_warp, &tot_unused);
            if (ready) {
                const int E = merged + ev_before;
                if (!s.active[a] || !s.active[b] || E >= max_frame) {
                    pending = false;  // a skip, whatever the cap
                } else if (E + pend_before < max_frame) {
                    pending = false;
                    if (counts[a] < max_body && counts[b] < max_body) {
                        merge_pair(s, a, b, density_merge, min_radius, counts);
                        event = true;
                    }
                }
                // otherwise the cap is undecided: wait for the earlier pairs
            }
            __syncthreads();  // this round's merges are visible to the next
            block_excl_count(pending, s_warp, &left);
        }
        int ev_total = 0;
        block_excl_count(event, s_warp, &ev_total);
        merged += ev_total;
    }
    if (t == 0) *n_merges = merged < max_frame ? merged : max_frame;
}

// ---- compaction ---------------------------------------------------------

// Destination row of every kept row (active with mass > 0), -1 for the rest:
// a ballot count per warp, a warp-wide decoupled look-back across tiles.
__global__ void __launch_bounds__(kCompThreads)
k_compact(int n, State s, int32_t* __restrict__ dest, uint32_t* look, uint32_t* tile_ctr,
          int* n_kept, int* err, const int* dn) {
    __shared__ int s_tile;
    n = dev_rows(n, dn);  // tiles past the rows keep nothing
    __shared__ uint32_t s_wtot[kCompThreads / 32];
    __shared__ uint32_t s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const int tile = s_tile;
    const int seg = tile * kCompTile + warp * (32 * kCompItems);
    unsigned ball[kCompItems];
    uint32_t wcount = 0;
#pragma unroll
    for (int k = 0; k < kCompItems; k++) {
        const int i = seg + k * 32 + lane;
        const bool keep = i < n && s.active[i] && s.mass[i] > 0.0;
        ball[k] = __ballot_sync(0xFFFFFFFFu, keep);
        wcount += __popc(ball[k]);
    }
    if (lane == 0) s_wtot[warp] = wcount;
    __syncthreads();
    if (warp == 0) {
        // warp-wide look-back: lane q reads predecessor j - q, so one L2
        // round trip covers 32 tiles; the words are consumed nearest first up
        // to the first inclusive prefix or the first unpublished word
        uint32_t tot = 0;
        for (int w = 0; w < kCompThreads / 32; w++) tot += s_wtot[w];
        uint32_t excl = 0;
        if (tile == 0) {
            if (lane == 0) atomicExch(&look[0], kCFlagPre | tot);
        } else {
            if (lane == 0) atomicExch(&look[tile], kCFlagAgg | tot);
            int j = tile - 1;
            uint32_t spins = 0;
            for (;;) {
                const uint32_t v = (j - lane >= 0) ? *(volatile uint32_t*)&look[j - lane] : 0u;
                const uint32_t f = v & ~kCValMask;
                // tile 0 always publishes a prefix: j - lane == 0 ends the chain
                const unsigned stop = __ballot_sync(0xFFFFFFFFu, f == kCFlagPre ||
                                                                     (f != 0 && j - lane == 0));
                const unsigned unpub = __ballot_sync(0xFFFFFFFFu, f == 0);
                const int first_stop = stop ? __ffs(stop) - 1 : 32;
                const int first_unpub = unpub ? __ffs(unpub) - 1 : 32;
                const bool done = first_stop < first_unpub;
                const int used = done ? first_stop + 1 : first_unpub;
                excl += __reduce_add_sync(0xFFFFFFFFu, lane < used ? (v & kCValMask) : 0u);
                if (done) break;
                j -= used;
                if (used == 0 && ++spins > kSpinLimit) {
                    if (lane == 0) dev_flag(err, kErrTimeout);
                    break;
                }
            }
            __threadfence();
            if (lane == 0) atomicExch(&look[tile], kCFlagPre | (excl + tot));
        }
        if (lane == 0) {
            s_base = excl;
            if (tile == (int)gridDim.x - 1) *n_kept = (int)(excl + tot);
        }
    }
    __syncthreads();
    uint32_t off = s_base;
    for (int w = 0; w < warp; w++) off += s_wtot[w];
#pragma unroll
    for (int k = 0; k < kCompItems; k++) {
        const int i = seg + k * 32 + lane;
        const bool keep = (ball[k] >> lane) & 1u;
        const uint32_t pos = off + __popc(ball[k] & lanemask_lt());
        off += __popc(ball[k]);
        if (i < n) dest[i] = keep ? (int32_t)pos : -1;
    }
}

// The kept rows' 15 fields moved to their destination rows: one thread per
// row, so every field's loads and stores of a warp are in flight together
// (the rows keep their order, so the stores of a warp are nearly contiguous).
__global__ void k_scatter_rows(int n, State s, State d, const int32_t* __restrict__ dest,
                               const int* dn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dev_rows(n, dn)) return;
    const int pos = dest[i];
    if (pos < 0) return;
    d.px[pos] = s.px[i]; d.py[pos] = s.py[i]; d.pz[pos] = s.pz[i];
    d.vx[pos] = s.vx[i]; d.vy[pos] = s.vy[i]; d.vz[pos] = s.vz[i];
    d.ax[pos] = s.ax[i]; d.ay[pos] = s.ay[i]; d.az[pos] = s.az[i];
    d.mass[pos] = s.mass[i]; d.radius[pos] = s.radius[i]; d.density[pos] = s.density[i];
    d.active[pos] = s.active[i]; d.collidable[pos] = s.collidable[i];
    d.ids[pos] = s.ids[i];
}

// dest: n destination rows (-1: removed); with `d` the kept rows are moved
// into d's rows 0 .. *n_kept - 1.  dn: optional device row count (<= n).
static void launch_compact(cudaStream_t st, CollideBufs& b, int n, const State& s,
                           const State* d, int32_t* dest, int* n_kept, int* err,
                           const int* dn = nullptr) {
    const int tiles = ceil_div(n, kCompTile);
    cudaMemsetAsync(b.look, 0, sizeof(uint32_t) * (size_t)tiles, st);
    cudaMemsetAsync(b.tile_ctr, 0, sizeof(uint32_t), st);
    k_compact<<<tiles, kCompThreads, 0, st>>>(n, s, dest, b.look, b.tile_ctr, n_kept, err, dn);
    if (d) k_scatter_rows<<<ceil_div(n, 256), 256, 0, st>>>(n, s, *d, dest, dn);
}

int compact_indices(cudaStream_t st, CollideBufs& b, int n, const uint8_t* active,
                    const double* mass, int32_t* dest, int* n_kept_dev, int* err) {
    if (n <= 0) return NB_OK;
    State s{};
    s.active = (uint8_t*)active;
    s.mass = (double*)mass;
    launch_compact(st, b, n, s, nullptr, dest, n_kept_dev, err);
    return cudaGetLastError() == cudaSuccess ? NB_OK : NB_ERR_CUDA;
}

// The collision stage with no host round trip, for a captured step: the
// pair count stays on the device (the merge block sorts the pairs itself)
// and the rows are counted by *dn, which the compaction's count replaces at
// the end.  It queries the force evaluation's tree (a.reuse_tree); a.n and
// a.n_active only bound the launches.
int collide_step_device(cudaStream_t st, CollideBufs& b, CollideArgs& a, int* dn) {
    if (!a.reuse_tree) return NB_ERR_INVALID_ARG;
    cudaMemsetAsync(a.n_pairs, 0, sizeof(int), st);
    if (a.n <= 0) return NB_OK;
    if (a.n_active > 0) {
        find_groups(st, a.tree, a.sbody, a.n_active, a.groups, a.n_groups, 2.25, 0);
        cudaMemsetAsync(a.group_ctr, 0, sizeof(unsigned), st);
        k_broad_phase_groups<<<a.sms * 4, kBpWarps * 32, 0, st>>>(
            a.s, a.vals0, a.tree, a.cube, a.groups, a.n_groups, a.group_ctr,
            b.pair_keys, b.pair_cap, a.n_pairs, a.err);
    }
    cudaMemsetAsync(b.merge_count, 0, sizeof(int) * (size_t)a.n, st);
    k_merge_rounds<<<1, kMergeThreads, 0, st>>>(a.s, b.pair_keys, b.pair_keys_alt, b.pair_cap,
                                                a.n_pairs, a.max_frame, a.max_body,
                                                a.density_merge, a.min_radius, b.merge_count,
                                                b.owner, a.n_merges, a.err);
    launch_compact(st, b, a.n, a.s, &a.s_alt, b.owner, a.n_kept, a.err, dn);
    cudaMemcpyAsync(dn, a.n_kept, sizeof(int), cudaMemcpyDeviceToDevice, st);
    return NB_OK;
}

int collide_step(cudaStream_t st, CollideBufs& b, CollideArgs& a, int* npairs, int* nmerge,
                 int* nkept) {
    int np = 0;
    int r = broad_phase(st, b, a, true, &np);
    if (r) return r;
    *npairs = np;
    *nmerge = 0;
    const int w = np < b.pair_cap ? np : b.pair_cap;
    cudaMemsetAsync(a.n_merges, 0, sizeof(int), st);
    if (w > 0) {
        cudaMemsetAsync(b.merge_count, 0, sizeof(int) * (size_t)a.n, st);
        k_merge_rounds<<<1, kMergeThreads, 0, st>>>(a.s, b.pair_keys, b.pair_keys_alt, w, nullptr,
                                                    a.max_frame, a.max_body, a.density_merge,
                                                    a.min_radius, b.merge_count, b.owner,
                                                    a.n_merges, a.err);
    }
    // the merge's owner words are free again: they hold the destination rows
    launch_compact(st, b, a.n, a.s, &a.s_alt, b.owner, a.n_kept, a.err);
    int host[2] = {0, 0};
    if (cudaMemcpyAsync(&host[0], a.n_kept, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&host[1], a.n_merges, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return NB_ERR_CUDA;
    *nkept = host[0];
    *nmerge = host[1];
    return NB_OK;
}

}  // namespace nb
