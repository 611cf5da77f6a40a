// tree.cu - parallel octree build from sorted Morton keys, and multipoles.
//
// Replaces tree_build_kernel<<<1,1>>> (engine/src/cuda/gpu_tree.cu:269-464,
// one thread inserting every body) with a fully parallel construction:
//   1. k_radix_tree: Karras' binary radix tree over the sorted 63-bit keys
//      (Karras 2012, "Maximizing parallelism in the construction of BVHs,
//      octrees and k-d trees"), one thread per internal node; equal keys are
//      split by index so the tree is always binary.
//   2. k_octree_mark: a binary node X is an octree node iff floor(d_X/3) >
//      floor(d_parent/3) (d = common prefix length): its body range is then
//      exactly an octree cell, the deepest one being level floor(d_X/3).
//      Single-child chains of the point-region octree collapse into it.  A
//      node is emitted when its octree parent holds more than leaf_cap
//      bodies; it is walk-internal when it also holds more than leaf_cap
//      bodies and is above level 21.  Its walk children are the exits of
//      its <= 3-deep binary subtree inside the same cell, in key order.
//   3. block scan of the child counts gives every walk-internal node a
//      contiguous child slot range; k_octree_emit writes the nodes.
//   4. k_multipole_leaves / k_multipole_climb: leaves from their bodies, then
//      bottom-up, the last child to arrive at a parent computes the parent
//      (arrival counters), so each node is reduced exactly once from its
//      children in child order: deterministic.
// With leaf_cap = 1 the walk tree is the reference's point-region octree
// (OctreeBuilder::insert_body, engine/src/physics/octree_builder.cpp:50-105)
// down to level 21, with chains collapsed.
#include "tree.cuh"

#include <algorithm>

namespace nb {

constexpr int kMarkThreads = 256;
constexpr int kMarkItems = 4;
constexpr int kMarkTile = kMarkThreads * kMarkItems;  // internal nodes per block

size_t tree_bytes(int cap) {
    size_t c = (size_t)(cap > 1 ? cap : 2);
    size_t b = 0;
    b += 2 * c * 4 + c * 4 + c * 4 + c + c * 4 + c + c * 4 + c * 4;  // binary tree
    b += (c / kMarkTile + 2) * 4;                                      // block sums
    b += 256;                                                          // align slack
    size_t w = 2 * c;
    b += w * 16 + w * 4 + w * 4 + w * 32 + w * 16 + w * 16 + w * 4 + 16;
    b += w * 4 + 16;                                                   // parent walk index
    b += 2 * w * 16;                                                   // body boxes
    b += c * 4 + 16;                                                   // leaf list
    return b + 16 * 64;
}

template <typename T>
static T* carve(char*& p, size_t count, size_t align = 16) {
    uintptr_t a = ((uintptr_t)p + align - 1) & ~(uintptr_t)(align - 1);
    p = (char*)(a + count * sizeof(T));
    return (T*)a;
}

void tree_carve(TreeBufs& t, void* base, int cap) {
    size_t c = (size_t)(cap > 1 ? cap : 2);
    size_t w = 2 * c;
    char* p = (char*)base;
    t.com = carve<double4>(p, w, 32);
    t.link = carve<int4>(p, w);
    t.q0 = carve<float4>(p, w);
    t.q1 = carve<float4>(p, w);
    t.blo = carve<float4>(p, w);
    t.bhi = carve<float4>(p, w);
    t.level = carve<int>(p, w);
    t.parent_bin = carve<int>(p, w);
    t.parent_walk = carve<int>(p, w);
    t.counter = carve<int>(p, w);
    t.n_nodes = carve<int>(p, 4);
    t.leaves = carve<int>(p, c);
    t.n_leaves = carve<int>(p, 4);
    t.bchild = carve<int>(p, 2 * c);
    t.bfirst = carve<int>(p, c);
    t.blast = carve<int>(p, c);
    t.bparent = carve<int>(p, c);
    t.child_base = carve<int>(p, c);
    t.walk_index = carve<int>(p, c);
    t.block_sums = carve<int>(p, c / kMarkTile + 2);
    t.bdelta = carve<uint8_t>(p, c);
    t.bnchild = carve<uint8_t>(p, c);
    t.capacity = cap;
}

// Common prefix length of sorted keys i and j in the 63-bit key space;
// equal keys continue with the index bits (>= 63); -1 out of range.
__device__ __forceinline__ int prefix_len(const uint64_t* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[i], b = k[j];
    if (a != b) return __clzll((long long)(a ^ b)) - 1;
    return 63 + __clz(i ^ j);
}

__global__ void k_radix_tree(int n, const uint64_t* __restrict__ keys, TreeBufs t, const int* dn) {
    n = dev_rows(n, dn);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int dl = prefix_len(keys, n, i, i - 1);
    int dr = prefix_len(keys, n, i, i + 1);
    int d = (dr > dl) ? 1 : -1;
    int dmin = min(dl, dr);
    int lmax = 2;
    while (prefix_len(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int s = lmax >> 1; s >= 1; s >>= 1)
        if (prefix_len(keys, n, i, i + (l + s) * d) > dmin) l += s;
    int j = i + l * d;
    int dnode = prefix_len(keys, n, i, j);
    int s = 0, step = l;
    do {
        step = (step + 1) >> 1;
        if (prefix_len(keys, n, i, i + (s + step) * d) > dnode) s += step;
    } while (step > 1);
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    int left = (first == gamma) ? ~gamma : gamma;
    int right = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    t.bchild[2 * i] = left;
    t.bchild[2 * i + 1] = right;
    t.bfirst[i] = first;
    t.blast[i] = last;
    t.bdelta[i] = (uint8_t)min(dnode, 63);
    if (left >= 0) t.bparent[left] = i;
    if (right >= 0) t.bparent[right] = i;
    if (i == 0) t.bparent[0] = -1;
}

__device__ __forceinline__ int lvl(const TreeBufs& t, int x) { return t.bdelta[x] / 3; }

// Walk-tree children (exits of the binary subtree inside node i's cell),
// visited in key order; calls f(child_code) for each.
template <typename F>
__device__ __forceinline__ void for_each_exit(const TreeBufs& t, int i, F f) {
    const int li = lvl(t, i);
    int stack[8];  // the subtree is at most 3 binary levels deep: <= 5 entries
    int sp = 0;
    stack[sp++] = t.bchild[2 * i + 1];
    stack[sp++] = t.bchild[2 * i];
    while (sp > 0) {
        int c = stack[--sp];
        if (c < 0 || lvl(t, c) > li) {
            f(c);
        } else {  // same cell: expand, right pushed first so left comes out first
            stack[sp++] = t.bchild[2 * c + 1];
            stack[sp++] = t.bchild[2 * c];
        }
    }
}

// Counting pass; the visiting order does not matter here.
__device__ int count_exits(const TreeBufs& t, int i) {
    int c = 0;
    for_each_exit(t, i, [&](int) { c++; });
    return c;
}

__device__ __forceinline__ bool walk_internal(const TreeBufs& t, int x, int leaf_cap) {
    return (t.blast[x] - t.bfirst[x] + 1) > leaf_cap && lvl(t, x) < 21;
}

__global__ void __launch_bounds__(kMarkThreads)
k_octree_mark(int n, TreeBufs t, int leaf_cap, const int* dn) {
    __shared__ int s_red[kMarkThreads / 32];
    const int m = dev_rows(n, dn) - 1;  // internal nodes (blocks past them sum 0)
    int local = 0;
    for (int k = 0; k < kMarkItems; k++) {
        int i = blockIdx.x * kMarkTile + k * kMarkThreads + threadIdx.x;
        if (i >= m) break;
        int P = t.bparent[i];
        int li = lvl(t, i);
        bool exists;
        if (P < 0) {
            exists = true;
        } else if (li <= lvl(t, P)) {
            exists = false;  // inside its parent's cell
        } else {
            int Y = P;  // climb to the octree node holding P
            while (t.bparent[Y] >= 0 && lvl(t, t.bparent[Y]) == lvl(t, Y)) Y = t.bparent[Y];
            exists = walk_internal(t, Y, leaf_cap);
        }
        int nc = (exists && walk_internal(t, i, leaf_cap)) ? count_exits(t, i) : 0;
        t.bnchild[i] = (uint8_t)nc;
        t.walk_index[i] = -1;
        local += nc;
    }
    local = warp_sum(local);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kMarkThreads / 32; w++) s += s_red[w];
        t.block_sums[blockIdx.x] = s;
    }
}

// Exclusive scan of the block sums in one block; writes the node count.
__global__ void k_scan_block_sums(int nblocks, TreeBufs t, int n, const int* dn) {
    __shared__ int s[1024];
    n = dev_rows(n, dn);
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nblocks; base += 1024) {
        int i = base + threadIdx.x;
        int v = (i < nblocks) ? t.block_sums[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int x = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += x;
            __syncthreads();
        }
        if (i < nblocks) t.block_sums[i] = carry + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *t.n_nodes = (n >= 2) ? 1 + carry : (n == 1 ? 1 : 0);
}

// Child slot of every walk-internal node: 1 + exclusive scan of bnchild.
__global__ void __launch_bounds__(kMarkThreads) k_octree_base(int n, TreeBufs t, const int* dn) {
    __shared__ int s_w[kMarkThreads / 32];
    const int m = dev_rows(n, dn) - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int off = 1 + t.block_sums[blockIdx.x];
    for (int k = 0; k < kMarkItems; k++) {
        int i = blockIdx.x * kMarkTile + k * kMarkThreads + threadIdx.x;
        int v = (i < m) ? t.bnchild[i] : 0;
        int inc = warp_incl_scan(v);
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        int wpre = 0, tot = 0;
        for (int w = 0; w < kMarkThreads / 32; w++) {
            int x = s_w[w];
            if (w < warp) wpre += x;
            tot += x;
        }
        if (i < m) t.child_base[i] = off + wpre + inc - v;
        off += tot;
        __syncthreads();
    }
}

__global__ void k_octree_emit(int n, TreeBufs t, int leaf_cap, const int* dn) {
    n = dev_rows(n, dn);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (n == 1) {
        if (i == 0) {
            t.link[0] = make_int4(-1, 0, 0, 1);
            t.level[0] = 0;
            t.parent_bin[0] = -1;
        }
        return;
    }
    if (i >= n - 1) return;
    if (i == 0) {
        bool wi = walk_internal(t, 0, leaf_cap);
        t.link[0] = make_int4(wi ? t.child_base[0] : -1, t.bnchild[0], 0, n);
        t.level[0] = lvl(t, 0);
        t.parent_bin[0] = -1;
        t.walk_index[0] = 0;
    }
    int nc = t.bnchild[i];
    if (nc == 0) return;
    const int li = lvl(t, i);
    int w = t.child_base[i];
    for_each_exit(t, i, [&](int c) {
        if (c < 0) {
            t.link[w] = make_int4(-1, 0, ~c, 1);
            t.level[w] = li + 1;
        } else {
            bool wi = walk_internal(t, c, leaf_cap);
            int cnt = t.blast[c] - t.bfirst[c] + 1;
            t.link[w] = make_int4(wi ? t.child_base[c] : -1, wi ? (int)t.bnchild[c] : 0,
                                  t.bfirst[c], cnt);
            t.level[w] = lvl(t, c);
            t.walk_index[c] = w;
        }
        t.parent_bin[w] = i;
        w++;
    });
}

// Moments of a set of point masses or child cells accumulated in one pass
// about a reference point r0 (the first member): M, S = sum m d, the second
// moments T = sum m d d^T (d = x - r0) and, for cells, the sum of the
// children's own traceless quadrupoles.  The centre of mass is r0 + S / M and
// the traceless quadrupole about it follows from the parallel-axis shift
// C = T - M D D^T (D = S / M), Q = 3 C - tr(C) I + sum Q_child; with r0 inside
// the cell the shift cancels nothing larger than the cell's own spread.
struct Moments {
    double M = 0, sx = 0, sy = 0, sz = 0;
    double txx = 0, tyy = 0, tzz = 0, txy = 0, txz = 0, tyz = 0;
    double qxx = 0, qyy = 0, qxy = 0, qxz = 0, qyz = 0;
    __device__ __forceinline__ void add(double m, double dx, double dy, double dz) {
        M += m;
        const double mx = m * dx, my = m * dy, mz = m * dz;
        sx += mx; sy += my; sz += mz;
        txx = fma(mx, dx, txx); tyy = fma(my, dy, tyy); tzz = fma(mz, dz, tzz);
        txy = fma(mx, dy, txy); txz = fma(mx, dz, txz); tyz = fma(my, dz, tyz);
    }
    // centre of mass (r0 when massless) and the quadrupole about it
    __device__ __forceinline__ void finish(double r0x, double r0y, double r0z, double4& com,
                                           float4& q0, float& qyz_out) const {
        double Dx = 0, Dy = 0, Dz = 0;
        if (M > 0) {
            Dx = sx / M; Dy = sy / M; Dz = sz / M;
        }
        const double cxx = txx - M * Dx * Dx, cyy = tyy - M * Dy * Dy, czz = tzz - M * Dz * Dz;
        const double cxy = txy - M * Dx * Dy, cxz = txz - M * Dx * Dz, cyz = tyz - M * Dy * Dz;
        com = make_double4(r0x + Dx, r0y + Dy, r0z + Dz, M);
        q0 = make_float4((float)(qxx + 2.0 * cxx - cyy - czz), (float)(qyy + 2.0 * cyy - cxx - czz),
                         (float)(qxy + 3.0 * cxy), (float)(qxz + 3.0 * cxz));
        qyz_out = (float)(qyz + 3.0 * cyz);
    }
};

// sys_half16: batched systems (keys carry the system in their top bits): the
// half-size of each system's cube times 2^4, the half-size its level-0 cell
// would have; null for one system in `cube`.
__device__ __forceinline__ int atomic_add_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(p), "r"(v)
                 : "memory");
    return old;
}

// Multipoles in two kernels.  k_multipole_leaves: every leaf reduces its
// bodies in one pass (a persistent grid-stride loop, nothing waits) and enters
// the leaf list.  k_multipole_climb: one thread per leaf, all resident at
// once, climbs; the last child to arrive at a parent reduces it from its
// children in child order, so the result does not depend on which thread
// arrives last (deterministic).  Per level a climb makes two dependent L2
// trips: the parent's link / level / parent words together with the
// acquire-release arrival atomic, then every child word in one loop.  (Computing the
// leaves inside the climbing threads left the last blocks' leaves waiting for
// resident blocks to drain, so the root finished a whole wave of climbs late.)
__global__ void __launch_bounds__(256)
k_multipole_leaves(TreeBufs t, const double4* __restrict__ sbody,
                   const float* __restrict__ srad, const double* __restrict__ cube,
                   const uint64_t* __restrict__ skeys, const double* __restrict__ sys_half16) {
    const int nn = *t.n_nodes;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nn; w += gridDim.x * blockDim.x) {
        const int4 lk = __ldg(&t.link[w]);
        const bool leaf = lk.y == 0;
        // every node's parent as a walk index, for the climb and the groups
        const int pbin = __ldg(&t.parent_bin[w]);
        t.parent_walk[w] = pbin >= 0 ? __ldg(&t.walk_index[pbin]) : -1;
        const unsigned am = __activemask();
        const unsigned lm = __ballot_sync(am, leaf);
        int slot = 0;
        const int lead = __ffs(am) - 1;
        if ((threadIdx.x & 31) == lead && lm) slot = atomicAdd(t.n_leaves, __popc(lm));
        slot = __shfl_sync(am, slot, lead);
        if (!leaf) continue;
        t.leaves[slot + __popc(lm & lanemask_lt())] = w;
        const double root_half =
            sys_half16 ? sys_half16[skeys[lk.z] >> kEnsSysShift] : cube[3];
        const double half = ldexp(root_half, -__ldg(&t.level[w]));
        const double4 p0 = sbody[lk.z];
        Moments mo;
        float rmax = 0.f;
        double lo[3] = {p0.x, p0.y, p0.z}, hi[3] = {p0.x, p0.y, p0.z};
#pragma unroll 4
        for (int b = lk.z; b < lk.z + lk.w; b++) {
            const double4 p = sbody[b];
            mo.add(p.w, p.x - p0.x, p.y - p0.y, p.z - p0.z);
            if (srad) rmax = fmaxf(rmax, srad[b]);
            lo[0] = fmin(lo[0], p.x); lo[1] = fmin(lo[1], p.y); lo[2] = fmin(lo[2], p.z);
            hi[0] = fmax(hi[0], p.x); hi[1] = fmax(hi[1], p.y); hi[2] = fmax(hi[2], p.z);
        }
        double4 com;
        float4 q0;
        float qyz;
        mo.finish(p0.x, p0.y, p0.z, com, q0, qyz);
        t.blo[w] = make_float4(__double2float_rd(lo[0]), __double2float_rd(lo[1]),
                               __double2float_rd(lo[2]), 0.f);
        t.bhi[w] = make_float4(__double2float_ru(hi[0]), __double2float_ru(hi[1]),
                               __double2float_ru(hi[2]), 0.f);
        t.com[w] = com;
        t.q0[w] = q0;
        t.q1[w] = make_float4(qyz, (float)half, rmax, 0.f);
    }
}

// A parent's child words are loaded kClimbUnroll children at a time (one L2
// round trip each batch): 4 children per batch at 128 registers (4 blocks
// of 128 per SM) measured 0.218 ms for the tree stage at 2^20 against 0.231
// with 2 per batch at 80 registers and 0.227 with all 8 at 255.
#ifndef NB_CLIMB_THREADS
#define NB_CLIMB_THREADS 128
#endif
#ifndef NB_CLIMB_MIN_BLOCKS
#define NB_CLIMB_MIN_BLOCKS 4
#endif
constexpr int kClimbThreads = NB_CLIMB_THREADS;
#ifndef NB_CLIMB_UNROLL
#define NB_CLIMB_UNROLL 4
#endif
constexpr int kClimbUnroll = NB_CLIMB_UNROLL;

__global__ void __launch_bounds__(kClimbThreads, NB_CLIMB_MIN_BLOCKS)
k_multipole_climb(TreeBufs t, const double* __restrict__ cube,
                  const uint64_t* __restrict__ skeys, const double* __restrict__ sys_half16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *t.n_leaves) return;
    int p = __ldg(&t.parent_walk[t.leaves[i]]);
    for (int guard = 0; p >= 0 && guard < 64; guard++) {  // <= 22 levels up
        const int4 pl = __ldg(&t.link[p]);
        const int plev = __ldg(&t.level[p]);
        const int pp = __ldg(&t.parent_walk[p]);
        // arrival: release orders this thread's node words before it, acquire
        // orders the children's words (released by their own arrivals) after
        if (atomic_add_acq_rel(&t.counter[p], 1) != pl.y - 1) return;
        const double root_half = sys_half16 ? sys_half16[skeys[pl.z] >> kEnsSysShift] : cube[3];
        const double2 r0a = __ldcg((const double2*)&t.com[pl.x]);
        const double r0z = __ldcg((const double*)&t.com[pl.x] + 2);
        Moments mo;
        float rmax = 0.f;
        float4 blo = make_float4(3e38f, 3e38f, 3e38f, 0.f);
        float4 bhi = make_float4(-3e38f, -3e38f, -3e38f, 0.f);
#pragma unroll kClimbUnroll
        for (int c = pl.x; c < pl.x + pl.y; c++) {
            const double2 a = __ldcg((const double2*)&t.com[c]);
            const double2 b = __ldcg((const double2*)&t.com[c] + 1);
            const float4 c0 = __ldcg(&t.q0[c]);
            const float4 c1 = __ldcg(&t.q1[c]);
            const float4 l = __ldcg(&t.blo[c]), h = __ldcg(&t.bhi[c]);
            mo.add(b.y, a.x - r0a.x, a.y - r0a.y, b.x - r0z);
            mo.qxx += c0.x; mo.qyy += c0.y; mo.qxy += c0.z; mo.qxz += c0.w; mo.qyz += c1.x;
            rmax = fmaxf(rmax, c1.z);
            blo.x = fminf(blo.x, l.x); blo.y = fminf(blo.y, l.y); blo.z = fminf(blo.z, l.z);
            bhi.x = fmaxf(bhi.x, h.x); bhi.y = fmaxf(bhi.y, h.y); bhi.z = fmaxf(bhi.z, h.z);
        }
        double4 com;
        float4 q0;
        float qyz;
        mo.finish(r0a.x, r0a.y, r0z, com, q0, qyz);
        t.blo[p] = blo;
        t.bhi[p] = bhi;
        t.com[p] = com;
        t.q0[p] = q0;
        t.q1[p] = make_float4(qyz, (float)ldexp(root_half, -plev), rmax, 0.f);
        p = pp;
    }
}

// Resident blocks of k_multipole_leaves on this device (its persistent grid).
static int leaves_grid() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_multipole_leaves, 256, 0);
        blocks = std::max(1, sms) * std::max(1, per_sm);
    }
    return blocks;
}

void tree_build(cudaStream_t st, const TreeBufs& t, int n, const uint64_t* skeys,
                const double4* sbody, const float* srad, const double* cube, int leaf_cap,
                int* err, const double* sys_half16, const int* dn) {
    (void)err;
    if (n <= 0) {
        cudaMemsetAsync(t.n_nodes, 0, sizeof(int), st);
        return;
    }
    const int m = n - 1;
    const int nblk = ceil_div(m > 0 ? m : 1, kMarkTile);
    if (m > 0) {
        k_radix_tree<<<ceil_div(m, 256), 256, 0, st>>>(n, skeys, t, dn);
        k_octree_mark<<<nblk, kMarkThreads, 0, st>>>(n, t, leaf_cap, dn);
    }
    k_scan_block_sums<<<1, 1024, 0, st>>>(m > 0 ? nblk : 0, t, n, dn);
    if (m > 0) k_octree_base<<<nblk, kMarkThreads, 0, st>>>(n, t, dn);
    k_octree_emit<<<ceil_div(m > 0 ? m : 1, 256), 256, 0, st>>>(n, t, leaf_cap, dn);
    cudaMemsetAsync(t.counter, 0, sizeof(int) * 2 * (size_t)n, st);
    cudaMemsetAsync(t.n_leaves, 0, sizeof(int), st);
    k_multipole_leaves<<<std::min(ceil_div(2 * n, 256), leaves_grid()), 256, 0, st>>>(
        t, sbody, srad, cube, skeys, sys_half16);
    // at most n leaves (each holds a body); the threads past the count return
    k_multipole_climb<<<ceil_div(n, kClimbThreads), kClimbThreads, 0, st>>>(t, cube, skeys,
                                                                             sys_half16);
}

}  // namespace nb
