// tree.cuh - octree construction and multipoles on the GPU.
#pragma once
#include "common.cuh"

namespace nb {

// Device buffers of the radix tree (over n active sorted keys) and of the
// walk tree (the octree with single-child chains collapsed and leaf buckets
// of at most `leaf_cap` bodies, children stored contiguously).
struct TreeBufs {
    // binary radix tree, n-1 internal nodes
    int* bchild;        // 2 per node: >= 0 internal node, < 0 leaf body ~c
    int* bfirst;        // first sorted position covered
    int* blast;         // last sorted position covered
    uint8_t* bdelta;    // common prefix length in the 63-bit key, capped at 63
    int* bparent;       // parent internal node, -1 for the root
    uint8_t* bnchild;   // walk-tree children of this node (0 unless walk-internal)
    int* child_base;    // walk index of the first child of a walk-internal node
    int* walk_index;    // walk index of an octree node, -1 otherwise
    int* block_sums;    // scan workspace
    // walk tree, up to 2n nodes
    int4* link;         // first_child (-1 leaf), n_child, body_first, body_count
    int* level;         // octree level of the node's (deepest) cell
    int* parent_bin;    // binary id of the parent octree node (-1 root)
    int* parent_walk;   // walk index of the parent node (-1 root; set by the multipole pass)
    double4* com;       // centre of mass (FP64) and mass
    float4* q0;         // Qxx, Qyy, Qxy, Qxz (traceless, about the COM)
    float4* q1;         // Qyz, cell half-size, max body radius, 0
    float4* blo;        // bounding box of the node's bodies (xyz, rounded outwards)
    float4* bhi;
    int* counter;       // bottom-up arrival counters
    int* leaves;        // walk index of every leaf (multipole pass, any order)
    int* n_leaves;      // device leaf count
    int* n_nodes;       // device node count
    int capacity;       // bodies
};

size_t tree_bytes(int capacity);
void tree_carve(TreeBufs& t, void* base, int capacity);

// Build the walk tree over n sorted keys (already in sorted order) with the
// bodies sorted in `sbody` (x, y, z, m).  cube: device (cx, cy, cz, half).
// srad may be null (then max radius is 0).  Batched systems: the keys hold
// the system index in bits 62..51 (four octree levels) and a 17-bit-per-axis
// Morton code in that system's own cube below; sys_half16[s] = that cube's
// half-size x 16 (cube is then unused).  dn: optional device body count
// replacing n when smaller (the launches stay sized for n).
void tree_build(cudaStream_t st, const TreeBufs& t, int n, const uint64_t* skeys,
                const double4* sbody, const float* srad, const double* cube, int leaf_cap,
                int* err, const double* sys_half16 = nullptr, const int* dn = nullptr);

}  // namespace nb
