// walk.cuh - Barnes-Hut tree walks.
#pragma once
#include "common.cuh"
#include "mac.cuh"
#include "tree.cuh"

namespace nb {

struct WalkArgs {
    int n;                      // active bodies, sorted positions [0, n)
    const double4* sbody;       // sorted x, y, z, m
    const float* srad;          // sorted radius (shell theorem), may be null
    const uint64_t* skeys;      // sorted keys (reference-order walk)
    const uint32_t* sidx;       // sorted position -> body row
    TreeBufs t;
    double theta2, eps2;
    double* ax;                 // outputs by body row
    double* ay;
    double* az;
    double* pot;                // potential by body row (may be null)
    int* front;                 // per-warp node stacks, front_cap ints each
    int front_cap;
    int2* groups;               // walk groups: body_first, body_count (<= group_size)
    int* n_groups;
    double pack;                // sibling packing box-growth limit (0: no packing)
    int group_span;             // >= 32: runs of group_size bodies inside cells of <=
                                // group_span bodies (find_groups); otherwise sibling packing
    int group_size;             // 32, or 64 with span groups: a lane holds two bodies
    // learned MAC / harvest
    const float* samag;         // |a| of each sorted body from the previous step
    const MacDev* mac;          // network image (learned mode)
    const float2* mac_node;     // per walk-tree node: screen term, log2 mass (learned mode)
    float mac_theta_hi2;        // band upper edge, (2h/d)^2
    float mac_budget;           // normalised log2 error budget (learned mode)
    MacRecord* records;         // harvest output
    int* n_records;
    int record_cap;
    unsigned mac_seed;          // harvest group sampling
    unsigned mac_sample;        // groups kept per 65536
    const int* sys_root;        // batched systems: walk-tree root of each system
                                // (indexed by the key's system field), else null
    unsigned* group_ctr;        // dynamic group counter (zeroed)
    unsigned long long* counters;  // [0] body-cell, [1] body-body interactions
    int* err;
};

struct WalkConfig {
    int blocks;        // persistent grid size
    int blocks_mac;    // persistent grid size of the learned-MAC walk
    int blocks_small;  // persistent grid size of the small-block geometric walk (shape 1)
    int blocks64;      // persistent grid sizes of the 64-body-group walks
    int blocks_mac64;
    int front_cap;
};

void walk_init(int sms, WalkConfig& cfg);
// Walk groups (sets of at most 32 consecutive sorted bodies), groups: >= n
// entries.  span >= 32: every walk-tree node holding at most `span` bodies
// whose parent holds more is cut into runs of 32 consecutive bodies.
// Otherwise: the octree nodes holding <= 32 bodies whose parent holds more,
// runs of such siblings packed while the packed box stays within `pack`
// times the larger part's (0: no packing), plus 32-body slices of level-21
// buckets that hold more than 32.
void find_groups(cudaStream_t st, const TreeBufs& t, const double4* sbody, int n, int2* groups,
                 int* n_groups, double pack, int span, int size = 32);
size_t walk_front_bytes(const WalkConfig& cfg);
// Group walk, FP32 monopole(+quadrupole) on FP64-differenced coordinates.
// mac: 0 geometric, 1 harvest, 2 learned (1 and 2 need quad, no shell, no
// potential, softening > 0).  shape (geometric quadrupole walk without shell
// theorem or potential): 0 = blocks of 8 warps, 1 = blocks of 4 warps (the
// same warps per SM).
void walk_group(cudaStream_t st, const WalkConfig& cfg, WalkArgs a, bool quad, bool shell,
                bool pot, int mac = 0, int shape = 0);
// Per-body FP64 walk with the reference's MAC, monopole, child order.
void walk_reference(cudaStream_t st, WalkArgs a, bool shell);

}  // namespace nb
