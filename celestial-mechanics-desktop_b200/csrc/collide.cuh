// collide.cuh - collision broad phase, merge and stream compaction.
#pragma once
#include <functional>

#include "bodies.cuh"
#include "tree.cuh"

namespace nb {

struct CollideBufs {
    int pair_cap;
    uint64_t* pair_keys;   // (lo << 32 | hi), sorted after broad_phase
    uint32_t* pair_vals;
    uint64_t* pair_keys_alt;
    uint32_t* pair_vals_alt;
    void* pair_sort_ws;
    int* merge_count;      // per row, merges this step
    int* owner;            // per row, the lowest pending pair touching it (merge rounds)
    uint32_t* look;        // compaction look-back words
    uint32_t* tile_ctr;
    int capacity;
};

struct CollideArgs {
    int n, n_active;
    State s, s_alt;
    uint64_t *keys0, *keys1;
    uint32_t *vals0, *vals1;
    void* sort_ws;
    TreeBufs tree;
    double4* sbody;
    float* srad;
    double* cube;
    int leaf_cap;
    int max_frame, max_body, density_merge;
    double min_radius;
    int *n_pairs, *n_kept, *n_merges;
    int* err;
    int sms;
    unsigned long long* bbox_ord;
    int* n_active_dev;
    // the force evaluation of this step left a tree of the current positions
    // (keys0/vals0 sorted, sbody/srad gathered, multipole pass with radii,
    // cube): the broad phase queries it instead of building its own
    bool reuse_tree = false;
    // walk-group buffers the broad phase (re)fills: >= n_active entries, the
    // device group count and a work counter
    int2* groups = nullptr;
    int* n_groups = nullptr;
    unsigned* group_ctr = nullptr;
};

int collide_alloc(CollideBufs& b, int capacity, const std::function<int(void**, size_t)>& alloc);
// All overlapping pairs of active, collidable rows, sorted; *np on the host.
// build_tree: the bounding cube is recomputed first (otherwise a.cube is
// current); with a.reuse_tree no key, sort or tree stage runs at all.
int broad_phase(cudaStream_t st, CollideBufs& b, CollideArgs& a, bool build_tree, int* np);
// Broad phase + merges + compaction of c.s into c.s_alt.
int collide_step(cudaStream_t st, CollideBufs& b, CollideArgs& a, int* npairs, int* nmerge,
                 int* nkept);
// The same stage with every count kept on the device, for a captured step:
// the rows are counted by *dn (replaced by the kept count at the end); needs
// a.reuse_tree; a.n / a.n_active bound the launches.
int collide_step_device(cudaStream_t st, CollideBufs& b, CollideArgs& a, int* dn);
// Destination rows of the order-preserving compaction (mask active && mass > 0).
int compact_indices(cudaStream_t st, CollideBufs& b, int n, const uint8_t* active,
                    const double* mass, int32_t* dest, int* n_kept_dev, int* err);

}  // namespace nb
