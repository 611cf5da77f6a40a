/*
 * nbody_b200.h - C ABI of the B200 (sm_100a) N-body force engine.
 *
 * The engine sits behind the desktop app's force-backend seam
 *   IPhysicsComputeBackend.ComputeForces(BodySoA bodies, double softening)
 *   (src/CelestialMechanics.Physics/Solvers/IPhysicsComputeBackend.cs:21-34)
 * and is reached from C# through P/Invoke.  Every entry point is plain C:
 * opaque handle, raw pointers, explicit sizes, int32 status.  No C++
 * exception crosses this boundary and there is no CPU fallback: when the
 * GPU path cannot run, the call returns a negative status and
 * nb_last_error() says why.
 *
 * Conventions shared by all entry points
 *   - G = 1 (AU, solar mass, time unit of the reference engine,
 *     engine/include/celestial/core/constants.hpp:26,29).
 *   - Host arrays are borrowed for the duration of the call only.
 *   - `active` is one byte per body (C# bool[] passed as byte*).
 *   - A handle owns one CUDA stream and its device buffers; it is not
 *     thread-safe, separate handles are independent.
 *   - Calls that take host arrays are synchronous: results are in the
 *     host arrays when the call returns.
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define NB_API __declspec(dllexport)
#else
#define NB_API __attribute__((visibility("default")))
#endif

typedef struct nb_engine nb_engine;

/* Status codes.  Precedent: the reference ABI returns int32 0 / negative
 * ErrorCode (engine/src/interop/native_api.cpp:30-55). */
enum nb_status {
    NB_OK = 0,
    NB_ERR_INVALID_ARG = -1,
    NB_ERR_CAPACITY = -2,       /* n above the handle's capacity            */
    NB_ERR_CUDA = -3,           /* a CUDA runtime call failed               */
    NB_ERR_TIMEOUT = -4,        /* a bounded device wait ran out            */
    NB_ERR_STACK_OVERFLOW = -5, /* tree-walk frontier overflow (the reference
                                   drops children silently, gpu_tree.cu:588) */
    NB_ERR_NO_DEVICE = -6,      /* no CUDA device / not an sm_100 device    */
    NB_ERR_NONFINITE = -7,      /* NaN/Inf in an input position or mass     */
    NB_ERR_STATE = -8           /* call out of order (e.g. no state set)    */
};

/* Force modes (low 4 bits of `flags`). */
enum nb_mode {
    NB_MODE_DIRECT = 0,          /* tiled O(n^2), FP32 pair math on FP64-differenced coords */
    NB_MODE_DIRECT_FP64 = 1,     /* tiled O(n^2), FP64 arithmetic of CpuParallelBackend     */
    NB_MODE_BARNES_HUT = 2,      /* warp-group tree walk, monopole+quadrupole, FP32 pairs   */
    NB_MODE_BARNES_HUT_REF = 3   /* per-body walk with the reference's MAC and monopole     */
};
#define NB_MODE_MASK 0xF
#define NB_FLAG_SHELL_THEOREM 0x10  /* IGravityModelAwareBackend.EnableShellTheorem          */
#define NB_FLAG_NO_QUADRUPOLE 0x20  /* monopole only in NB_MODE_BARNES_HUT                   */
#define NB_FLAG_COLLISIONS 0x40     /* nb_step: broad phase + merge + compaction per step    */
#define NB_FLAG_LEARNED_MAC 0x80    /* NB_MODE_BARNES_HUT: MLP opening criterion              */
/* nb_step: each step is Yoshida's 4th-order composition of three KDK
 * sub-steps of w1 dt, w0 dt, w1 dt, w1 = 1 / (2 - 2^(1/3)), w0 = -2^(1/3) w1
 * (IntegratorType::Yoshida4: engine/include/celestial/sim/yoshida.hpp:8-27,
 * Engine::cpu_yoshida_substep, engine/src/sim/engine.cpp:685-746), three
 * force evaluations per step. */
#define NB_FLAG_YOSHIDA4 0x100
/* nb_step: adaptive time step (AdaptiveTimestep::compute_dt, engine/src/sim/
 * adaptive_timestep.cpp:12-17, applied after every step as Engine::step does,
 * engine/src/sim/engine.cpp:268-272): after each step dt becomes
 * clamp(eta sqrt(softening / a_max), dt_min, dt_max), a_max the largest |a|
 * over active bodies (dt_max when a_max or softening is 0).  The first step
 * after nb_set_state or a NB_PARAM_ADAPTIVE_* change uses nb_step's dt; the
 * current dt is read with nb_get_adaptive_dt.  Steps run one by one (no
 * captured graph: dt changes every step). */
#define NB_FLAG_ADAPTIVE_DT 0x200
/* NB_MODE_DIRECT_FP64 only: the rounding and summation order of another of
 * the desktop app's CPU backends instead of CpuParallelBackend's, so that a
 * user of that backend gets its bits.
 *   NB_FLAG_ORDER_SIMD: SimdSingleThreadBackend (SimdSingleThreadBackend.cs:
 *     43-165), which is also the native engine's CPU brute force
 *     (Engine::compute_cpu_brute_forces, engine/src/sim/engine.cpp:649-674):
 *     coefficient m * ((inv * inv) * inv), sources summed in row order.
 *   NB_FLAG_ORDER_PAIRWISE: CpuSingleThreadBackend's Newton's-third-law loop
 *     (CpuSingleThreadBackend.cs:50-159): the same coefficient; a body's
 *     acceleration is its running sum over lower rows plus its running sum
 *     over higher rows.
 * With NB_FLAG_SHELL_THEOREM those backends run CpuParallelBackend's
 * arithmetic, and so do these flags. */
#define NB_FLAG_ORDER_SIMD 0x400
#define NB_FLAG_ORDER_PAIRWISE 0x800

/* Parameter ids for nb_set_param_f64 / nb_set_param_i32. */
enum nb_param {
    NB_PARAM_THETA = 1,            /* f64, opening angle, default 0.5                         */
    NB_PARAM_LEAF_CAPACITY = 2,    /* i32, bodies per leaf bucket of the walk tree, 1..64,
                                      default 24                                              */
    NB_PARAM_MAX_MERGES_FRAME = 3, /* i32, default 64 (simulation_config.hpp:57)               */
    NB_PARAM_MAX_MERGES_BODY = 4,  /* i32, default 2  (simulation_config.hpp:58)               */
    NB_PARAM_MIN_RADIUS = 5,       /* f64, density-model floor for merged radii, default 1e-6
                                      (engine/include/celestial/physics/density_model.hpp:12) */
    NB_PARAM_DENSITY_MERGE = 6,    /* i32, 1 = density-preserving merge radius (default 1)     */
    NB_PARAM_TIMING = 7,           /* i32, 1 = record per-stage CUDA events (default 1)        */
    NB_PARAM_MAC_BUDGET = 8,       /* f64, learned MAC: max predicted log10 rel. error         */
    NB_PARAM_GROUP_BODIES = 9,     /* i32, bodies per walk group with span groups: 64 (default;
                                      each warp lane holds two bodies) or 32; the shell-theorem,
                                      potential and small-block walks use 32                  */
    NB_PARAM_GROUP_PACK = 10,      /* f64, pack sibling cells into one walk group while the
                                      packed box is at most this many times the larger part's
                                      box; 0 = no packing (default 2.25)                       */
    NB_PARAM_MAC_THETA_LO = 11,    /* f64, learned MAC: cells with 2h/d below this are accepted
                                      geometrically (default 0.35)                            */
    NB_PARAM_MAC_THETA_HI = 12,    /* f64, learned MAC: cells with 2h/d at or above this are
                                      opened; in between the network decides (default 1.0)   */
    NB_PARAM_MAC_SCREEN_QUANTILE = 13, /* f64, learned MAC: quantile of |network - screen| over
                                      the training set that sets the linear screen's margin;
                                      0 = no screen (default 0.8, used by the next fit)       */
    NB_PARAM_ENS_DIRECT_SHAPE = 14, /* i32, ensembles: direct-sum tile shape 0..8 (threads x
                                      targets/thread: 64x1 64x2 64x4 128x1 128x2 128x4 256x1
                                      256x2 256x4; default 4), normally set by nb_ens_autotune */
    NB_PARAM_MAC_AUDIT_INTERVAL = 15, /* i32, learned MAC in nb_step: every this many steps the
                                      accelerations are audited against the FP64 direct sum on
                                      sampled bodies; 0 = never (default).  Setting it also
                                      clears a fallback                                        */
    NB_PARAM_MAC_AUDIT_SAMPLES = 16, /* i32, bodies per audit (default 1024)                   */
    NB_PARAM_MAC_AUDIT_RMS = 17,   /* f64, an audit whose rms relative error exceeds this
                                      switches the handle to the geometric MAC at
                                      NB_PARAM_THETA (default 1e-3)                           */
    /* NB_FLAG_ADAPTIVE_DT (AdaptiveTimestepConfig, engine/include/celestial/sim/
     * simulation_config.hpp:73-79); setting one restarts from nb_step's dt */
    NB_PARAM_ADAPTIVE_ETA = 18,    /* f64, safety factor eta (default 0.01)                  */
    NB_PARAM_ADAPTIVE_DT_MIN = 19, /* f64, floor (default 1e-8)                               */
    NB_PARAM_ADAPTIVE_DT_MAX = 20, /* f64, ceiling (default 0.01)                             */
    NB_PARAM_ENS_WALK_SHAPE = 22,  /* i32, ensembles: tree-branch walk block shape, 0 = 8 warps
                                      x 3 blocks per SM, 1 = 4 warps x 6 (default 0), normally
                                      set by nb_ens_autotune_tree                            */
    NB_PARAM_GROUP_SPAN = 21       /* i32, 0 or 32..1024: walk groups are runs of 32
                                      consecutive sorted bodies cut from the walk-tree cells
                                      holding at most this many bodies whose parent holds
                                      more (full warps; a group's box stays inside a cell of
                                      at most this many bodies; default 1024); 0: octree
                                      cells of <= 32 bodies with NB_PARAM_GROUP_PACK sibling
                                      packing                                                */
};

/* Indices into nb_get_timings() output (milliseconds, CUDA events).
 * Mirrors BarnesHutBackend.LastBuildTimeMs/LastTraversalTimeMs/LastTotalTimeMs
 * (src/CelestialMechanics.Physics/Solvers/BarnesHutBackend.cs:101-107). */
enum nb_timing {
    NB_T_BUILD = 0,     /* bbox + keys + sort + tree + multipoles */
    NB_T_TRAVERSAL = 1, /* walk or direct sum                     */
    NB_T_TOTAL = 2,     /* whole last force evaluation            */
    NB_T_SORT = 3,      /* keys + radix sort                      */
    NB_T_TREE = 4,      /* radix tree + octree + multipoles       */
    NB_T_COLLIDE = 5,   /* last collision stage: broad phase, merges,
                           compaction (NB_FLAG_COLLISIONS)        */
    NB_T_COUNT = 6
};

/* Indices into nb_get_counters() output. */
enum nb_counter {
    NB_C_CELL_INTERACTIONS = 0,     /* body-cell (multipole) interactions, last evaluation */
    NB_C_BODY_INTERACTIONS = 1,     /* body-body interactions, last evaluation              */
    NB_C_NODES = 2,                 /* walk-tree nodes                                      */
    NB_C_ACTIVE = 3,                /* active bodies in the last evaluation                 */
    NB_C_PAIRS = 4,                 /* collision pairs found, last step                     */
    NB_C_MERGES = 5,                /* merges performed, last step                          */
    NB_C_OVERFLOWS = 6,             /* walk frontier overflows (non-zero means an error)    */
    NB_C_GROUPS = 7,                /* walk groups (warps' body sets), last evaluation       */
    NB_C_MAX_GROUP_WORK = 8,        /* longest interaction list of one group (load balance)  */
    NB_C_MAC_EVALS = 9,             /* learned MAC: (group, cell) rows the network evaluated */
    NB_C_MAC_AUDITS = 10,           /* learned MAC: audits run since the interval was set    */
    NB_C_MAC_FALLBACK = 11,         /* learned MAC: 1 once an audit switched to geometric    */
    NB_C_COUNT = 12
};

/* ---- lifetime -------------------------------------------------------- */

/* Create a handle on CUDA device `device` able to hold `capacity` bodies.
 * Replaces construction of a backend in NBodySolver.SelectBackend
 * (src/CelestialMechanics.Physics/Solvers/NBodySolver.cs:451-484). */
NB_API int32_t nb_create(int32_t capacity, int32_t device, nb_engine** out);
NB_API int32_t nb_destroy(nb_engine* h);
/* Message of the last failed call on this handle (static storage per handle).
 * Precedent: celestial_get_last_error_message (native_api.h:292-294). */
NB_API const char* nb_last_error(const nb_engine* h);
NB_API int32_t nb_set_param_f64(nb_engine* h, int32_t param, double value);
NB_API int32_t nb_set_param_i32(nb_engine* h, int32_t param, int32_t value);
NB_API int32_t nb_get_timings(const nb_engine* h, double* out, int32_t n);
NB_API int32_t nb_get_counters(const nb_engine* h, int64_t* out, int32_t n);
/* The time step the next NB_FLAG_ADAPTIVE_DT step will take (0 before the
 * first adaptive step; AdaptiveTimestep::current_dt,
 * engine/include/celestial/sim/adaptive_timestep.hpp:26). */
NB_API int32_t nb_get_adaptive_dt(const nb_engine* h, double* dt);
/* Largest |a| over the active bodies of the device state
 * (Engine::compute_max_acceleration, engine/src/sim/engine.cpp:468-501). */
NB_API int32_t nb_max_acceleration(nb_engine* h, double* a_max);
/* Rows of the device state and how many are active (ParticleSystem::count
 * and the active count, engine/src/interop/native_api.cpp:217-220,393-396). */
NB_API int32_t nb_get_body_count(const nb_engine* h, int32_t* n, int32_t* n_active);
/* cudaStream_t of the handle, for callers that time with CUDA events. */
NB_API void* nb_stream(nb_engine* h);
NB_API const char* nb_version(void);

/* ---- the seam --------------------------------------------------------- */

/* IPhysicsComputeBackend.ComputeForces(BodySoA, softening)
 * (IPhysicsComputeBackend.cs:33; arithmetic of CpuParallelBackend.cs:99-142
 * and GravityKernel.cs:9-33).  Writes acc for all i in [0,n): active i get
 * the sum over active j != i, inactive i get 0.  radius may be NULL unless
 * NB_FLAG_SHELL_THEOREM is set. */
NB_API int32_t nb_compute_forces(nb_engine* h, int32_t n,
                                 const double* px, const double* py, const double* pz,
                                 const double* mass, const double* radius,
                                 const uint8_t* active, double softening, int32_t flags,
                                 double* ax, double* ay, double* az);

/* ---- device-resident state (ISoAIntegrator path) ---------------------- */

/* Upload a BodySoA (BodySoA.cs:39-175).  old_ax/ay/az, radius, density and
 * collidable may be NULL (zeros / 0 / 0 / all collidable). */
NB_API int32_t nb_set_state(nb_engine* h, int32_t n,
                            const double* px, const double* py, const double* pz,
                            const double* vx, const double* vy, const double* vz,
                            const double* mass, const double* radius, const double* density,
                            const uint8_t* active, const uint8_t* collidable,
                            const double* old_ax, const double* old_ay, const double* old_az);
/* Download state; any pointer may be NULL.  `ids` receives each row's
 * original body index (rows move when compaction removes merged bodies). */
NB_API int32_t nb_get_state(nb_engine* h, int32_t* n_out,
                            double* px, double* py, double* pz,
                            double* vx, double* vy, double* vz,
                            double* ax, double* ay, double* az,
                            double* mass, double* radius, uint8_t* active, int32_t* ids);
/* n_steps of SoAVerletIntegrator.Step (SoAVerletIntegrator.cs:48-116) on
 * device-resident state: half kick, drift, forces, half kick.  With
 * NB_FLAG_COLLISIONS each step then runs broad phase, merge
 * (collision_resolver.cpp:20-100 semantics) and order-preserving compaction
 * (compact_kernel.cu:39 mask).  A call of several collisional Barnes-Hut
 * steps (geometric MAC) keeps every count on the device between its steps:
 * the result is the same as one call per step, and NB_C_PAIRS / NB_C_MERGES
 * then hold the last step's counts. */
NB_API int32_t nb_step(nb_engine* h, int32_t n_steps, double dt, double softening,
                       int32_t flags);
/* Energy/momentum diagnostics of the device state, FP64
 * (EnergyCalculator.cs:16-78, NewtonianGravity.cs:68-77, energy_tracker.cpp:194-240).
 * out[0..12]: KE, PE, E, Px, Py, Pz, Lx, Ly, Lz, COMx, COMy, COMz, M.
 * PE is the exact pairwise sum when pe_mode == 0, the tree potential
 * 1/2 sum m_i phi_i when pe_mode == 1. */
NB_API int32_t nb_diagnostics(nb_engine* h, double softening, int32_t pe_mode, double* out13);
/* ForceErrorAnalyzer.CompareForces metric (ForceErrorAnalyzer.cs:67-134)
 * of the device acc against an FP64 direct sum over all active sources,
 * for `n_samples` bodies drawn uniformly with `seed` (all bodies if
 * n_samples <= 0 or >= n).  out3: mean, max, rms relative error. */
NB_API int32_t nb_force_error(nb_engine* h, int32_t n_samples, uint64_t seed,
                              double softening, int32_t flags, double* out3);

/* ---- single stages on host arrays (integer-stage parity) -------------- */

/* Morton keys.  mode 0: per-axis AABB normalisation and the (2^21-1)
 * scale of morton_code_kernel (morton_kernel.cu:11-45, morton.hpp:13-35);
 * idx[i] = i, inactive keys = ~0.  mode 1: octree-aligned keys in the cube
 * (cx,cy,cz,half) = cube4, or the bounding cube of the active bodies
 * (gpu_tree.cu:163-167) when cube4 == NULL; cube4_out (may be NULL)
 * receives the cube used. */
NB_API int32_t nb_morton_keys(nb_engine* h, int32_t n,
                              const double* px, const double* py, const double* pz,
                              const uint8_t* active, int32_t mode, const double* cube4,
                              uint64_t* keys, int32_t* idx, double* cube4_out);
/* Stable sort of (key, value) pairs by key, in place; replaces
 * launch_radix_sort (morton_kernel.cu:185-230) with a stable sort. */
NB_API int32_t nb_sort_pairs(nb_engine* h, int32_t n, uint64_t* keys, int32_t* values);
/* Stable sort of (key, value) pairs that live in DEVICE memory, in place,
 * without allocating any device memory.  No counterpart in the reference:
 * it serves callers that cannot call cudaMalloc - hosts whose device memory
 * is all owned by their own pool allocator, and latency-critical paths where
 * cudaMalloc's device-wide synchronisation is not acceptable.  The scratch is
 * a fixed 21.0 MB __device__ array inside the library, held by every GPU
 * that loads it until the process exits; n above NB_NOALLOC_SORT_MAX is
 * rejected with NB_ERR_CAPACITY.  The first call on a device looks up that
 * array's address (make it before any stream capture).  All calls share the
 * one array: calls that overlap on the GPU (other streams, other threads)
 * race and must be serialised by the caller.  `stream` is a cudaStream_t
 * (NULL: the legacy default stream); the call returns when the sort is done. */
#define NB_NOALLOC_SORT_MAX 1048576
NB_API int32_t nb_sort_pairs_noalloc(uint64_t* keys, int32_t* values, int32_t n, void* stream);
/* Build the octree of the active bodies in cube4 (NULL: bounding cube) and
 * export it, replacing tree_build_kernel (gpu_tree.cu:269-464) and
 * OctreeBuilder::build (octree_builder.cpp:8-135).  Nodes are in walk order
 * (children contiguous).  Per node: level, first_child (-1 for leaves),
 * n_children, body_first, body_count (in sorted order), mass, com[3],
 * quad[6] (Qxx,Qyy,Qzz,Qxy,Qxz,Qyz).  sorted_idx receives the body index
 * of each sorted position.  Any output pointer may be NULL.  *n_nodes is
 * set to the node count; when it exceeds max_nodes nothing else is written
 * and NB_ERR_CAPACITY is returned. */
NB_API int32_t nb_build_octree(nb_engine* h, int32_t n,
                               const double* px, const double* py, const double* pz,
                               const double* mass, const uint8_t* active,
                               const double* cube4, int32_t leaf_capacity, int32_t max_nodes,
                               int32_t* n_nodes, int32_t* level, int32_t* first_child,
                               int32_t* n_children, int32_t* body_first, int32_t* body_count,
                               double* node_mass, double* com3, float* quad6,
                               int32_t* sorted_idx, uint64_t* sorted_keys);
/* Order-preserving compaction indices: dest[i] = destination row of body i
 * or -1 when it is removed (mask is_active && mass > 0, compact_kernel.cu:39);
 * *n_kept = survivors. */
NB_API int32_t nb_compact_indices(nb_engine* h, int32_t n, const uint8_t* active,
                                  const double* mass, int32_t* dest, int32_t* n_kept);
/* Collision broad phase: all pairs of active, collidable bodies with
 * |xi-xj|^2 < (ri+rj)^2, as (lo, hi) sorted lexicographically
 * (collision_kernel.cu:16-64 test, CollisionResolver::sort_pairs order).
 * *n_pairs is the true count even when it exceeds max_pairs (then only
 * max_pairs are written and NB_ERR_CAPACITY is returned). */
NB_API int32_t nb_broad_phase(nb_engine* h, int32_t n,
                              const double* px, const double* py, const double* pz,
                              const double* radius, const uint8_t* active,
                              const uint8_t* collidable, int32_t max_pairs,
                              int32_t* pair_lo, int32_t* pair_hi, int32_t* n_pairs);

/* ---- learned multipole acceptance criterion --------------------------- */
/* No reference counterpart: these replace the geometric opening test
 * (engine/src/cuda/gpu_tree.cu:567-569, BarnesHutBackend.cs:431-447) inside
 * the band theta_lo <= 2h/d < theta_hi by an MLP 8-64-64-1 (BF16 tensor-core
 * tiles, FP32 accumulate) that predicts log2 of the cell's monopole +
 * quadrupole force error relative to the group's smallest |a|; the cell is
 * accepted when the prediction is below NB_PARAM_MAC_BUDGET (log10).  Enable
 * with NB_FLAG_LEARNED_MAC in nb_step / nb_compute_forces. */
#define NB_MAC_PARAMS 4801  /* W1 8x64, b1 64, W2 64x64, b2 64, w3 64, b3 1 */
#define NB_MAC_NORM 18      /* feature means[8], feature stds[8], target mean, target std */

/* Harvest training samples from the device state: one Barnes-Hut force
 * evaluation with the geometric test at theta_lo (it updates the state's
 * accelerations) that records, for a `sample_frac` share of the walk groups,
 * every candidate cell in the band with its exact FP64 error target.  Up to
 * max_records records per call; samples are appended to the handle's
 * training set (16,777,216 rows).  Needs an acceleration estimate from a
 * previous force evaluation. */
NB_API int32_t nb_mac_harvest(nb_engine* h, int32_t max_records, double sample_frac,
                              uint64_t seed, double softening, int32_t* n_added);
/* Size of the training set, and a copy (X: n x 8 features, Y: n targets;
 * either may be NULL). */
NB_API int32_t nb_mac_dataset(nb_engine* h, int32_t* n, float* X, float* Y);
NB_API int32_t nb_mac_clear(nb_engine* h);
/* Train on the handle's set with Adam (MSE on normalised log2 errors); the
 * first call fixes the normalisation and initialises the weights from seed.
 * loss_per_epoch (may be NULL) receives the mean normalised loss per epoch. */
NB_API int32_t nb_mac_train(nb_engine* h, int32_t epochs, int32_t batch, double lr, uint64_t seed,
                            double* loss_per_epoch);
/* Parameters: NB_MAC_PARAMS weights followed by NB_MAC_NORM normalisation. */
NB_API int32_t nb_mac_set_params(nb_engine* h, const float* params, int32_t n);
NB_API int32_t nb_mac_get_params(nb_engine* h, float* params, int32_t n);
/* Gradient (NB_MAC_PARAMS floats) of the mean squared error over the given
 * rows with the current parameters, computed by the training kernel.  The
 * kernel sums its partials in a fixed order, so gradients and trainings are
 * bitwise reproducible on one device. */
NB_API int32_t nb_mac_gradient(nb_engine* h, const float* X, const float* Y, int32_t n,
                               float* grad, double* loss);
/* Predictions (log2 error units) of the walk's inference routine. */
NB_API int32_t nb_mac_predict(nb_engine* h, const float* X, int32_t n, float* y);

/* The last audit of the learned MAC inside nb_step (NB_PARAM_MAC_AUDIT_*):
 * its rms and max relative force error against the FP64 direct sum, the
 * audits run and whether the handle has fallen back to the geometric MAC. */
NB_API int32_t nb_mac_audit_state(nb_engine* h, double* rms, double* max_err, int64_t* audits,
                                  int32_t* fallback);

/* Linear screen in front of the network: in the band the walk first forms
 * s = w . x_norm + b (x_norm: features normalised as the network's input,
 * s in normalised target units); s < budget - margin accepts, s > budget +
 * margin opens, and only in between the network is evaluated.  Cells of one
 * body are accepted without either (their monopole is exact).
 * nb_mac_fit_screen fits w, b by least squares to the network's own
 * predictions on the multi-body rows of the training set and sets margin to
 * the NB_PARAM_MAC_SCREEN_QUANTILE quantile of the residuals; nb_mac_train
 * calls it at the end, nb_mac_set_params switches the screen off (margin =
 * +inf) until a fit or nb_mac_set_screen. */
#define NB_MAC_SCREEN 10  /* w[8], b, margin */
NB_API int32_t nb_mac_fit_screen(nb_engine* h);
NB_API int32_t nb_mac_get_screen(nb_engine* h, float* screen, int32_t n);
NB_API int32_t nb_mac_set_screen(nb_engine* h, const float* screen, int32_t n);

/* ---- batched ensembles of independent systems -------------------------- */
/* No reference counterpart (the reference steps one system per
 * NBodySolver.Step, src/CelestialMechanics.Physics/Solvers/NBodySolver.cs:
 * 290-391).  An ensemble holds many independent systems of uneven size, each
 * with G = 1 gravity among its own bodies only.  Systems of at most ds_max_n
 * bodies are summed directly (FP32 pair forces on FP64-differenced
 * coordinates, compensated); larger ones use the Barnes-Hut group walk
 * (NB_PARAM_THETA, default 0.5, monopole + quadrupole) over one shared sort
 * and tree.  One velocity-Verlet step of all systems is one CUDA-graph launch.
 * Arrays are the systems' bodies concatenated in the order of `sizes`. */
typedef struct nb_ensemble nb_ensemble;

/* At most 4096 systems above ds_max_n. */
NB_API int32_t nb_ens_create(int32_t n_systems, const int32_t* sizes, int32_t ds_max_n,
                             int32_t device, nb_ensemble** out);
NB_API int32_t nb_ens_destroy(nb_ensemble* h);
NB_API const char* nb_ens_last_error(const nb_ensemble* h);
/* systems, direct systems, tree systems, bodies, direct bodies, tree bodies */
NB_API int32_t nb_ens_info(const nb_ensemble* h, int64_t* out, int32_t n);
/* NB_PARAM_THETA (f64); NB_PARAM_LEAF_CAPACITY, NB_PARAM_ENS_DIRECT_SHAPE,
 * NB_PARAM_ENS_WALK_SHAPE, NB_PARAM_GROUP_SPAN, NB_PARAM_GROUP_BODIES (i32) */
NB_API int32_t nb_ens_set_param_f64(nb_ensemble* h, int32_t param, double value);
NB_API int32_t nb_ens_set_param_i32(nb_ensemble* h, int32_t param, int32_t value);
/* Positions, velocities, masses; accelerations are unknown until the first
 * force evaluation (nb_ens_step does one first when needed). */
NB_API int32_t nb_ens_set_state(nb_ensemble* h, const double* px, const double* py,
                                const double* pz, const double* vx, const double* vy,
                                const double* vz, const double* mass);
/* Any pointer may be NULL. */
NB_API int32_t nb_ens_get_state(nb_ensemble* h, double* px, double* py, double* pz, double* vx,
                                double* vy, double* vz, double* ax, double* ay, double* az);
/* Accelerations at the current positions. */
NB_API int32_t nb_ens_compute_forces(nb_ensemble* h, double softening);
/* n_steps velocity-Verlet steps (SoAVerletIntegrator.cs:48-116 per system),
 * one graph launch each. */
NB_API int32_t nb_ens_step(nb_ensemble* h, int32_t n_steps, double dt, double softening);
/* Times every direct tile shape on the current state (3 runs each, CUDA
 * events) and keeps the fastest; ms_per_shape (9 entries, may be NULL) gets
 * the times, -1 for a shape that cannot run. */
NB_API int32_t nb_ens_autotune(nb_ensemble* h, double softening, int32_t* shape,
                               double* ms_per_shape);
/* Times the tree branch (keys, sort, tree, walk of every tree system) on the
 * current state for each walk block shape (NB_PARAM_ENS_WALK_SHAPE 0, 1) and
 * walk-group span (NB_PARAM_GROUP_SPAN 0, 256, 512, 1024) with 32-body groups,
 * and for shape 0 with spans 256, 512, 1024 and 64-body groups
 * (NB_PARAM_GROUP_BODIES), 3 runs each with CUDA events, and keeps the
 * fastest: choice k < 8 is shape k / 4 with the k % 4-th span, choice 8 + j
 * is shape 0 with the (j + 1)-th span and 64-body groups.  Spans at or above
 * the smallest tree system's body count are skipped (time -1).
 * ms_per_choice (NB_ENS_TREE_CHOICES entries, may be NULL) gets the times.
 * The tree systems' accelerations are then those of the choice. */
#define NB_ENS_TREE_CHOICES 11
NB_API int32_t nb_ens_autotune_tree(nb_ensemble* h, double softening, int32_t* choice,
                                    double* ms_per_choice);
/* Per system (in `sizes` order): rms and max relative error of the current
 * accelerations against an FP64 direct sum on up to `samples` bodies. */
NB_API int32_t nb_ens_force_error(nb_ensemble* h, int32_t samples, uint64_t seed,
                                  double softening, double* rms, double* max_err);
/* Per system: total, kinetic and softened potential energy (FP64). */
NB_API int32_t nb_ens_energy(nb_ensemble* h, double softening, double* energy, double* kinetic,
                             double* potential);
/* direct pairs per evaluation, tree body-cell and body-body interactions of
 * the last evaluation, graph launches so far, direct work items, direct shape,
 * tree walk shape, walk-group span */
NB_API int32_t nb_ens_get_counters(const nb_ensemble* h, int64_t* out, int32_t n);
/* Device time per step of the last nb_ens_step (or of the last evaluation). */
NB_API int32_t nb_ens_get_timings(const nb_ensemble* h, double* ms_per_step);

#ifdef __cplusplus
}
#endif

#endif /* NBODY_B200_H */
