// engine.cu - the C ABI (include/nbody_b200.h): handle, device buffers and
// the force / step pipelines.
//
// The handle replaces the reference's global Engine* behind its C ABI
// (engine/src/interop/native_api.cpp:9,30-124) and the GpuPool buffers
// (engine/src/memory/gpu_pool.cu:79-124): one CUDA stream and fixed-capacity
// device arrays per handle, allocated once in nb_create, so no call allocates
// device memory on the hot path.  Every entry point returns a status; no C++
// exception leaves this file; there is no CPU fallback.
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "bodies.cuh"
#include "collide.cuh"
#include "diag.cuh"
#include "direct.cuh"
#include "sort.cuh"
#include "tree.cuh"
#include "walk.cuh"
#include "mac_train.cuh"

#include <algorithm>
#include <cmath>
#include <random>

namespace {

// Device scalars of a handle (one allocation).
struct Scal {
    unsigned long long bbox_ord[6];
    int n_active;
    unsigned group_ctr;
    int n_groups;
    double cube[4];
    double cube_in[4];
    int err[nb::kErrCount];
    unsigned long long counters[4];
    double diag[16];
    int n_pairs;
    int n_kept;
    int n_merges;
    int n_rows;  // current row count of a captured collisional step
    unsigned long long amax2;  // bits of the largest |a|^2 (adaptive dt)
};

}  // namespace

struct nb_engine {
    int device = 0;
    int sms = 148;
    int capacity = 0;
    cudaStream_t st = nullptr;
    char err_msg[512] = {0};
    // parameters
    double theta = 0.5;
    int leaf_cap = 24;  // walk-tree leaf bucket (bodies): 24 measured fastest of 4..32
    int max_merges_frame = 64;
    int max_merges_body = 2;
    double min_radius = 1e-6;
    int density_merge = 1;
    int timing = 1;
    double mac_budget = -3.0;
    // bodies per walk group: 64 (two per lane) measured 5 % faster on the
    // learned and 3 % on the geometric walk at equal error at N = 2^20
    // (span groups only; sibling-packed groups stay at 32)
    int group_bodies = 64;
    double group_pack = 2.25;
    // walk groups: runs of group_bodies bodies cut from cells of <= group_span bodies; 1024
    // measured fastest of 0 (sibling packing), 64 .. 1024 at N = 2^20 (learned /
    // geometric / theta 0.5 steps/s: 303 / 255 / 142 with packing, 329 / 297 / 157)
    int group_span = 1024;
    // adaptive time step (AdaptiveTimestepConfig defaults)
    double adapt_eta = 0.01, adapt_dt_min = 1e-8, adapt_dt_max = 0.01;
    double adapt_dt = 0.0;  // the next adaptive step's dt; 0 = take nb_step's dt
    // learned MAC
    double mac_theta_lo = 0.35, mac_theta_hi = 1.0;
    // residual quantile that sets the screen margin: at N = 2^20 and equal
    // rms, 0.8 measured 1 % faster than 0.9 and 4 % faster than 0.97 (fewer
    // rows reach the network)
    double mac_screen_q = 0.8;
    // sampled FP64 audit of the learned MAC inside nb_step, geometric fallback
    int mac_audit_every = 0, mac_audit_samples = 1024, mac_since_audit = 0;
    double mac_audit_rms_max = 1e-3, mac_audit_last_rms = 0.0, mac_audit_last_max = 0.0;
    int64_t mac_audits = 0;
    bool mac_fallback = false;
    float mac_screen[nb::kMacScreen] = {0, 0, 0, 0, 0, 0, 0, 0, 0, INFINITY};
    bool mac_ready = false;               // parameters trained or set
    float mac_norm_host[nb::kMacNorm] = {0};
    nb::MacDev* mac_dev = nullptr;        // BF16 fragment image for the walk
    float2* mac_node = nullptr;           // per-node screen terms (learned walk)
    float *mac_P = nullptr, *mac_m = nullptr, *mac_v = nullptr, *mac_G = nullptr;
    float *mac_norm = nullptr, *mac_loss = nullptr;
    float* mac_part = nullptr;            // per-block gradient partials (training)
    int mac_adam_step = 0;
    float* samag = nullptr;               // sorted |a| of the previous step
    // training set (allocated by the first harvest)
    float *mac_X = nullptr, *mac_Y = nullptr;
    int mac_n = 0, mac_cap = 0;
    nb::MacRecord* mac_rec = nullptr;
    nb::MacRecord* mac_rec2 = nullptr;    // records in a fixed order
    uint64_t *mac_rk0 = nullptr, *mac_rk1 = nullptr;
    uint32_t *mac_rv0 = nullptr, *mac_rv1 = nullptr;
    void* mac_rws = nullptr;
    int mac_rec_cap = 0;
    int* mac_counts = nullptr;            // [0] records, [1] accepted samples
    // device-resident state
    int n = 0;
    int n_active = 0;
    bool has_state = false;
    nb::State s{};
    nb::State s_alt{};  // compaction target
    // work buffers
    uint64_t *keys0 = nullptr, *keys1 = nullptr;
    uint32_t *vals0 = nullptr, *vals1 = nullptr;
    void* sort_ws = nullptr;
    double4* sbody = nullptr;
    double4* rows4 = nullptr;             // (x, y, z, m) by row, for the gather
    float* amag_rows = nullptr;           // |a| of the previous step by row
    float* srad = nullptr;
    void* tree_mem = nullptr;
    nb::TreeBufs tree{};
    nb::WalkConfig wcfg{};
    int* front = nullptr;
    double* rows = nullptr;
    double* part = nullptr;
    double* phi = nullptr;
    int32_t* targets = nullptr;
    int2* groups = nullptr;
    double* tgt_out = nullptr;
    double* tgt_part = nullptr;           // FP64 force-error chunk partials
    double* aud_part = nullptr;           // audit chunk partials
    nb::CollideBufs col{};
    Scal* scal = nullptr;
    std::vector<void*> allocs;
    // timing
    cudaEvent_t ev[6] = {};
    // captured single step (CUDA graph) and the parameters it was captured with
    cudaGraphExec_t graph_exec = nullptr;
    struct GraphKey {
        int flags, n, n_active, leaf_cap, span, bodies;
        double dt, eps, theta, pack, mac_lo, mac_hi, mac_budget;
        const double* state;  // the state arrays swap after a compaction
        bool operator==(const GraphKey& o) const {
            return flags == o.flags && n == o.n && n_active == o.n_active &&
                   leaf_cap == o.leaf_cap && span == o.span && bodies == o.bodies && dt == o.dt &&
                   eps == o.eps && theta == o.theta &&
                   pack == o.pack && mac_lo == o.mac_lo && mac_hi == o.mac_hi &&
                   mac_budget == o.mac_budget && state == o.state;
        }
    } graph_key{};
    // the collisional step captured twice, from each state buffer into the
    // other (compaction alternates them): cstate[k] is graph k's source
    // buffer; n and n_active in ckey are the launch bounds of the capture
    cudaGraphExec_t cgraph[2] = {nullptr, nullptr};
    GraphKey ckey{};
    const double* cstate[2] = {nullptr, nullptr};
    struct MergeKey {
        int max_frame, max_body, density;
        double min_radius;
        bool operator==(const MergeKey& o) const {
            return max_frame == o.max_frame && max_body == o.max_body && density == o.density &&
                   min_radius == o.min_radius;
        }
    } cmerge{};
    bool ev_valid = false;
    bool ev_tree = false;
    bool ev_collide = false;   // ev[4], ev[5] bracket the last collision stage
    bool tree_current = false; // the last force evaluation left a tree (with radii) of the
                               // current positions: keys0/vals0, sbody/srad, tree, cube
    double timings[NB_T_COUNT] = {0};
    int64_t counters[NB_C_COUNT] = {0};
};

namespace {

int fail(nb_engine* h, int code, const char* fmt, ...) {
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err_msg, sizeof(h->err_msg), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define NB_CUDA(h, call)                                                                \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail((h), NB_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int dalloc(nb_engine* h, T** p, size_t count) {
    size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
        return fail(h, NB_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    h->allocs.push_back(q);
    *p = (T*)q;
    return NB_OK;
}

int alloc_state(nb_engine* h, nb::State& s, int cap) {
    int r = NB_OK;
    double** d[] = {&s.px, &s.py, &s.pz, &s.vx, &s.vy, &s.vz, &s.ax, &s.ay, &s.az,
                    &s.mass, &s.radius, &s.density};
    for (double** p : d)
        if ((r = dalloc(h, p, cap))) return r;
    if ((r = dalloc(h, &s.active, cap))) return r;
    if ((r = dalloc(h, &s.collidable, cap))) return r;
    return dalloc(h, &s.ids, cap);
}

// Collect the device error word and the last CUDA error after a sync.
int check_device(nb_engine* h) {
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) return fail(h, NB_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, NB_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    int err[nb::kErrCount];
    e = cudaMemcpy(err, h->scal->err, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(h, NB_ERR_CUDA, "error word: %s", cudaGetErrorString(e));
    cudaMemsetAsync(h->scal->err, 0, sizeof(err), h->st);
    if (err[nb::kErrNonFinite]) return fail(h, NB_ERR_NONFINITE, "non-finite position or mass");
    if (err[nb::kErrTimeout]) return fail(h, NB_ERR_TIMEOUT, "a bounded device wait expired");
    if (err[nb::kErrOverflow])
        return fail(h, NB_ERR_STACK_OVERFLOW, "tree-walk frontier overflow");
    if (err[nb::kErrCapacity]) return fail(h, NB_ERR_CAPACITY, "device buffer capacity exceeded");
    return NB_OK;
}

int upload(nb_engine* h, void* dst, const void* src, size_t bytes) {
    if (!src || bytes == 0) return NB_OK;
    NB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->st));
    return NB_OK;
}

int download(nb_engine* h, void* dst, const void* src, size_t bytes) {
    if (!dst || bytes == 0) return NB_OK;
    NB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->st));
    return NB_OK;
}

int check_n(nb_engine* h, int n) {
    if (n < 0) return fail(h, NB_ERR_INVALID_ARG, "n = %d is negative", n);
    if (n > h->capacity)
        return fail(h, NB_ERR_CAPACITY, "n = %d exceeds the handle capacity %d", n, h->capacity);
    return NB_OK;
}

void record(nb_engine* h, int k) {
    if (h->timing) cudaEventRecord(h->ev[k], h->st);
}

// Forces for the current device rows.  kick: fuse the first half kick and
// the drift of a Verlet step into the bounding-box pass.  dn (Barnes-Hut
// modes only): the rows are counted on the device (a captured collisional
// step); h->n and h->n_active then only bound the launches, and the sorted
// stages take the active count the bounding-box pass writes.
int force_pipeline(nb_engine* h, int flags, double eps, bool kick, double dt,
                   const int* dn = nullptr) {
    const int mode = flags & NB_MODE_MASK;
    const bool shell = (flags & NB_FLAG_SHELL_THEOREM) != 0;
    // the collision broad phase reuses this evaluation's tree, which then
    // needs the radii (sorted, and each node's largest radius)
    const bool radii = shell || (flags & NB_FLAG_COLLISIONS) != 0;
    const int n = h->n;
    Scal* sc = h->scal;
    h->tree_current = false;
    record(h, 0);
    nb::launch_kick_drift_bbox(h->st, n, h->s, kick, dt, sc->bbox_ord, &sc->n_active, sc->err,
                               dn);
    cudaMemsetAsync(sc->counters, 0, sizeof(sc->counters), h->st);
    h->ev_tree = false;
    const int* dna = dn ? &sc->n_active : nullptr;
    if (dn && mode != NB_MODE_BARNES_HUT)
        return fail(h, NB_ERR_INVALID_ARG, "device row counts need NB_MODE_BARNES_HUT");
    if (mode == NB_MODE_DIRECT_FP64) {
        record(h, 1);
        record(h, 2);
        const int order = (flags & NB_FLAG_ORDER_PAIRWISE) ? nb::kOrderPairwise
                          : (flags & NB_FLAG_ORDER_SIMD)   ? nb::kOrderSimd
                                                           : nb::kOrderParallel;
        nb::direct_fp64(h->st, n, h->s.px, h->s.py, h->s.pz, h->s.mass, h->s.radius,
                        h->s.active, eps, shell, order, h->s.ax, h->s.ay, h->s.az);
        record(h, 3);
        h->counters[NB_C_BODY_INTERACTIONS] = (int64_t)h->n_active * (h->n_active - 1);
        h->counters[NB_C_CELL_INTERACTIONS] = 0;
        h->ev_valid = h->timing != 0;
        return NB_OK;
    }
    const int na = h->n_active;
    const bool learned = (flags & NB_FLAG_LEARNED_MAC) != 0;
    if (learned && (mode != NB_MODE_BARNES_HUT || shell || (flags & NB_FLAG_NO_QUADRUPOLE) ||
                    !(eps > 0.0)))
        return fail(h, NB_ERR_INVALID_ARG,
                    "the learned MAC needs NB_MODE_BARNES_HUT with quadrupoles, no shell "
                    "theorem and softening > 0");
    if (learned && !h->mac_ready)
        return fail(h, NB_ERR_STATE, "the learned MAC has no trained parameters");
    nb::launch_cube(h->st, sc->bbox_ord, nullptr, sc->cube);
    // the keys kernel also writes each row's (x, y, z, m) record and, for the
    // learned MAC, the previous step's |a| (before the buffer is zeroed)
    nb::launch_keys_cube(h->st, n, h->s, sc->cube, h->keys0, h->vals0, (uint32_t*)h->sort_ws,
                         h->rows4, learned ? h->amag_rows : nullptr, dn);
    nb::sort_pairs(h->st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, true, sc->err,
                   h->sms, dn);
    nb::launch_gather(h->st, na, h->s, h->vals0, h->sbody, radii ? h->srad : nullptr,
                      learned ? h->samag : nullptr, h->rows4, h->amag_rows, dna);
    nb::launch_zero_acc(h->st, n, h->s, dn);
    record(h, 1);
    if (mode == NB_MODE_DIRECT) {
        record(h, 2);
        // the walk tree's memory is idle in this mode and holds the chunk partials
        nb::direct_fp32(h->st, na, h->sbody, h->srad, h->vals0, eps, shell, h->s.ax, h->s.ay,
                        h->s.az, &sc->counters[1], h->tree_mem, nb::tree_bytes(h->capacity),
                        &sc->group_ctr, h->sms);
    } else if (mode == NB_MODE_BARNES_HUT || mode == NB_MODE_BARNES_HUT_REF) {
        const bool ref = mode == NB_MODE_BARNES_HUT_REF;
        nb::tree_build(h->st, h->tree, na, h->keys0, h->sbody, radii ? h->srad : nullptr, sc->cube,
                       ref ? 1 : h->leaf_cap, sc->err, nullptr, dna);
        h->ev_tree = true;
        h->tree_current = radii;
        record(h, 2);
        nb::WalkArgs a{};
        a.n = na;
        a.sbody = h->sbody;
        a.srad = h->srad;
        a.skeys = h->keys0;
        a.sidx = h->vals0;
        a.t = h->tree;
        a.eps2 = eps * eps;
        a.ax = h->s.ax;
        a.ay = h->s.ay;
        a.az = h->s.az;
        a.pot = nullptr;
        a.front = h->front;
        a.group_ctr = &sc->group_ctr;
        a.groups = h->groups;
        a.n_groups = &sc->n_groups;
        a.pack = h->group_pack;
        a.group_span = h->group_span;
        a.group_size = h->group_bodies;
        a.counters = sc->counters;
        a.err = sc->err;
        if (ref) {
            const double te = h->theta < 0.2 ? 0.2 : h->theta;  // barnes_hut_solver.cpp:16
            a.theta2 = te * te;
            nb::walk_reference(h->st, a, shell);
        } else if (learned) {
            // geometric below theta_lo, open from theta_hi, the network in between
            a.theta2 = h->mac_theta_lo * h->mac_theta_lo;
            a.mac_theta_hi2 = (float)(h->mac_theta_hi * h->mac_theta_hi);
            a.samag = h->samag;
            a.mac = h->mac_dev;
            nb::mac_node_terms(h->st, h->tree, na, h->mac_dev, h->mac_node);
            a.mac_node = h->mac_node;
            a.mac_budget = (float)((h->mac_budget * 3.321928094887362 - h->mac_norm_host[16]) /
                                   h->mac_norm_host[17]);
            nb::walk_group(h->st, h->wcfg, a, true, false, false, 2);
        } else {
            a.theta2 = h->theta * h->theta;
            nb::walk_group(h->st, h->wcfg, a, (flags & NB_FLAG_NO_QUADRUPOLE) == 0, shell, false);
        }
    } else {
        return fail(h, NB_ERR_INVALID_ARG, "unknown force mode %d", mode);
    }
    record(h, 3);
    h->ev_valid = h->timing != 0;
    return NB_OK;
}

// Yoshida 4th-order sub-step multipliers, computed as the reference computes
// them (YoshidaCoefficients, engine/include/celestial/sim/yoshida.hpp:19-24)
constexpr double kCbrt2 = 1.2599210498948732;
constexpr double kYoshidaW1 = 1.0 / (2.0 - kCbrt2);
constexpr double kYoshidaW0 = -kCbrt2 / (2.0 - kCbrt2);
constexpr double kYoshidaSub[3] = {kYoshidaW1, kYoshidaW0, kYoshidaW1};

// The sub-step time steps of one step: dt itself, or Yoshida's three.
int sub_steps(int flags, double dt, double* sub) {
    if (!(flags & NB_FLAG_YOSHIDA4)) {
        sub[0] = dt;
        return 1;
    }
    for (int s = 0; s < 3; s++) sub[s] = kYoshidaSub[s] * dt;
    return 3;
}

// Capture one device step (forces + second half kick) as a CUDA graph, or
// reuse the captured one when nothing it depends on changed.  Per-stage
// timing events are not recorded inside the graph.
int step_graph(nb_engine* h, int flags, double dt, double eps) {
    const nb_engine::GraphKey key{flags,           h->n,           h->n_active,
                                  h->leaf_cap,     h->group_span,  h->group_bodies,
                                  dt,              eps,
                                  h->theta,        h->group_pack,  h->mac_theta_lo,
                                  h->mac_theta_hi, h->mac_budget,  h->s.px};
    if (h->graph_exec && key == h->graph_key) return NB_OK;
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    NB_CUDA(h, cudaStreamSynchronize(h->st));
    const int timing = h->timing;
    h->timing = 0;
    cudaGraph_t g = nullptr;
    NB_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    double sub[3];
    const int ns = sub_steps(flags, dt, sub);
    int r = NB_OK;
    for (int k = 0; k < ns && r == NB_OK; k++) {
        r = force_pipeline(h, flags, eps, true, sub[k]);
        if (r == NB_OK) nb::launch_kick(h->st, h->n, h->s, sub[k]);
    }
    const cudaError_t e = cudaStreamEndCapture(h->st, &g);
    h->timing = timing;
    if (r != NB_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(h, NB_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&h->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        h->graph_exec = nullptr;
        return fail(h, NB_ERR_CUDA, "step graph: %s", cudaGetErrorString(ei));
    }
    h->graph_key = key;
    return NB_OK;
}

void collect_counters(nb_engine* h) {
    unsigned long long c[4];
    if (cudaMemcpy(c, h->scal->counters, sizeof(c), cudaMemcpyDeviceToHost) == cudaSuccess) {
        h->counters[NB_C_CELL_INTERACTIONS] = (int64_t)c[0];
        h->counters[NB_C_BODY_INTERACTIONS] = (int64_t)c[1];
        h->counters[NB_C_MAX_GROUP_WORK] = (int64_t)c[2];
        h->counters[NB_C_MAC_EVALS] = (int64_t)c[3];
    }
    int nn = 0;
    if (h->ev_tree && cudaMemcpy(&nn, h->tree.n_nodes, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess)
        h->counters[NB_C_NODES] = nn;
    int ng = 0;
    if (h->ev_tree && cudaMemcpy(&ng, &h->scal->n_groups, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess)
        h->counters[NB_C_GROUPS] = ng;
    h->counters[NB_C_ACTIVE] = h->n_active;
}

int count_active_host(const uint8_t* a, int n) {
    int c = 0;
    for (int i = 0; i < n; i++) c += a[i] != 0;
    return c;
}

// Upload positions / masses / radii / active into the device rows (the
// host-array entry points stage through the state arrays).
int stage_bodies(nb_engine* h, int n, const double* px, const double* py, const double* pz,
                 const double* mass, const double* radius, const uint8_t* active) {
    int r;
    if ((r = check_n(h, n))) return r;
    if (n > 0 && (!px || !py || !pz || !active))
        return fail(h, NB_ERR_INVALID_ARG, "null position or active array");
    const size_t d = sizeof(double) * (size_t)n;
    if ((r = upload(h, h->s.px, px, d)) || (r = upload(h, h->s.py, py, d)) ||
        (r = upload(h, h->s.pz, pz, d)) || (r = upload(h, h->s.active, active, (size_t)n)))
        return r;
    if (mass) {
        if ((r = upload(h, h->s.mass, mass, d))) return r;
    } else {
        NB_CUDA(h, cudaMemsetAsync(h->s.mass, 0, d, h->st));
    }
    if (radius) {
        if ((r = upload(h, h->s.radius, radius, d))) return r;
    } else {
        NB_CUDA(h, cudaMemsetAsync(h->s.radius, 0, d, h->st));
    }
    h->n = n;
    h->n_active = n > 0 ? count_active_host(active, n) : 0;
    h->has_state = false;
    return NB_OK;
}

}  // namespace

extern "C" {

NB_API const char* nb_version(void) { return "nbody_b200 1.0 (sm_100a)"; }

NB_API int32_t nb_create(int32_t capacity, int32_t device, nb_engine** out) {
    if (!out) return NB_ERR_INVALID_ARG;
    *out = nullptr;
    if (capacity <= 0) return NB_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return NB_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return NB_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return NB_ERR_NO_DEVICE;
    if (prop.major != 10) return NB_ERR_NO_DEVICE;  // built for sm_100a only
    nb_engine* h = new (std::nothrow) nb_engine();
    if (!h) return NB_ERR_CAPACITY;
    h->device = device;
    h->sms = prop.multiProcessorCount;
    h->capacity = capacity;
    int r = NB_OK;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return NB_ERR_CUDA;
    }
    nb::sort_init();
    nb::walk_init(h->sms, h->wcfg);
    const size_t cap = (size_t)capacity;
    do {
        if ((r = alloc_state(h, h->s, capacity))) break;
        if ((r = alloc_state(h, h->s_alt, capacity))) break;
        if ((r = dalloc(h, &h->keys0, cap)) || (r = dalloc(h, &h->keys1, cap))) break;
        if ((r = dalloc(h, &h->vals0, cap)) || (r = dalloc(h, &h->vals1, cap))) break;
        if ((r = dalloc(h, (char**)&h->sort_ws, nb::sort_workspace_bytes(capacity)))) break;
        if ((r = dalloc(h, &h->sbody, cap)) || (r = dalloc(h, &h->srad, cap))) break;
        if ((r = dalloc(h, &h->rows4, cap)) || (r = dalloc(h, &h->amag_rows, cap))) break;
        if ((r = dalloc(h, (char**)&h->tree_mem, nb::tree_bytes(capacity)))) break;
        nb::tree_carve(h->tree, h->tree_mem, capacity);
        if ((r = dalloc(h, (char**)&h->front, nb::walk_front_bytes(h->wcfg)))) break;
        if ((r = dalloc(h, &h->rows, cap)) || (r = dalloc(h, &h->phi, cap))) break;
        if ((r = dalloc(h, (char**)&h->part, nb::diag_partial_bytes(capacity)))) break;
        if ((r = dalloc(h, &h->targets, cap)) || (r = dalloc(h, &h->tgt_out, 3 * cap))) break;
        if ((r = dalloc(h, (char**)&h->tgt_part, nb::direct_targets_scratch_bytes(h->sms)))) break;
        if ((r = dalloc(h, (char**)&h->aud_part, nb::audit_targets_scratch_bytes(h->sms)))) break;
        if ((r = dalloc(h, &h->groups, cap))) break;
        if ((r = dalloc(h, &h->samag, cap))) break;
        if ((r = dalloc(h, &h->mac_node, 2 * cap))) break;
        if ((r = dalloc(h, &h->mac_dev, 1))) break;
        if ((r = dalloc(h, &h->mac_P, nb::kMacParams)) || (r = dalloc(h, &h->mac_m, nb::kMacParams)) ||
            (r = dalloc(h, &h->mac_v, nb::kMacParams)) || (r = dalloc(h, &h->mac_G, nb::kMacParams)))
            break;
        if ((r = dalloc(h, &h->mac_norm, nb::kMacNorm)) || (r = dalloc(h, &h->mac_loss, 4))) break;
        if ((r = dalloc(h, &h->mac_counts, 4))) break;
        if ((r = dalloc(h, (char**)&h->mac_part, nb::mac_grad_partial_bytes(h->sms)))) break;
        if ((r = nb::collide_alloc(h->col, capacity, [h](void** p, size_t b) {
                 return dalloc(h, (char**)p, b);
             })))
            break;
        if ((r = dalloc(h, &h->scal, 1))) break;
        if (cudaMemset(h->scal, 0, sizeof(Scal)) != cudaSuccess) { r = NB_ERR_CUDA; break; }
        for (auto& e : h->ev)
            if (cudaEventCreate(&e) != cudaSuccess) { r = NB_ERR_CUDA; break; }
    } while (0);
    if (r != NB_OK) {
        nb_destroy(h);
        return r;
    }
    *out = h;
    return NB_OK;
}

NB_API int32_t nb_destroy(nb_engine* h) {
    if (!h) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (void* p : h->allocs) cudaFree(p);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    for (auto& g : h->cgraph)
        if (g) cudaGraphExecDestroy(g);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return NB_OK;
}

NB_API const char* nb_last_error(const nb_engine* h) { return h ? h->err_msg : "null handle"; }

NB_API void* nb_stream(nb_engine* h) { return h ? (void*)h->st : nullptr; }

NB_API int32_t nb_set_param_f64(nb_engine* h, int32_t p, double v) {
    if (!h) return NB_ERR_INVALID_ARG;
    switch (p) {
        case NB_PARAM_THETA:
            if (!(v >= 0.0)) return fail(h, NB_ERR_INVALID_ARG, "theta must be >= 0");
            h->theta = v;
            return NB_OK;
        case NB_PARAM_MIN_RADIUS: h->min_radius = v; return NB_OK;
        case NB_PARAM_MAC_BUDGET: h->mac_budget = v; return NB_OK;
        case NB_PARAM_MAC_THETA_LO:
            if (!(v > 0.0 && v < 2.0)) return fail(h, NB_ERR_INVALID_ARG, "theta_lo must be in (0, 2)");
            h->mac_theta_lo = v;
            return NB_OK;
        case NB_PARAM_MAC_THETA_HI:
            if (!(v > 0.0 && v < 4.0)) return fail(h, NB_ERR_INVALID_ARG, "theta_hi must be in (0, 4)");
            h->mac_theta_hi = v;
            return NB_OK;
        case NB_PARAM_MAC_AUDIT_RMS:
            if (!(v > 0.0)) return fail(h, NB_ERR_INVALID_ARG, "audit rms bound must be > 0");
            h->mac_audit_rms_max = v;
            return NB_OK;
        case NB_PARAM_ADAPTIVE_ETA:
            if (!(v > 0.0)) return fail(h, NB_ERR_INVALID_ARG, "eta must be > 0");
            h->adapt_eta = v;
            h->adapt_dt = 0.0;
            return NB_OK;
        case NB_PARAM_ADAPTIVE_DT_MIN:
        case NB_PARAM_ADAPTIVE_DT_MAX: {
            const double lo = p == NB_PARAM_ADAPTIVE_DT_MIN ? v : h->adapt_dt_min;
            const double hi = p == NB_PARAM_ADAPTIVE_DT_MAX ? v : h->adapt_dt_max;
            if (!(lo > 0.0 && lo <= hi)) return fail(h, NB_ERR_INVALID_ARG, "need 0 < dt_min <= dt_max");
            h->adapt_dt_min = lo;
            h->adapt_dt_max = hi;
            h->adapt_dt = 0.0;
            return NB_OK;
        }
        case NB_PARAM_MAC_SCREEN_QUANTILE:
            if (!(v >= 0.0 && v <= 1.0)) return fail(h, NB_ERR_INVALID_ARG, "screen quantile must be in [0, 1]");
            h->mac_screen_q = v;
            return NB_OK;
        case NB_PARAM_GROUP_PACK:
            if (!(v >= 0.0 && v <= 64.0)) return fail(h, NB_ERR_INVALID_ARG, "group packing must be 0..64");
            h->group_pack = v;
            return NB_OK;
        default: return fail(h, NB_ERR_INVALID_ARG, "unknown f64 parameter %d", p);
    }
}

NB_API int32_t nb_set_param_i32(nb_engine* h, int32_t p, int32_t v) {
    if (!h) return NB_ERR_INVALID_ARG;
    switch (p) {
        case NB_PARAM_LEAF_CAPACITY:
            if (v < 1 || v > 64) return fail(h, NB_ERR_INVALID_ARG, "leaf capacity must be 1..64");
            h->leaf_cap = v;
            return NB_OK;
        case NB_PARAM_MAX_MERGES_FRAME: h->max_merges_frame = v; return NB_OK;
        case NB_PARAM_MAX_MERGES_BODY: h->max_merges_body = v; return NB_OK;
        case NB_PARAM_DENSITY_MERGE: h->density_merge = v; return NB_OK;
        case NB_PARAM_TIMING: h->timing = v; return NB_OK;
        case NB_PARAM_MAC_AUDIT_INTERVAL:
            if (v < 0) return fail(h, NB_ERR_INVALID_ARG, "audit interval must be >= 0");
            h->mac_audit_every = v;
            h->mac_since_audit = 0;
            h->mac_audits = 0;
            h->mac_fallback = false;
            return NB_OK;
        case NB_PARAM_MAC_AUDIT_SAMPLES:
            if (v < 1) return fail(h, NB_ERR_INVALID_ARG, "audit samples must be >= 1");
            h->mac_audit_samples = v;
            return NB_OK;
        case NB_PARAM_GROUP_SPAN:
            if (v != 0 && (v < 32 || v > 1024))
                return fail(h, NB_ERR_INVALID_ARG, "group span must be 0 or 32..1024");
            h->group_span = v;
            return NB_OK;
        case NB_PARAM_GROUP_BODIES:
            if (v != 32 && v != 64) return fail(h, NB_ERR_INVALID_ARG, "group size must be 32 or 64");
            h->group_bodies = v;
            return NB_OK;
        default: return fail(h, NB_ERR_INVALID_ARG, "unknown i32 parameter %d", p);
    }
}

NB_API int32_t nb_get_timings(const nb_engine* hc, double* out, int32_t n) {
    nb_engine* h = const_cast<nb_engine*>(hc);
    if (!h || !out) return NB_ERR_INVALID_ARG;
    if (h->ev_valid) {
        float t[3] = {0, 0, 0};
        cudaEventSynchronize(h->ev[3]);
        cudaEventElapsedTime(&t[0], h->ev[0], h->ev[1]);
        cudaEventElapsedTime(&t[1], h->ev[1], h->ev[2]);
        cudaEventElapsedTime(&t[2], h->ev[2], h->ev[3]);
        h->timings[NB_T_SORT] = t[0];
        h->timings[NB_T_TREE] = t[1];
        h->timings[NB_T_BUILD] = t[0] + t[1];
        h->timings[NB_T_TRAVERSAL] = t[2];
        h->timings[NB_T_TOTAL] = t[0] + t[1] + t[2];
        h->ev_valid = false;
    }
    if (h->ev_collide) {
        float tc = 0.f;
        cudaEventSynchronize(h->ev[5]);
        cudaEventElapsedTime(&tc, h->ev[4], h->ev[5]);
        h->timings[NB_T_COLLIDE] = tc;
        h->ev_collide = false;
    }
    for (int i = 0; i < n && i < NB_T_COUNT; i++) out[i] = h->timings[i];
    return NB_OK;
}

NB_API int32_t nb_get_counters(const nb_engine* h, int64_t* out, int32_t n) {
    if (!h || !out) return NB_ERR_INVALID_ARG;
    for (int i = 0; i < n && i < NB_C_COUNT; i++) out[i] = h->counters[i];
    return NB_OK;
}

NB_API int32_t nb_get_adaptive_dt(const nb_engine* h, double* dt) {
    if (!h || !dt) return NB_ERR_INVALID_ARG;
    *dt = h->adapt_dt;
    return NB_OK;
}

NB_API int32_t nb_get_body_count(const nb_engine* h, int32_t* n, int32_t* n_active) {
    if (!h || !n || !n_active) return NB_ERR_INVALID_ARG;
    *n = h->n;
    *n_active = h->n_active;
    return NB_OK;
}

NB_API int32_t nb_compute_forces(nb_engine* h, int32_t n, const double* px, const double* py,
                                 const double* pz, const double* mass, const double* radius,
                                 const uint8_t* active, double softening, int32_t flags,
                                 double* ax, double* ay, double* az) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, NB_ERR_CUDA, "cudaSetDevice");
    if ((flags & NB_FLAG_SHELL_THEOREM) && !radius)
        return fail(h, NB_ERR_INVALID_ARG, "shell theorem needs radii");
    if (!mass && n > 0) return fail(h, NB_ERR_INVALID_ARG, "null mass array");
    if (n > 0 && (!ax || !ay || !az)) return fail(h, NB_ERR_INVALID_ARG, "null output array");
    int r;
    if ((r = stage_bodies(h, n, px, py, pz, mass, radius, active))) return r;
    if (n == 0) return NB_OK;
    if ((r = force_pipeline(h, flags, softening, false, 0.0))) return r;
    const size_t d = sizeof(double) * (size_t)n;
    if ((r = download(h, ax, h->s.ax, d)) || (r = download(h, ay, h->s.ay, d)) ||
        (r = download(h, az, h->s.az, d)))
        return r;
    if ((r = check_device(h))) return r;
    collect_counters(h);
    return NB_OK;
}

NB_API int32_t nb_set_state(nb_engine* h, int32_t n, const double* px, const double* py,
                            const double* pz, const double* vx, const double* vy, const double* vz,
                            const double* mass, const double* radius, const double* density,
                            const uint8_t* active, const uint8_t* collidable,
                            const double* oax, const double* oay, const double* oaz) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, NB_ERR_CUDA, "cudaSetDevice");
    int r;
    if (n > 0 && (!vx || !vy || !vz || !mass))
        return fail(h, NB_ERR_INVALID_ARG, "null velocity or mass array");
    if ((r = stage_bodies(h, n, px, py, pz, mass, radius, active))) return r;
    const size_t d = sizeof(double) * (size_t)n;
    if ((r = upload(h, h->s.vx, vx, d)) || (r = upload(h, h->s.vy, vy, d)) ||
        (r = upload(h, h->s.vz, vz, d)))
        return r;
    double* acc[3] = {h->s.ax, h->s.ay, h->s.az};
    const double* old[3] = {oax, oay, oaz};
    for (int k = 0; k < 3; k++) {
        if (old[k]) {
            if ((r = upload(h, acc[k], old[k], d))) return r;
        } else {
            NB_CUDA(h, cudaMemsetAsync(acc[k], 0, d, h->st));
        }
    }
    if (density) {
        if ((r = upload(h, h->s.density, density, d))) return r;
    } else {
        NB_CUDA(h, cudaMemsetAsync(h->s.density, 0, d, h->st));
    }
    if (collidable) {
        if ((r = upload(h, h->s.collidable, collidable, (size_t)n))) return r;
    } else {
        NB_CUDA(h, cudaMemsetAsync(h->s.collidable, 1, (size_t)n, h->st));
    }
    std::vector<int32_t> ids((size_t)n);
    for (int i = 0; i < n; i++) ids[i] = i;
    if ((r = upload(h, h->s.ids, ids.data(), sizeof(int32_t) * (size_t)n))) return r;
    if ((r = check_device(h))) return r;
    h->has_state = true;
    h->adapt_dt = 0.0;
    return NB_OK;
}

NB_API int32_t nb_get_state(nb_engine* h, int32_t* n_out, double* px, double* py, double* pz,
                            double* vx, double* vy, double* vz, double* ax, double* ay,
                            double* az, double* mass, double* radius, uint8_t* active,
                            int32_t* ids) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NB_ERR_STATE, "no device-resident state");
    cudaSetDevice(h->device);
    const int n = h->n;
    if (n_out) *n_out = n;
    const size_t d = sizeof(double) * (size_t)n;
    int r;
    if ((r = download(h, px, h->s.px, d)) || (r = download(h, py, h->s.py, d)) ||
        (r = download(h, pz, h->s.pz, d)) || (r = download(h, vx, h->s.vx, d)) ||
        (r = download(h, vy, h->s.vy, d)) || (r = download(h, vz, h->s.vz, d)) ||
        (r = download(h, ax, h->s.ax, d)) || (r = download(h, ay, h->s.ay, d)) ||
        (r = download(h, az, h->s.az, d)) || (r = download(h, mass, h->s.mass, d)) ||
        (r = download(h, radius, h->s.radius, d)) ||
        (r = download(h, active, h->s.active, (size_t)n)) ||
        (r = download(h, ids, h->s.ids, sizeof(int32_t) * (size_t)n)))
        return r;
    return check_device(h);
}

namespace {

int force_error_stats(nb_engine* h, int32_t n_samples, uint64_t seed, double softening,
                      double* out3, bool sorted = false);

// The collision stage's arguments for the current state.
nb::CollideArgs collide_args(nb_engine* h) {
    nb::CollideArgs c{};
    c.n = h->n;
    c.n_active = h->n_active;
    c.s = h->s;
    c.s_alt = h->s_alt;
    c.keys0 = h->keys0; c.keys1 = h->keys1; c.vals0 = h->vals0; c.vals1 = h->vals1;
    c.sort_ws = h->sort_ws;
    c.tree = h->tree;
    c.sbody = h->sbody;
    c.srad = h->srad;
    c.cube = h->scal->cube;
    c.leaf_cap = h->leaf_cap;
    c.max_frame = h->max_merges_frame;
    c.max_body = h->max_merges_body;
    c.density_merge = h->density_merge;
    c.min_radius = h->min_radius;
    c.n_pairs = &h->scal->n_pairs;
    c.n_kept = &h->scal->n_kept;
    c.n_merges = &h->scal->n_merges;
    c.err = h->scal->err;
    c.sms = h->sms;
    c.bbox_ord = h->scal->bbox_ord;
    c.n_active_dev = &h->scal->n_active;
    // the second half kick moved no body: the force evaluation's tree
    // (Barnes-Hut modes) still describes the positions
    c.reuse_tree = h->tree_current;
    c.groups = h->groups;
    c.n_groups = &h->scal->n_groups;
    c.group_ctr = &h->scal->group_ctr;
    return c;
}

// Capture one collisional step (sub-steps, kicks, collision stage) from the
// current state buffer into the other, every count on the device.
int capture_collide_step(nb_engine* h, int flags, double dt, double eps, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    NB_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int* dn = &h->scal->n_rows;
    double sub[3];
    const int ns = sub_steps(flags, dt, sub);
    int r = NB_OK;
    for (int k = 0; k < ns && r == NB_OK; k++) {
        r = force_pipeline(h, flags, eps, true, sub[k], dn);
        if (r == NB_OK) nb::launch_kick(h->st, h->n, h->s, sub[k], dn);
    }
    if (r == NB_OK) {
        nb::CollideArgs c = collide_args(h);
        if (nb::collide_step_device(h->st, h->col, c, dn) != NB_OK)
            r = fail(h, NB_ERR_INVALID_ARG, "captured collision stage needs the step's tree");
    }
    h->tree_current = false;
    const cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (r != NB_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(h, NB_ERR_CUDA, "collision step capture: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        *out = nullptr;
        return fail(h, NB_ERR_CUDA, "collision step graph: %s", cudaGetErrorString(ei));
    }
    return NB_OK;
}

// n_steps collisional Barnes-Hut steps (geometric MAC) as replays of the two
// captured steps: nothing returns to the host between steps.  The captures
// are kept while the parameters match and the rows stay within 1/32 below
// the bounds they were captured with (the launches are sized by the bounds).
int run_collide_graphs(nb_engine* h, int n_steps, double dt, double eps, int flags) {
    nb_engine::GraphKey key{flags,           h->n,           h->n_active,
                            h->leaf_cap,     h->group_span,  h->group_bodies,
                            dt,              eps,
                            h->theta,        h->group_pack,  h->mac_theta_lo,
                            h->mac_theta_hi, h->mac_budget,  nullptr};
    const nb_engine::MergeKey mk{h->max_merges_frame, h->max_merges_body, h->density_merge,
                                 h->min_radius};
    nb_engine::GraphKey have = h->ckey;
    const bool fits = h->cgraph[0] && h->cgraph[1] && h->n <= have.n &&
                      h->n >= have.n - have.n / 32 && h->n_active <= have.n_active &&
                      (h->s.px == h->cstate[0] || h->s.px == h->cstate[1]) && mk == h->cmerge;
    have.n = key.n;
    have.n_active = key.n_active;
    int r = NB_OK;
    if (!(fits && have == key)) {
        for (auto& g : h->cgraph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        NB_CUDA(h, cudaStreamSynchronize(h->st));
        const int timing = h->timing;
        h->timing = 0;
        // capture from buffer A into B, then from B into A; the two swaps
        // leave the state where it was
        for (int k = 0; k < 2; k++) {
            h->cstate[k] = h->s.px;
            if (r == NB_OK) r = capture_collide_step(h, flags, dt, eps, &h->cgraph[k]);
            std::swap(h->s, h->s_alt);
        }
        h->timing = timing;
        if (r) {
            for (auto& g : h->cgraph)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
            return r;
        }
        h->ckey = key;
        h->cmerge = mk;
    }
    NB_CUDA(h, cudaMemcpyAsync(&h->scal->n_rows, &h->n, sizeof(int), cudaMemcpyHostToDevice,
                               h->st));
    const int first = h->s.px == h->cstate[0] ? 0 : 1;
    for (int k = 0; k < n_steps; k++)
        NB_CUDA(h, cudaGraphLaunch(h->cgraph[(first + k) & 1], h->st));
    if (n_steps & 1) std::swap(h->s, h->s_alt);
    h->tree_current = false;
    h->ev_valid = false;
    h->ev_collide = false;
    int cnt[4] = {0, 0, 0, 0};  // n_pairs, n_kept, n_merges, n_rows
    if ((r = download(h, cnt, &h->scal->n_pairs, sizeof(cnt)))) return r;
    r = check_device(h);  // synchronises: cnt holds the last step's counts
    h->n = cnt[3];
    h->n_active = cnt[3];  // compaction keeps exactly the active rows
    h->counters[NB_C_PAIRS] = cnt[0];
    h->counters[NB_C_MERGES] = cnt[2];
    if (r) return r;
    collect_counters(h);
    return NB_OK;
}

// n_steps Verlet steps with one flag set (no audits).
int run_steps(nb_engine* h, int n_steps, double dt, double softening, int flags) {
    const bool collide = (flags & NB_FLAG_COLLISIONS) != 0;
    int r;
    if (collide && n_steps > 1 && (flags & NB_MODE_MASK) == NB_MODE_BARNES_HUT &&
        !(flags & NB_FLAG_LEARNED_MAC))
        return run_collide_graphs(h, n_steps, dt, softening, flags);
    if (!collide && n_steps > 1) {
        // Multi-step calls replay one captured step (a CUDA graph) n times;
        // the row and active counts do not change without collisions.
        if ((r = step_graph(h, flags, dt, softening))) return r;
        for (int k = 0; k < n_steps; k++)
            NB_CUDA(h, cudaGraphLaunch(h->graph_exec, h->st));
        if ((r = check_device(h))) return r;
        collect_counters(h);
        return NB_OK;
    }
    double sub[3];
    const int ns = sub_steps(flags, dt, sub);
    for (int k = 0; k < n_steps * ns; k++) {
        const double sdt = sub[k % ns];
        if ((r = force_pipeline(h, flags, softening, true, sdt))) return r;
        nb::launch_kick(h->st, h->n, h->s, sdt);
        // collisions are detected and resolved once per step, on the state at
        // the end of the step (after the last Yoshida sub-step): the C# solver
        // runs CollisionDetector after the whole integrator step
        // (NBodySolver.cs:408-430) and the reference engine's GPU paths after
        // the last sub-step (engine.cpp:1160-1190)
        if (collide && k % ns == ns - 1) {
            nb::CollideArgs c = collide_args(h);
            int npairs = 0, nmerge = 0, nkept = 0;
            record(h, 4);
            if ((r = nb::collide_step(h->st, h->col, c, &npairs, &nmerge, &nkept)))
                return fail(h, r, "collision step failed");
            record(h, 5);
            h->ev_collide = h->timing != 0;
            h->tree_current = false;  // the state rows are compacted below
            std::swap(h->s, h->s_alt);
            h->n = nkept;
            h->n_active = nkept;
            h->counters[NB_C_PAIRS] = npairs;
            h->counters[NB_C_MERGES] = nmerge;
            if ((r = check_device(h))) return r;
        }
    }
    if ((r = check_device(h))) return r;
    collect_counters(h);
    return NB_OK;
}

}  // namespace

namespace {

// AdaptiveTimestep::update after a step (engine/src/sim/adaptive_timestep.cpp:
// 12-23): a_max = sqrt of the largest |a|^2 over the active rows.
int adaptive_update(nb_engine* h, double softening) {
    nb::max_acc2(h->st, h->n, h->s, &h->scal->amax2, h->sms);
    unsigned long long bits = 0;
    int r;
    if ((r = download(h, &bits, &h->scal->amax2, sizeof(bits))) || (r = check_device(h))) return r;
    double a2;
    std::memcpy(&a2, &bits, sizeof(a2));
    const double a_max = std::sqrt(a2);
    if (a_max <= 0.0 || softening <= 0.0) {
        h->adapt_dt = h->adapt_dt_max;
    } else {
        const double dt_new = h->adapt_eta * std::sqrt(softening / a_max);
        h->adapt_dt = std::clamp(dt_new, h->adapt_dt_min, h->adapt_dt_max);
    }
    return NB_OK;
}

}  // namespace

NB_API int32_t nb_step(nb_engine* h, int32_t n_steps, double dt, double softening, int32_t flags) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NB_ERR_STATE, "nb_step before nb_set_state");
    if (n_steps < 0) return fail(h, NB_ERR_INVALID_ARG, "negative step count");
    cudaSetDevice(h->device);
    const bool learned = (flags & NB_FLAG_LEARNED_MAC) != 0;
    const bool audit = learned && h->mac_audit_every > 0;
    const bool adaptive = (flags & NB_FLAG_ADAPTIVE_DT) != 0;
    int r, left = n_steps;
    while (left > 0) {
        // after a failed audit the learned MAC falls back to the geometric test
        const int f = (learned && h->mac_fallback) ? (flags & ~NB_FLAG_LEARNED_MAC) : flags;
        int k = audit ? std::min(left, h->mac_audit_every - h->mac_since_audit) : left;
        if (adaptive) k = 1;  // dt changes after every step
        const double dstep = (adaptive && h->adapt_dt > 0.0) ? h->adapt_dt : dt;
        if ((r = run_steps(h, k, dstep, softening, f))) return r;
        if (adaptive && (r = adaptive_update(h, softening))) return r;
        left -= k;
        if (!audit) continue;
        h->mac_since_audit += k;
        if (h->mac_since_audit >= h->mac_audit_every) {
            h->mac_since_audit = 0;
            // without collisions the last force evaluation's sorted copy of
            // the active bodies holds the current positions: the audit sums
            // run on it
            const bool sorted = (f & NB_MODE_MASK) != NB_MODE_DIRECT_FP64 &&
                                (f & NB_FLAG_COLLISIONS) == 0;
            double st[3];
            if ((r = force_error_stats(h, h->mac_audit_samples, 0x5EEDull + (uint64_t)h->mac_audits,
                                       softening, st, sorted)))
                return r;
            h->mac_audits++;
            h->mac_audit_last_rms = st[2];
            h->mac_audit_last_max = st[1];
            if (st[2] > h->mac_audit_rms_max) h->mac_fallback = true;
        }
    }
    h->counters[NB_C_MAC_AUDITS] = h->mac_audits;
    h->counters[NB_C_MAC_FALLBACK] = h->mac_fallback ? 1 : 0;
    return NB_OK;
}

NB_API int32_t nb_max_acceleration(nb_engine* h, double* a_max) {
    if (!h || !a_max) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NB_ERR_STATE, "no device-resident state");
    cudaSetDevice(h->device);
    nb::max_acc2(h->st, h->n, h->s, &h->scal->amax2, h->sms);
    unsigned long long bits = 0;
    int r;
    if ((r = download(h, &bits, &h->scal->amax2, sizeof(bits))) || (r = check_device(h))) return r;
    double a2;
    std::memcpy(&a2, &bits, sizeof(a2));
    *a_max = std::sqrt(a2);
    return NB_OK;
}

NB_API int32_t nb_diagnostics(nb_engine* h, double softening, int32_t pe_mode, double* out13) {
    if (!h || !out13) return NB_ERR_INVALID_ARG;
    if (!h->has_state) return fail(h, NB_ERR_STATE, "no device-resident state");
    cudaSetDevice(h->device);
    int r;
    if (pe_mode == 1) {
        // tree potential: a walk with the potential accumulated
        const int n = h->n;
        Scal* sc = h->scal;
        nb::launch_kick_drift_bbox(h->st, n, h->s, false, 0.0, sc->bbox_ord, &sc->n_active, sc->err);
        nb::launch_cube(h->st, sc->bbox_ord, nullptr, sc->cube);
        nb::launch_keys_cube(h->st, n, h->s, sc->cube, h->keys0, h->vals0, (uint32_t*)h->sort_ws);
        nb::sort_pairs(h->st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, true, sc->err, h->sms);
        nb::launch_gather(h->st, h->n_active, h->s, h->vals0, h->sbody, nullptr);
        nb::tree_build(h->st, h->tree, h->n_active, h->keys0, h->sbody, nullptr, sc->cube,
                       h->leaf_cap, sc->err);
        NB_CUDA(h, cudaMemsetAsync(h->phi, 0, sizeof(double) * (size_t)n, h->st));
        // the walk writes acc too: keep the state's acc in the alt buffers
        nb::WalkArgs a{};
        a.n = h->n_active;
        a.sbody = h->sbody;
        a.sidx = h->vals0;
        a.skeys = h->keys0;
        a.t = h->tree;
        a.theta2 = h->theta * h->theta;
        a.eps2 = softening * softening;
        a.ax = h->s_alt.ax;
        a.ay = h->s_alt.ay;
        a.az = h->s_alt.az;
        a.pot = h->phi;
        a.front = h->front;
        a.group_ctr = &sc->group_ctr;
        a.groups = h->groups;
        a.n_groups = &sc->n_groups;
        a.pack = h->group_pack;
        a.group_span = h->group_span;
        a.group_size = h->group_bodies;
        a.counters = nullptr;
        a.err = sc->err;
        nb::walk_group(h->st, h->wcfg, a, true, false, true);
    }
    double out[12];
    nb::diagnostics(h->st, h->n, h->s, softening, pe_mode, h->phi, h->rows, h->part, h->scal->diag);
    if ((r = download(h, out, h->scal->diag, sizeof(out)))) return r;
    if ((r = check_device(h))) return r;
    const double M = out[10];
    out13[0] = out[0];
    out13[1] = out[11];
    out13[2] = out[0] + out[11];
    for (int k = 0; k < 6; k++) out13[3 + k] = out[1 + k];
    for (int k = 0; k < 3; k++) out13[9 + k] = M > 0 ? out[7 + k] / M : 0.0;
    out13[12] = M;
    return NB_OK;
}

namespace {

// ForceErrorAnalyzer statistics of the handle's current accelerations on
// n_samples sampled active bodies against the FP64 direct sum: mean, max, rms.
// out[3 k + axis] = acceleration of row targets[k]
__global__ void k_gather_acc(int ns, const int32_t* __restrict__ targets,
                             const double* __restrict__ ax, const double* __restrict__ ay,
                             const double* __restrict__ az, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    const int i = targets[k];
    out[3 * k] = ax[i];
    out[3 * k + 1] = ay[i];
    out[3 * k + 2] = az[i];
}

// sorted: the last force evaluation's sorted copy of the active bodies holds
// the current positions, and the sums may run on it (the learned MAC's audit)
int force_error_stats(nb_engine* h, int32_t n_samples, uint64_t seed, double softening,
                      double* out3, bool sorted) {
    const int n = h->n;
    int r;
    // SplitMix64-driven partial Fisher-Yates: uniform sample without replacement
    uint64_t x = seed;
    auto next = [&x]() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    std::vector<int32_t> cand;
    int ns;
    if (h->n_active == n && n_samples > 0 && n_samples < n) {
        // every row active: the candidates are 0 .. n-1, so the shuffle only
        // records the positions it touched (the same draws and the same
        // sample as on the full list, without reading the active flags)
        ns = n_samples;
        std::unordered_map<int32_t, int32_t> moved;
        moved.reserve(2 * (size_t)ns);
        auto at = [&moved](int32_t k) {
            auto it = moved.find(k);
            return it == moved.end() ? k : it->second;
        };
        cand.resize(ns);
        for (int k = 0; k < ns; k++) {
            const int32_t j = (int32_t)(k + next() % (uint64_t)(n - k));
            const int32_t vk = at(k), vj = at(j);
            moved[j] = vk;
            cand[k] = vj;
        }
    } else {
        std::vector<uint8_t> act((size_t)n);
        if ((r = download(h, act.data(), h->s.active, (size_t)n))) return r;
        if ((r = check_device(h))) return r;
        cand.reserve((size_t)n);
        for (int i = 0; i < n; i++)
            if (act[i]) cand.push_back(i);
        ns = (n_samples <= 0 || n_samples >= (int)cand.size()) ? (int)cand.size() : n_samples;
        if (ns < (int)cand.size())
            for (int k = 0; k < ns; k++) {
                uint64_t j = k + next() % (uint64_t)(cand.size() - k);
                std::swap(cand[k], cand[j]);
            }
        cand.resize(ns);
    }
    if ((r = upload(h, h->targets, cand.data(), sizeof(int32_t) * (size_t)ns))) return r;
    if (!sorted || !nb::audit_targets(h->st, h->n_active, h->sbody, h->s, softening, ns,
                                      h->targets, h->tgt_out, h->aud_part, h->sms))
        nb::direct_targets(h->st, n, h->s, softening, ns, h->targets, h->tgt_out, h->tgt_part,
                           h->sms);
    std::vector<double> ref((size_t)ns * 3), ax, ay, az;
    if ((r = download(h, ref.data(), h->tgt_out, sizeof(double) * 3 * (size_t)ns))) return r;
    const bool gathered = 3 * (size_t)ns <= (size_t)h->capacity;  // fits the key scratch
    if (gathered) {
        // only the sampled rows' accelerations cross PCIe
        double* g = (double*)h->keys1;
        k_gather_acc<<<nb::ceil_div(ns, 256), 256, 0, h->st>>>(ns, h->targets, h->s.ax, h->s.ay,
                                                               h->s.az, g);
        ax.resize(3 * (size_t)ns);
        if ((r = download(h, ax.data(), g, sizeof(double) * 3 * (size_t)ns))) return r;
    } else {
        ax.resize(n);
        ay.resize(n);
        az.resize(n);
        if ((r = download(h, ax.data(), h->s.ax, sizeof(double) * (size_t)n)) ||
            (r = download(h, ay.data(), h->s.ay, sizeof(double) * (size_t)n)) ||
            (r = download(h, az.data(), h->s.az, sizeof(double) * (size_t)n)))
            return r;
    }
    if ((r = check_device(h))) return r;
    // ForceErrorAnalyzer.CompareForces statistics (ForceErrorAnalyzer.cs:100-134)
    double se = 0, se2 = 0, mx = 0;
    int c = 0;
    for (int k = 0; k < ns; k++) {
        const int i = cand[k];
        const double ex = ref[3 * k], ey = ref[3 * k + 1], ez = ref[3 * k + 2];
        const double em = sqrt(ex * ex + ey * ey + ez * ez);
        if (em < 1e-30) continue;
        const double gx = gathered ? ax[3 * k] : ax[i];
        const double gy = gathered ? ax[3 * k + 1] : ay[i];
        const double gz = gathered ? ax[3 * k + 2] : az[i];
        const double dx = gx - ex, dy = gy - ey, dz = gz - ez;
        const double e = sqrt(dx * dx + dy * dy + dz * dz) / em;
        se += e;
        se2 += e * e;
        if (e > mx) mx = e;
        c++;
    }
    out3[0] = c ? se / c : 0;
    out3[1] = mx;
    out3[2] = c ? sqrt(se2 / c) : 0;
    return NB_OK;
}

}  // namespace

NB_API int32_t nb_force_error(nb_engine* h, int32_t n_samples, uint64_t seed, double softening,
                              int32_t flags, double* out3) {
    (void)flags;
    if (!h || !out3) return NB_ERR_INVALID_ARG;
    if (!h->has_state && h->n == 0) return fail(h, NB_ERR_STATE, "no bodies on the device");
    cudaSetDevice(h->device);
    return force_error_stats(h, n_samples, seed, softening, out3);
}

NB_API int32_t nb_mac_audit_state(nb_engine* h, double* rms, double* max_err, int64_t* audits,
                                  int32_t* fallback) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (rms) *rms = h->mac_audit_last_rms;
    if (max_err) *max_err = h->mac_audit_last_max;
    if (audits) *audits = h->mac_audits;
    if (fallback) *fallback = h->mac_fallback ? 1 : 0;
    return NB_OK;
}

NB_API int32_t nb_morton_keys(nb_engine* h, int32_t n, const double* px, const double* py,
                              const double* pz, const uint8_t* active, int32_t mode,
                              const double* cube4, uint64_t* keys, int32_t* idx,
                              double* cube4_out) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (mode != 0 && mode != 1) return fail(h, NB_ERR_INVALID_ARG, "mode must be 0 or 1");
    cudaSetDevice(h->device);
    int r;
    if ((r = stage_bodies(h, n, px, py, pz, nullptr, nullptr, active))) return r;
    if (n == 0) return NB_OK;
    Scal* sc = h->scal;
    nb::launch_kick_drift_bbox(h->st, n, h->s, false, 0.0, sc->bbox_ord, &sc->n_active, sc->err);
    if (mode == 0) {
        nb::launch_keys_aabb(h->st, n, h->s, sc->bbox_ord, h->keys0, h->vals0);
    } else {
        if (cube4 && (r = upload(h, sc->cube_in, cube4, sizeof(double) * 4))) return r;
        nb::launch_cube(h->st, sc->bbox_ord, cube4 ? sc->cube_in : nullptr, sc->cube);
        nb::launch_keys_cube(h->st, n, h->s, sc->cube, h->keys0, h->vals0, (uint32_t*)h->sort_ws);
        if ((r = download(h, cube4_out, sc->cube, sizeof(double) * 4))) return r;
    }
    if ((r = download(h, keys, h->keys0, sizeof(uint64_t) * (size_t)n)) ||
        (r = download(h, idx, h->vals0, sizeof(int32_t) * (size_t)n)))
        return r;
    return check_device(h);
}

NB_API int32_t nb_sort_pairs(nb_engine* h, int32_t n, uint64_t* keys, int32_t* values) {
    if (!h) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    int r;
    if ((r = check_n(h, n))) return r;
    if (n <= 1) return NB_OK;
    if ((r = upload(h, h->keys0, keys, sizeof(uint64_t) * (size_t)n)) ||
        (r = upload(h, h->vals0, values, sizeof(int32_t) * (size_t)n)))
        return r;
    nb::sort_pairs(h->st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, false,
                   h->scal->err, h->sms);
    if ((r = download(h, keys, h->keys0, sizeof(uint64_t) * (size_t)n)) ||
        (r = download(h, values, h->vals0, sizeof(int32_t) * (size_t)n)))
        return r;
    h->has_state = false;
    return check_device(h);
}

NB_API int32_t nb_build_octree(nb_engine* h, int32_t n, const double* px, const double* py,
                               const double* pz, const double* mass, const uint8_t* active,
                               const double* cube4, int32_t leaf_capacity, int32_t max_nodes,
                               int32_t* n_nodes, int32_t* level, int32_t* first_child,
                               int32_t* n_children, int32_t* body_first, int32_t* body_count,
                               double* node_mass, double* com3, float* quad6,
                               int32_t* sorted_idx, uint64_t* sorted_keys) {
    if (!h || !n_nodes) return NB_ERR_INVALID_ARG;
    if (leaf_capacity < 1 || leaf_capacity > 64)
        return fail(h, NB_ERR_INVALID_ARG, "leaf capacity must be 1..64");
    cudaSetDevice(h->device);
    int r;
    if ((r = stage_bodies(h, n, px, py, pz, mass, nullptr, active))) return r;
    *n_nodes = 0;
    if (n == 0) return NB_OK;
    Scal* sc = h->scal;
    nb::launch_kick_drift_bbox(h->st, n, h->s, false, 0.0, sc->bbox_ord, &sc->n_active, sc->err);
    if (cube4 && (r = upload(h, sc->cube_in, cube4, sizeof(double) * 4))) return r;
    nb::launch_cube(h->st, sc->bbox_ord, cube4 ? sc->cube_in : nullptr, sc->cube);
    nb::launch_keys_cube(h->st, n, h->s, sc->cube, h->keys0, h->vals0, (uint32_t*)h->sort_ws);
    nb::sort_pairs(h->st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, true, sc->err,
                   h->sms);
    const int na = h->n_active;
    nb::launch_gather(h->st, na, h->s, h->vals0, h->sbody, nullptr);
    nb::tree_build(h->st, h->tree, na, h->keys0, h->sbody, nullptr, sc->cube, leaf_capacity,
                   sc->err);
    int nn = 0;
    if ((r = download(h, &nn, h->tree.n_nodes, sizeof(int)))) return r;
    if ((r = check_device(h))) return r;
    *n_nodes = nn;
    if (nn > max_nodes) return fail(h, NB_ERR_CAPACITY, "%d nodes > max_nodes %d", nn, max_nodes);
    std::vector<int4> link((size_t)nn);
    std::vector<double4> com((size_t)nn);
    std::vector<float4> q0((size_t)nn), q1((size_t)nn);
    std::vector<int> lev((size_t)nn);
    if ((r = download(h, link.data(), h->tree.link, sizeof(int4) * (size_t)nn)) ||
        (r = download(h, com.data(), h->tree.com, sizeof(double4) * (size_t)nn)) ||
        (r = download(h, q0.data(), h->tree.q0, sizeof(float4) * (size_t)nn)) ||
        (r = download(h, q1.data(), h->tree.q1, sizeof(float4) * (size_t)nn)) ||
        (r = download(h, lev.data(), h->tree.level, sizeof(int) * (size_t)nn)) ||
        (r = download(h, sorted_idx, h->vals0, sizeof(int32_t) * (size_t)n)) ||
        (r = download(h, sorted_keys, h->keys0, sizeof(uint64_t) * (size_t)n)))
        return r;
    if ((r = check_device(h))) return r;
    for (int k = 0; k < nn; k++) {
        if (level) level[k] = lev[k];
        if (first_child) first_child[k] = link[k].x;
        if (n_children) n_children[k] = link[k].y;
        if (body_first) body_first[k] = link[k].z;
        if (body_count) body_count[k] = link[k].w;
        if (node_mass) node_mass[k] = com[k].w;
        if (com3) {
            com3[3 * k] = com[k].x;
            com3[3 * k + 1] = com[k].y;
            com3[3 * k + 2] = com[k].z;
        }
        if (quad6) {
            const float qxx = q0[k].x, qyy = q0[k].y;
            const float v[6] = {qxx, qyy, -(qxx + qyy), q0[k].z, q0[k].w, q1[k].x};
            for (int j = 0; j < 6; j++) quad6[6 * k + j] = v[j];
        }
    }
    h->ev_tree = true;
    return NB_OK;
}

NB_API int32_t nb_compact_indices(nb_engine* h, int32_t n, const uint8_t* active,
                                  const double* mass, int32_t* dest, int32_t* n_kept) {
    if (!h || !n_kept) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    int r;
    if ((r = check_n(h, n))) return r;
    *n_kept = 0;
    if (n == 0) return NB_OK;
    if ((r = upload(h, h->s.active, active, (size_t)n)) ||
        (r = upload(h, h->s.mass, mass, sizeof(double) * (size_t)n)))
        return r;
    int kept = 0;
    if ((r = nb::compact_indices(h->st, h->col, n, h->s.active, h->s.mass, (int32_t*)h->vals1,
                                 &h->scal->n_kept, h->scal->err)))
        return fail(h, r, "compaction failed");
    if ((r = download(h, dest, h->vals1, sizeof(int32_t) * (size_t)n)) ||
        (r = download(h, &kept, &h->scal->n_kept, sizeof(int))))
        return r;
    if ((r = check_device(h))) return r;
    *n_kept = kept;
    h->has_state = false;
    return NB_OK;
}

NB_API int32_t nb_broad_phase(nb_engine* h, int32_t n, const double* px, const double* py,
                              const double* pz, const double* radius, const uint8_t* active,
                              const uint8_t* collidable, int32_t max_pairs, int32_t* pair_lo,
                              int32_t* pair_hi, int32_t* n_pairs) {
    if (!h || !n_pairs || !radius) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    int r;
    if ((r = stage_bodies(h, n, px, py, pz, nullptr, radius, active))) return r;
    *n_pairs = 0;
    if (n == 0) return NB_OK;
    if (collidable) {
        if ((r = upload(h, h->s.collidable, collidable, (size_t)n))) return r;
    } else {
        NB_CUDA(h, cudaMemsetAsync(h->s.collidable, 1, (size_t)n, h->st));
    }
    // the broad phase reads masses only through the tree: give every body
    // unit mass so no cell is skipped as empty
    std::vector<double> ones((size_t)n, 1.0);
    if ((r = upload(h, h->s.mass, ones.data(), sizeof(double) * (size_t)n))) return r;
    Scal* sc = h->scal;
    nb::CollideArgs c{};
    c.n = n;
    c.n_active = h->n_active;
    c.s = h->s;
    c.s_alt = h->s_alt;
    c.keys0 = h->keys0; c.keys1 = h->keys1; c.vals0 = h->vals0; c.vals1 = h->vals1;
    c.sort_ws = h->sort_ws;
    c.tree = h->tree;
    c.sbody = h->sbody;
    c.srad = h->srad;
    c.cube = sc->cube;
    c.leaf_cap = h->leaf_cap;
    c.n_pairs = &sc->n_pairs;
    c.err = sc->err;
    c.sms = h->sms;
    c.bbox_ord = sc->bbox_ord;
    c.n_active_dev = &sc->n_active;
    c.groups = h->groups;
    c.n_groups = &sc->n_groups;
    c.group_ctr = &sc->group_ctr;
    int np = 0;
    if ((r = nb::broad_phase(h->st, h->col, c, true, &np)))
        return fail(h, r, "broad phase failed");
    if ((r = check_device(h))) return r;
    *n_pairs = np;
    const int w = np < max_pairs ? np : max_pairs;
    if (w > 0) {
        std::vector<uint64_t> pk((size_t)w);
        if ((r = download(h, pk.data(), h->col.pair_keys, sizeof(uint64_t) * (size_t)w))) return r;
        if ((r = check_device(h))) return r;
        for (int k = 0; k < w; k++) {
            if (pair_lo) pair_lo[k] = (int32_t)(pk[k] >> 32);
            if (pair_hi) pair_hi[k] = (int32_t)(pk[k] & 0xFFFFFFFFu);
        }
    }
    h->has_state = false;
    if (np > max_pairs) return fail(h, NB_ERR_CAPACITY, "%d pairs > max_pairs %d", np, max_pairs);
    return NB_OK;
}

// ---- learned MAC ------------------------------------------------------------

NB_API int32_t nb_mac_harvest(nb_engine* h, int32_t max_records, double sample_frac,
                              uint64_t seed, double softening, int32_t* n_added) {
    if (!h || !n_added) return NB_ERR_INVALID_ARG;
    *n_added = 0;
    if (!h->has_state) return fail(h, NB_ERR_STATE, "harvest needs device-resident state");
    if (max_records <= 0 || !(sample_frac > 0.0 && sample_frac <= 1.0) || !(softening > 0.0))
        return fail(h, NB_ERR_INVALID_ARG, "bad harvest arguments");
    cudaSetDevice(h->device);
    int r;
    if (!h->mac_X) {
        h->mac_cap = 1 << 24;
        if ((r = dalloc(h, &h->mac_X, (size_t)h->mac_cap * nb::kMacIn)) ||
            (r = dalloc(h, &h->mac_Y, (size_t)h->mac_cap)))
            return r;
    }
    if (h->mac_rec_cap < max_records) {
        const size_t m = (size_t)max_records;
        if ((r = dalloc(h, &h->mac_rec, m)) || (r = dalloc(h, &h->mac_rec2, m)) ||
            (r = dalloc(h, &h->mac_rk0, m)) || (r = dalloc(h, &h->mac_rk1, m)) ||
            (r = dalloc(h, &h->mac_rv0, m)) || (r = dalloc(h, &h->mac_rv1, m)) ||
            (r = dalloc(h, (char**)&h->mac_rws, nb::sort_workspace_bytes(max_records))))
            return r;
        h->mac_rec_cap = max_records;
    }
    const int n = h->n, na = h->n_active;
    Scal* sc = h->scal;
    nb::launch_kick_drift_bbox(h->st, n, h->s, false, 0.0, sc->bbox_ord, &sc->n_active, sc->err);
    nb::launch_cube(h->st, sc->bbox_ord, nullptr, sc->cube);
    nb::launch_keys_cube(h->st, n, h->s, sc->cube, h->keys0, h->vals0, (uint32_t*)h->sort_ws);
    nb::sort_pairs(h->st, n, h->keys0, h->vals0, h->keys1, h->vals1, h->sort_ws, true, sc->err, h->sms);
    nb::launch_gather(h->st, na, h->s, h->vals0, h->sbody, nullptr, h->samag);
    nb::launch_zero_acc(h->st, n, h->s);
    nb::tree_build(h->st, h->tree, na, h->keys0, h->sbody, nullptr, sc->cube, h->leaf_cap, sc->err);
    NB_CUDA(h, cudaMemsetAsync(h->mac_counts, 0, sizeof(int) * 4, h->st));
    nb::WalkArgs a{};
    a.n = na;
    a.sbody = h->sbody;
    a.skeys = h->keys0;
    a.sidx = h->vals0;
    a.t = h->tree;
    a.eps2 = softening * softening;
    a.ax = h->s.ax;
    a.ay = h->s.ay;
    a.az = h->s.az;
    a.front = h->front;
    a.group_ctr = &sc->group_ctr;
    a.groups = h->groups;
    a.n_groups = &sc->n_groups;
    a.pack = h->group_pack;
    a.group_span = h->group_span;
    a.group_size = h->group_bodies;
    a.counters = sc->counters;
    a.err = sc->err;
    a.theta2 = h->mac_theta_lo * h->mac_theta_lo;
    a.mac_theta_hi2 = (float)(h->mac_theta_hi * h->mac_theta_hi);
    a.samag = h->samag;
    a.records = h->mac_rec;
    a.n_records = &h->mac_counts[0];
    a.record_cap = max_records;
    a.mac_seed = (unsigned)(seed ^ (seed >> 32));
    a.mac_sample = (unsigned)std::min(65536.0, std::ceil(sample_frac * 65536.0));
    nb::walk_group(h->st, h->wcfg, a, true, false, false, 1);
    int nrec = 0;
    if ((r = download(h, &nrec, &h->mac_counts[0], sizeof(int)))) return r;
    if ((r = check_device(h))) return r;
    nrec = std::min(nrec, max_records);
    // a fixed record order (the walk appends them in warp order): the
    // training set, and so the trained network, do not depend on scheduling
    nb::mac_sort_records(h->st, nrec, h->mac_rec, h->mac_rec2, h->mac_rk0, h->mac_rv0,
                         h->mac_rk1, h->mac_rv1, h->mac_rws, &h->mac_counts[1], sc->err, h->sms);
    int got = 0;
    if ((r = download(h, &got, &h->mac_counts[1], sizeof(int)))) return r;
    if ((r = check_device(h))) return r;
    nb::mac_targets(h->st, got, h->mac_rec2, h->sbody, h->tree, softening, h->mac_X, h->mac_Y,
                    &h->mac_counts[2], h->mac_n, h->mac_cap);
    if ((r = check_device(h))) return r;
    got = std::min(got, h->mac_cap - h->mac_n);
    h->mac_n += got;
    *n_added = got;
    return NB_OK;
}

NB_API int32_t nb_mac_dataset(nb_engine* h, int32_t* n, float* X, float* Y) {
    if (!h || !n) return NB_ERR_INVALID_ARG;
    *n = h->mac_n;
    if (h->mac_n == 0) return NB_OK;
    int r;
    if ((r = download(h, X, h->mac_X, sizeof(float) * nb::kMacIn * (size_t)h->mac_n)) ||
        (r = download(h, Y, h->mac_Y, sizeof(float) * (size_t)h->mac_n)))
        return r;
    return check_device(h);
}

NB_API int32_t nb_mac_clear(nb_engine* h) {
    if (!h) return NB_ERR_INVALID_ARG;
    h->mac_n = 0;
    return NB_OK;
}

namespace {

// The screen block (normalised units) and its raw-feature form with the
// normalisation folded in: scr_w[k] = w[k] / std[k], scr_b = b - sum w[k]
// mean[k] / std[k] (inv_std as the device forms it, 1.f / std).
int mac_upload_screen(nb_engine* h) {
    constexpr int kIn = nb::kMacIn;
    float blk[nb::kMacScreen + kIn + 1];
    std::copy(h->mac_screen, h->mac_screen + nb::kMacScreen, blk);
    double b = h->mac_screen[kIn];
    for (int k = 0; k < kIn; k++) {
        const float inv = 1.f / h->mac_norm_host[kIn + k];
        blk[nb::kMacScreen + k] = h->mac_screen[k] * inv;
        b -= (double)h->mac_screen[k] * h->mac_norm_host[k] * inv;
    }
    blk[nb::kMacScreen + kIn] = (float)b;
    static_assert(offsetof(nb::MacDev, scr_w) == offsetof(nb::MacDev, lin_w) + sizeof(float) * nb::kMacScreen,
                  "screen block layout");
    return upload(h, h->mac_dev->lin_w, blk, sizeof(blk));
}

int mac_upload_params(nb_engine* h, const float* P, const float* norm) {
    int r;
    if ((r = upload(h, h->mac_P, P, sizeof(float) * nb::kMacParams)) ||
        (r = upload(h, h->mac_norm, norm, sizeof(float) * nb::kMacNorm)))
        return r;
    NB_CUDA(h, cudaMemsetAsync(h->mac_m, 0, sizeof(float) * nb::kMacParams, h->st));
    NB_CUDA(h, cudaMemsetAsync(h->mac_v, 0, sizeof(float) * nb::kMacParams, h->st));
    h->mac_adam_step = 0;
    std::copy(norm, norm + nb::kMacNorm, h->mac_norm_host);
    nb::mac_image(h->st, h->mac_P, h->mac_norm, h->mac_dev);
    // a new network invalidates the screen: off until the next fit
    std::fill(h->mac_screen, h->mac_screen + nb::kMacScreen, 0.f);
    h->mac_screen[nb::kMacScreen - 1] = INFINITY;
    int r2 = mac_upload_screen(h);
    return r2 ? r2 : check_device(h);
}

// Least-squares fit of the screen to the network's predictions on (a strided
// sample of) the multi-body rows of the training set; margin = the chosen
// quantile of |residual| in normalised target units.
int mac_fit_screen(nb_engine* h) {
    float sc[nb::kMacScreen] = {0, 0, 0, 0, 0, 0, 0, 0, 0, INFINITY};
    const int n = h->mac_n;
    constexpr int kIn = nb::kMacIn;
    if (h->mac_screen_q > 0.0 && n >= 64) {
        const int m = std::min(n, 1 << 18);
        const int stride = n / m;
        float *dX = nullptr, *dy = nullptr;
        NB_CUDA(h, cudaMalloc(&dX, sizeof(float) * kIn * (size_t)m));
        if (cudaMalloc(&dy, sizeof(float) * (size_t)m) != cudaSuccess) {
            cudaFree(dX);
            return fail(h, NB_ERR_CUDA, "screen fit: out of device memory");
        }
        cudaMemcpy2DAsync(dX, sizeof(float) * kIn, h->mac_X, sizeof(float) * kIn * (size_t)stride,
                          sizeof(float) * kIn, (size_t)m, cudaMemcpyDeviceToDevice, h->st);
        nb::mac_predict(h->st, dX, m, h->mac_dev, dy);
        std::vector<float> X((size_t)m * kIn), y((size_t)m);
        int r = download(h, X.data(), dX, sizeof(float) * X.size());
        if (!r) r = download(h, y.data(), dy, sizeof(float) * y.size());
        if (!r) r = check_device(h);
        cudaFree(dX);
        cudaFree(dy);
        if (r) return r;
        const float* nm = h->mac_norm_host;
        float inv[kIn];
        for (int k = 0; k < kIn; k++) inv[k] = 1.f / nm[kIn + k];
        // normal equations over [x_norm, 1]
        double A[kIn + 1][kIn + 2] = {};
        std::vector<float> fn((size_t)m * kIn);
        std::vector<double> yn((size_t)m);
        std::vector<char> use((size_t)m);
        int rows = 0;
        for (int i = 0; i < m; i++) {
            const float* xi = &X[(size_t)i * kIn];
            use[i] = xi[4] > 0.5f;  // log2(count): one-body cells never reach the screen
            if (!use[i]) continue;
            double v[kIn + 1];
            for (int k = 0; k < kIn; k++) v[k] = fn[(size_t)i * kIn + k] = (xi[k] - nm[k]) * inv[k];
            v[kIn] = 1.0;
            yn[i] = ((double)y[i] - nm[2 * kIn]) / nm[2 * kIn + 1];
            for (int a = 0; a <= kIn; a++) {
                for (int b = 0; b <= kIn; b++) A[a][b] += v[a] * v[b];
                A[a][kIn + 1] += v[a] * yn[i];
            }
            rows++;
        }
        if (rows >= 64) {
            for (int a = 0; a <= kIn; a++) A[a][a] += 1e-9 * (A[a][a] + 1.0);
            // Gaussian elimination with partial pivoting
            for (int c = 0; c <= kIn; c++) {
                int piv = c;
                for (int r1 = c + 1; r1 <= kIn; r1++)
                    if (std::fabs(A[r1][c]) > std::fabs(A[piv][c])) piv = r1;
                for (int k = 0; k <= kIn + 1; k++) std::swap(A[c][k], A[piv][k]);
                for (int r1 = 0; r1 <= kIn; r1++) {
                    if (r1 == c) continue;
                    const double f = A[r1][c] / A[c][c];
                    for (int k = c; k <= kIn + 1; k++) A[r1][k] -= f * A[c][k];
                }
            }
            float w[kIn + 1];
            for (int a = 0; a <= kIn; a++) w[a] = (float)(A[a][kIn + 1] / A[a][a]);
            std::vector<double> res;
            res.reserve(rows);
            for (int i = 0; i < m; i++) {
                if (!use[i]) continue;
                float s1 = w[kIn];
                for (int k = 0; k < kIn; k++) s1 = std::fma(w[k], fn[(size_t)i * kIn + k], s1);
                res.push_back(std::fabs(yn[i] - (double)s1));
            }
            const size_t q = std::min(res.size() - 1, (size_t)(h->mac_screen_q * (double)res.size()));
            std::nth_element(res.begin(), res.begin() + q, res.end());
            bool finite = std::isfinite(res[q]);
            for (int a = 0; a <= kIn; a++) finite = finite && std::isfinite(w[a]);
            if (finite) {
                std::copy(w, w + kIn + 1, sc);
                sc[kIn + 1] = (float)(res[q] * 1.0001 + 1e-6);
            }
        }
    }
    std::copy(sc, sc + nb::kMacScreen, h->mac_screen);
    int r = mac_upload_screen(h);
    return r ? r : check_device(h);
}

}  // namespace

NB_API int32_t nb_mac_set_params(nb_engine* h, const float* params, int32_t n) {
    if (!h || !params || n != nb::kMacParams + nb::kMacNorm) return NB_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    for (int k = 0; k < nb::kMacIn + 1; k++)
        if (!(params[nb::kMacParams + nb::kMacIn + k] > 0.f) && k < nb::kMacIn)
            return fail(h, NB_ERR_INVALID_ARG, "feature scales must be positive");
    if (!(params[nb::kMacParams + nb::kMacNorm - 1] > 0.f))
        return fail(h, NB_ERR_INVALID_ARG, "target scale must be positive");
    int r = mac_upload_params(h, params, params + nb::kMacParams);
    if (r) return r;
    h->mac_ready = true;
    h->mac_fallback = false;
    return NB_OK;
}

NB_API int32_t nb_mac_get_params(nb_engine* h, float* out, int32_t n) {
    if (!h || !out || n != nb::kMacParams + nb::kMacNorm) return NB_ERR_INVALID_ARG;
    if (!h->mac_ready) return fail(h, NB_ERR_STATE, "no learned-MAC parameters");
    cudaSetDevice(h->device);
    int r;
    if ((r = download(h, out, h->mac_P, sizeof(float) * nb::kMacParams))) return r;
    std::copy(h->mac_norm_host, h->mac_norm_host + nb::kMacNorm, out + nb::kMacParams);
    return check_device(h);
}

NB_API int32_t nb_mac_train(nb_engine* h, int32_t epochs, int32_t batch, double lr, uint64_t seed,
                            double* loss_per_epoch) {
    if (!h || epochs < 0 || batch < 32 || !(lr > 0.0)) return NB_ERR_INVALID_ARG;
    const int n = h->mac_n;
    if (n < batch) return fail(h, NB_ERR_STATE, "%d samples < batch %d", n, batch);
    cudaSetDevice(h->device);
    int r = NB_OK;
    if (!h->mac_ready) {
        // normalisation from the data, He-uniform initial weights
        std::vector<float> X((size_t)n * nb::kMacIn), Y((size_t)n);
        if ((r = download(h, X.data(), h->mac_X, sizeof(float) * X.size())) ||
            (r = download(h, Y.data(), h->mac_Y, sizeof(float) * Y.size())) || (r = check_device(h)))
            return r;
        float norm[nb::kMacNorm];
        for (int k = 0; k <= nb::kMacIn; k++) {
            double s = 0, s2 = 0;
            for (int i = 0; i < n; i++) {
                const double v = k < nb::kMacIn ? X[(size_t)i * nb::kMacIn + k] : Y[i];
                s += v;
                s2 += v * v;
            }
            const double mean = s / n, var = std::max(s2 / n - mean * mean, 0.0);
            const float sd = (float)std::max(std::sqrt(var), 1e-3);
            if (k < nb::kMacIn) {
                norm[k] = (float)mean;
                norm[nb::kMacIn + k] = sd;
            } else {
                norm[2 * nb::kMacIn] = (float)mean;
                norm[2 * nb::kMacIn + 1] = sd;
            }
        }
        std::vector<float> P(nb::kMacParams, 0.f);
        std::mt19937_64 rng(seed);
        auto fill = [&](int off, int count, int fan_in) {
            std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
            for (int i = 0; i < count; i++) P[off + i] = u(rng);
        };
        fill(nb::kMacW1, nb::kMacIn * nb::kMacHid, nb::kMacIn);
        fill(nb::kMacW2, nb::kMacHid * nb::kMacHid, nb::kMacHid);
        fill(nb::kMacW3, nb::kMacHid, nb::kMacHid);
        if ((r = mac_upload_params(h, P.data(), norm))) return r;
        h->mac_ready = true;
    }
    int* order = nullptr;
    NB_CUDA(h, cudaMalloc(&order, sizeof(int) * (size_t)n));
    std::vector<int> perm((size_t)n);
    for (int i = 0; i < n; i++) perm[i] = i;
    std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + 1);
    for (int e = 0; e < epochs && r == NB_OK; e++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        if ((r = upload(h, order, perm.data(), sizeof(int) * (size_t)n))) break;
        cudaMemsetAsync(h->mac_loss, 0, sizeof(float), h->st);
        for (int row0 = 0; row0 < n; row0 += batch) {
            const int rows = std::min(batch, n - row0);
            nb::mac_grad(h->st, h->mac_X, h->mac_Y, order, row0, rows, h->mac_P, h->mac_dev,
                         h->mac_G, h->mac_loss, h->sms, h->mac_part, h->scal->err);
            nb::mac_adam(h->st, h->mac_P, h->mac_G, h->mac_m, h->mac_v, ++h->mac_adam_step, (float)lr);
            nb::mac_image(h->st, h->mac_P, h->mac_norm, h->mac_dev);
        }
        float loss = 0.f;
        if ((r = download(h, &loss, h->mac_loss, sizeof(float)))) break;
        if ((r = check_device(h))) break;
        if (loss_per_epoch) loss_per_epoch[e] = (double)loss / n;
    }
    cudaStreamSynchronize(h->st);
    cudaFree(order);
    if (r == NB_OK) r = mac_fit_screen(h);
    h->mac_fallback = false;
    return r;
}

NB_API int32_t nb_mac_fit_screen(nb_engine* h) {
    if (!h) return NB_ERR_INVALID_ARG;
    if (!h->mac_ready) return fail(h, NB_ERR_STATE, "no learned-MAC parameters");
    cudaSetDevice(h->device);
    return mac_fit_screen(h);
}

NB_API int32_t nb_mac_get_screen(nb_engine* h, float* screen, int32_t n) {
    if (!h || !screen || n != nb::kMacScreen) return NB_ERR_INVALID_ARG;
    std::copy(h->mac_screen, h->mac_screen + nb::kMacScreen, screen);
    return NB_OK;
}

NB_API int32_t nb_mac_set_screen(nb_engine* h, const float* screen, int32_t n) {
    if (!h || !screen || n != nb::kMacScreen) return NB_ERR_INVALID_ARG;
    if (!h->mac_ready) return fail(h, NB_ERR_STATE, "no learned-MAC parameters");
    for (int k = 0; k < nb::kMacScreen - 1; k++)
        if (!std::isfinite(screen[k])) return fail(h, NB_ERR_INVALID_ARG, "screen weights must be finite");
    if (!(screen[nb::kMacScreen - 1] >= 0.f))
        return fail(h, NB_ERR_INVALID_ARG, "screen margin must be >= 0 (+inf = off)");
    cudaSetDevice(h->device);
    std::copy(screen, screen + nb::kMacScreen, h->mac_screen);
    int r = mac_upload_screen(h);
    return r ? r : check_device(h);
}

NB_API int32_t nb_mac_gradient(nb_engine* h, const float* X, const float* Y, int32_t n,
                               float* grad, double* loss) {
    if (!h || !X || !Y || !grad || n <= 0) return NB_ERR_INVALID_ARG;
    if (!h->mac_ready) return fail(h, NB_ERR_STATE, "no learned-MAC parameters");
    cudaSetDevice(h->device);
    float *dX = nullptr, *dY = nullptr;
    int* dO = nullptr;
    NB_CUDA(h, cudaMalloc(&dX, sizeof(float) * (size_t)n * (nb::kMacIn + 1) + sizeof(int) * (size_t)n));
    dY = dX + (size_t)n * nb::kMacIn;
    dO = (int*)(dY + n);
    std::vector<int> ord((size_t)n);
    for (int i = 0; i < n; i++) ord[i] = i;
    int r;
    if (!(r = upload(h, dX, X, sizeof(float) * (size_t)n * nb::kMacIn)) &&
        !(r = upload(h, dY, Y, sizeof(float) * (size_t)n)) &&
        !(r = upload(h, dO, ord.data(), sizeof(int) * (size_t)n))) {
        cudaMemsetAsync(h->mac_loss, 0, sizeof(float), h->st);
        nb::mac_grad(h->st, dX, dY, dO, 0, n, h->mac_P, h->mac_dev, h->mac_G,
                     h->mac_loss, h->sms, h->mac_part, h->scal->err);
        float l = 0.f;
        if (!(r = download(h, grad, h->mac_G, sizeof(float) * nb::kMacParams)) &&
            !(r = download(h, &l, h->mac_loss, sizeof(float))) && !(r = check_device(h)) && loss)
            *loss = (double)l / n;
    }
    cudaStreamSynchronize(h->st);
    cudaFree(dX);
    return r;
}

NB_API int32_t nb_mac_predict(nb_engine* h, const float* X, int32_t n, float* y) {
    if (!h || !X || !y || n <= 0) return NB_ERR_INVALID_ARG;
    if (!h->mac_ready) return fail(h, NB_ERR_STATE, "no learned-MAC parameters");
    cudaSetDevice(h->device);
    float* dX = nullptr;
    NB_CUDA(h, cudaMalloc(&dX, sizeof(float) * (size_t)n * (nb::kMacIn + 1)));
    int r;
    if (!(r = upload(h, dX, X, sizeof(float) * (size_t)n * nb::kMacIn))) {
        nb::mac_predict(h->st, dX, n, h->mac_dev, dX + (size_t)n * nb::kMacIn);
        if (!(r = download(h, y, dX + (size_t)n * nb::kMacIn, sizeof(float) * (size_t)n)))
            r = check_device(h);
    }
    cudaStreamSynchronize(h->st);
    cudaFree(dX);
    return r;
}

}  // extern "C"
