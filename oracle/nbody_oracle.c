/*
 * nbody_oracle.c - CPU restatement of the reference's N-body force path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests,
 * the smoke check and the benchmark's CPU-baseline leg load this library;
 * the engine never does.  Parity of this file with the reference itself is
 * pinned by tests/test_oracle_ref.py against oracle/_ref (the reference's
 * own C++ sources compiled in place) and against the reference's
 * known-answer tests.
 *
 * Built with -ffp-contract=off so that every FP64 expression rounds
 * exactly as the C# / C++ reference code does (RyuJIT does not contract
 * a*b+c into an FMA either).
 */
#include "nbody_oracle.h"

#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static void set_threads(int32_t threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

/* GravityKernel.AccelerationCoeffFromSource (GravityKernel.cs:9-33). */
static double accel_coeff(double dist_sq, double src_mass, double src_radius, double eps2,
                          int32_t shell) {
    if (!shell || src_radius <= 0.0) {
        double inv = 1.0 / sqrt(dist_sq + eps2);
        return src_mass * inv * inv * inv;
    }
    double dist = sqrt(dist_sq);
    if (dist < src_radius) {
        double denom = src_radius * src_radius + eps2;
        double inv_denom_sqrt = 1.0 / sqrt(denom);
        return src_mass * inv_denom_sqrt / denom;
    }
    double inv = 1.0 / sqrt(dist_sq + eps2);
    return src_mass * inv * inv * inv;
}

/* Body i of CpuParallelBackend.ComputeForces (CpuParallelBackend.cs:99-142):
 * sequential j order, skip self and inactive sources. */
static void direct_one(int32_t i, int32_t n, const double* px, const double* py,
                       const double* pz, const double* m, const double* radius,
                       const uint8_t* active, double eps2, int32_t shell, double* oax,
                       double* oay, double* oaz) {
    double xi = px[i], yi = py[i], zi = pz[i];
    double axi = 0.0, ayi = 0.0, azi = 0.0;
    for (int32_t j = 0; j < n; j++) {
        if (j == i || !active[j]) continue;
        double dx = xi - px[j];
        double dy = yi - py[j];
        double dz = zi - pz[j];
        double raw = dx * dx + dy * dy + dz * dz;
        double c = accel_coeff(raw, m[j], radius ? radius[j] : 0.0, eps2, shell);
        axi -= c * dx;
        ayi -= c * dy;
        azi -= c * dz;
    }
    *oax = axi;
    *oay = ayi;
    *oaz = azi;
}

void or_direct_forces(int32_t n, const double* px, const double* py, const double* pz,
                      const double* m, const double* radius, const uint8_t* active,
                      double eps, int32_t shell, double* ax, double* ay, double* az,
                      int32_t threads) {
    double eps2 = eps * eps;
    set_threads(threads);
    /* Array.Clear of the acceleration buffers (CpuParallelBackend.cs:92-94). */
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) {
            ax[i] = ay[i] = az[i] = 0.0;
            continue;
        }
        direct_one(i, n, px, py, pz, m, radius, active, eps2, shell, &ax[i], &ay[i], &az[i]);
    }
}

void or_direct_forces_targets(int32_t n, const double* px, const double* py, const double* pz,
                              const double* m, const double* radius, const uint8_t* active,
                              double eps, int32_t shell, int32_t n_t, const int32_t* targets,
                              double* ax, double* ay, double* az, int32_t threads) {
    double eps2 = eps * eps;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int32_t t = 0; t < n_t; t++) {
        int32_t i = targets[t];
        if (!active[i]) {
            ax[t] = ay[t] = az[t] = 0.0;
            continue;
        }
        direct_one(i, n, px, py, pz, m, radius, active, eps2, shell, &ax[t], &ay[t], &az[t]);
    }
}

/* SimdSingleThreadBackend.ComputeForces (SimdSingleThreadBackend.cs:43-165):
 * sources in chunks of Vector<double>.Count lanes (4: 256-bit vectors), per
 * lane dist2 = ((dx*dx + dy*dy) + dz*dz) + eps2, invDist = 1 / sqrt(dist2),
 * invDist3 = (invDist*invDist)*invDist, factor = m_j * invDist3 (not the
 * ((m*inv)*inv)*inv of GravityKernel); the lanes are then subtracted from
 * the scalar sums in lane order (self and inactive lanes skipped), the tail
 * runs the same arithmetic in scalar code.  The lane width therefore does
 * not change a single bit.  The same arithmetic and order are the native
 * engine's CPU brute force (Engine::compute_cpu_brute_forces, global
 * softening, engine/src/sim/engine.cpp:649-674).  With the shell theorem the
 * backend runs CpuSingleThreadBackend's shell loop, whose arithmetic is
 * CpuParallelBackend's. */
#define OR_SIMD_LANES 4
void or_direct_forces_simd(int32_t n, const double* px, const double* py, const double* pz,
                           const double* m, const double* radius, const uint8_t* active,
                           double eps, int32_t shell, double* ax, double* ay, double* az,
                           int32_t threads) {
    if (shell) {
        or_direct_forces(n, px, py, pz, m, radius, active, eps, 1, ax, ay, az, threads);
        return;
    }
    const double eps2 = eps * eps;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < n; i++) {
        ax[i] = ay[i] = az[i] = 0.0;
        if (!active[i]) continue;
        const double xi = px[i], yi = py[i], zi = pz[i];
        double axi = 0.0, ayi = 0.0, azi = 0.0;
        int32_t j = 0;
        const int32_t vec_limit = n - (n % OR_SIMD_LANES);
        for (; j < vec_limit; j += OR_SIMD_LANES) {
            double fx[OR_SIMD_LANES], fdx[OR_SIMD_LANES], fdy[OR_SIMD_LANES], fdz[OR_SIMD_LANES];
            for (int k = 0; k < OR_SIMD_LANES; k++) {
                const double dx = xi - px[j + k], dy = yi - py[j + k], dz = zi - pz[j + k];
                const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
                const double inv = 1.0 / sqrt(dist2);
                const double inv3 = inv * inv * inv;
                fx[k] = m[j + k] * inv3;
                fdx[k] = dx;
                fdy[k] = dy;
                fdz[k] = dz;
            }
            for (int k = 0; k < OR_SIMD_LANES; k++) {
                const int32_t jk = j + k;
                if (jk == i || !active[jk]) continue;
                axi -= fx[k] * fdx[k];
                ayi -= fx[k] * fdy[k];
                azi -= fx[k] * fdz[k];
            }
        }
        for (; j < n; j++) {
            if (j == i || !active[j]) continue;
            const double dx = xi - px[j], dy = yi - py[j], dz = zi - pz[j];
            const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            const double inv = 1.0 / sqrt(dist2);
            const double inv3 = inv * inv * inv;
            const double f = m[j] * inv3;
            axi -= f * dx;
            ayi -= f * dy;
            azi -= f * dz;
        }
        ax[i] = axi;
        ay[i] = ayi;
        az[i] = azi;
    }
}

/* CpuSingleThreadBackend.ComputeForces (CpuSingleThreadBackend.cs:50-159).
 * Without the shell theorem: the O(n^2/2) Newton's-third-law loop - for
 * each active i and each active j > i one factor pair m_j*invDist3,
 * m_i*invDist3 (invDist3 = (inv*inv)*inv); i's sum over j > i is kept in a
 * register and added to ax[i] at the end of row i, while j receives
 * +m_i*invDist3*dx directly in ax[j] during earlier rows.  So a body's
 * acceleration is (sum over lower partners, in order) + (sum over higher
 * partners, in order): a different summation order from CpuParallel's single
 * running sum.  With the shell theorem: the CpuParallel loop. Serial. */
void or_direct_forces_pairwise(int32_t n, const double* px, const double* py, const double* pz,
                               const double* m, const double* radius, const uint8_t* active,
                               double eps, int32_t shell, double* ax, double* ay, double* az) {
    if (shell) {
        or_direct_forces(n, px, py, pz, m, radius, active, eps, 1, ax, ay, az, 1);
        return;
    }
    const double eps2 = eps * eps;
    for (int32_t i = 0; i < n; i++) ax[i] = ay[i] = az[i] = 0.0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        const double xi = px[i], yi = py[i], zi = pz[i], mi = m[i];
        double axi = 0.0, ayi = 0.0, azi = 0.0;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j]) continue;
            const double dx = xi - px[j], dy = yi - py[j], dz = zi - pz[j];
            const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            const double inv = 1.0 / sqrt(dist2);
            const double inv3 = inv * inv * inv;
            const double f_ij = m[j] * inv3, f_ji = mi * inv3;
            axi -= f_ij * dx;
            ayi -= f_ij * dy;
            azi -= f_ij * dz;
            ax[j] += f_ji * dx;
            ay[j] += f_ji * dy;
            az[j] += f_ji * dz;
        }
        ax[i] += axi;
        ay[i] += ayi;
        az[i] += azi;
    }
}

/* One of the three direct-sum orders: 0 CpuParallelBackend, 1 the SIMD
 * backend / native engine, 2 CpuSingleThreadBackend. */
void or_direct_forces_order(int32_t n, const double* px, const double* py, const double* pz,
                            const double* m, const double* radius, const uint8_t* active,
                            double eps, int32_t shell, int32_t order, double* ax, double* ay,
                            double* az, int32_t threads) {
    if (order == 1)
        or_direct_forces_simd(n, px, py, pz, m, radius, active, eps, shell, ax, ay, az, threads);
    else if (order == 2)
        or_direct_forces_pairwise(n, px, py, pz, m, radius, active, eps, shell, ax, ay, az);
    else
        or_direct_forces(n, px, py, pz, m, radius, active, eps, shell, ax, ay, az, threads);
}

/* Bounding box over active bodies (BarnesHutBackend.cs:150-170). */
void or_bbox(int32_t n, const double* px, const double* py, const double* pz,
             const uint8_t* active, double* out6) {
    double mnx = 1.7976931348623157e308, mny = mnx, mnz = mnx;
    double mxx = -1.7976931348623157e308, mxy = mxx, mxz = mxx;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        if (px[i] < mnx) mnx = px[i];
        if (py[i] < mny) mny = py[i];
        if (pz[i] < mnz) mnz = pz[i];
        if (px[i] > mxx) mxx = px[i];
        if (py[i] > mxy) mxy = py[i];
        if (pz[i] > mxz) mxz = pz[i];
    }
    out6[0] = mnx; out6[1] = mny; out6[2] = mnz;
    out6[3] = mxx; out6[4] = mxy; out6[5] = mxz;
}

/* Cube with margin (octree_builder.cpp:29-35; gpu_tree.cu:163-167). */
void or_cube_from_bbox(const double* b, double* cube4) {
    double cx = (b[0] + b[3]) * 0.5;
    double cy = (b[1] + b[4]) * 0.5;
    double cz = (b[2] + b[5]) * 0.5;
    double ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
    double e = ex;
    if (ey > e) e = ey;
    if (ez > e) e = ez;
    double h = e * 0.5;
    if (h < 1e-10) h = 1e-10;
    h *= 1.001;
    cube4[0] = cx; cube4[1] = cy; cube4[2] = cz; cube4[3] = h;
}

/* expand_bits_21 (engine/include/celestial/cuda/morton.hpp:13-21). */
uint64_t or_expand_bits_21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

static uint64_t encode3(uint64_t x, uint64_t y, uint64_t z) {
    return (or_expand_bits_21(x) << 2) | (or_expand_bits_21(y) << 1) | or_expand_bits_21(z);
}

static double clamp01(double u) { return fmax(0.0, fmin(1.0, u)); }

/* morton_code_kernel + launch_morton_codes (morton_kernel.cu:11-76) and
 * morton_from_unit (morton.hpp:29-35): per-axis AABB, scale 2^21-1,
 * truncation. */
void or_morton_aabb(int32_t n, const double* px, const double* py, const double* pz,
                    const uint8_t* active, const double* b, uint64_t* keys, int32_t* idx) {
    double rx = b[3] - b[0], ry = b[4] - b[1], rz = b[5] - b[2];
    double ix = (rx > 1e-30) ? 1.0 / rx : 0.0;
    double iy = (ry > 1e-30) ? 1.0 / ry : 0.0;
    double iz = (rz > 1e-30) ? 1.0 / rz : 0.0;
    const double scale = 2097151.0;
    for (int32_t i = 0; i < n; i++) {
        idx[i] = i;
        if (!active[i]) {
            keys[i] = ~0ull;
            continue;
        }
        double ux = clamp01((px[i] - b[0]) * ix);
        double uy = clamp01((py[i] - b[1]) * iy);
        double uz = clamp01((pz[i] - b[2]) * iz);
        keys[i] = encode3((uint64_t)(ux * scale), (uint64_t)(uy * scale), (uint64_t)(uz * scale));
    }
}

/* Octree-aligned quantisation: bit (20-l) of q is the level-(l+1) octant
 * bit of OctreeNode::octant_for (octree_node.hpp:53-59) up to rounding at
 * cell planes. */
static uint64_t quant_cube(double p, double lo, double inv2h) {
    double u = clamp01((p - lo) * inv2h);
    uint64_t q = (uint64_t)(u * 2097152.0);
    return q > 2097151ull ? 2097151ull : q;
}

void or_morton_cube(int32_t n, const double* px, const double* py, const double* pz,
                    const uint8_t* active, const double* c, uint64_t* keys, int32_t* idx) {
    double inv2h = 1.0 / (2.0 * c[3]);
    double lx = c[0] - c[3], ly = c[1] - c[3], lz = c[2] - c[3];
    for (int32_t i = 0; i < n; i++) {
        idx[i] = i;
        if (!active[i]) {
            keys[i] = ~0ull;
            continue;
        }
        keys[i] = encode3(quant_cube(px[i], lx, inv2h), quant_cube(py[i], ly, inv2h),
                          quant_cube(pz[i], lz, inv2h));
    }
}

/* Stable LSD radix sort, 8 bits x 8 passes. */
void or_stable_sort(int32_t n, uint64_t* keys, int32_t* values) {
    if (n <= 1) return;
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int32_t* v2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    uint64_t* ks = keys;
    int32_t* vs = values;
    uint64_t* kd = k2;
    int32_t* vd = v2;
    for (int pass = 0; pass < 8; pass++) {
        int shift = pass * 8;
        size_t count[257];
        memset(count, 0, sizeof(count));
        for (int32_t i = 0; i < n; i++) count[((ks[i] >> shift) & 0xFF) + 1]++;
        for (int d = 0; d < 256; d++) count[d + 1] += count[d];
        for (int32_t i = 0; i < n; i++) {
            size_t p = count[(ks[i] >> shift) & 0xFF]++;
            kd[p] = ks[i];
            vd[p] = vs[i];
        }
        uint64_t* tk = ks; ks = kd; kd = tk;
        int32_t* tv = vs; vs = vd; vd = tv;
    }
    /* 8 passes: result is back in the caller's arrays. */
    free(k2);
    free(v2);
}

/* ---- point-region octree by insertion (octree_builder.cpp:8-135) ------ */

typedef struct {
    double* c4;
    double* mass;
    double* com;
    int32_t* ch;
    int32_t* body;
    uint8_t* leaf;
    int32_t count, cap;
    double min_node_size;
    int overflow;
} pool_t;

static int32_t pool_alloc(pool_t* p, double cx, double cy, double cz, double h) {
    if (p->count >= p->cap) {
        p->overflow = 1;
        return -1;
    }
    int32_t k = p->count++;
    p->c4[4 * k + 0] = cx; p->c4[4 * k + 1] = cy; p->c4[4 * k + 2] = cz; p->c4[4 * k + 3] = h;
    p->mass[k] = 0.0;
    p->com[3 * k] = p->com[3 * k + 1] = p->com[3 * k + 2] = 0.0;
    for (int o = 0; o < 8; o++) p->ch[8 * k + o] = -1;
    p->body[k] = -1;
    p->leaf[k] = 0;
    return k;
}

/* OctreeBuilder::update_mass (octree_builder.cpp:124-133). */
static void update_mass(pool_t* p, int32_t k, double bm, double bx, double by, double bz) {
    double nm = p->mass[k] + bm;
    if (nm > 0.0) {
        double inv = 1.0 / nm;
        p->com[3 * k + 0] = (p->com[3 * k + 0] * p->mass[k] + bx * bm) * inv;
        p->com[3 * k + 1] = (p->com[3 * k + 1] * p->mass[k] + by * bm) * inv;
        p->com[3 * k + 2] = (p->com[3 * k + 2] * p->mass[k] + bz * bm) * inv;
    }
    p->mass[k] = nm;
}

static void insert_body(pool_t* p, int32_t k, int32_t bi, double bx, double by, double bz,
                        double bm);

/* OctreeBuilder::insert_into_child (octree_builder.cpp:107-122),
 * OctreeNode::octant_for / child_center (octree_node.hpp:53-67). */
static void insert_into_child(pool_t* p, int32_t k, int32_t bi, double bx, double by,
                              double bz, double bm) {
    const double* c = &p->c4[4 * k];
    int oct = 0;
    if (bx >= c[0]) oct |= 1;
    if (by >= c[1]) oct |= 2;
    if (bz >= c[2]) oct |= 4;
    int32_t child = p->ch[8 * k + oct];
    if (child == -1) {
        double q = c[3] * 0.5;
        double ccx = c[0] + ((oct & 1) ? q : -q);
        double ccy = c[1] + ((oct & 2) ? q : -q);
        double ccz = c[2] + ((oct & 4) ? q : -q);
        child = pool_alloc(p, ccx, ccy, ccz, c[3] * 0.5);
        if (child < 0) return;
        p->ch[8 * k + oct] = child;
    }
    insert_body(p, child, bi, bx, by, bz, bm);
}

/* OctreeBuilder::insert_body (octree_builder.cpp:50-105). */
static void insert_body(pool_t* p, int32_t k, int32_t bi, double bx, double by, double bz,
                        double bm) {
    if (p->overflow) return;
    if (p->mass[k] == 0.0 && p->body[k] == -1) {
        p->body[k] = bi;
        p->leaf[k] = 1;
        p->mass[k] = bm;
        p->com[3 * k] = bx; p->com[3 * k + 1] = by; p->com[3 * k + 2] = bz;
        return;
    }
    if (p->leaf[k]) {
        if (p->c4[4 * k + 3] * 0.5 < p->min_node_size) {
            double total = p->mass[k] + bm;
            p->com[3 * k + 0] = (p->com[3 * k + 0] * p->mass[k] + bx * bm) / total;
            p->com[3 * k + 1] = (p->com[3 * k + 1] * p->mass[k] + by * bm) / total;
            p->com[3 * k + 2] = (p->com[3 * k + 2] * p->mass[k] + bz * bm) / total;
            p->mass[k] = total;
            return;
        }
        int32_t eb = p->body[k];
        double em = p->mass[k];
        double ex = p->com[3 * k], ey = p->com[3 * k + 1], ez = p->com[3 * k + 2];
        p->body[k] = -1;
        p->leaf[k] = 0;
        p->mass[k] = 0.0;
        p->com[3 * k] = p->com[3 * k + 1] = p->com[3 * k + 2] = 0.0;
        insert_into_child(p, k, eb, ex, ey, ez, em);
        insert_into_child(p, k, bi, bx, by, bz, bm);
        update_mass(p, k, em, ex, ey, ez);
        update_mass(p, k, bm, bx, by, bz);
        return;
    }
    insert_into_child(p, k, bi, bx, by, bz, bm);
    update_mass(p, k, bm, bx, by, bz);
}

int32_t or_octree_build(int32_t n, const double* px, const double* py, const double* pz,
                        const double* m, const uint8_t* active, double min_node_size,
                        int32_t cap, double* center4, double* mass, double* com3,
                        int32_t* children8, int32_t* body, uint8_t* is_leaf) {
    pool_t p = {center4, mass, com3, children8, body, is_leaf, 0, cap, min_node_size, 0};
    if (n <= 0) return 0;
    double b[6], c[4];
    or_bbox(n, px, py, pz, active, b);
    or_cube_from_bbox(b, c);
    int32_t root = pool_alloc(&p, c[0], c[1], c[2], c[3]);
    if (root < 0) return -1;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        insert_body(&p, root, i, px[i], py[i], pz[i], m[i]);
        if (p.overflow) return -1;
    }
    return p.count;
}

/* BarnesHutSolver::compute_force_on_body (barnes_hut_solver.cpp:230-286);
 * leaves use GravityKernel with the shell theorem when `shell`
 * (BarnesHutBackend.cs:410-424). */
static void bh_body(const pool_t* p, int32_t k, int32_t bi, double bx, double by, double bz,
                    const double* radius, double eps2, double theta2, int32_t shell,
                    double* ax, double* ay, double* az) {
    double nm = p->mass[k];
    if (nm == 0.0) return;
    double dx = bx - p->com[3 * k];
    double dy = by - p->com[3 * k + 1];
    double dz = bz - p->com[3 * k + 2];
    double d2 = dx * dx + dy * dy + dz * dz;
    if (p->leaf[k]) {
        if (p->body[k] == bi) return;
        double f;
        if (shell) {
            double r = p->body[k] >= 0 && radius ? radius[p->body[k]] : 0.0;
            f = accel_coeff(d2, nm, r, eps2, 1);
        } else {
            double inv = 1.0 / sqrt(d2 + eps2);
            double inv3 = inv * inv * inv;
            f = nm * inv3;
        }
        *ax -= f * dx;
        *ay -= f * dy;
        *az -= f * dz;
        return;
    }
    double h = p->c4[4 * k + 3];
    double s2 = 4.0 * h * h;
    if (d2 > 0.0 && s2 < theta2 * d2) {
        double inv = 1.0 / sqrt(d2 + eps2);
        double inv3 = inv * inv * inv;
        double f = nm * inv3;
        *ax -= f * dx;
        *ay -= f * dy;
        *az -= f * dz;
        return;
    }
    for (int o = 0; o < 8; o++) {
        int32_t c = p->ch[8 * k + o];
        if (c != -1) bh_body(p, c, bi, bx, by, bz, radius, eps2, theta2, shell, ax, ay, az);
    }
}

void or_bh_forces(int32_t n, const double* px, const double* py, const double* pz,
                  const double* radius, const uint8_t* active, double eps, double theta,
                  int32_t shell, const double* center4, const double* mass, const double* com3,
                  const int32_t* children8, const int32_t* body, const uint8_t* is_leaf,
                  double* ax, double* ay, double* az, int32_t threads) {
    pool_t p = {(double*)center4, (double*)mass, (double*)com3, (int32_t*)children8,
                (int32_t*)body, (uint8_t*)is_leaf, 0, 0, 0.0, 0};
    double te = theta < 0.2 ? 0.2 : theta;
    double eps2 = eps * eps, theta2 = te * te;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t i = 0; i < n; i++) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (active[i]) bh_body(&p, 0, i, px[i], py[i], pz[i], radius, eps2, theta2, shell, &a0, &a1, &a2);
        ax[i] = a0;
        ay[i] = a1;
        az[i] = a2;
    }
}

/* build_active_mask_kernel + exclusive scan (compact_kernel.cu:31-40,191-256). */
int32_t or_compact_indices(int32_t n, const uint8_t* active, const double* mass, int32_t* dest) {
    int32_t w = 0;
    for (int32_t i = 0; i < n; i++) dest[i] = (active[i] && mass[i] > 0.0) ? w++ : -1;
    return w;
}

/* Overlap test of broad_phase_collision_kernel (collision_kernel.cu:40-52),
 * applied to every pair; (lo, hi) order of CollisionResolver::sort_pairs. */
int32_t or_broad_phase(int32_t n, const double* px, const double* py, const double* pz,
                       const double* radius, const uint8_t* active, const uint8_t* collidable,
                       int32_t max_pairs, int32_t* lo, int32_t* hi) {
    int32_t cnt = 0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i] || (collidable && !collidable[i])) continue;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j] || (collidable && !collidable[j])) continue;
            double dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
            double d2 = dx * dx + dy * dy + dz * dz;
            double sr = radius[i] + radius[j];
            if (d2 < sr * sr) {
                if (cnt < max_pairs) {
                    lo[cnt] = i;
                    hi[cnt] = j;
                }
                cnt++;
            }
        }
    }
    return cnt;
}

/* The same pair list as or_broad_phase (the all-pairs test of
 * collision_kernel.cu:40-52, pairs in (lo, hi) lexicographic order), with the
 * rows split over OpenMP threads: a counting pass, an exclusive scan of the
 * row counts, then a filling pass.  For config-size inputs. */
int32_t or_broad_phase_parallel(int32_t n, const double* px, const double* py, const double* pz,
                                const double* radius, const uint8_t* active,
                                const uint8_t* collidable, int32_t max_pairs, int32_t* lo,
                                int32_t* hi, int32_t threads) {
    int64_t* start = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t i = 0; i < n; i++) {
        if (!active[i] || (collidable && !collidable[i])) continue;
        int64_t c = 0;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j] || (collidable && !collidable[j])) continue;
            double dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
            double d2 = dx * dx + dy * dy + dz * dz;
            double sr = radius[i] + radius[j];
            if (d2 < sr * sr) c++;
        }
        start[i + 1] = c;
    }
    for (int32_t i = 0; i < n; i++) start[i + 1] += start[i];
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t i = 0; i < n; i++) {
        int64_t k = start[i];
        if (k == start[i + 1]) continue;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j] || (collidable && !collidable[j])) continue;
            double dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
            double d2 = dx * dx + dy * dy + dz * dz;
            double sr = radius[i] + radius[j];
            if (d2 < sr * sr) {
                if (k < max_pairs) {
                    lo[k] = i;
                    hi[k] = j;
                }
                k++;
            }
        }
    }
    const int64_t total = start[n];
    free(start);
    return total > 2147483647 ? 2147483647 : (int32_t)total;
}

/* DensityModel (density_model.cpp:10-22). */
static double dm_density(double mass, double radius, double min_radius) {
    double r = (radius > min_radius) ? radius : min_radius;
    double volume = (4.0 / 3.0) * M_PI * r * r * r;
    if (volume < 1e-30) return 0.0;
    return mass / volume;
}
static double dm_radius(double mass, double density, double min_radius) {
    if (density < 1e-30 || mass < 1e-30) return min_radius;
    double r = cbrt(3.0 * mass / (4.0 * M_PI * density));
    return (r > min_radius) ? r : min_radius;
}

/* CollisionResolver::resolve (Merge mode) + resolve_merge
 * (collision_resolver.cpp:20-100, 190-250). */
int32_t or_resolve_merges(int32_t n, double* px, double* py, double* pz, double* vx,
                          double* vy, double* vz, double* m, double* radius, double* density,
                          uint8_t* active, int32_t n_pairs, const int32_t* lo, const int32_t* hi,
                          int32_t max_per_frame, int32_t max_per_body, int32_t density_merge,
                          double min_radius) {
    int32_t* counts = (int32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
    int32_t total = 0;
    for (int32_t k = 0; k < n_pairs; k++) {
        int32_t a = lo[k], b = hi[k];
        if (!active[a] || !active[b]) continue;
        if (total >= max_per_frame) continue;
        if (counts[a] >= max_per_body || counts[b] >= max_per_body) continue;
        double ma = m[a], mb = m[b], M = ma + mb;
        if (!(M < 1e-30)) {
            double vxm = (ma * vx[a] + mb * vx[b]) / M;
            double vym = (ma * vy[a] + mb * vy[b]) / M;
            double vzm = (ma * vz[a] + mb * vz[b]) / M;
            double pxm = (ma * px[a] + mb * px[b]) / M;
            double pym = (ma * py[a] + mb * py[b]) / M;
            double pzm = (ma * pz[a] + mb * pz[b]) / M;
            int32_t s = (ma >= mb) ? a : b;
            int32_t v = (ma >= mb) ? b : a;
            double rm;
            if (density_merge && density) {
                double sd = density[s];
                if (sd < 1e-30) sd = dm_density(m[s], radius[s], min_radius);
                rm = dm_radius(M, sd, min_radius);
            } else {
                double ra3 = radius[a] * radius[a] * radius[a];
                double rb3 = radius[b] * radius[b] * radius[b];
                rm = cbrt(ra3 + rb3);
            }
            px[s] = pxm; py[s] = pym; pz[s] = pzm;
            vx[s] = vxm; vy[s] = vym; vz[s] = vzm;
            m[s] = M;
            radius[s] = rm;
            if (density) density[s] = dm_density(M, rm, min_radius);
            active[v] = 0;
        }
        int32_t surv = (m[a] > 0 && active[a]) ? a : b;
        counts[surv]++;
        total++;
    }
    free(counts);
    return total;
}

/* SoAVerletIntegrator.Step (SoAVerletIntegrator.cs:48-116) with a direct
 * sum of the given order (or_direct_forces_order) as the backend.  With
 * order 1 this is also the native engine's CPU brute-force Leapfrog step
 * (Engine::step_cpu_brute_force, engine/src/sim/engine.cpp:753-800: half
 * kick with the previous acceleration, drift, forces, half kick, rotate). */
void or_verlet_direct_order(int32_t n, double* px, double* py, double* pz, double* vx,
                            double* vy, double* vz, double* ax, double* ay, double* az,
                            const double* m, const uint8_t* active, double eps, double dt,
                            int32_t steps, int32_t order, int32_t threads) {
    double half = 0.5 * dt;
    double* nx = (double*)malloc(sizeof(double) * (size_t)n * 3);
    double* ny = nx + n;
    double* nz = ny + n;
    for (int32_t s = 0; s < steps; s++) {
        for (int32_t i = 0; i < n; i++) {
            if (!active[i]) continue;
            vx[i] += half * ax[i];
            vy[i] += half * ay[i];
            vz[i] += half * az[i];
        }
        for (int32_t i = 0; i < n; i++) {
            if (!active[i]) continue;
            px[i] += dt * vx[i];
            py[i] += dt * vy[i];
            pz[i] += dt * vz[i];
        }
        or_direct_forces_order(n, px, py, pz, m, NULL, active, eps, 0, order, nx, ny, nz,
                               threads);
        for (int32_t i = 0; i < n; i++) {
            if (!active[i]) continue;
            vx[i] += half * nx[i];
            vy[i] += half * ny[i];
            vz[i] += half * nz[i];
        }
        memcpy(ax, nx, sizeof(double) * (size_t)n);
        memcpy(ay, ny, sizeof(double) * (size_t)n);
        memcpy(az, nz, sizeof(double) * (size_t)n);
    }
    free(nx);
}

/* SoAVerletIntegrator.Step with the CpuParallelBackend direct sum. */
void or_verlet_direct(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                      double* vz, double* ax, double* ay, double* az, const double* m,
                      const uint8_t* active, double eps, double dt, int32_t steps,
                      int32_t threads) {
    or_verlet_direct_order(n, px, py, pz, vx, vy, vz, ax, ay, az, m, active, eps, dt, steps, 0,
                           threads);
}

/* Engine::step_yoshida4_cpu_brute_force (engine/src/sim/engine.cpp:1057-1066):
 * per step, three Engine::cpu_yoshida_substep calls (engine.cpp:685-746:
 * half kick with the previous acceleration, drift, forces, half kick,
 * rotate) with sub_dt = SUB_DT[s] * dt, SUB_DT = {w1, w0, w1} of
 * YoshidaCoefficients (engine/include/celestial/sim/yoshida.hpp:19-24);
 * each sub-step is the Verlet step above, with the direct sum as forces. */
void or_yoshida_direct_order(int32_t n, double* px, double* py, double* pz, double* vx,
                             double* vy, double* vz, double* ax, double* ay, double* az,
                             const double* m, const uint8_t* active, double eps, double dt,
                             int32_t steps, int32_t order, int32_t threads) {
    const double cbrt2 = 1.2599210498948732;
    const double w1 = 1.0 / (2.0 - cbrt2);
    const double w0 = -cbrt2 / (2.0 - cbrt2);
    const double sub[3] = {w1, w0, w1};
    for (int32_t s = 0; s < steps; s++)
        for (int k = 0; k < 3; k++)
            or_verlet_direct_order(n, px, py, pz, vx, vy, vz, ax, ay, az, m, active, eps,
                                   sub[k] * dt, 1, order, threads);
}

void or_yoshida_direct(int32_t n, double* px, double* py, double* pz, double* vx, double* vy,
                       double* vz, double* ax, double* ay, double* az, const double* m,
                       const uint8_t* active, double eps, double dt, int32_t steps,
                       int32_t threads) {
    or_yoshida_direct_order(n, px, py, pz, vx, vy, vz, ax, ay, az, m, active, eps, dt, steps, 0,
                            threads);
}

/* AdaptiveTimestep::compute_dt (engine/src/sim/adaptive_timestep.cpp:12-17)
 * from Engine::compute_max_acceleration's CPU loop (engine/src/sim/
 * engine.cpp:491-501): the next dt after a step. */
double or_adaptive_dt(int32_t n, const double* ax, const double* ay, const double* az,
                      const uint8_t* active, double eps, double eta, double dt_min,
                      double dt_max) {
    double max_a2 = 0.0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        const double a2 = ax[i] * ax[i] + ay[i] * ay[i] + az[i] * az[i];
        if (a2 > max_a2) max_a2 = a2;
    }
    const double a_max = sqrt(max_a2);
    if (a_max <= 0.0 || eps <= 0.0) return dt_max;
    const double v = eta * sqrt(eps / a_max);
    return v < dt_min ? dt_min : (v > dt_max ? dt_max : v);
}

/* EnergyCalculator.ComputeKE/ComputePE/ComputeMomentum/ComputeAngularMomentum
 * (EnergyCalculator.cs:16-78); pair PE of NewtonianGravity.cs:68-77. */
void or_energy(int32_t n, const double* px, const double* py, const double* pz,
               const double* vx, const double* vy, const double* vz, const double* m,
               const uint8_t* active, double eps, double* o, int32_t threads) {
    double ke = 0, P[3] = {0, 0, 0}, L[3] = {0, 0, 0}, C[3] = {0, 0, 0}, M = 0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        double v2 = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
        ke += 0.5 * m[i] * v2;
        double mvx = vx[i] * m[i], mvy = vy[i] * m[i], mvz = vz[i] * m[i];
        P[0] += mvx; P[1] += mvy; P[2] += mvz;
        L[0] += py[i] * mvz - pz[i] * mvy;
        L[1] += pz[i] * mvx - px[i] * mvz;
        L[2] += px[i] * mvy - py[i] * mvx;
        C[0] += m[i] * px[i]; C[1] += m[i] * py[i]; C[2] += m[i] * pz[i];
        M += m[i];
    }
    double eps2 = eps * eps;
    double* row = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        double s = 0.0;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j]) continue;
            double rx = px[j] - px[i], ry = py[j] - py[i], rz = pz[j] - pz[i];
            double d2 = rx * rx + ry * ry + rz * rz + eps2;
            s += -1.0 * m[i] * m[j] / sqrt(d2);
        }
        row[i] = s;
    }
    double pe = 0.0;
    for (int32_t i = 0; i < n; i++) pe += row[i];
    free(row);
    o[0] = ke; o[1] = pe; o[2] = ke + pe;
    o[3] = P[0]; o[4] = P[1]; o[5] = P[2];
    o[6] = L[0]; o[7] = L[1]; o[8] = L[2];
    o[9] = M > 0 ? C[0] / M : 0; o[10] = M > 0 ? C[1] / M : 0; o[11] = M > 0 ? C[2] / M : 0;
    o[12] = M;
}

/* The native engine's EnergyTracker::compute (engine/src/profile/
 * energy_tracker.cpp:8-90): one pass over the active bodies for KE
 * (0.5*m*v2), momentum m*v, angular momentum m*(r x v), total mass and the
 * mass-weighted position sums, then the pair potential -m_i*m_j/sqrt(r2+eps2)
 * subtracted from one running total in (i, j > i) order.  out13 as
 * or_energy's. */
void or_energy_tracker(int32_t n, const double* px, const double* py, const double* pz,
                       const double* vx, const double* vy, const double* vz, const double* m,
                       const uint8_t* active, double eps, double* o) {
    const double eps2 = eps * eps;
    double ke = 0, P[3] = {0, 0, 0}, L[3] = {0, 0, 0}, C[3] = {0, 0, 0}, M = 0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        const double mi = m[i];
        const double vxi = vx[i], vyi = vy[i], vzi = vz[i];
        const double pxi = px[i], pyi = py[i], pzi = pz[i];
        const double v2 = vxi * vxi + vyi * vyi + vzi * vzi;
        ke += 0.5 * mi * v2;
        P[0] += mi * vxi;
        P[1] += mi * vyi;
        P[2] += mi * vzi;
        L[0] += mi * (pyi * vzi - pzi * vyi);
        L[1] += mi * (pzi * vxi - pxi * vzi);
        L[2] += mi * (pxi * vyi - pyi * vxi);
        M += mi;
        C[0] += mi * pxi;
        C[1] += mi * pyi;
        C[2] += mi * pzi;
    }
    double pe = 0.0;
    for (int32_t i = 0; i < n; i++) {
        if (!active[i]) continue;
        for (int32_t j = i + 1; j < n; j++) {
            if (!active[j]) continue;
            const double dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
            const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            pe -= m[i] * m[j] / sqrt(dist2);
        }
    }
    o[0] = ke; o[1] = pe; o[2] = ke + pe;
    o[3] = P[0]; o[4] = P[1]; o[5] = P[2];
    o[6] = L[0]; o[7] = L[1]; o[8] = L[2];
    o[9] = M > 0 ? C[0] / M : 0; o[10] = M > 0 ? C[1] / M : 0; o[11] = M > 0 ? C[2] / M : 0;
    o[12] = M;
}

/* ForceErrorAnalyzer.CompareForces statistics (ForceErrorAnalyzer.cs:100-134). */
int32_t or_force_error(int32_t n, const double* ax, const double* ay, const double* az,
                       const double* rx, const double* ry, const double* rz,
                       const uint8_t* active, double* out3) {
    double s = 0, s2 = 0, mx = 0;
    int32_t c = 0;
    for (int32_t i = 0; i < n; i++) {
        if (active && !active[i]) continue;
        double em = sqrt(rx[i] * rx[i] + ry[i] * ry[i] + rz[i] * rz[i]);
        if (em < 1e-30) continue;
        double dx = ax[i] - rx[i], dy = ay[i] - ry[i], dz = az[i] - rz[i];
        double e = sqrt(dx * dx + dy * dy + dz * dz) / em;
        s += e;
        s2 += e * e;
        if (e > mx) mx = e;
        c++;
    }
    out3[0] = c ? s / c : 0;
    out3[1] = mx;
    out3[2] = c ? sqrt(s2 / c) : 0;
    return c;
}
