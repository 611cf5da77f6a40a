// common.cuh - shared device helpers of the B200 N-body engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nbody_b200.h"

namespace nb {

// 1/sqrt(x), one approximate MUFU instruction with denormal inputs flushed to
// zero (the pair kernels only pass r^2 + eps^2, far from the denormal range,
// or guard r^2 = 0 themselves).
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Packed pairs of FP32 values (sm_100 f32x2 arithmetic): one instruction
// applies the same IEEE-rounded operation to both halves.
using f32x2 = unsigned long long;
__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Batched systems: keys = system (12 bits, bits 62..51) | 3 x 17-bit Morton.
constexpr int kEnsSysShift = 51;
constexpr int kEnsSysBits = 12;
constexpr int kEnsAxisBits = 17;

constexpr int kSMs = 148;            // B200; the launch code queries the real count
constexpr int kWarp = 32;
constexpr uint64_t kInactiveKey = ~0ull;
// Iteration cap of every device spin-wait; past it the waiter records
// NB_ERR_TIMEOUT in the handle's error word and gives up.
constexpr uint32_t kSpinLimit = 1u << 22;

// Device error word layout: one int per status, set to 1 by atomicExch.
enum DevErr { kErrTimeout = 0, kErrOverflow = 1, kErrCapacity = 2, kErrNonFinite = 3, kErrCount = 4 };

__device__ __forceinline__ void dev_flag(int* err, int which) {
    if (err) atomicExch(err + which, 1);
}

// Order-preserving bijection double <-> uint64 (total order of finite values),
// so that min/max of doubles become integer atomicMin/atomicMax: exact and
// independent of the order in which blocks arrive.
__device__ __forceinline__ unsigned long long dbl_to_ord(double x) {
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_to_dbl(unsigned long long u) {
    u = (u & 0x8000000000000000ull) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
    return __longlong_as_double((long long)u);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}
// Inclusive warp scan of an int.
__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 21-bit spread to every third bit (same bit pattern as the reference's
// expand_bits_21, engine/include/celestial/cuda/morton.hpp:13-21, written as
// a PDEP-style shift/mask ladder).
__host__ __device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Inverse of spread21.
__host__ __device__ __forceinline__ uint32_t compact21(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v | (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v | (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v | (v >> 8)) & 0x1F0000FF0000FFull;
    v = (v | (v >> 16)) & 0x1F00000000FFFFull;
    v = (v | (v >> 32)) & 0x1FFFFFull;
    return (uint32_t)v;
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Rows of a launch sized on the host for n rows: with a device count `dn`
// (a count that only shrinks inside a captured multi-step graph, e.g. the
// rows left by the last compaction) the smaller of the two.
__device__ __forceinline__ int dev_rows(int n, const int* dn) { return dn ? min(n, *dn) : n; }

}  // namespace nb
