// direct.cuh - softened O(n^2) direct sums.
#pragma once
#include "common.cuh"

namespace nb {

// Rounding and summation orders of the desktop app's CPU backends.
enum DirectOrder { kOrderParallel = 0, kOrderSimd = 1, kOrderPairwise = 2 };

// FP64, rows in caller order, bit-identical to the CPU backend `order`
// names (CpuParallelBackend, SimdSingleThreadBackend / the native engine's
// CPU brute force, CpuSingleThreadBackend).
void direct_fp64(cudaStream_t st, int n, const double* px, const double* py, const double* pz,
                 const double* m, const double* rad, const uint8_t* act, double eps, bool shell,
                 int order, double* ax, double* ay, double* az);
// FP32 pair math over the n sorted (active) bodies; writes rows sidx[k].
// scratch: device memory for the per-chunk FP64 partial sums (3 x n doubles
// per source chunk; at least 24 n bytes); ctr: a device work-queue counter.
void direct_fp32(cudaStream_t st, int n, const double4* sbody, const float* srad,
                 const uint32_t* sidx, double eps, bool shell, double* ax, double* ay,
                 double* az, unsigned long long* counter, void* scratch, size_t scratch_bytes,
                 unsigned* ctr, int sms);

}  // namespace nb
