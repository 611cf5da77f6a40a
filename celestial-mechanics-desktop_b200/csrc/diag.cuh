// diag.cuh - energy / momentum diagnostics, the sampled FP64 force-error sums
// and the learned MAC's audit sums.
#pragma once
#include "bodies.cuh"

namespace nb {

size_t diag_partial_bytes(int capacity);
// out12: KE, Px, Py, Pz, Lx, Ly, Lz, sum m x, sum m y, sum m z, M, PE.
// pe_mode 0: exact pair sum; 1: 1/2 sum m_i phi_i from `phi` (by row).
void diagnostics(cudaStream_t st, int n, const State& s, double eps, int pe_mode,
                 const double* phi, double* rows, double* part, double* out12);
// FP64 direct-sum accelerations of rows targets[0 .. nt) into out3 (xyz per
// target); scratch: direct_targets_scratch_bytes(sms).
size_t direct_targets_scratch_bytes(int sms);
// *out = bits of the largest |a|^2 over the active rows (0 when none > 0).
void max_acc2(cudaStream_t st, int n, const State& s, unsigned long long* out, int sms);
void direct_targets(cudaStream_t st, int n, const State& s, double eps, int nt,
                    const int32_t* targets, double* out3, double* scratch, int sms);
// The learned MAC's audit sums: accelerations of rows targets[0 .. nt) from
// the ns Morton-sorted active bodies of the last force evaluation (sbody,
// current positions), FP32 pair terms on tile-differenced FP64 coordinates
// with FP64 accumulation (within ~1e-6 relative of direct_targets).  eps > 0.
// Returns false (nothing launched) when the sample does not fit the scratch.
size_t audit_targets_scratch_bytes(int sms);
bool audit_targets(cudaStream_t st, int ns, const double4* sbody, const State& s, double eps,
                   int nt, const int32_t* targets, double* out3, double* scratch, int sms);

}  // namespace nb
