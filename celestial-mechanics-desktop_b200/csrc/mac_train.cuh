// mac_train.cuh - training-side pieces of the learned MAC.
#pragma once
#include "mac.cuh"
#include "tree.cuh"

namespace nb {

// Normalisation block: 8 feature means, 8 feature stds, target mean, target std.
constexpr int kMacNorm = 2 * kMacIn + 2;

// Sort harvest records by (usable, body, node) into `sorted`; *n_valid = the
// usable ones, which come first.  Buffers of nrec entries; ws for nrec keys.
void mac_sort_records(cudaStream_t st, int nrec, const MacRecord* rec, MacRecord* sorted,
                      uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, void* ws,
                      int* n_valid, int* err, int sms);
// Targets of the first nrec (usable, sorted) records, written to rows
// out_off + r.
void mac_targets(cudaStream_t st, int nrec, const MacRecord* rec, const double4* sbody,
                 const TreeBufs& t, double eps, float* X, float* Y, int* n_out, int out_off,
                 int out_cap);
void mac_image(cudaStream_t st, const float* P, const float* norm, MacDev* w);
// Gradient of the mean squared error of rows order[row0 .. row0+nrows) into
// grad (kMacParams floats, overwritten); the sum of squared errors is added
// to *loss.  part: mac_grad_partial_bytes(sms) of scratch.  The result is
// bitwise reproducible (no floating-point atomics).
size_t mac_grad_partial_bytes(int sms);
// P: the FP32 master parameters (the tensor-core kernel stages W1, W2 from
// them as BF16); err: the device error word (a bounded wait that expired).
void mac_grad(cudaStream_t st, const float* X, const float* Y, const int* order, int row0,
              int nrows, const float* P, const MacDev* w, float* grad, float* loss, int sms,
              float* part, int* err);
// The tcgen05 training kernel (mac_tc.cu): one CTA of 128 threads per SM.
__global__ void k_mac_train_tc(const float* __restrict__ X, const float* __restrict__ Y,
                               const int* __restrict__ order, int row0, int nrows,
                               const float* __restrict__ P, const MacDev* __restrict__ w,
                               float inv_batch, float* __restrict__ part, int acc_floats,
                               int loss_index, int* err);
size_t mac_train_tc_smem();
void mac_adam(cudaStream_t st, float* P, const float* G, float* m, float* v, int step, float lr);
void mac_predict(cudaStream_t st, const float* X, int n, const MacDev* w, float* out);
// Per walk-tree node (2n slots, *t.n_nodes used): screen term and log2 mass.
void mac_node_terms(cudaStream_t st, const TreeBufs& t, int n, const MacDev* w, float2* out);

}  // namespace nb
