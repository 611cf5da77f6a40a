// sort.cuh - stable one-sweep LSD radix sort of (uint64, uint32) pairs.
#pragma once
#include "common.cuh"

namespace nb {

void sort_init();
size_t sort_workspace_bytes(int capacity);
// Returns the first failing status of the call's own memsets and launches.
// dn: optional device count replacing n when smaller (launches sized for n).
cudaError_t sort_pairs(cudaStream_t st, int n, uint64_t* k0, uint32_t* v0, uint64_t* k1,
                       uint32_t* v1, void* ws, bool hist_ready, int* err, int sms,
                       const int* dn = nullptr);

}  // namespace nb
