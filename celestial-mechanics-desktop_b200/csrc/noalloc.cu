// noalloc.cu - a stable (uint64 key, int32 value) sort that allocates no
// device memory: nb_sort_pairs_noalloc.
//
// Who needs it: callers whose device memory is all owned by their own pool
// allocator (a framework's caching allocator, an application that reserves
// every byte at start-up), and callers on a latency-critical path where a
// cudaMalloc - which can synchronise the whole device - is not acceptable.
// They hand in device buffers they already own and get them back sorted.
//
// How: the sort's scratch (ping-pong key/value buffers, the 8 digit
// histograms, the per-tile look-back words, an error word) lives in one
// file-scope __device__ array of kScratchBytes.  Every GPU that loads this
// library holds that array until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on each device
// looks the address up with cudaGetSymbolAddress (with that device current)
// and caches it; that first call should therefore come before any stream
// capture.  The sort kernels are the same ones nb_sort_pairs launches.
#include <mutex>

#include "sort.cuh"

namespace {

// Largest n accepted: 1,048,576 pairs (the Barnes-Hut workload's body count).
constexpr int kNoAllocMaxN = 1 << 20;
constexpr size_t kAltKeysOff = 0;
constexpr size_t kAltValsOff = kAltKeysOff + sizeof(uint64_t) * kNoAllocMaxN;
constexpr size_t kWsOff = kAltValsOff + sizeof(uint32_t) * kNoAllocMaxN;
// sort workspace for kNoAllocMaxN keys: 8 x 256 histogram words, 8 tile
// counters, 8 passes x 1024 tiles (of the smallest tile, 1024 keys) x 256
// look-back words (checked at set-up)
constexpr size_t kWsBytes = sizeof(uint32_t) * (8 * 256 + 8 + 8 * 1024 * 256) + 4096;
constexpr size_t kErrOff = (kWsOff + kWsBytes + 255) & ~(size_t)255;
constexpr size_t kScratchBytes = kErrOff + 256;  // about 21.0 MB

__device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

struct DeviceScratch {
    unsigned char* base = nullptr;  // device address of g_sort_scratch
    int sms = 0;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
DeviceScratch g_scratch[kMaxDevices];

// Once per device, with that device current: the array's device address.
int32_t scratch_for_current_device(DeviceScratch* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return NB_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch& d = g_scratch[dev];
    if (!d.base) {
        if (nb::sort_workspace_bytes(kNoAllocMaxN) > kWsBytes) return NB_ERR_CAPACITY;
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return NB_ERR_CUDA;
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return NB_ERR_CUDA;
        nb::sort_init();
        d.sms = sms;
        d.base = (unsigned char*)p;
    }
    *out = d;
    return NB_OK;
}

}  // namespace

extern "C" NB_API int32_t nb_sort_pairs_noalloc(uint64_t* keys, int32_t* values, int32_t n,
                                                void* stream) {
    if (n > kNoAllocMaxN) return NB_ERR_CAPACITY;  // beyond the fixed scratch
    if (n < 0 || (n > 0 && (!keys || !values))) return NB_ERR_INVALID_ARG;
    if (n <= 1) return NB_OK;
    DeviceScratch d;
    int32_t r = scratch_for_current_device(&d);
    if (r != NB_OK) return r;
    cudaStream_t st = (cudaStream_t)stream;
    int* err = (int*)(d.base + kErrOff);
    // The array keeps the previous call's contents: the error word must start
    // clear; sort_pairs clears its own histogram, tile-counter and look-back
    // words before use.  Only this call's own memsets, launches and copies are
    // checked: an error that earlier, unrelated work left pending in the CUDA
    // runtime is neither reported as this call's nor cleared.
    if (cudaMemsetAsync(err, 0, sizeof(int) * nb::kErrCount, st) != cudaSuccess) return NB_ERR_CUDA;
    if (nb::sort_pairs(st, n, keys, (uint32_t*)values, (uint64_t*)(d.base + kAltKeysOff),
                       (uint32_t*)(d.base + kAltValsOff), d.base + kWsOff, false, err,
                       d.sms) != cudaSuccess)
        return NB_ERR_CUDA;
    int host_err[nb::kErrCount] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(host_err, err, sizeof(host_err), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return NB_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return NB_ERR_CUDA;
    if (host_err[nb::kErrTimeout]) return NB_ERR_TIMEOUT;
    return NB_OK;
}
