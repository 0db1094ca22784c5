// Allocation-free sort entry point.
//
// bz_sort_pairs_noalloc runs the same stable onesweep radix sort as the engine (bz_sort.cu),
// but takes its scratch -- the ping-pong key/value buffers, the digit histograms, the tile
// tickets, the look-back words and the error flag -- from one fixed array in device memory
// declared below, instead of from cudaMalloc.  It is meant for callers that may not allocate
// device memory at all: a host application that reserves all of HBM for its own pool or
// arena at start-up (so a cudaMalloc from a plug-in fails, or bypasses the pool's
// accounting), and step loops where cudaMalloc/cudaFree are too costly (cudaFree waits for
// the whole device).  The handle-based API cannot serve them: bz_create allocates the
// engine's buffers.
//
// The array is a module global: every process that loads this library holds it on each
// device it uses, until exit.  All calls on a device share it and it keeps the contents of
// the last call; the sort clears what must start at zero (histograms, tile tickets, error
// flag) and tags its look-back words with a per-call epoch, so stale words from an earlier
// call are never read as current ones.
#include <mutex>

#include "bz_common.cuh"
#include "bz_kernels.h"
#include "bzgrav.h"

namespace {

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

constexpr size_t kMaxKeys = BZ_SORT_NOALLOC_MAX_KEYS;
constexpr size_t kTileItems = 4096;  // onesweep tile; checked against sort_tile_items()
constexpr size_t kStateWords = (kMaxKeys + kTileItems - 1) / kTileItems * 256;

constexpr size_t kOffKeys = 0;
constexpr size_t kOffVals = align_up(kOffKeys + 8 * kMaxKeys);
constexpr size_t kOffState = align_up(kOffVals + 4 * kMaxKeys);
constexpr size_t kOffHist = align_up(kOffState + 8 * kStateWords);
constexpr size_t kOffBase = align_up(kOffHist + 4 * 8 * 256);
constexpr size_t kOffTicket = align_up(kOffBase + 4 * 8 * 256);
constexpr size_t kOffEpoch = align_up(kOffTicket + 4 * 8);
constexpr size_t kOffTrivial = align_up(kOffEpoch + 4);
constexpr size_t kOffErr = align_up(kOffTrivial + 4 * 8);
constexpr size_t kScratchBytes = align_up(kOffErr + 4);  // 12.6 MiB for 2^20 keys

// The scratch.  In host code this name is only a host-side stand-in for the symbol: the
// device address comes from cudaGetSymbolAddress, once per device (scratch_on_device).
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_addr[bz::kMaxDevices] = {};

// Device address of the scratch on device `dev`, which must be current.  The first call on
// a device resolves it (this may load the module on that device); later calls reuse it.
cudaError_t scratch_on_device(int dev, unsigned char** out)
{
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess)
            return e;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// True when p is memory the current device `dev` can read and write as a kernel operand.
bool device_accessible(const void* p, int dev)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged)
        return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

} // namespace

extern "C" bz_status bz_sort_pairs_noalloc(uint64_t* keys, uint32_t* values, int64_t n,
                                           int key_bits, uint64_t stream)
{
    if (n < 0 || n > static_cast<int64_t>(kMaxKeys))
        return BZ_INVALID_ARGUMENT;
    if (key_bits < 8 || key_bits > 64 || key_bits % 8 != 0)
        return BZ_INVALID_ARGUMENT;
    if (n <= 1)
        return BZ_OK;  // nothing to order
    if (keys == nullptr || values == nullptr)
        return BZ_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(keys) % alignof(uint64_t) != 0 ||
        reinterpret_cast<uintptr_t>(values) % alignof(uint32_t) != 0)
        return BZ_INVALID_ARGUMENT;
    if (static_cast<size_t>(bz::sort_tile_items()) != kTileItems ||
        bz::sort_state_words(static_cast<int>(n)) > kStateWords)
        return BZ_INTERNAL_ERROR;

    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= bz::kMaxDevices)
        return BZ_CUDA_ERROR;
    // Host pointers must never reach the kernels: reject anything the device cannot address.
    if (!device_accessible(keys, dev) || !device_accessible(values, dev))
        return BZ_INVALID_ARGUMENT;

    unsigned char* base = nullptr;
    if (scratch_on_device(dev, &base) != cudaSuccess)
        return BZ_CUDA_ERROR;

    bz::SortWorkspace ws{};
    ws.keys_alt = reinterpret_cast<unsigned long long*>(base + kOffKeys);
    ws.vals_alt = reinterpret_cast<uint32_t*>(base + kOffVals);
    ws.state = reinterpret_cast<unsigned long long*>(base + kOffState);
    ws.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    ws.base = reinterpret_cast<uint32_t*>(base + kOffBase);
    ws.ticket = reinterpret_cast<uint32_t*>(base + kOffTicket);
    ws.epoch = reinterpret_cast<uint32_t*>(base + kOffEpoch);
    ws.trivial = reinterpret_cast<int*>(base + kOffTrivial);
    ws.max_tiles = static_cast<int>(kStateWords / 256);
    int* err = reinterpret_cast<int*>(base + kOffErr);

    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess)
        return BZ_CUDA_ERROR;
    bz::launch_radix_sort(reinterpret_cast<unsigned long long*>(keys), values,
                          static_cast<int>(n), key_bits, ws, err, s);
    if (cudaGetLastError() != cudaSuccess)
        return BZ_CUDA_ERROR;
    int host_err = 0;
    if (cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return BZ_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess)
        return BZ_CUDA_ERROR;
    return host_err ? BZ_DEVICE_LIMIT : BZ_OK;
}
