// Stable LSD radix sort of (u64 key, u32 value) pairs: one histogram pass over the keys for
// all digit positions, then one single-pass ("onesweep") kernel per 8-bit digit that ranks a
// 4096-key tile in shared memory, obtains its global digit offsets through decoupled
// look-back, and scatters.  Replaces thrust::sort_by_key in
// engine/physics/octree/cuda/linear/OctBuild.inl:96 (CUB radix sort, stable), with which it
// agrees bit for bit (same stable order).
//
// HBM-bound: 8 B read per key for the histogram, then 12 B read + 12 B written per pair and
// digit pass.  Look-back waits are bounded (kErrSortSpin) instead of unbounded spins.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIter = 16;                     // keys per lane
constexpr int kTile = kWarps * 32 * kIter;    // 4096 keys per tile
constexpr unsigned long long kFlagAgg = 1ull << 30;
constexpr unsigned long long kFlagPrefix = 2ull << 30;
constexpr unsigned long long kValueMask = (1ull << 30) - 1;

__global__ void k_sort_init(SortWorkspace ws)
{
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x)
        ws.hist[i] = 0;
    if (threadIdx.x < 8)
        ws.ticket[threadIdx.x] = 0;
    if (threadIdx.x == 0)
        ws.epoch[0] += 1;
}

__global__ void __launch_bounds__(kThreads) k_histogram(const unsigned long long* __restrict__ keys,
                                                         int n, int passes, SortWorkspace ws)
{
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += kThreads)
        (&h[0][0])[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const unsigned long long k = keys[i];
        for (int p = 0; p < passes; ++p)
            atomicAdd(&h[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) {
        const uint32_t v = (&h[0][0])[i];
        if (v)
            atomicAdd(&ws.hist[i], v);
    }
}

// One block per digit position: exclusive scan of its 256 counts; flags passes in which a
// single digit holds every key (such a pass is the identity and is skipped).
__global__ void k_scan_hist(int n, SortWorkspace ws)
{
    __shared__ uint32_t s[256];
    const int p = blockIdx.x, d = threadIdx.x;
    const uint32_t c = ws.hist[p * 256 + d];
    s[d] = c;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        const uint32_t t = d >= o ? s[d - o] : 0u;
        __syncthreads();
        s[d] += t;
        __syncthreads();
    }
    ws.base[p * 256 + d] = s[d] - c;
    if (d == 0)
        ws.trivial[p] = 0;
    __syncthreads();
    if (c == static_cast<uint32_t>(n))
        ws.trivial[p] = 1;
}

__device__ __forceinline__ unsigned long long load_state(const unsigned long long* p)
{
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void store_state(unsigned long long* p, unsigned long long v)
{
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

struct PassSmem {
    unsigned long long keys[kTile];
    uint32_t vals[kTile];
    uint32_t warp_hist[kWarps][256];
    uint32_t tile_excl[256];
    uint32_t global_off[256];
    uint32_t scan[256];
    int tile;
};

__global__ void __launch_bounds__(kThreads) k_onesweep(unsigned long long* keys_a, uint32_t* vals_a,
                                                        unsigned long long* keys_b,
                                                        uint32_t* vals_b, int n, int pass,
                                                        SortWorkspace ws, int* err)
{
    if (ws.trivial[pass])
        return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem& sm = *reinterpret_cast<PassSmem*>(smem_raw);
    int np = 0;
    for (int p = 0; p < pass; ++p)
        np += ws.trivial[p] ? 0 : 1;
    const unsigned long long* src_k = (np & 1) ? keys_b : keys_a;
    const uint32_t* src_v = (np & 1) ? vals_b : vals_a;
    unsigned long long* dst_k = (np & 1) ? keys_a : keys_b;
    uint32_t* dst_v = (np & 1) ? vals_a : vals_b;

    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    if (tid == 0)
        sm.tile = static_cast<int>(atomicAdd(&ws.ticket[pass], 1u));
    for (int i = tid; i < kWarps * 256; i += kThreads)
        (&sm.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const int tile = sm.tile;
    const long long base = static_cast<long long>(tile) * kTile;
    const int shift = 8 * pass;
    const unsigned lt = lanemask_lt();

    unsigned long long kr[kIter];
    uint32_t vr[kIter];
    uint32_t rank[kIter];
#pragma unroll
    for (int k = 0; k < kIter; ++k) {
        const long long idx = base + w * (32 * kIter) + k * 32 + lane;
        const bool valid = idx < n;
        kr[k] = valid ? src_k[idx] : 0ull;
        vr[k] = valid ? src_v[idx] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kIter; ++k) {
        const long long idx = base + w * (32 * kIter) + k * 32 + lane;
        const bool valid = idx < n;
        const unsigned d = static_cast<unsigned>((kr[k] >> shift) & 255u);
        const unsigned peers = __match_any_sync(kFullMask, valid ? d : 256u + lane);
        if (valid)
            rank[k] = sm.warp_hist[w][d] + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1)
            sm.warp_hist[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Per digit: warp offsets within the tile and the tile's count.
    const int d = tid;
    uint32_t cnt = 0;
    for (int ww = 0; ww < kWarps; ++ww) {
        const uint32_t c = sm.warp_hist[ww][d];
        sm.warp_hist[ww][d] = cnt;
        cnt += c;
    }
    // Decoupled look-back for this digit (one thread per digit).
    const unsigned long long tag = (static_cast<unsigned long long>(ws.epoch[0] * 8u + pass)) << 32;
    unsigned long long* st = ws.state;
    uint32_t excl = 0;
    if (tile == 0) {
        store_state(&st[d], tag | kFlagPrefix | cnt);
    } else {
        store_state(&st[static_cast<size_t>(tile) * 256 + d], tag | kFlagAgg | cnt);
        int t = tile - 1;
        int spins = 0;
        while (t >= 0) {
            const unsigned long long v = load_state(&st[static_cast<size_t>(t) * 256 + d]);
            if ((v & 0xffffffff00000000ull) != tag || (v & (3ull << 30)) == 0) {
                if (++spins > kSpinLimit) {
                    raise_error(err, kErrSortSpin);
                    break;
                }
                if (spins > 32)
                    __nanosleep(32);
                continue;
            }
            excl += static_cast<uint32_t>(v & kValueMask);
            if (v & kFlagPrefix)
                break;
            --t;
        }
        store_state(&st[static_cast<size_t>(tile) * 256 + d], tag | kFlagPrefix | (excl + cnt));
    }
    sm.global_off[d] = ws.base[pass * 256 + d] + excl;
    // Tile-local exclusive scan over digits (for staging in shared memory).
    sm.scan[d] = cnt;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        const uint32_t t = d >= o ? sm.scan[d - o] : 0u;
        __syncthreads();
        sm.scan[d] += t;
        __syncthreads();
    }
    sm.tile_excl[d] = sm.scan[d] - cnt;
    __syncthreads();

#pragma unroll
    for (int k = 0; k < kIter; ++k) {
        const long long idx = base + w * (32 * kIter) + k * 32 + lane;
        if (idx < n) {
            const unsigned dd = static_cast<unsigned>((kr[k] >> shift) & 255u);
            const uint32_t pos = sm.tile_excl[dd] + sm.warp_hist[w][dd] + rank[k];
            sm.keys[pos] = kr[k];
            sm.vals[pos] = vr[k];
        }
    }
    __syncthreads();
    const int tile_n = static_cast<int>(min(static_cast<long long>(kTile), n - base));
    for (int j = tid; j < tile_n; j += kThreads) {
        const unsigned long long key = sm.keys[j];
        const unsigned dd = static_cast<unsigned>((key >> shift) & 255u);
        const uint32_t out = sm.global_off[dd] + (static_cast<uint32_t>(j) - sm.tile_excl[dd]);
        dst_k[out] = key;
        dst_v[out] = sm.vals[j];
    }
}

// After the passes the data sits in the alternate buffers when an odd number of passes ran;
// copy it back so callers always find it in (keys, vals).
__global__ void k_fixup(unsigned long long* keys_a, uint32_t* vals_a,
                        const unsigned long long* keys_b, const uint32_t* vals_b, int n,
                        int passes, SortWorkspace ws)
{
    int np = 0;
    for (int p = 0; p < passes; ++p)
        np += ws.trivial[p] ? 0 : 1;
    if ((np & 1) == 0)
        return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        keys_a[i] = keys_b[i];
        vals_a[i] = vals_b[i];
    }
}

} // namespace

int sort_tile_items() { return kTile; }

size_t sort_state_words(int n)
{
    const size_t tiles = (static_cast<size_t>(n) + kTile - 1) / kTile;
    return (tiles < 1 ? 1 : tiles) * 256;
}

void launch_radix_sort(unsigned long long* keys, uint32_t* vals, int n, int bits,
                       SortWorkspace& ws, int* err, cudaStream_t s)
{
    if (n <= 1)
        return;
    const int passes = (bits + 7) / 8;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    count_launch();
    k_sort_init<<<1, 256, 0, s>>>(ws);
    int hb = (n + kThreads - 1) / kThreads;
    hb = hb < 2 * sms ? hb : 2 * sms;
    count_launch();
    k_histogram<<<hb, kThreads, 0, s>>>(keys, n, passes, ws);
    count_launch();
    k_scan_hist<<<passes, 256, 0, s>>>(n, ws);
    const int tiles = (n + kTile - 1) / kTile;
    const size_t smem = sizeof(PassSmem);
    // function attributes belong to the device's context: set once per device
    static std::atomic<bool> attr_set[kMaxDevices];
    if (dev < 0 || dev >= kMaxDevices || !attr_set[dev].load()) {
        cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        if (dev >= 0 && dev < kMaxDevices)
            attr_set[dev].store(true);
    }
    for (int p = 0; p < passes; ++p) {
        count_launch();
        k_onesweep<<<tiles, kThreads, smem, s>>>(keys, vals, ws.keys_alt, ws.vals_alt, n, p, ws,
                                                 err);
    }
    int fb = (n + 255) / 256;
    fb = fb < 4 * sms ? fb : 4 * sms;
    count_launch();
    k_fixup<<<fb, 256, 0, s>>>(keys, vals, ws.keys_alt, ws.vals_alt, n, passes, ws);
}

} // namespace bz
