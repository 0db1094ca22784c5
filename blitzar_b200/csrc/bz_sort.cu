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

// `job` (optional) names the arrays and the count on the device; the host-side arguments are
// then only the capacity the grid was sized for.
__global__ void __launch_bounds__(kThreads) k_histogram(const unsigned long long* __restrict__ keys,
                                                         int n, int passes, SortWorkspace ws,
                                                         const SortJob* __restrict__ job)
{
    if (job) {
        keys = job->ka;
        n = job->n;
    }
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
__global__ void k_scan_hist(int n, SortWorkspace ws, const SortJob* __restrict__ job)
{
    if (job)
        n = job->n;
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
                                                        SortWorkspace ws, int* err,
                                                        const SortJob* __restrict__ job)
{
    if (ws.trivial[pass])
        return;
    if (job) {
        keys_a = job->ka;
        vals_a = job->va;
        keys_b = job->kb;
        vals_b = job->vb;
        n = job->n;
    }
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
    const int shift = 8 * pass;
    const unsigned lt = lanemask_lt();
    // Persistent blocks take tiles in ticket order until the (device-side) count is covered:
    // a tile's look-back waits only on tiles taken earlier by running blocks.  A grid sized
    // for a larger capacity than the job costs a few idle blocks, not a wave per tile.
    for (;;) {
    if (tid == 0)
        sm.tile = static_cast<int>(atomicAdd(&ws.ticket[pass], 1u));
    for (int i = tid; i < kWarps * 256; i += kThreads)
        (&sm.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const int tile = sm.tile;
    const long long base = static_cast<long long>(tile) * kTile;
    if (base >= n)
        return;  // no later tile waits for this one

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
    // a grid with a block for every tile of this count takes no second ticket
    if (static_cast<long long>(gridDim.x) * kTile >= n)
        return;
    __syncthreads();  // the next tile reuses the shared memory
    }
}

// After the passes the data sits in the alternate buffers when an odd number of passes ran;
// copy it back so callers always find it in (keys, vals).
__global__ void k_fixup(unsigned long long* keys_a, uint32_t* vals_a,
                        const unsigned long long* keys_b, const uint32_t* vals_b, int n,
                        int passes, SortWorkspace ws, const SortJob* __restrict__ job)
{
    if (job) {
        keys_a = job->ka;
        vals_a = job->va;
        keys_b = job->kb;
        vals_b = job->vb;
        n = job->n;
    }
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

namespace {

// The passes for a grid of capacity n; with `job` the device-held arrays and count decide the
// work.
void enqueue_sort(unsigned long long* keys, uint32_t* vals, int n, int bits, SortWorkspace& ws,
                  int* err, cudaStream_t s, const SortJob* job)
{
    const int passes = (bits + 7) / 8;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    count_launch();
    k_sort_init<<<1, 256, 0, s>>>(ws);
    int hb = (n + kThreads - 1) / kThreads;
    hb = hb < 2 * sms ? hb : 2 * sms;
    count_launch();
    k_histogram<<<hb, kThreads, 0, s>>>(keys, n, passes, ws, job);
    count_launch();
    k_scan_hist<<<passes, 256, 0, s>>>(n, ws, job);
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
    // persistent grid: the resident blocks (at most one per tile)
    static std::atomic<int> resident[kMaxDevices];
    int per_sm = dev >= 0 && dev < kMaxDevices ? resident[dev].load() : 0;
    if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_onesweep, kThreads, smem);
        per_sm = per_sm > 0 ? per_sm : 1;
        if (dev >= 0 && dev < kMaxDevices)
            resident[dev].store(per_sm);
    }
    const int grid = tiles < per_sm * sms ? tiles : per_sm * sms;
    for (int p = 0; p < passes; ++p) {
        count_launch();
        k_onesweep<<<grid, kThreads, smem, s>>>(keys, vals, ws.keys_alt, ws.vals_alt, n, p, ws,
                                                err, job);
    }
    int fb = (n + 255) / 256;
    fb = fb < 4 * sms ? fb : 4 * sms;
    count_launch();
    k_fixup<<<fb, 256, 0, s>>>(keys, vals, ws.keys_alt, ws.vals_alt, n, passes, ws, job);
}

} // namespace

void launch_radix_sort(unsigned long long* keys, uint32_t* vals, int n, int bits,
                       SortWorkspace& ws, int* err, cudaStream_t s)
{
    if (n <= 1)
        return;
    enqueue_sort(keys, vals, n, bits, ws, err, s, nullptr);
}

// ---- nearly sorted inputs -------------------------------------------------------------------
// Between two steps of a simulation the particles move little, so the keys arrive (in the
// previous step's sorted order) almost sorted.  The adaptive sort splits the positions into
// U, those not locally out of order (key neither below any of the kWindow keys before it nor
// above any of the kWindow keys after it), and F, the rest; checks that U is sorted (a window
// of one misses runs of particles that moved past a run of others together); sorts F (small)
// with the radix sort;
// and merges the two by (key, original position).  Because the values are the original
// positions 0..n-1, that order is exactly the stable order of the full sort.  When U is not
// sorted or F exceeds its capacity, the full radix sort runs instead.  The choice is made on
// the device: every kernel is always launched (the step stays one captured graph), and the
// kernels of the path not taken return at once.
namespace {

constexpr int kInvItems = 16;
constexpr int kInvChunk = kThreads * kInvItems;  // positions per flag/compaction block
constexpr int kMergeSeg = 256;                  // in-order positions per merge segment
constexpr int kWindow = 8;                      // neighbours compared on each side

// Flags the out-of-order positions of a chunk (staged with its halo in shared memory) and
// counts them per block.
__global__ void __launch_bounds__(kThreads) k_inv_flag(const unsigned long long* __restrict__ keys, int n,
                                                        unsigned char* __restrict__ flag,
                                                        int* __restrict__ block_sums)
{
    __shared__ unsigned long long sk[kInvChunk + 2 * kWindow];
    const int base = blockIdx.x * kInvChunk;
    for (int j = threadIdx.x; j < kInvChunk + 2 * kWindow; j += kThreads) {
        const int i = base - kWindow + j;
        // outside [0, n) the halo can neither be below a key before it nor above one after it
        sk[j] = i < 0 ? 0ull : (i >= n ? ~0ull : keys[i]);
    }
    __syncthreads();
    // a chunk sorted together with its halo has nothing out of order
    bool unsorted = false;
    for (int j = threadIdx.x; j + 1 < kInvChunk + 2 * kWindow; j += kThreads)
        unsorted = unsorted || sk[j] > sk[j + 1];
    if (!__syncthreads_or(unsorted)) {
        for (int j = threadIdx.x; j < kInvChunk; j += kThreads)
            if (base + j < n)
                flag[base + j] = 0;
        if (threadIdx.x == 0)
            block_sums[blockIdx.x] = 0;
        return;
    }
    int c = 0;
    for (int it = 0; it < kInvItems; ++it) {
        const int j = it * kThreads + threadIdx.x;
        const int i = base + j;
        if (i >= n)
            break;
        const unsigned long long v = sk[j + kWindow];
        bool f = false;
#pragma unroll
        for (int w = 1; w <= kWindow; ++w)
            f = f || v < sk[j + kWindow - w] || v > sk[j + kWindow + w];
        flag[i] = f ? 1 : 0;
        c += f ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(kFullMask, c, o);
    __shared__ int ws[kWarps];
    if ((threadIdx.x & 31) == 0)
        ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kWarps; ++w)
            t += ws[w];
        block_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the block counts in one block; ctl[0] = out-of-order count, ctl[1] = 0.
__global__ void __launch_bounds__(1024) k_inv_scan(int* __restrict__ block_sums, int blocks,
                                                   int* __restrict__ ctl)
{
    __shared__ int carry;
    __shared__ int ws[32];
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < blocks; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < blocks ? block_sums[i] : 0;
        const int x = warp_incl_scan(v);
        if (lane == 31)
            ws[warp] = x;
        __syncthreads();
        if (warp == 0)
            ws[lane] = warp_incl_scan(ws[lane]);
        __syncthreads();
        const int before = (warp > 0 ? ws[warp - 1] : 0) + carry;
        if (i < blocks)
            block_sums[i] = before + x - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl[0] = carry;
        ctl[1] = 0;
    }
}

// Stable split into U (ukeys/uvals, in order) and F (fkeys/fvals, the first `cap` of them).
__global__ void __launch_bounds__(kThreads) k_inv_emit(const unsigned long long* __restrict__ keys,
                                                        const uint32_t* __restrict__ vals,
                                                        const unsigned char* __restrict__ flag, int n,
                                                        const int* __restrict__ block_offsets, int cap,
                                                        const int* __restrict__ ctl,
                                                        unsigned long long* __restrict__ ukeys,
                                                        uint32_t* __restrict__ uvals,
                                                        unsigned long long* __restrict__ fkeys,
                                                        uint32_t* __restrict__ fvals)
{
    const int base = blockIdx.x * kInvChunk;
    const int fb0 = block_offsets[blockIdx.x];
    const int fb1 = blockIdx.x + 1 < gridDim.x ? block_offsets[blockIdx.x + 1] : ctl[0];
    if (fb0 == fb1) {  // nothing out of order here: a shifted copy into U
        for (int i = base + threadIdx.x; i < min(base + kInvChunk, n); i += kThreads) {
            ukeys[i - fb0] = keys[i];
            uvals[i - fb0] = vals[i];
        }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ int ws[kWarps];
    __shared__ int carry;
    if (threadIdx.x == 0)
        carry = block_offsets[blockIdx.x];
    __syncthreads();
    for (int it = 0; it < kInvItems; ++it) {
        const int i = base + it * kThreads + threadIdx.x;
        const int f = i < n ? flag[i] : 0;
        const int x = warp_incl_scan(f);
        if (lane == 31)
            ws[warp] = x;
        __syncthreads();
        int before = carry;
        for (int w = 0; w < warp; ++w)
            before += ws[w];
        if (i < n) {
            const int fb = before + x - f;  // out-of-order positions before i
            if (f) {
                if (fb < cap) {
                    fkeys[fb] = keys[i];
                    fvals[fb] = vals[i];
                }
            } else {
                ukeys[i - fb] = keys[i];
                uvals[i - fb] = vals[i];
            }
        }
        __syncthreads();
        if (threadIdx.x == kThreads - 1)
            carry = before + x;
        __syncthreads();
    }
}

// ctl[1] |= 1 when U is not sorted.  Each thread checks a run of kVerifyRun consecutive keys
// (16-byte loads) and the pair across the run's end.
constexpr int kVerifyRun = 16;
__global__ void __launch_bounds__(kThreads) k_inv_verify(const unsigned long long* __restrict__ ukeys,
                                                          int n, int* __restrict__ ctl)
{
    const long long m = n - ctl[0];
    bool bad = false;
    const long long stride = static_cast<long long>(gridDim.x) * kThreads * kVerifyRun;
    for (long long s0 = (static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x) * kVerifyRun;
         s0 + 1 < m; s0 += stride) {
        if (s0 + kVerifyRun < m) {
            const ulonglong2* p = reinterpret_cast<const ulonglong2*>(ukeys + s0);  // 128-byte aligned
            unsigned long long prev = 0;
#pragma unroll
            for (int q = 0; q < kVerifyRun / 2; ++q) {
                const ulonglong2 v = p[q];
                bad = bad || (q > 0 && prev > v.x) || v.x > v.y;
                prev = v.y;
            }
            bad = bad || prev > ukeys[s0 + kVerifyRun];
        } else {
            for (long long j = s0; j + 1 < m; ++j)
                bad = bad || ukeys[j] > ukeys[j + 1];
        }
    }
    if (__any_sync(kFullMask, bad) && (threadIdx.x & 31) == 0)
        atomicOr(&ctl[1], 1);
}

// Picks the radix sort's job: the out-of-order pairs (fast path; ctl[3] = 0) or all pairs
// (ctl[3] = n).  ctl[2] = the fast path's out-of-order count.
__global__ void k_inv_mode(int n, int cap, int* __restrict__ ctl, SortJob* __restrict__ job,
                           SortJob fast_job, SortJob full_job)
{
    const bool fast = ctl[1] == 0 && ctl[0] <= cap;
    ctl[2] = fast ? ctl[0] : 0;
    ctl[3] = fast ? 0 : n;
    fast_job.n = ctl[0];
    *job = fast ? fast_job : full_job;
}

// Entries of the sorted (k, v)[lo, hi) ordered before (key, val) by (key, value), plus lo.
__device__ __forceinline__ int rank_in(const unsigned long long* __restrict__ k,
                                       const uint32_t* __restrict__ v, int lo, int hi,
                                       unsigned long long key, uint32_t val)
{
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const unsigned long long km = k[mid];
        if (km < key || (km == key && v[mid] < val))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Fast path: an in-order pair at U index j lands at j + (F pairs before it); an out-of-order
// pair at F index q lands at q + (U pairs before it).  A segment of kMergeSeg U pairs first
// bounds the F range that can fall inside it (usually empty).
__global__ void __launch_bounds__(kThreads) k_inv_merge(const unsigned long long* __restrict__ ukeys,
                                                         const uint32_t* __restrict__ uvals,
                                                         const unsigned long long* __restrict__ fkeys,
                                                         const uint32_t* __restrict__ fvals, int n,
                                                         const int* __restrict__ ctl,
                                                         unsigned long long* __restrict__ keys,
                                                         uint32_t* __restrict__ vals)
{
    if (ctl[3] != 0)
        return;  // the full sort ran
    const int nf = ctl[2], m = n - nf;
    const int useg = (m + kMergeSeg - 1) / kMergeSeg;
    const int fseg = (nf + kThreads - 1) / kThreads;
    __shared__ int s_lo, s_hi;
    for (int sgi = blockIdx.x; sgi < useg + fseg; sgi += gridDim.x) {
        if (sgi < useg) {
            const int j0 = sgi * kMergeSeg;
            const int j1 = min(j0 + kMergeSeg, m) - 1;
            if (threadIdx.x == 0) {
                s_lo = nf ? rank_in(fkeys, fvals, 0, nf, ukeys[j0], uvals[j0]) : 0;
                s_hi = nf ? rank_in(fkeys, fvals, 0, nf, ukeys[j1], uvals[j1]) : 0;
            }
            __syncthreads();
            const int lo = s_lo, hi = s_hi;
            for (int j = j0 + threadIdx.x; j <= j1; j += kThreads) {
                const unsigned long long key = ukeys[j];
                const uint32_t val = uvals[j];
                const int before = lo == hi ? lo : rank_in(fkeys, fvals, lo, hi, key, val);
                keys[j + before] = key;
                vals[j + before] = val;
            }
            __syncthreads();
        } else {
            const int q = (sgi - useg) * kThreads + threadIdx.x;
            if (q < nf) {
                const unsigned long long key = fkeys[q];
                const uint32_t val = fvals[q];
                const int pos = q + rank_in(ukeys, uvals, 0, m, key, val);
                keys[pos] = key;
                vals[pos] = val;
            }
        }
    }
}

} // namespace

int adaptive_sort_blocks(int n) { return n > 0 ? (n + kInvChunk - 1) / kInvChunk : 1; }
int adaptive_sort_cap(int n) { return n / 8 > 4096 ? n / 8 : 4096; }

void launch_radix_sort_adaptive(unsigned long long* keys, uint32_t* vals, int n, int bits,
                                SortWorkspace& ws, AdaptiveSortWorkspace& aws, int* err,
                                cudaStream_t s)
{
    if (n <= 1)
        return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = adaptive_sort_blocks(n);
    count_launch(3);
    k_inv_flag<<<blocks, kThreads, 0, s>>>(keys, n, aws.flag, aws.block_sums);
    k_inv_scan<<<1, 1024, 0, s>>>(aws.block_sums, blocks, aws.ctl);
    k_inv_emit<<<blocks, kThreads, 0, s>>>(keys, vals, aws.flag, n, aws.block_sums, aws.cap,
                                           aws.ctl, ws.keys_alt, ws.vals_alt, aws.fkeys, aws.fvals);
    int vb = (n + kThreads - 1) / kThreads;
    vb = vb < 4 * sms ? vb : 4 * sms;
    count_launch(2);
    k_inv_verify<<<vb, kThreads, 0, s>>>(ws.keys_alt, n, aws.ctl);
    const SortJob fast_job{aws.fkeys, aws.fvals, aws.falt_keys, aws.falt_vals, 0};
    const SortJob full_job{keys, vals, ws.keys_alt, ws.vals_alt, n};
    k_inv_mode<<<1, 1, 0, s>>>(n, aws.cap, aws.ctl, aws.job, fast_job, full_job);
    // one radix sort: of F in place on the fast path, else of all of (keys, vals)
    enqueue_sort(keys, vals, n, bits, ws, err, s, aws.job);
    count_launch();
    k_inv_merge<<<8 * sms, kThreads, 0, s>>>(ws.keys_alt, ws.vals_alt, aws.fkeys, aws.fvals, n,
                                             aws.ctl, keys, vals);
}

} // namespace bz
