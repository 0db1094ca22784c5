// Adaptive linear octree over Morton-sorted particles: top-down topology (one kernel per
// level, decoupled look-back over the level's child counts, no host round trip) and a single
// bottom-up moments kernel (last-arriving child computes its parent).
//
// This file is compiled with --fmad=false: the FP64 moment sums must round exactly as written
// (fixed order, no contraction) so that node moments are bit-identical to the oracle's.
//
// Replaces the reference's level loop with a host sync per level
// (engine/physics/octree/cuda/linear/OctBuild.inl:156-199, OctLeafKernels.inl:7-81,
// OctParentKernels.inl:7-103, OctLinkKernels.inl): same idea (node = Morton cell, children
// from the next 3 key bits, FP64 mass/COM), but leaves are adaptive (<= leaf_cap particles),
// children of a node are contiguous (breadth-first layout, no `next` links needed) and the
// moments include the quadrupole.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;
constexpr unsigned long long kAgg = 1ull << 30;
constexpr unsigned long long kPrefix = 2ull << 30;
constexpr unsigned long long kMask = (1ull << 30) - 1;

__global__ void k_tree_init(TreeArrays t, int n)
{
    const int i = threadIdx.x;
    if (i < kMaxLevels + 2) {
        t.lvl_first[i] = 0;
        t.lvl_count[i] = 0;
        t.lvl_split[i] = 0;
        t.ticket[i] = 0;
    }
    if (i == 0) {
        t.lvl_count[0] = 1;
        t.lvl_split[0] = 1;  // the root level goes the general way
        t.n_nodes[0] = 1;
        t.start[0] = 0;
        t.count[0] = n;
        t.parent[0] = -1;
        t.level[0] = 0;
        t.arrive[0] = 0;
    }
}

__device__ __forceinline__ int lower_bound_digit(const unsigned long long* __restrict__ keys,
                                                 int lo, int hi, int shift, unsigned d)
{
    // first i in [lo, hi) with digit(i) >= d (digits are non-decreasing inside a cell)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const unsigned dm = static_cast<unsigned>((keys[mid] >> shift) & 7u);
        if (dm < d)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long vload(const unsigned long long* p)
{
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void vstore(unsigned long long* p, unsigned long long v)
{
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Split every node of level `l` with more than leaf_cap particles into its non-empty octant
// cells.  Children of the level are appended in (parent, octant) order.  On the top levels
// (few, very large nodes) TPN = 8 threads serve one node: thread d (1..7) finds the first
// particle whose digit is >= d, so the seven binary searches run side by side; deeper levels
// use one thread per node.  Look-back tiles are indexed in units of kLookbackNodes nodes.
constexpr int kLookbackNodes = kThreads / 8;

template <int TPN>
__global__ void __launch_bounds__(kThreads) k_tree_level(const unsigned long long* __restrict__ keys,
                                                          int l, int leaf_cap, int max_level,
                                                          int min_split, TreeArrays t, int* err)
{
    constexpr int kNodesPerTile = kThreads / TPN;
    __shared__ int s_tile;
    __shared__ int s_scan[kThreads / 32];
    __shared__ int s_prefix;
    const int first = t.lvl_first[l];
    const int level_splits = t.lvl_split[l];  // loaded with the level's range, one round trip
    // after a capacity overflow the recorded count can exceed the arrays: clamp
    const int cnt = min(t.lvl_count[l], t.cap - first);
    if (cnt <= 0)
        return;
    const int next_first = first + cnt;
    if (level_splits == 0 && l >= min_split) {
        // no node of this level holds more than a leaf: all are leaves, no children, no scan
        for (int i = blockIdx.x * kThreads + threadIdx.x; i < cnt; i += gridDim.x * kThreads) {
            t.child[first + i] = -1;
            t.nchild[first + i] = 0;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            t.lvl_first[l + 1] = next_first;
            t.lvl_count[l + 1] = 0;
            t.n_nodes[0] = min(next_first, t.cap);
        }
        return;
    }
    const int ntiles = (cnt + kNodesPerTile - 1) / kNodesPerTile;
    unsigned long long* lb = t.lookback + (first / kLookbackNodes + 2 * l);
    const int shift = 3 * (max_level - l - 1);
    const int slot = threadIdx.x / TPN, sub = threadIdx.x % TPN, lane = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0)
            s_tile = static_cast<int>(atomicAdd(&t.ticket[l], 1u));
        __syncthreads();
        const int tile = s_tile;
        __syncthreads();
        if (tile >= ntiles)
            break;
        const int k = first + tile * kNodesPerTile + slot;
        int s0 = 0, c0 = 0;
        bool split = false;
        int bsub = 0;
        int b[9];
        if (k < next_first) {
            s0 = t.start[k];
            c0 = t.count[k];
            // levels above min_split always split (ensembles: they separate the systems)
            split = (c0 > leaf_cap || l < min_split) && l < max_level;
            if (TPN == 8) {
                if (split && sub > 0)
                    bsub = lower_bound_digit(keys, s0, s0 + c0, shift, static_cast<unsigned>(sub));
            } else if (split) {
                // the seven searches advance in lockstep, so each step's seven loads are in
                // flight together (one memory round trip per step, not one per search step)
                int lo[8], hi[8];
#pragma unroll
                for (int d = 1; d < 8; ++d) {
                    lo[d] = s0;
                    hi[d] = s0 + c0;
                }
                for (int step = 0; step < 32; ++step) {
                    bool open = false;
#pragma unroll
                    for (int d = 1; d < 8; ++d) {
                        if (lo[d] < hi[d]) {
                            const int mid = (lo[d] + hi[d]) >> 1;
                            const unsigned dm = static_cast<unsigned>((keys[mid] >> shift) & 7u);
                            if (dm < static_cast<unsigned>(d))
                                lo[d] = mid + 1;
                            else
                                hi[d] = mid;
                            open = true;
                        }
                    }
                    if (!open)
                        break;
                }
#pragma unroll
                for (int d = 1; d < 8; ++d)
                    b[d] = lo[d];
            }
        }
        if (TPN == 8) {
#pragma unroll
            for (int d = 1; d < 8; ++d)
                b[d] = __shfl_sync(kFullMask, bsub, (lane & ~7) + d);
        }
        b[0] = s0;
        b[8] = s0 + c0;
        int nch = 0;
        if (split && sub == 0) {
#pragma unroll
            for (int d = 0; d < 8; ++d)
                nch += b[d + 1] > b[d] ? 1 : 0;
        }
        // block scan of child counts (only the leader of each node contributes): warp scans,
        // then one warp scans the warp totals
        const int wincl = warp_incl_scan(nch);
        const int warp = threadIdx.x >> 5;
        if (lane == 31)
            s_scan[warp] = wincl;
        __syncthreads();
        if (threadIdx.x < 32) {
            int v = threadIdx.x < kThreads / 32 ? s_scan[threadIdx.x] : 0;
            v = warp_incl_scan(v);
            if (threadIdx.x < kThreads / 32)
                s_scan[threadIdx.x] = v;
        }
        __syncthreads();
        const int incl = wincl + (warp > 0 ? s_scan[warp - 1] : 0);
        const int total = s_scan[kThreads / 32 - 1];
        if (threadIdx.x == 0) {
            unsigned long long excl = 0;
            if (tile == 0) {
                vstore(&lb[0], kPrefix | static_cast<unsigned long long>(total));
            } else {
                vstore(&lb[tile], kAgg | static_cast<unsigned long long>(total));
                int tt = tile - 1, spins = 0;
                while (tt >= 0) {
                    const unsigned long long v = vload(&lb[tt]);
                    if ((v & (3ull << 30)) == 0) {
                        if (++spins > kSpinLimit) {
                            raise_error(err, kErrTreeSpin);
                            break;
                        }
                        if (spins > 32)
                            __nanosleep(32);
                        continue;
                    }
                    excl += v & kMask;
                    if (v & kPrefix)
                        break;
                    --tt;
                }
                vstore(&lb[tile], kPrefix | (excl + static_cast<unsigned long long>(total)));
            }
            s_prefix = static_cast<int>(excl);
            if (tile == ntiles - 1) {
                const int children = static_cast<int>(excl) + total;
                t.lvl_first[l + 1] = next_first;
                t.lvl_count[l + 1] = children;
                t.n_nodes[0] = min(next_first + children, t.cap);
                if (next_first + children > t.cap)
                    raise_error(err, kErrTreeCapacity);
            }
        }
        __syncthreads();
        int cmax = 0;
        if (k < next_first && sub == 0) {
            int c = next_first + s_prefix + incl - nch;
            if (split && c + nch > t.cap)
                nch = 0;  // capacity exceeded (error raised above): keep the node a leaf
            t.child[k] = nch > 0 ? c : -1;
            t.nchild[k] = nch;
            if (nch > 0) {
#pragma unroll
                for (int d = 0; d < 8; ++d) {
                    if (b[d + 1] > b[d]) {
                        t.start[c] = b[d];
                        t.count[c] = b[d + 1] - b[d];
                        t.parent[c] = k;
                        t.level[c] = l + 1;
                        t.arrive[c] = 0;
                        cmax = max(cmax, b[d + 1] - b[d]);
                        ++c;
                    }
                }
            }
        }
        // a child larger than a leaf lets the next level split: flag it (plain stores of the
        // same value, which no thread waits for, instead of contended atomics)
        if (__any_sync(kFullMask, cmax > leaf_cap) && lane == 0)
            t.lvl_split[l + 1] = 1;
        __syncthreads();
    }
}

// Leaves of the deepest level are never visited by k_tree_level (it stops at max_level), so
// their child fields are written here before the moments pass reads them.
__global__ void k_tree_finish_last(TreeArrays t, int max_level)
{
    const int first = t.lvl_first[max_level];
    const int cnt = min(t.lvl_count[max_level], t.cap - first);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        t.child[first + i] = -1;
        t.nchild[first + i] = 0;
    }
}

// QUAD = false (monopole walks): the second moments are left zero, without their pass.
template <bool QUAD>
__device__ void leaf_moments(const float4* __restrict__ pos4, int k, TreeArrays& t)
{
    const int s = t.start[k], e = s + t.count[k];
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    double tm = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = s; i < e; ++i) {
        const float4 p = pos4[i];
        mn[0] = fminf(mn[0], p.x);
        mn[1] = fminf(mn[1], p.y);
        mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x);
        mx[1] = fmaxf(mx[1], p.y);
        mx[2] = fmaxf(mx[2], p.z);
        tm += (double)p.w;
        sx += (double)p.w * (double)p.x;
        sy += (double)p.w * (double)p.y;
        sz += (double)p.w * (double)p.z;
    }
    const double cx = tm > 0.0 ? sx / tm : 0.5 * ((double)mn[0] + (double)mx[0]);
    const double cy = tm > 0.0 ? sy / tm : 0.5 * ((double)mn[1] + (double)mx[1]);
    const double cz = tm > 0.0 ? sz / tm : 0.5 * ((double)mn[2] + (double)mx[2]);
    double q[6] = {0, 0, 0, 0, 0, 0};
    for (int i = s; QUAD && i < e; ++i) {
        const float4 p = pos4[i];
        const double dx = (double)p.x - cx, dy = (double)p.y - cy, dz = (double)p.z - cz;
        const double w = (double)p.w;
        q[0] += w * dx * dx;
        q[1] += w * dx * dy;
        q[2] += w * dx * dz;
        q[3] += w * dy * dy;
        q[4] += w * dy * dz;
        q[5] += w * dz * dz;
    }
    t.m64[k] = tm;
    t.s64[3 * k] = sx;
    t.s64[3 * k + 1] = sy;
    t.s64[3 * k + 2] = sz;
    if (QUAD) {  // the FP64 centre and second moments feed only the parents' second moments
        t.c64[3 * k] = cx;
        t.c64[3 * k + 1] = cy;
        t.c64[3 * k + 2] = cz;
        for (int j = 0; j < 6; ++j)
            t.q64[6 * k + j] = q[j];
    }
    t.box0[k] = make_float4(mn[0], mn[1], mn[2], __int_as_float(s));
    t.box1[k] = make_float4(mx[0], mx[1], mx[2], __int_as_float(-(e - s)));
    t.mono[k] = make_float4((float)cx, (float)cy, (float)cz, (float)tm);
    t.quadA[k] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    t.quadB[k] = make_float2((float)q[4], (float)q[5]);
}

template <bool QUAD>
__device__ void internal_moments(int k, TreeArrays& t)
{
    const int c0 = t.child[k], nc = t.nchild[k];
    // Both passes are unrolled over the (at most 8) children with predication, so the loads of
    // all children issue together and one climb step costs about one memory round trip; the
    // sums still run in octant order.
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    double tm = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (j < nc) {
            const int c = c0 + j;
            const float4 b0 = __ldcg(&t.box0[c]);
            const float4 b1 = __ldcg(&t.box1[c]);
            mn[0] = fminf(mn[0], b0.x);
            mn[1] = fminf(mn[1], b0.y);
            mn[2] = fminf(mn[2], b0.z);
            mx[0] = fmaxf(mx[0], b1.x);
            mx[1] = fmaxf(mx[1], b1.y);
            mx[2] = fmaxf(mx[2], b1.z);
            tm += __ldcg(&t.m64[c]);
            sx += __ldcg(&t.s64[3 * c]);
            sy += __ldcg(&t.s64[3 * c + 1]);
            sz += __ldcg(&t.s64[3 * c + 2]);
        }
    }
    const double cx = tm > 0.0 ? sx / tm : 0.5 * ((double)mn[0] + (double)mx[0]);
    const double cy = tm > 0.0 ? sy / tm : 0.5 * ((double)mn[1] + (double)mx[1]);
    const double cz = tm > 0.0 ? sz / tm : 0.5 * ((double)mn[2] + (double)mx[2]);
    double q[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (QUAD && j < nc) {
            const int c = c0 + j;
            const double dx = __ldcg(&t.c64[3 * c]) - cx;
            const double dy = __ldcg(&t.c64[3 * c + 1]) - cy;
            const double dz = __ldcg(&t.c64[3 * c + 2]) - cz;
            const double w = __ldcg(&t.m64[c]);
            q[0] += __ldcg(&t.q64[6 * c]) + w * dx * dx;
            q[1] += __ldcg(&t.q64[6 * c + 1]) + w * dx * dy;
            q[2] += __ldcg(&t.q64[6 * c + 2]) + w * dx * dz;
            q[3] += __ldcg(&t.q64[6 * c + 3]) + w * dy * dy;
            q[4] += __ldcg(&t.q64[6 * c + 4]) + w * dy * dz;
            q[5] += __ldcg(&t.q64[6 * c + 5]) + w * dz * dz;
        }
    }
    t.m64[k] = tm;
    t.s64[3 * k] = sx;
    t.s64[3 * k + 1] = sy;
    t.s64[3 * k + 2] = sz;
    if (QUAD) {  // the FP64 centre and second moments feed only the parents' second moments
        t.c64[3 * k] = cx;
        t.c64[3 * k + 1] = cy;
        t.c64[3 * k + 2] = cz;
        for (int j = 0; j < 6; ++j)
            t.q64[6 * k + j] = q[j];
    }
    t.box0[k] = make_float4(mn[0], mn[1], mn[2], __int_as_float(c0));
    t.box1[k] = make_float4(mx[0], mx[1], mx[2], __int_as_float(nc));
    t.mono[k] = make_float4((float)cx, (float)cy, (float)cz, (float)tm);
    t.quadA[k] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    t.quadB[k] = make_float2((float)q[4], (float)q[5]);
}

// One thread per leaf computes its moments, then climbs: the child that arrives last at a
// parent (atomic counter) computes the parent from all children in octant order.
template <bool QUAD>
__global__ void __launch_bounds__(kThreads) k_tree_moments(const float4* __restrict__ pos4,
                                                            TreeArrays t)
{
    const int nn = t.n_nodes[0];
    for (int k = blockIdx.x * kThreads + threadIdx.x; k < nn; k += gridDim.x * kThreads) {
        if (t.nchild[k] != 0)
            continue;
        leaf_moments<QUAD>(pos4, k, t);
        int node = k;
        for (;;) {
            const int p = t.parent[node];
            if (p < 0)
                break;
            // release this node's moments and, for the last child, acquire its siblings'
            int old;
            asm volatile("atom.add.acq_rel.gpu.s32 %0, [%1], 1;" : "=r"(old) : "l"(&t.arrive[p]) : "memory");
            if (old != t.nchild[p] - 1)
                break;
            internal_moments<QUAD>(p, t);
            node = p;
        }
    }
}


// clear_arrive: the arrival counters are not fresh from a build (a refit of an existing tree)
void enqueue_moments(const float4* pos4, TreeArrays& t, int sms, cudaStream_t s, bool quad,
                     bool clear_arrive)
{
    if (clear_arrive)
        cudaMemsetAsync(t.arrive, 0, sizeof(int) * static_cast<size_t>(t.cap), s);
    long long mb = (static_cast<long long>(t.cap) + kThreads - 1) / kThreads;
    if (mb > 16LL * sms)
        mb = 16LL * sms;
    count_launch();
    if (quad)
        k_tree_moments<true><<<static_cast<int>(mb), kThreads, 0, s>>>(pos4, t);
    else
        k_tree_moments<false><<<static_cast<int>(mb), kThreads, 0, s>>>(pos4, t);
}

} // namespace

void launch_tree_refit(const float4* pos4, TreeArrays& t, cudaStream_t s, bool quad)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    enqueue_moments(pos4, t, sms, s, quad, true);
}

size_t tree_lookback_words(int cap) { return static_cast<size_t>(cap) / kLookbackNodes + 2 * kMaxLevels + 8; }

void launch_tree_build(const unsigned long long* sorted_keys, const float4* pos4, int n,
                       int leaf_cap, int max_level, TreeArrays& t, int* err, cudaStream_t s,
                       int min_split, bool quad)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaMemsetAsync(t.lookback, 0, tree_lookback_words(t.cap) * sizeof(unsigned long long), s);
    count_launch();
    k_tree_init<<<1, 32, 0, s>>>(t, n);
    // Level l holds at most min(8^l, n) nodes; the persistent grid covers that with tiles.
    for (int l = 0; l < max_level; ++l) {
        long long bound = 1;
        for (int j = 0; j < l && bound < n; ++j)
            bound *= 8;
        if (bound > n)
            bound = n;
        const bool wide = bound <= 4096;  // top levels: few, large nodes
        const long long per_tile = wide ? kThreads / 8 : kThreads;
        long long blocks = (bound + per_tile - 1) / per_tile;
        // the tiles are latency-bound (loads, scan, look-back): fill the SMs (8 blocks each)
        if (blocks > 8LL * sms)
            blocks = 8LL * sms;
        count_launch();
        if (wide)
            k_tree_level<8><<<static_cast<int>(blocks), kThreads, 0, s>>>(sorted_keys, l, leaf_cap,
                                                                          max_level, min_split, t, err);
        else
            k_tree_level<1><<<static_cast<int>(blocks), kThreads, 0, s>>>(sorted_keys, l, leaf_cap,
                                                                          max_level, min_split, t, err);
    }
    count_launch();
    k_tree_finish_last<<<sms, 256, 0, s>>>(t, max_level);
    enqueue_moments(pos4, t, sms, s, quad, false);
}

} // namespace bz

// ---- reference-mode topology ------------------------------------------------------------
// The reference's linear octree for its own keys.  Its bit spread keeps 10 bits per axis, so
// keys are < 2^30, while the leaf prefix is key >> 3*(21 - leafDepth) with leafDepth <= 11
// for any n below 16*8^11: every key has prefix 0, the build yields exactly one leaf holding
// all particles in sorted order, the parent loop never runs and that leaf is the root
// (engine/physics/octree/cuda/linear/OctBuild.inl:109-199).  This kernel builds that node as
// buildLinearOctreeLeafNodesKernel does (OctLeafKernels.inl:7-81): FP32 tight box, FP64 mass
// and weighted position sums in sorted order.  The reference is compiled with nvcc's default
// contraction, so its `w += x * m` sums and `0.5f * ext + 1e-6f` execute as fused
// multiply-adds; they are written as explicit fmas here (this file is otherwise compiled
// without contraction).
namespace bz {
namespace {
__global__ void k_reference_leaf(const float* __restrict__ x, const float* __restrict__ y,
                                 const float* __restrict__ z, const float* __restrict__ m,
                                 const uint32_t* __restrict__ sorted_index, int n, float* hot8)
{
    if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
    float mn[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float mx[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int j = 0; j < n; ++j) {
        const uint32_t p = sorted_index[j];
        const float px = x[p], py = y[p], pz = z[p], pm = m[p];
        mn[0] = fminf(mn[0], px);
        mn[1] = fminf(mn[1], py);
        mn[2] = fminf(mn[2], pz);
        mx[0] = fmaxf(mx[0], px);
        mx[1] = fmaxf(mx[1], py);
        mx[2] = fmaxf(mx[2], pz);
        tm += (double)pm;
        wx = __fma_rn((double)px, (double)pm, wx);
        wy = __fma_rn((double)py, (double)pm, wy);
        wz = __fma_rn((double)pz, (double)pm, wz);
    }
    const float cx = 0.5f * (mn[0] + mx[0]);
    const float cy = 0.5f * (mn[1] + mx[1]);
    const float cz = 0.5f * (mn[2] + mx[2]);
    const float half = __fmaf_rn(0.5f, fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]), 1.0e-6f);
    hot8[0] = cx;
    hot8[1] = cy;
    hot8[2] = cz;
    hot8[3] = half;
    hot8[4] = (float)tm;
    hot8[5] = tm > 0.0 ? (float)(wx / tm) : cx;
    hot8[6] = tm > 0.0 ? (float)(wy / tm) : cy;
    hot8[7] = tm > 0.0 ? (float)(wz / tm) : cz;
}
} // namespace

void launch_reference_leaf(const float* x, const float* y, const float* z, const float* m,
                           const uint32_t* sorted_index, int n, float* hot8, cudaStream_t s)
{
    count_launch();
    k_reference_leaf<<<1, 32, 0, s>>>(x, y, z, m, sorted_index, n, hot8);
}

} // namespace bz
