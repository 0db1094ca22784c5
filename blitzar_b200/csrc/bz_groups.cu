// Target groups for the group walk, cut from the octree.
//
// A group is at most gmax <= kGroupMax (one warp) consecutive sorted particles that the walk treats
// as one target box.  Fixed chunks of 32 consecutive Morton-ordered particles can straddle
// distant branches where the particles are sparse, and such a group's box (hence its list of
// opened nodes) grows without bound.  Groups are instead runs of consecutive sibling subtrees:
// for every node holding more than gmax particles, its children are visited in order;
// a child with more than gmax particles forms its own groups (recursively), and the
// other children are packed greedily into runs of at most gmax particles.  A small child
// whose particles are spread wide compared with its distance from the system's centre of mass
// ("sparse", below) is cut further in the same way, down to single particles.  A leaf above
// the limit (possible only at the depth limit) is cut into chunks of gmax.  A root with
// at most gmax particles is one group.  Every group is thus a contiguous particle range
// inside one node's box, and groups come out in sorted (Morton) order.
//
// Construction is one flag per group start (written by the node that owns the run) followed
// by an order-preserving compaction, so the table is deterministic.  The oracle restates the
// same rule (or_tree_groups).
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;                 // flags per thread: one 16-byte load
constexpr int kChunk = kThreads * kItems;  // flags per compaction block

constexpr float kSparseRatio = 0.5f;

// The system root of node k: its ancestor at root_level (node 0, the tree root, when
// root_level = 0).
__device__ __forceinline__ int system_root(const TreeArrays& t, int k, int root_level)
{
    if (root_level == 0)
        return 0;
    for (int guard = 0; guard <= kMaxLevels + 1 && t.level[k] > root_level; ++guard)
        k = t.parent[k];
    return k;
}

// A node with at most gmax particles is "sparse" when its tight box is wider than
// kSparseRatio times its distance from its system's centre of mass: its particles are spread
// over a region comparable to their distance from the bulk of the mass, and one box around all
// of them would make the walk open almost the whole tree.  A system root is never sparse.
// Evaluated with round-to-nearest intrinsics (no contraction), as the oracle does.
__device__ __forceinline__ bool node_sparse(const TreeArrays& t, int k, int root_level, float cx,
                                            float cy, float cz)
{
    if (t.level[k] <= root_level)
        return false;
    const float4 b0 = t.box0[k];
    const float4 b1 = t.box1[k];
    const float ex = __fsub_rn(b1.x, b0.x), ey = __fsub_rn(b1.y, b0.y), ez = __fsub_rn(b1.z, b0.z);
    const float e = fmaxf(ex, fmaxf(ey, ez));
    const float dx = fmaxf(fmaxf(__fsub_rn(b0.x, cx), __fsub_rn(cx, b1.x)), 0.0f);
    const float dy = fmaxf(fmaxf(__fsub_rn(b0.y, cy), __fsub_rn(cy, b1.y)), 0.0f);
    const float dz = fmaxf(fmaxf(__fsub_rn(b0.z, cz), __fsub_rn(cz, b1.z)), 0.0f);
    const float d = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    return e > __fmul_rn(kSparseRatio, d);
}

// A node is split (its particles do not all share one group) when it holds more than gmax
// particles, or when it is sparse and its parent is split.
__device__ bool node_split(const TreeArrays& t, int k, int gmax, int root_level, float cx, float cy,
                           float cz)
{
    int j = k;
    for (int guard = 0; guard <= kMaxLevels + 1; ++guard) {
        if (t.count[j] > gmax)
            return true;
        if (!node_sparse(t, j, root_level, cx, cy, cz))
            return false;
        j = t.parent[j];
        if (j < 0)
            return false;
    }
    return false;
}

__global__ void __launch_bounds__(kThreads) k_group_flags(TreeArrays t, int n, int gmax,
                                                           int root_level, unsigned char* __restrict__ flag)
{
    const int nodes = *t.n_nodes;
    for (int k = blockIdx.x * kThreads + threadIdx.x; k < nodes; k += gridDim.x * kThreads) {
        const int lev = t.level[k];
        if (lev < root_level)
            continue;  // above the systems: they cut their own groups
        const int cnt = t.count[k];
        const int st = t.start[k];
        const int nch = t.nchild[k];
        if (lev == root_level && cnt <= gmax) {
            flag[st] = 1;  // a small system is one group
            continue;
        }
        const float4 com = t.mono[system_root(t, k, root_level)];
        if (!node_split(t, k, gmax, root_level, com.x, com.y, com.z))
            continue;
        if (nch == 0) {
            // a split leaf: chunks of gmax, or single particles when sparse
            const int step = cnt > gmax ? gmax : 1;
            for (int i = 0; i < cnt; i += step)
                flag[st + i] = 1;
            continue;
        }
        const int c0 = t.child[k];
        int run = 0;
        for (int c = c0; c < c0 + nch; ++c) {
            const int cc = t.count[c];
            if (cc > gmax || node_sparse(t, c, root_level, com.x, com.y, com.z)) {
                run = 0;  // the child cuts its own groups
                continue;
            }
            if (run == 0 || run + cc > gmax) {
                flag[t.start[c]] = 1;
                run = 0;
            }
            run += cc;
        }
    }
}

// Ensembles: the node of each system's root, by system id (key bits 54..62).
__global__ void k_system_roots(TreeArrays t, int root_level, const unsigned long long* __restrict__ keys,
                               int* __restrict__ sysroot)
{
    const int nodes = *t.n_nodes;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nodes; k += gridDim.x * blockDim.x)
        if (t.level[k] == root_level && t.count[k] > 0)
            sysroot[static_cast<int>(keys[t.start[k]] >> 54)] = k;
}

// Flags set among the 16 bytes of v (each byte 0 or 1).
__device__ __forceinline__ int flags_in(const uint4 v)
{
    return __popc(v.x & 0x01010101u) + __popc(v.y & 0x01010101u) + __popc(v.z & 0x01010101u) +
           __popc(v.w & 0x01010101u);
}

__global__ void __launch_bounds__(kThreads) k_flag_count(const unsigned char* __restrict__ flag, int n,
                                                          int* __restrict__ block_sums)
{
    // the flag array is zero past n up to a whole chunk: every thread reads its 16 bytes
    const uint4 v = reinterpret_cast<const uint4*>(flag + static_cast<size_t>(blockIdx.x) * kChunk)[threadIdx.x];
    int c = flags_in(v);
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(kFullMask, c, o);
    __shared__ int ws[kThreads / 32];
    if ((threadIdx.x & 31) == 0)
        ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kThreads / 32; ++w)
            s += ws[w];
        block_sums[blockIdx.x] = s;
    }
}

// Exclusive scan of the block sums in one block; also writes the group count.
__global__ void __launch_bounds__(1024) k_flag_scan(int* __restrict__ block_sums, int blocks,
                                                     int* __restrict__ ngroups)
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
        int x = warp_incl_scan(v);
        if (lane == 31)
            ws[warp] = x;
        __syncthreads();
        if (warp == 0) {
            const int y = warp_incl_scan(ws[lane]);
            ws[lane] = y;
        }
        __syncthreads();
        const int before = (warp > 0 ? ws[warp - 1] : 0) + carry;
        if (i < blocks)
            block_sums[i] = before + x - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *ngroups = carry;
}

// Writes the sorted index of every flagged position at its rank, plus the end sentinel n.  Thread
// t of a block takes the 16 consecutive flags at t * 16 of the block's chunk: a warp scan of the
// threads' counts and one scan of the warp totals place every flag.
__global__ void __launch_bounds__(kThreads) k_flag_emit(const unsigned char* __restrict__ flag, int n,
                                                         const int* __restrict__ block_offsets,
                                                         const int* __restrict__ ngroups,
                                                         int* __restrict__ gstart,
                                                         int* __restrict__ groot,
                                                         const unsigned long long* __restrict__ keys,
                                                         const int* __restrict__ sysroot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * kChunk + threadIdx.x * kItems;
    const uint4 v = reinterpret_cast<const uint4*>(flag + static_cast<size_t>(blockIdx.x) * kChunk)[threadIdx.x];
    const int c = flags_in(v);
    const int incl = warp_incl_scan(c);
    __shared__ int ws[kThreads / 32];
    if (lane == 31)
        ws[warp] = incl;
    __syncthreads();
    int before = block_offsets[blockIdx.x] + incl - c;
    for (int w = 0; w < warp; ++w)
        before += ws[w];
    if (c > 0) {
        const unsigned words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            if ((words[j >> 2] >> (8 * (j & 3))) & 1u) {
                const int idx = base + j;  // flags are zero past n
                gstart[before] = idx;
                groot[before] = sysroot ? sysroot[static_cast<int>(keys[idx] >> 54)] : 0;
                ++before;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        gstart[*ngroups] = n;
}

int sms_now()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

} // namespace

int group_count_blocks(int n) { return (n + kChunk - 1) / kChunk > 0 ? (n + kChunk - 1) / kChunk : 1; }
size_t group_flag_bytes(int n) { return static_cast<size_t>(group_count_blocks(n)) * kChunk; }

void launch_groups(const TreeArrays& t, int n, int gmax, int root_level,
                   const unsigned long long* keys, GroupTable& g, cudaStream_t s)
{
    gmax = gmax < 1 ? 1 : (gmax > kGroupMax ? kGroupMax : gmax);
    cudaMemsetAsync(g.flag, 0, group_flag_bytes(n), s);
    const int sms = sms_now();
    int fb = (t.cap + kThreads - 1) / kThreads;
    fb = fb < 8 * sms ? fb : 8 * sms;
    count_launch();
    k_group_flags<<<fb > 0 ? fb : 1, kThreads, 0, s>>>(t, n, gmax, root_level, g.flag);
    if (root_level > 0) {
        count_launch();
        k_system_roots<<<fb > 0 ? fb : 1, kThreads, 0, s>>>(t, root_level, keys, g.sysroot);
    }
    const int blocks = group_count_blocks(n);
    count_launch();
    k_flag_count<<<blocks, kThreads, 0, s>>>(g.flag, n, g.block_sums);
    count_launch();
    k_flag_scan<<<1, 1024, 0, s>>>(g.block_sums, blocks, g.ngroups);
    count_launch();
    k_flag_emit<<<blocks, kThreads, 0, s>>>(g.flag, n, g.block_sums, g.ngroups, g.gstart, g.groot,
                                            keys, root_level > 0 ? g.sysroot : nullptr);
}

} // namespace bz
