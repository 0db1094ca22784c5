// Bounding boxes and 63-bit Morton keys.
//
// Replaces the reference's thrust::transform_reduce bbox + buildMortonCodesKernel
// (engine/physics/octree/cuda/linear/OctBuild.inl:64-86, OctKeyKernels.inl:22-46): the box is
// reduced on the device (no host round trip) and the key kernel reads it from device memory,
// so the whole step can live in one CUDA graph.  HBM-bound: 24 B read + 12 B written per
// particle in production mode.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;

__global__ void k_bbox_init(BoxF64* box)
{
    if (threadIdx.x < 3) {
        box->mn[threadIdx.x] = 0xffffffffffffffffull;
        box->mx[threadIdx.x] = 0ull;
    }
}

// Block-reduced FP64 min/max, one atomic per block and axis.  Min/max are exact, so the
// result does not depend on the reduction order.
__global__ void __launch_bounds__(kThreads) k_bbox_f64(const double* __restrict__ x,
                                                        const double* __restrict__ y,
                                                        const double* __restrict__ z, int n,
                                                        BoxF64* box)
{
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const double p[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = fmin(mn[a], p[a]);
            mx[a] = fmax(mx[a], p[a]);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fmin(mn[a], __shfl_xor_sync(kFullMask, mn[a], o));
            mx[a] = fmax(mx[a], __shfl_xor_sync(kFullMask, mx[a], o));
        }
    }
    __shared__ double smn[3][kThreads / 32], smx[3][kThreads / 32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            smn[a][w] = mn[a];
            smx[a][w] = mx[a];
        }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int a = threadIdx.x;
        double m0 = smn[a][0], m1 = smx[a][0];
        for (int k = 1; k < kThreads / 32; ++k) {
            m0 = fmin(m0, smn[a][k]);
            m1 = fmax(m1, smx[a][k]);
        }
        if (m0 <= m1) {
            atomicMin(&box->mn[a], ordered_from_double(m0));
            atomicMax(&box->mx[a], ordered_from_double(m1));
        }
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long v)
{
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__device__ __forceinline__ unsigned long long quantise21(double p, double origin, double scale)
{
    double t = floor(__dmul_rn(__dsub_rn(p, origin), scale));
    t = t >= 0.0 ? t : 0.0;  // also maps NaN to 0
    t = fmin(t, 2097151.0);
    return static_cast<unsigned long long>(t);
}

// Production key: floor((p - origin) * 2^21 / size) per axis, interleaved x<<2 | y<<1 | z.
// Every key prefix of 3l bits is then an exact geometric cell of the cube at level l.
__global__ void __launch_bounds__(kThreads) k_keys63(const double* __restrict__ x,
                                                      const double* __restrict__ y,
                                                      const double* __restrict__ z, int n,
                                                      const BoxF64* __restrict__ box,
                                                      double periodic_len,
                                                      unsigned long long* __restrict__ keys,
                                                      uint32_t* __restrict__ perm)
{
    double o[3], size;
    if (periodic_len > 0.0) {
        o[0] = o[1] = o[2] = 0.0;
        size = periodic_len;
    } else {
        double mn[3], mx[3];
        for (int a = 0; a < 3; ++a) {
            mn[a] = double_from_ordered(box->mn[a]);
            mx[a] = double_from_ordered(box->mx[a]);
        }
        size = fmax(fmax(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
        if (!(size > 0.0))
            size = 1.0;
        for (int a = 0; a < 3; ++a)
            o[a] = mn[a];
    }
    const double scale = __ddiv_rn(2097152.0, size);
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const unsigned long long qx = quantise21(x[i], o[0], scale);
        const unsigned long long qy = quantise21(y[i], o[1], scale);
        const unsigned long long qz = quantise21(z[i], o[2], scale);
        keys[i] = (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz);
        perm[i] = static_cast<uint32_t>(i);
    }
}

// ---- reference-compatible keys ---------------------------------------------------------

__device__ __forceinline__ unsigned ordered_from_float(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_from_ordered(unsigned u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_bbox32_init(unsigned* b)
{
    if (threadIdx.x < 3) {
        b[threadIdx.x] = 0xffffffffu;
        b[3 + threadIdx.x] = 0u;
    }
}

__global__ void __launch_bounds__(kThreads) k_bbox_f32(const float* __restrict__ x,
                                                        const float* __restrict__ y,
                                                        const float* __restrict__ z, int n,
                                                        unsigned* b)
{
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        mn[0] = fminf(mn[0], x[i]);
        mn[1] = fminf(mn[1], y[i]);
        mn[2] = fminf(mn[2], z[i]);
        mx[0] = fmaxf(mx[0], x[i]);
        mx[1] = fmaxf(mx[1], y[i]);
        mx[2] = fmaxf(mx[2], z[i]);
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(kFullMask, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(kFullMask, mx[a], o));
        }
        if ((threadIdx.x & 31) == 0 && mn[a] <= mx[a]) {
            atomicMin(&b[a], ordered_from_float(mn[a]));
            atomicMax(&b[3 + a], ordered_from_float(mx[a]));
        }
    }
}

// The reference's bit spread (engine/physics/octree/morton/OctMortonCodes.inl:7-14): 10-bit
// masks on a 32-bit word, so only bits 0..9 of each 21-bit coordinate survive.
__device__ __forceinline__ unsigned long long ref_spread(unsigned v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return static_cast<unsigned long long>(v);
}

// OctKeyKernels.inl:31-45.  The reference is compiled with nvcc's default contraction, so
// `n * 2097151.0f + 0.5f` executes as one fused multiply-add there; it is written as an
// explicit fma here, and every other operation with _rn intrinsics so that nothing else is
// contracted.
__device__ __forceinline__ unsigned ref_quantise(float p, float mn, float inv)
{
    const float t = fminf(fmaxf(__fmul_rn(__fsub_rn(p, mn), inv), 0.0f), 1.0f);
    const unsigned q = static_cast<unsigned>(__fmaf_rn(t, 2097151.0f, 0.5f));
    return q < 2097151u ? q : 2097151u;
}

__global__ void __launch_bounds__(kThreads) k_keys_reference(const float* __restrict__ x,
                                                              const float* __restrict__ y,
                                                              const float* __restrict__ z,
                                                              int n, const unsigned* b,
                                                              unsigned long long* keys,
                                                              uint32_t* perm)
{
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = float_from_ordered(b[a]);
        mx[a] = float_from_ordered(b[3 + a]);
    }
    const float invX = __fdiv_rn(1.0f, fmaxf(__fsub_rn(mx[0], mn[0]), 1.0e-12f));
    const float invY = __fdiv_rn(1.0f, fmaxf(__fsub_rn(mx[1], mn[1]), 1.0e-12f));
    const float invZ = __fdiv_rn(1.0f, fmaxf(__fsub_rn(mx[2], mn[2]), 1.0e-12f));
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const unsigned qx = ref_quantise(x[i], mn[0], invX);
        const unsigned qy = ref_quantise(y[i], mn[1], invY);
        const unsigned qz = ref_quantise(z[i], mn[2], invZ);
        keys[i] = (ref_spread(qx) << 2) | (ref_spread(qy) << 1) | ref_spread(qz);
        perm[i] = static_cast<uint32_t>(i);
    }
}

// ---- ensembles: per-system boxes and keys (system id in the top 9 bits, 18 bits per axis)

__device__ __forceinline__ int system_of(const long long* __restrict__ offsets, int systems, int id)
{
    int lo = 0, hi = systems;  // offsets[lo] <= id < offsets[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (offsets[mid] <= id)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_sys_box_init(BoxF64* boxes, int systems)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < systems; s += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            boxes[s].mn[a] = 0xffffffffffffffffull;
            boxes[s].mx[a] = 0ull;
        }
}

// Per-system FP64 min/max.  Particles of a system are contiguous in both the caller's and the
// sorted order, so a warp usually holds one system: it then reduces by shuffles and issues one
// atomic per axis; mixed warps fall back to per-lane atomics.  Exact either way.
__global__ void __launch_bounds__(kThreads) k_sys_bbox(const double* __restrict__ x,
                                                        const double* __restrict__ y,
                                                        const double* __restrict__ z,
                                                        const int* __restrict__ id, int n,
                                                        const long long* __restrict__ offsets,
                                                        int systems, BoxF64* boxes)
{
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * kThreads; base < n; base += gridDim.x * kThreads) {
        const int i = base + threadIdx.x;
        const bool valid = i < n;
        const int sys = valid ? system_of(offsets, systems, id[i]) : -1;
        double p[3] = {0.0, 0.0, 0.0};
        if (valid) {
            p[0] = x[i];
            p[1] = y[i];
            p[2] = z[i];
        }
        const int s0 = __shfl_sync(kFullMask, sys, 0);
        const bool uniform = __all_sync(kFullMask, !valid || sys == s0) && s0 >= 0;
        if (uniform) {
            for (int a = 0; a < 3; ++a) {
                double mn = valid ? p[a] : 1e300, mx = valid ? p[a] : -1e300;
                for (int o = 16; o > 0; o >>= 1) {
                    mn = fmin(mn, __shfl_xor_sync(kFullMask, mn, o));
                    mx = fmax(mx, __shfl_xor_sync(kFullMask, mx, o));
                }
                if (lane == 0) {
                    atomicMin(&boxes[s0].mn[a], ordered_from_double(mn));
                    atomicMax(&boxes[s0].mx[a], ordered_from_double(mx));
                }
            }
        } else if (valid) {
            for (int a = 0; a < 3; ++a) {
                atomicMin(&boxes[sys].mn[a], ordered_from_double(p[a]));
                atomicMax(&boxes[sys].mx[a], ordered_from_double(p[a]));
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_keys_ensemble(const double* __restrict__ x,
                                                             const double* __restrict__ y,
                                                             const double* __restrict__ z,
                                                             const int* __restrict__ id, int n,
                                                             const long long* __restrict__ offsets,
                                                             int systems,
                                                             const BoxF64* __restrict__ boxes,
                                                             unsigned long long* __restrict__ keys,
                                                             uint32_t* __restrict__ perm)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const int sys = system_of(offsets, systems, id[i]);
        const BoxF64 b = boxes[sys];
        double o[3], mx[3];
        for (int a = 0; a < 3; ++a) {
            o[a] = double_from_ordered(b.mn[a]);
            mx[a] = double_from_ordered(b.mx[a]);
        }
        double size = fmax(fmax(mx[0] - o[0], mx[1] - o[1]), mx[2] - o[2]);
        if (!(size > 0.0))
            size = 1.0;
        const double scale = __ddiv_rn(262144.0, size);
        const double p[3] = {x[i], y[i], z[i]};
        unsigned long long q[3];
        for (int a = 0; a < 3; ++a) {
            double t = floor(__dmul_rn(__dsub_rn(p[a], o[a]), scale));
            t = t >= 0.0 ? t : 0.0;
            q[a] = static_cast<unsigned long long>(fmin(t, 262143.0));
        }
        keys[i] = (static_cast<unsigned long long>(sys) << 54) | (spread21(q[0]) << 2) |
                  (spread21(q[1]) << 1) | spread21(q[2]);
        perm[i] = static_cast<uint32_t>(i);
    }
}

int grid_for(int n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int want = (n + kThreads - 1) / kThreads;
    const int cap = sms * 8;
    return want < 1 ? 1 : (want < cap ? want : cap);
}

} // namespace

void launch_bbox_f64(const double* x, const double* y, const double* z, int n, BoxF64* box,
                     cudaStream_t s)
{
    count_launch();
    k_bbox_init<<<1, 32, 0, s>>>(box);
    count_launch();
    k_bbox_f64<<<grid_for(n), kThreads, 0, s>>>(x, y, z, n, box);
}

void launch_keys_ensemble(const double* x, const double* y, const double* z, const int* id, int n,
                          const long long* offsets, int systems, BoxF64* boxes,
                          unsigned long long* keys, uint32_t* perm, cudaStream_t s)
{
    count_launch();
    k_sys_box_init<<<(systems + 255) / 256, 256, 0, s>>>(boxes, systems);
    count_launch();
    k_sys_bbox<<<grid_for(n), kThreads, 0, s>>>(x, y, z, id, n, offsets, systems, boxes);
    count_launch();
    k_keys_ensemble<<<grid_for(n), kThreads, 0, s>>>(x, y, z, id, n, offsets, systems, boxes, keys, perm);
}

void launch_keys63(const double* x, const double* y, const double* z, int n,
                   const BoxF64* box, double periodic_len, unsigned long long* keys,
                   uint32_t* perm, cudaStream_t s)
{
    count_launch();
    k_keys63<<<grid_for(n), kThreads, 0, s>>>(x, y, z, n, box, periodic_len, keys, perm);
}

void launch_keys_reference(const float* x, const float* y, const float* z, int n,
                           unsigned* bbox_ordered6, unsigned long long* keys, uint32_t* perm,
                           cudaStream_t s)
{
    count_launch();
    k_bbox32_init<<<1, 32, 0, s>>>(bbox_ordered6);
    count_launch();
    k_bbox_f32<<<grid_for(n), kThreads, 0, s>>>(x, y, z, n, bbox_ordered6);
    count_launch();
    k_keys_reference<<<grid_for(n), kThreads, 0, s>>>(x, y, z, n, bbox_ordered6, keys, perm);
}

} // namespace bz
