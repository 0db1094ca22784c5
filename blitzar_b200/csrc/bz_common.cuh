// Shared device helpers for the bzgrav CUDA kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bz {

// ---- device-side error bits (collected in one int per handle; the host turns any set bit
// into a bz_status instead of letting a kernel hang or trap).
enum DeviceError : int {
    kErrWalkStack = 1,      // group walk traversal stack would overflow
    kErrSortSpin = 2,       // radix-sort look-back gave up waiting for a predecessor tile
    kErrTreeCapacity = 4,   // more octree nodes than the preallocated capacity
    kErrTreeSpin = 8,       // octree level look-back gave up waiting
    kErrBulkWait = 16,      // a bulk-copy or MMA mbarrier wait ran out of time
    kErrListCapacity = 32,  // an interaction list exceeded its shared-memory capacity
};

constexpr unsigned kFullMask = 0xffffffffu;
// Upper bound on polls of a flag written by another block / the copy engine.  Each poll
// backs off with __nanosleep, so this bounds a wait at roughly a few hundred milliseconds.
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ void raise_error(int* err, int bit) { atomicOr(err, bit); }

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFullMask, v, o);
        if (lane >= o)
            v += t;
    }
    return v;
}

// The acceleration clamp of the reference (clampAcceleration, engine/physics/core/cuda/
// prelude/CudForceKernels.inl:7-14): a vector longer than max_acc is scaled to that length.
__device__ __forceinline__ void clamp_acceleration(float& x, float& y, float& z, float max_acc)
{
    const float norm = sqrtf(x * x + y * y + z * z);
    if (norm > max_acc && norm > 1e-12f) {
        const float s = max_acc / norm;
        x *= s;
        y *= s;
        z *= s;
    }
}

// Ordered-integer images of doubles so that atomicMin/atomicMax on unsigned long long give
// the IEEE order (used for the FP64 bounding box).
__device__ __forceinline__ unsigned long long ordered_from_double(double d)
{
    unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(d));
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double double_from_ordered(unsigned long long u)
{
    u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(u));
#else
    double d;
    __builtin_memcpy(&d, &u, sizeof(d));
    return d;
#endif
}

// ---- mbarrier + bulk copy (global -> shared, into this CTA only) -------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Returns true once the phase with the given parity has completed.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase has not completed sleeps (up to ns
// nanoseconds, or until the phase completes) instead of polling, leaving its issue slots to
// the other warps of the SM.
__device__ __forceinline__ bool mbar_try_wait_suspend(unsigned long long* bar, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: suspends on the mbarrier and gives up after about a second of device time
// (global timer), raising kErrBulkWait.
constexpr uint64_t kWaitLimitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity, int* err)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_ns();
    do {
        if (mbar_try_wait_suspend(bar, parity, 20000u))
            return true;
    } while (global_ns() - t0 < kWaitLimitNs);
    raise_error(err, kErrBulkWait);
    return false;
}

// 1-D bulk copy global -> shared completing on an mbarrier (cp.async.bulk, non-tensor,
// into this CTA only).  dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float rsqrt_approx(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Error-free transformation a + b = s + e (Knuth two-sum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

} // namespace bz
