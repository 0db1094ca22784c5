// Adaptive block time steps: power-of-two levels, hierarchical kick-drift-kick.
//
// A particle on level k takes steps of dt_k = dt_max / 2^k.  One block step of dt_max runs
// 2^L substeps of dt_max / 2^L, where L is the finest level present at the start of the
// block.  At substep s a particle of level k opens a step (half kick with its cached
// acceleration) when s is a multiple of 2^(L-k); every particle drifts; a particle closes its
// step when s + 1 is such a multiple: its force is evaluated at the new positions (the walk
// skips groups without such a particle), it receives the closing half kick and picks its next
// level.  The level rule is the reference's (engine/physics/core/cuda/integration/
// CudAdaptive.inl:42-71): stable dt = min(dt_max, eta sqrt(eps / |a|), eta eps / |v|) and the
// smallest level whose dt does not exceed it, capped at the maximum level.  A particle may
// only move to a coarser level at a time its coarser step is aligned with; within a block it
// is also capped at the block's level L.  At the end of a block every particle is closed, so
// block steps compose exactly like plain leapfrog steps (level 0 for everyone reproduces the
// plain KDK step bit for bit).
//
// Levels and cached accelerations are stored by caller index, so the per-substep re-sort
// (which permutes the state) leaves them in place.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;

int grid_for(int n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int b = (n + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b < 8 * sms ? b : 8 * sms);
}

__device__ __forceinline__ int choose_level(float ax, float ay, float az, double vx, double vy,
                                            double vz, float eta, float eps, float dt_max,
                                            int max_level)
{
    const float safe = fmaxf(eps, 1.0e-6f);
    const float am = sqrtf(ax * ax + ay * ay + az * az);
    const float vm = static_cast<float>(sqrt(vx * vx + vy * vy + vz * vz));
    const float adt = am > 1.0e-6f ? eta * sqrtf(safe / am) : dt_max;
    const float vdt = vm > 1.0e-6f ? eta * safe / vm : dt_max;
    const float stable = fminf(dt_max, fminf(adt, vdt));
    for (int l = 0; l <= max_level; ++l)
        if (dt_max / static_cast<float>(1u << l) <= stable)
            return l;
    return max_level;
}

// Levels allowed to change at the end of substep s (boundary s + 1 of a block of 2^L):
// the coarsest level aligned with that boundary.
__device__ __forceinline__ int aligned_level(int boundary, int L)
{
    if (boundary >= (1 << L))
        return 0;
    return L - (__ffs(boundary) - 1);
}

// After a force evaluation of every particle (set-up, or the end of a block): cache the
// accelerations by caller index and pick each particle's level.
__global__ void __launch_bounds__(kThreads) k_adaptive_init(const float* __restrict__ ax,
                                                             const float* __restrict__ ay,
                                                             const float* __restrict__ az,
                                                             const double* __restrict__ vx,
                                                             const double* __restrict__ vy,
                                                             const double* __restrict__ vz,
                                                             const int* __restrict__ id, int n,
                                                             AdaptiveParams p, AdaptiveState a)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const int c = id[i];
        a.ax[c] = ax[i];
        a.ay[c] = ay[i];
        a.az[c] = az[i];
        a.level[c] = static_cast<unsigned char>(
            choose_level(ax[i], ay[i], az[i], vx[i], vy[i], vz[i], p.eta, p.eps,
                         static_cast<float>(p.dt_max), p.max_level));
    }
}

__global__ void k_level_max(const unsigned char* __restrict__ level, int n, int* __restrict__ out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, static_cast<int>(level[i]));
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(kFullMask, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(out, m);
}

// Opening half kicks of the particles whose step starts at substep s, then the drift of all.
__global__ void __launch_bounds__(kThreads) k_adaptive_open_drift(double* __restrict__ x,
                                                                   double* __restrict__ y,
                                                                   double* __restrict__ z,
                                                                   double* __restrict__ vx,
                                                                   double* __restrict__ vy,
                                                                   double* __restrict__ vz,
                                                                   const int* __restrict__ id, int n,
                                                                   AdaptiveParams p, AdaptiveState a,
                                                                   int s, int L)
{
    const double sub = p.dt_max / static_cast<double>(1 << L);
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const int c = id[i];
        const int k = min(static_cast<int>(a.level[c]), L);
        double ux = vx[i], uy = vy[i], uz = vz[i];
        if ((s & ((1 << (L - k)) - 1)) == 0) {
            const double h = 0.5 * p.dt_max / static_cast<double>(1 << k);
            ux += static_cast<double>(a.ax[c]) * h;
            uy += static_cast<double>(a.ay[c]) * h;
            uz += static_cast<double>(a.az[c]) * h;
            vx[i] = ux;
            vy[i] = uy;
            vz[i] = uz;
        }
        x[i] += ux * sub;
        y[i] += uy * sub;
        z[i] += uz * sub;
    }
}

// Which sorted slots close their step at boundary s + 1.
__global__ void __launch_bounds__(kThreads) k_adaptive_active(const int* __restrict__ id, int n,
                                                               AdaptiveState a, int s, int L,
                                                               unsigned char* __restrict__ active)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const int k = min(static_cast<int>(a.level[id[i]]), L);
        active[i] = ((s + 1) & ((1 << (L - k)) - 1)) == 0 ? 1 : 0;
    }
}

// Closing half kicks with the fresh accelerations, cache them, pick the next levels.
__global__ void __launch_bounds__(kThreads) k_adaptive_close(const float* __restrict__ ax,
                                                              const float* __restrict__ ay,
                                                              const float* __restrict__ az,
                                                              double* __restrict__ vx,
                                                              double* __restrict__ vy,
                                                              double* __restrict__ vz,
                                                              const int* __restrict__ id,
                                                              const unsigned char* __restrict__ active,
                                                              int n, AdaptiveParams p,
                                                              AdaptiveState a, int s, int L)
{
    unsigned long long count = 0;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        if (!active[i])
            continue;
        ++count;
        const int c = id[i];
        const int k = min(static_cast<int>(a.level[c]), L);
        const double h = 0.5 * p.dt_max / static_cast<double>(1 << k);
        const double ux = vx[i] + static_cast<double>(ax[i]) * h;
        const double uy = vy[i] + static_cast<double>(ay[i]) * h;
        const double uz = vz[i] + static_cast<double>(az[i]) * h;
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        a.ax[c] = ax[i];
        a.ay[c] = ay[i];
        a.az[c] = az[i];
        const int want = choose_level(ax[i], ay[i], az[i], ux, uy, uz, p.eta, p.eps,
                                      static_cast<float>(p.dt_max), p.max_level);
        const int lo = aligned_level(s + 1, L);  // coarsest level this boundary allows
        const int hi = (s + 1 >= (1 << L)) ? p.max_level : L;  // no finer than the block's L
        a.level[c] = static_cast<unsigned char>(min(max(want, lo), hi));
    }
    for (int o = 16; o > 0; o >>= 1)
        count += __shfl_xor_sync(kFullMask, count, o);
    if ((threadIdx.x & 31) == 0 && count)
        atomicAdd(a.updates, count);
}

} // namespace

void launch_adaptive_init(const float* ax, const float* ay, const float* az, const double* vx,
                          const double* vy, const double* vz, const int* id, int n,
                          const AdaptiveParams& p, const AdaptiveState& a, cudaStream_t s)
{
    count_launch();
    k_adaptive_init<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, vx, vy, vz, id, n, p, a);
}

void launch_level_max(const unsigned char* level, int n, int* out, cudaStream_t s)
{
    cudaMemsetAsync(out, 0, sizeof(int), s);
    count_launch();
    k_level_max<<<grid_for(n), kThreads, 0, s>>>(level, n, out);
}

void launch_adaptive_open_drift(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                                const int* id, int n, const AdaptiveParams& p, const AdaptiveState& a,
                                int sub, int L, cudaStream_t s)
{
    count_launch();
    k_adaptive_open_drift<<<grid_for(n), kThreads, 0, s>>>(x, y, z, vx, vy, vz, id, n, p, a, sub, L);
}

void launch_adaptive_active(const int* id, int n, const AdaptiveState& a, int sub, int L,
                            unsigned char* active, cudaStream_t s)
{
    count_launch();
    k_adaptive_active<<<grid_for(n), kThreads, 0, s>>>(id, n, a, sub, L, active);
}

void launch_adaptive_close(const float* ax, const float* ay, const float* az, double* vx, double* vy,
                           double* vz, const int* id, const unsigned char* active, int n,
                           const AdaptiveParams& p, const AdaptiveState& a, int sub, int L,
                           cudaStream_t s)
{
    count_launch();
    k_adaptive_close<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, vx, vy, vz, id, active, n, p, a, sub, L);
}

} // namespace bz
