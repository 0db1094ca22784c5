// Particle state maintenance: permutation into Morton order, FP64 leapfrog kick/drift and
// scatters back to the caller's particle order.
//
// The reference keeps FP32 state and runs leapfrog as KDK with two force evaluations per step
// (engine/physics/core/cuda/integration/CudOctreeGpuIntegrators.inl:121-195, kernels in
// CudParticleKernels.inl:94-220).  Here positions and velocities are FP64, the force from the
// end of one step is reused as the first kick of the next (one evaluation per step, the same
// trajectory), and the state is physically re-ordered by the sort each step so that every
// later kernel streams it in Morton order.
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
    int b = (n + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b < sms * 8 ? b : sms * 8);
}

struct PermuteArgs {
    const double* src[6];
    double* dst[6];
};

__global__ void __launch_bounds__(kThreads) k_permute(const uint32_t* __restrict__ perm, int n,
                                                       PermuteArgs a, int nd,
                                                       const float* __restrict__ msrc,
                                                       float* __restrict__ mdst,
                                                       const int* __restrict__ idsrc,
                                                       int* __restrict__ iddst,
                                                       float4* __restrict__ pos4)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const uint32_t j = perm[i];
        double v[6];
#pragma unroll
        for (int c = 0; c < 6; ++c)
            if (c < nd) {
                v[c] = a.src[c][j];
                a.dst[c][i] = v[c];
            }
        const float m = msrc[j];
        mdst[i] = m;
        iddst[i] = idsrc[j];
        pos4[i] = make_float4(static_cast<float>(v[0]), static_cast<float>(v[1]),
                              static_cast<float>(v[2]), m);
    }
}

// Closing half kick.  With (bx, by, bz) (the mesh leg's accelerations from the second stream)
// the accelerations are first completed in place, a = clamp(a + b), as k_add3 would.
__global__ void __launch_bounds__(kThreads) k_kick(double* __restrict__ vx, double* __restrict__ vy,
                                                    double* __restrict__ vz,
                                                    float* __restrict__ ax,
                                                    float* __restrict__ ay,
                                                    float* __restrict__ az, int n,
                                                    const double* __restrict__ dt_half,
                                                    const float* __restrict__ bx,
                                                    const float* __restrict__ by,
                                                    const float* __restrict__ bz, float max_acc)
{
    const double h = *dt_half;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        float a[3] = {ax[i], ay[i], az[i]};
        if (bx) {
            a[0] += bx[i];
            a[1] += by[i];
            a[2] += bz[i];
            clamp_acceleration(a[0], a[1], a[2], max_acc);
            ax[i] = a[0];
            ay[i] = a[1];
            az[i] = a[2];
        }
        vx[i] += static_cast<double>(a[0]) * h;
        vy[i] += static_cast<double>(a[1]) * h;
        vz[i] += static_cast<double>(a[2]) * h;
    }
}

__device__ __forceinline__ double wrap_periodic(double x, double L)
{
    if (L <= 0.0)
        return x;
    x -= L * floor(x / L);
    return x >= L ? 0.0 : x;
}

// Kick with the cached acceleration (kick_frac x dt: half for leapfrog, whole for symplectic
// Euler), full drift with the kicked velocity, periodic wrap; for open boundaries the FP64 box
// of the drifted positions is reduced in the same pass.
__global__ void __launch_bounds__(kThreads) k_kick_drift(double* __restrict__ x,
                                                          double* __restrict__ y,
                                                          double* __restrict__ z,
                                                          double* __restrict__ vx,
                                                          double* __restrict__ vy,
                                                          double* __restrict__ vz,
                                                          const float* __restrict__ ax,
                                                          const float* __restrict__ ay,
                                                          const float* __restrict__ az, int n,
                                                          const double* __restrict__ dtp,
                                                          double L, BoxF64* box,
                                                          const float* __restrict__ mass,
                                                          float4* __restrict__ pos4, double kick_frac)
{
    const double dt = *dtp;
    const double h = kick_frac * dt;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const double ux = vx[i] + static_cast<double>(ax[i]) * h;
        const double uy = vy[i] + static_cast<double>(ay[i]) * h;
        const double uz = vz[i] + static_cast<double>(az[i]) * h;
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        const double p[3] = {wrap_periodic(x[i] + ux * dt, L), wrap_periodic(y[i] + uy * dt, L),
                             wrap_periodic(z[i] + uz * dt, L)};
        x[i] = p[0];
        y[i] = p[1];
        z[i] = p[2];
        if (pos4)  // FP32 copy in the current (pre-sort) order, as k_permute converts it
            pos4[i] = make_float4(static_cast<float>(p[0]), static_cast<float>(p[1]),
                                  static_cast<float>(p[2]), mass[i]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = fmin(mn[a], p[a]);
            mx[a] = fmax(mx[a], p[a]);
        }
    }
    if (box == nullptr)
        return;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fmin(mn[a], __shfl_xor_sync(kFullMask, mn[a], o));
            mx[a] = fmax(mx[a], __shfl_xor_sync(kFullMask, mx[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a)
            if (mn[a] <= mx[a]) {
                atomicMin(&box->mn[a], ordered_from_double(mn[a]));
                atomicMax(&box->mx[a], ordered_from_double(mx[a]));
            }
}

__global__ void k_box_reset(BoxF64* box)
{
    if (threadIdx.x < 3) {
        box->mn[threadIdx.x] = 0xffffffffffffffffull;
        box->mx[threadIdx.x] = 0ull;
    }
}

__global__ void __launch_bounds__(kThreads) k_scatter3(const float* __restrict__ ax,
                                                        const float* __restrict__ ay,
                                                        const float* __restrict__ az,
                                                        const int* __restrict__ id, int n,
                                                        float* __restrict__ out)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const int o = id[i];
        out[o] = ax[i];
        out[n + o] = ay[i];
        out[2 * n + o] = az[i];
    }
}

__global__ void __launch_bounds__(kThreads) k_f64_to_f32(const double* __restrict__ s,
                                                          float* __restrict__ d, int n)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads)
        d[i] = static_cast<float>(s[i]);
}

} // namespace

void launch_permute(const uint32_t* perm, int n, const double* const* src, double* const* dst,
                    int ndouble, const float* msrc, float* mdst, const int* idsrc, int* iddst,
                    float4* pos4, double periodic_len, cudaStream_t s)
{
    (void)periodic_len;
    PermuteArgs a{};
    for (int c = 0; c < ndouble && c < 6; ++c) {
        a.src[c] = src[c];
        a.dst[c] = dst[c];
    }
    count_launch();
    k_permute<<<grid_for(n), kThreads, 0, s>>>(perm, n, a, ndouble, msrc, mdst, idsrc, iddst, pos4);
}

void launch_kick(double* vx, double* vy, double* vz, float* ax, float* ay, float* az, int n,
                 const double* dt_half, cudaStream_t s, const float* bx, const float* by,
                 const float* bz, float max_acc)
{
    count_launch();
    k_kick<<<grid_for(n), kThreads, 0, s>>>(vx, vy, vz, ax, ay, az, n, dt_half, bx, by, bz,
                                            max_acc);
}

void launch_kick_drift(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                       const float* ax, const float* ay, const float* az, int n,
                       const double* dt, double periodic_len, BoxF64* box, cudaStream_t s,
                       const float* mass, float4* pos4, double kick_frac)
{
    if (box) {
        count_launch();
        k_box_reset<<<1, 32, 0, s>>>(box);
    }
    count_launch();
    k_kick_drift<<<grid_for(n), kThreads, 0, s>>>(x, y, z, vx, vy, vz, ax, ay, az, n, dt,
                                                  periodic_len, box, mass, pos4, kick_frac);
}

void launch_scatter3(const float* ax, const float* ay, const float* az, const int* id, int n,
                     float* out_soa3, cudaStream_t s)
{
    count_launch();
    k_scatter3<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, id, n, out_soa3);
}

namespace {
__global__ void __launch_bounds__(kThreads) k_add3(float* __restrict__ ax, float* __restrict__ ay,
                                                   float* __restrict__ az, const float* __restrict__ bx,
                                                   const float* __restrict__ by,
                                                   const float* __restrict__ bz, int n,
                                                   float max_acc)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        float x = ax[i] + bx[i], y = ay[i] + by[i], z = az[i] + bz[i];
        clamp_acceleration(x, y, z, max_acc);
        ax[i] = x;
        ay[i] = y;
        az[i] = z;
    }
}
} // namespace

namespace {
__global__ void __launch_bounds__(kThreads) k_refresh_pos4(const double* __restrict__ x,
                                                           const double* __restrict__ y,
                                                           const double* __restrict__ z,
                                                           const float* __restrict__ m, int n,
                                                           float4* __restrict__ pos4)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads)
        pos4[i] = make_float4(static_cast<float>(x[i]), static_cast<float>(y[i]),
                              static_cast<float>(z[i]), m[i]);
}
} // namespace

void launch_refresh_pos4(const double* x, const double* y, const double* z, const float* m, int n,
                         float4* pos4, cudaStream_t s)
{
    count_launch();
    k_refresh_pos4<<<grid_for(n), kThreads, 0, s>>>(x, y, z, m, n, pos4);
}

void launch_add3(float* ax, float* ay, float* az, const float* bx, const float* by, const float* bz,
                 int n, float max_acc, cudaStream_t s)
{
    count_launch();
    k_add3<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, bx, by, bz, n, max_acc);
}

void launch_f64_to_f32(const double* src, float* dst, int n, cudaStream_t s)
{
    count_launch();
    k_f64_to_f32<<<grid_for(n), kThreads, 0, s>>>(src, dst, n);
}

namespace {

constexpr int kEnergyBlocks = 1024;

// Per-block FP64 partial sums of {sum m v^2 / 2, sum m phi / 2, sum m vx, sum m vy, sum m vz};
// blocks write their partials and a single block adds them in block order (deterministic).
__global__ void __launch_bounds__(kThreads) k_energy_partials(
    const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
    const float* __restrict__ m, const float* __restrict__ pot, int n, double* __restrict__ part)
{
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const double mi = m[i];
        const double x = vx[i], y = vy[i], z = vz[i];
        acc[0] += 0.5 * mi * (x * x + y * y + z * z);
        if (pot)
            acc[1] += 0.5 * mi * static_cast<double>(pot[i]);
        acc[2] += mi * x;
        acc[3] += mi * y;
        acc[4] += mi * z;
    }
    __shared__ double red[5][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(kFullMask, v, o);
        if (lane == 0)
            red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w)
            v += red[threadIdx.x][w];
        part[threadIdx.x * kEnergyBlocks + blockIdx.x] = v;
    }
}

__global__ void k_energy_final(const double* __restrict__ part, int blocks, double* __restrict__ out)
{
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int b = 0; b < blocks; ++b)
            v += part[threadIdx.x * kEnergyBlocks + b];
        out[threadIdx.x] = v;
    }
}

} // namespace

size_t energy_scratch_doubles() { return 5 * static_cast<size_t>(kEnergyBlocks) + 8; }

void launch_energy(const double* vx, const double* vy, const double* vz, const float* m,
                   const float* pot, int n, double* scratch, cudaStream_t s)
{
    int blocks = grid_for(n);
    blocks = blocks < kEnergyBlocks ? blocks : kEnergyBlocks;
    count_launch();
    k_energy_partials<<<blocks, kThreads, 0, s>>>(vx, vy, vz, m, pot, n, scratch);
    count_launch();
    k_energy_final<<<1, 32, 0, s>>>(scratch, blocks, scratch + 5 * kEnergyBlocks);
}

} // namespace bz
