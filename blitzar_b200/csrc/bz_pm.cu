// Periodic particle-mesh (long-range) leg of TreePM:
//   CIC deposit (float atomics onto the mesh, Morton-sorted particles for locality)
//   -> cuFFT R2C -> Green's function with Gaussian split, CIC window deconvolution and the
//      1/M^3 normalisation folded in (normalisation constant in FP64)
//   -> cuFFT C2R -> potential
//   -> per-particle CIC interpolation of the centred-difference gradient, fused: the three
//      gradient meshes of the reference are never written.
// Formulas follow the reference CPU templates driven with a periodic grid
// (engine/physics/treepm/deposit/TpmAssignment.inl:104-199,
//  engine/physics/treepm/field/TpmField.inl:6-89): mesh node i sits at i*h, density is
// mass/h^3, phi_k = 4 pi e^{-k^2 r_s^2} rho_k / (k^2 max(W, 0.08)), W = prod sinc^4(k h/2),
// acceleration = +centred difference of that phi.
#include <cufft.h>

#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

struct PmPlan {
    int mesh = 0;
    double box = 0.0;
    double rsplit = 0.0;
    float* rho = nullptr;          // M^3, later reused for phi
    cufftComplex* spec = nullptr;  // M*M*(M/2+1)
    double* green = nullptr;       // M*M*(M/2+1) precomputed Green x window x normalisation
    cufftHandle r2c = 0, c2r = 0;
    size_t bytes = 0;
};

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void cic_axis(float coord, float inv_h, int mesh, int& i0, int& i1,
                                         float& w0, float& w1)
{
    const float raw = coord * inv_h;
    const float m = static_cast<float>(mesh);
    const float s = raw - floorf(raw / m) * m;
    const float fl = floorf(s);
    int a = static_cast<int>(fl);
    a = a >= mesh ? a - mesh : (a < 0 ? a + mesh : a);
    i0 = a;
    i1 = a + 1 == mesh ? 0 : a + 1;
    w1 = s - fl;
    w0 = 1.0f - w1;
}

__global__ void __launch_bounds__(kThreads) k_deposit(const float4* __restrict__ pos4, int n,
                                                       int mesh, float inv_h, float inv_h3,
                                                       float* __restrict__ rho)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const float4 p = pos4[i];
        int x0, x1, y0, y1, z0, z1;
        float wx0, wx1, wy0, wy1, wz0, wz1;
        cic_axis(p.x, inv_h, mesh, x0, x1, wx0, wx1);
        cic_axis(p.y, inv_h, mesh, y0, y1, wy0, wy1);
        cic_axis(p.z, inv_h, mesh, z0, z1, wz0, wz1);
        const float m = p.w * inv_h3;
        const size_t M = static_cast<size_t>(mesh);
        const size_t r00 = (static_cast<size_t>(z0) * M + y0) * M, r01 = (static_cast<size_t>(z0) * M + y1) * M;
        const size_t r10 = (static_cast<size_t>(z1) * M + y0) * M, r11 = (static_cast<size_t>(z1) * M + y1) * M;
        atomicAdd(&rho[r00 + x0], m * wx0 * wy0 * wz0);
        atomicAdd(&rho[r00 + x1], m * wx1 * wy0 * wz0);
        atomicAdd(&rho[r01 + x0], m * wx0 * wy1 * wz0);
        atomicAdd(&rho[r01 + x1], m * wx1 * wy1 * wz0);
        atomicAdd(&rho[r10 + x0], m * wx0 * wy0 * wz1);
        atomicAdd(&rho[r10 + x1], m * wx1 * wy0 * wz1);
        atomicAdd(&rho[r11 + x0], m * wx0 * wy1 * wz1);
        atomicAdd(&rho[r11 + x1], m * wx1 * wy1 * wz1);
    }
}

__device__ __forceinline__ double sinc_d(double v) { return fabs(v) < 1.0e-5 ? 1.0 : sin(v) / v; }

// Green x deconvolution x 1/M^3, once per plan (depends only on mesh, box, r_s).
__global__ void k_green_table(int mesh, double box, double rsplit, double* green)
{
    const int hx = mesh / 2 + 1;
    const size_t total = static_cast<size_t>(mesh) * mesh * hx;
    const double h = box / mesh;
    const double ks = 2.0 * 3.14159265358979323846 / (mesh * h);
    const double norm = 1.0 / (static_cast<double>(mesh) * mesh * mesh);
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(idx % hx);
        const size_t pl = idx / hx;
        const int y = static_cast<int>(pl % mesh);
        const int z = static_cast<int>(pl / mesh);
        const int sy = y <= mesh / 2 ? y : y - mesh;
        const int sz = z <= mesh / 2 ? z : z - mesh;
        const double kx = x * ks, ky = sy * ks, kz = sz * ks;
        const double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 <= 1.0e-12) {
            green[idx] = 0.0;
            continue;
        }
        double wx = sinc_d(0.5 * kx * h), wy = sinc_d(0.5 * ky * h), wz = sinc_d(0.5 * kz * h);
        wx = wx * wx * wx * wx;
        wy = wy * wy * wy * wy;
        wz = wz * wz * wz * wz;
        double W = wx * wy * wz;
        if (W < 0.08)
            W = 0.08;
        green[idx] = 4.0 * 3.14159265358979323846 * exp(-k2 * rsplit * rsplit) / (k2 * W) * norm;
    }
}

__global__ void __launch_bounds__(kThreads) k_apply_green(cufftComplex* __restrict__ spec,
                                                           const double* __restrict__ green,
                                                           size_t total)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * kThreads) {
        const float g = static_cast<float>(green[i]);
        cufftComplex c = spec[i];
        c.x *= g;
        c.y *= g;
        spec[i] = c;
    }
}

// Interpolate the centred-difference gradient of phi with the CIC stencil.
__global__ void __launch_bounds__(kThreads) k_interp_gradient(const float4* __restrict__ pos4,
                                                               int n, int mesh, float inv_h,
                                                               const float* __restrict__ phi,
                                                               float* __restrict__ ax,
                                                               float* __restrict__ ay,
                                                               float* __restrict__ az)
{
    const float half_inv_h = 0.5f * inv_h;
    const size_t M = static_cast<size_t>(mesh);
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const float4 p = pos4[i];
        int xs[2], ys[2], zs[2];
        float wx[2], wy[2], wz[2];
        cic_axis(p.x, inv_h, mesh, xs[0], xs[1], wx[0], wx[1]);
        cic_axis(p.y, inv_h, mesh, ys[0], ys[1], wy[0], wy[1]);
        cic_axis(p.z, inv_h, mesh, zs[0], zs[1], wz[0], wz[1]);
        const int xm = xs[0] == 0 ? mesh - 1 : xs[0] - 1, xp = xs[1] + 1 == mesh ? 0 : xs[1] + 1;
        const int ym = ys[0] == 0 ? mesh - 1 : ys[0] - 1, yp = ys[1] + 1 == mesh ? 0 : ys[1] + 1;
        const int zm = zs[0] == 0 ? mesh - 1 : zs[0] - 1, zp = zs[1] + 1 == mesh ? 0 : zs[1] + 1;
        const int xa[4] = {xm, xs[0], xs[1], xp};
        const int ya[4] = {ym, ys[0], ys[1], yp};
        const int za[4] = {zm, zs[0], zs[1], zp};
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const size_t row = (static_cast<size_t>(za[c + 1]) * M + ya[b + 1]) * M;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const float w = wx[a] * wy[b] * wz[c];
                    const float dxp = __ldg(&phi[row + xa[a + 2]]) - __ldg(&phi[row + xa[a]]);
                    const float dyp = __ldg(&phi[(static_cast<size_t>(za[c + 1]) * M + ya[b + 2]) * M + xa[a + 1]]) -
                                      __ldg(&phi[(static_cast<size_t>(za[c + 1]) * M + ya[b]) * M + xa[a + 1]]);
                    const float dzp = __ldg(&phi[(static_cast<size_t>(za[c + 2]) * M + ya[b + 1]) * M + xa[a + 1]]) -
                                      __ldg(&phi[(static_cast<size_t>(za[c]) * M + ya[b + 1]) * M + xa[a + 1]]);
                    gx = fmaf(w, dxp, gx);
                    gy = fmaf(w, dyp, gy);
                    gz = fmaf(w, dzp, gz);
                }
            }
        ax[i] = gx * half_inv_h;
        ay[i] = gy * half_inv_h;
        az[i] = gz * half_inv_h;
    }
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

} // namespace

PmPlan* pm_create(int mesh, double box, double rsplit, cudaStream_t s, int* cuda_err)
{
    PmPlan* p = new PmPlan();
    p->mesh = mesh;
    p->box = box;
    p->rsplit = rsplit;
    const size_t cells = static_cast<size_t>(mesh) * mesh * mesh;
    const size_t half = static_cast<size_t>(mesh) * mesh * (mesh / 2 + 1);
    *cuda_err = 0;
    if (cudaMalloc(&p->rho, cells * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->spec, half * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc(&p->green, half * sizeof(double)) != cudaSuccess) {
        *cuda_err = 1;
        pm_destroy(p);
        return nullptr;
    }
    if (cufftPlan3d(&p->r2c, mesh, mesh, mesh, CUFFT_R2C) != CUFFT_SUCCESS ||
        cufftPlan3d(&p->c2r, mesh, mesh, mesh, CUFFT_C2R) != CUFFT_SUCCESS) {
        *cuda_err = 2;
        pm_destroy(p);
        return nullptr;
    }
    cufftSetStream(p->r2c, s);
    cufftSetStream(p->c2r, s);
    size_t ws1 = 0, ws2 = 0;
    cufftGetSize(p->r2c, &ws1);
    cufftGetSize(p->c2r, &ws2);
    p->bytes = cells * sizeof(float) + half * (sizeof(cufftComplex) + sizeof(double)) + ws1 + ws2;
    count_launch();
    k_green_table<<<sm_count() * 4, 256, 0, s>>>(mesh, box, rsplit, p->green);
    return p;
}

void pm_destroy(PmPlan* p)
{
    if (!p)
        return;
    if (p->r2c)
        cufftDestroy(p->r2c);
    if (p->c2r)
        cufftDestroy(p->c2r);
    cudaFree(p->rho);
    cudaFree(p->spec);
    cudaFree(p->green);
    delete p;
}

size_t pm_bytes(const PmPlan* p) { return p ? p->bytes : 0; }
float* pm_mesh(PmPlan* p) { return p->rho; }

void pm_deposit(PmPlan* p, const float4* pos4, int n, cudaStream_t s)
{
    const int M = p->mesh;
    const size_t cells = static_cast<size_t>(M) * M * M;
    const double h = p->box / M;
    const float inv_h = static_cast<float>(1.0 / h);
    const float inv_h3 = static_cast<float>(1.0 / (h * h * h));
    const int sms = sm_count();
    cudaMemsetAsync(p->rho, 0, cells * sizeof(float), s);
    int b = (n + kThreads - 1) / kThreads;
    b = b < sms * 8 ? b : sms * 8;
    count_launch();
    k_deposit<<<b, kThreads, 0, s>>>(pos4, n, M, inv_h, inv_h3, p->rho);
}

int pm_solve(PmPlan* p, cudaStream_t s)
{
    const int M = p->mesh;
    const size_t half = static_cast<size_t>(M) * M * (M / 2 + 1);
    if (cufftExecR2C(p->r2c, p->rho, p->spec) != CUFFT_SUCCESS)
        return 1;
    count_launch();
    k_apply_green<<<sm_count() * 4, kThreads, 0, s>>>(p->spec, p->green, half);
    if (cufftExecC2R(p->c2r, p->spec, p->rho) != CUFFT_SUCCESS)
        return 2;
    return 0;
}

void pm_interp(PmPlan* p, const float4* pos4, int n, float* ax, float* ay, float* az,
               cudaStream_t s)
{
    const int M = p->mesh;
    const float inv_h = static_cast<float>(1.0 / (p->box / M));
    const int sms = sm_count();
    int b = (n + kThreads - 1) / kThreads;
    b = b < sms * 8 ? b : sms * 8;
    count_launch();
    k_interp_gradient<<<b, kThreads, 0, s>>>(pos4, n, M, inv_h, p->rho, ax, ay, az);
}

int pm_forces(PmPlan* p, const float4* pos4, int n, float* ax, float* ay, float* az,
              cudaStream_t s)
{
    pm_deposit(p, pos4, n, s);
    const int rc = pm_solve(p, s);
    if (rc)
        return rc;
    pm_interp(p, pos4, n, ax, ay, az, s);
    return 0;
}

} // namespace bz
