// Periodic particle-mesh (long-range) leg of TreePM.
//
//   deposit  : mass assignment of order p (2 CIC, 3 TSC, 4 PCS) onto an M^3 mesh.  Each block
//              takes 2048 consecutive Morton-sorted particles, accumulates them into a
//              shared-memory tile covering their stencils (shared atomics), then adds the tile
//              to the mesh (one global atomic per tile cell instead of p^3 per particle);
//              blocks whose stencils do not fit a tile use global atomics directly.
//   solve    : cuFFT R2C -> Green's function with Gaussian split, window deconvolution and 1/M^3
//              (precomputed in FP64) -> one of
//              - the potential (reference centred differences, then a gradient kernel into an
//                interleaved float4 force mesh);
//              - fused in the same k-space pass, the three spectral gradients i k phi_k ->
//                three cuFFT C2R -> interleaved float4 force mesh;
//              - the potential alone (one C2R): analytic differentiation, below.
//   interp   : the same order-p stencil gathers the force mesh at each particle; with analytic
//              differentiation it gathers the potential with the gradient of the stencil
//              weights, a = sum_c phi_c grad W(x - x_c), so that one inverse transform and a
//              scalar mesh replace three transforms and a four-component mesh.
//
// Formulas follow the reference CPU templates driven with a periodic grid
// (engine/physics/treepm/deposit/TpmAssignment.inl:39-199, engine/physics/treepm/field/
// TpmField.inl:6-89): node i at i*h, density mass/h^3, phi_k = 4 pi e^{-k^2 r_s^2} rho_k /
// (k^2 max(W, floor)), W = prod sinc^{2p}(k h / 2), acceleration = +gradient of that phi.
// The reference's PCS stencil starts at floor(s + 0.5) - 1 and so drops the node floor(s) - 1
// when frac(s) >= 0.5; here every order uses the full support (TSC: nearest node +-1, CIC and
// PCS: floor(s) - (p/2 - 1) ... floor(s) + p/2).
#include <cufft.h>

#include <cmath>

#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

struct PmPlan {
    int mesh = 0;
    double box = 0.0;
    double rsplit = 0.0;
    int order = 2;
    int gradient = 0;          // 0 centred differences of phi (reference), 1 spectral, 2 analytic
    double floor = 0.08;
    float* rho = nullptr;      // M^3: density, then potential (centred-difference mode)
    cufftComplex* spec = nullptr;     // M*M*(M/2+1)
    cufftComplex* spec3 = nullptr;    // 3 x M*M*(M/2+1) spectral gradients
    float* field3 = nullptr;          // 3 x M^3 spectral gradient meshes
    float4* force = nullptr;          // M^3 interleaved force mesh {ax, ay, az, 0}
    float* green = nullptr;           // M*M*(M/2+1), computed in FP64
    cufftHandle r2c = 0, c2r = 0;
    size_t bytes = 0;
    const IsoGrid* iso = nullptr;     // isolated mesh: grid on the device, Green in the solve
    int* err = nullptr;               // device error bits (bounded waits of the staged gathers)
};

namespace {

constexpr int kThreads = 256;
constexpr int kTileCells = 12000;      // 47 KB of float accumulators (static shared memory <= 48 KB)

__device__ __forceinline__ float tsc_w(float d)
{
    const float a = fabsf(d);
    if (a < 0.5f)
        return 0.75f - a * a;
    if (a < 1.5f) {
        const float t = 1.5f - a;
        return 0.5f * t * t;
    }
    return 0.0f;
}
__device__ __forceinline__ float pcs_w(float d)
{
    const float a = fabsf(d);
    if (a < 1.0f)
        return (4.0f - 6.0f * a * a + 3.0f * a * a * a) * (1.0f / 6.0f);
    if (a < 2.0f) {
        const float t = 2.0f - a;
        return t * t * t * (1.0f / 6.0f);
    }
    return 0.0f;
}

// Mesh frame of a plan: periodic meshes start at 0 with a fixed cell; an isolated mesh reads
// its origin and cell from the device-held grid of the current force evaluation.
struct MeshFrame {
    float ox, oy, oz, inv_h;
};
__device__ __forceinline__ MeshFrame mesh_frame(const IsoGrid* iso, float inv_h)
{
    if (iso)
        return MeshFrame{iso->origin[0], iso->origin[1], iso->origin[2], iso->inv_h};
    return MeshFrame{0.0f, 0.0f, 0.0f, inv_h};
}

// Stencil of order P along one axis: first (unwrapped) node index and P weights.  coord is
// the position relative to the mesh origin; for an isolated mesh the particles lie in its
// central half, so the periodic fold below never applies there.
template <int P>
__device__ __forceinline__ int stencil(float coord, float inv_h, int mesh, float* w)
{
    const float raw = coord * inv_h;
    const float m = static_cast<float>(mesh);
    const float s = raw - floorf(raw / m) * m;  // [0, M]
    if (P == 2) {
        const float fl = floorf(s);
        const float f = s - fl;
        w[0] = 1.0f - f;
        w[1] = f;
        return static_cast<int>(fl);
    } else if (P == 3) {
        const float c = floorf(s + 0.5f);
        w[0] = tsc_w(s - (c - 1.0f));
        w[1] = tsc_w(s - c);
        w[2] = tsc_w(s - (c + 1.0f));
        return static_cast<int>(c) - 1;
    } else {
        const float fl = floorf(s);
        w[0] = pcs_w(s - (fl - 1.0f));
        w[1] = pcs_w(s - fl);
        w[2] = pcs_w(s - (fl + 1.0f));
        w[3] = pcs_w(s - (fl + 2.0f));
        return static_cast<int>(fl) - 1;
    }
}

// Derivatives of the weights with respect to the particle coordinate in cells.
__device__ __forceinline__ float tsc_dw(float d)
{
    const float a = fabsf(d);
    if (a < 0.5f)
        return -2.0f * d;
    if (a < 1.5f)
        return -copysignf(1.5f - a, d);  // -(1.5 - |d|) sign(d)
    return 0.0f;
}
__device__ __forceinline__ float pcs_dw(float d)
{
    const float a = fabsf(d);
    if (a < 1.0f)
        return d * (1.5f * a - 2.0f);
    if (a < 2.0f) {
        const float t = 2.0f - a;
        return -copysignf(0.5f * t * t, d);  // -(2 - |d|)^2 / 2 sign(d)
    }
    return 0.0f;
}

// As stencil<P>, with the derivatives dw of the weights (per cell of coordinate).
template <int P>
__device__ __forceinline__ int stencil_d(float coord, float inv_h, int mesh, float* w, float* dw)
{
    const float raw = coord * inv_h;
    const float m = static_cast<float>(mesh);
    const float s = raw - floorf(raw / m) * m;
    if (P == 2) {
        const float fl = floorf(s);
        const float f = s - fl;
        w[0] = 1.0f - f;
        w[1] = f;
        dw[0] = -1.0f;
        dw[1] = 1.0f;
        return static_cast<int>(fl);
    } else if (P == 3) {
        const float c = floorf(s + 0.5f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            w[k] = tsc_w(s - (c - 1.0f + k));
            dw[k] = tsc_dw(s - (c - 1.0f + k));
        }
        return static_cast<int>(c) - 1;
    } else {
        const float fl = floorf(s);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            w[k] = pcs_w(s - (fl - 1.0f + k));
            dw[k] = pcs_dw(s - (fl - 1.0f + k));
        }
        return static_cast<int>(fl) - 1;
    }
}

__device__ __forceinline__ int wrapm(int i, int m)
{
    i %= m;
    return i < 0 ? i + m : i;
}

// Index i + d, d in [-m, m], wrapped into [0, m).
__device__ __forceinline__ int wrap1(int i, int m) { return i < 0 ? i + m : (i >= m ? i - m : i); }

// Weight of stencil column q (a lane's own column) without indexing a register array.
template <int P>
__device__ __forceinline__ float column_weight(const float* w, int q)
{
    float r = 0.0f;
#pragma unroll
    for (int a = 0; a < P; ++a)
        r = q == a ? w[a] : r;
    return r;
}

template <int P>
__global__ void __launch_bounds__(kThreads) k_deposit_tiled(const float4* __restrict__ pos4, int n,
                                                             int chunk, int mesh, float inv_h_fixed,
                                                             float inv_h3_fixed, const IsoGrid* iso,
                                                             float* __restrict__ rho)
{
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed);
    const float inv_h = fr.inv_h;
    const float inv_h3 = iso ? 1.0f / (iso->h * iso->h * iso->h) : inv_h3_fixed;
    // The tile accumulates in 32-bit fixed point: integer shared-memory atomics are native and
    // about three times the rate of float ones, and integer sums are exact and independent of
    // the order of the additions.  The block's scale 2^k keeps any cell sum below 2^31 / 1.01: a
    // cell receives at most (largest 1-D weight)^3 x sum |m| / h^3 from the chunk, and the
    // rounding of at most chunk x P^3 contributions adds less than 2^15.  One unit is then
    // below 2 x 1.01 x (largest weight)^3 x sum |m| / h^3 / 2^31: with at most 512 particles a
    // chunk, a few 1e-7 of a mean cell.
    __shared__ int tile[kTileCells];
    __shared__ int s_lo[3], s_hi[3];
    __shared__ float s_mass, s_scale, s_unscale;
    const int base = blockIdx.x * chunk;
    const int end = min(base + chunk, n);
    if (threadIdx.x < 3) {
        s_lo[threadIdx.x] = 1 << 30;
        s_hi[threadIdx.x] = -(1 << 30);
    }
    if (threadIdx.x == 0)
        s_mass = 0.0f;
    __syncthreads();
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    float msum = 0.0f;
    for (int i = base + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos4[i];
        float w[P];
        const int b[3] = {stencil<P>(p.x - fr.ox, inv_h, mesh, w), stencil<P>(p.y - fr.oy, inv_h, mesh, w),
                          stencil<P>(p.z - fr.oz, inv_h, mesh, w)};
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], b[a]);
            hi[a] = max(hi[a], b[a] + P - 1);
        }
        msum += fabsf(p.w);
    }
    for (int a = 0; a < 3; ++a) {
        atomicMin(&s_lo[a], lo[a]);
        atomicMax(&s_hi[a], hi[a]);
    }
    for (int o = 16; o > 0; o >>= 1)
        msum += __shfl_xor_sync(kFullMask, msum, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(&s_mass, msum);
    __syncthreads();
    if (threadIdx.x == 0) {
        constexpr float kWmax3 = P == 2 ? 1.0f : (P == 3 ? 0.421875f : 0.2962963f);
        const float bound = s_mass * inv_h3 * kWmax3 * 1.01f;  // margin for float rounding
        int k = 0;
        if (bound > 0.0f) {
            int e = 0;
            frexpf(bound, &e);  // bound < 2^e
            k = min(max(31 - e, -120), 120);
        }
        s_scale = ldexpf(1.0f, k);
        s_unscale = ldexpf(1.0f, -k);
    }
    const int ex = s_hi[0] - s_lo[0] + 1, ey = s_hi[1] - s_lo[1] + 1, ez = s_hi[2] - s_lo[2] + 1;
    const bool tiled = ex > 0 && ey > 0 && ez > 0 && static_cast<long long>(ex) * ey * ez <= kTileCells;
    const int ox = s_lo[0], oy = s_lo[1], oz = s_lo[2];
    if (tiled)
        for (int c = threadIdx.x; c < ex * ey * ez; c += kThreads)
            tile[c] = 0;
    __syncthreads();
    const float scale = s_scale, unscale = s_unscale;
    const size_t M = static_cast<size_t>(mesh);
    for (int i = base + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos4[i];
        float wx[P], wy[P], wz[P];
        const int bx = stencil<P>(p.x - fr.ox, inv_h, mesh, wx);
        const int by = stencil<P>(p.y - fr.oy, inv_h, mesh, wy);
        const int bz = stencil<P>(p.z - fr.oz, inv_h, mesh, wz);
        const float m = p.w * inv_h3;
#pragma unroll
        for (int c = 0; c < P; ++c)
#pragma unroll
            for (int b = 0; b < P; ++b) {
                const float wzy = m * wz[c] * wy[b];
#pragma unroll
                for (int a = 0; a < P; ++a) {
                    const float v = wzy * wx[a];
                    if (tiled) {
                        atomicAdd(&tile[((bz + c - oz) * ey + (by + b - oy)) * ex + (bx + a - ox)],
                                  __float2int_rn(v * scale));
                    } else {
                        const size_t g = (static_cast<size_t>(wrapm(bz + c, mesh)) * M + wrapm(by + b, mesh)) * M +
                                         wrapm(bx + a, mesh);
                        atomicAdd(&rho[g], v);
                    }
                }
            }
    }
    if (!tiled)
        return;
    __syncthreads();
    // Flush the tile row by row.  Where a row segment is contiguous in the mesh (no periodic
    // wrap) and 16-byte aligned, four cells go in one vector atomic (red.global.add.v4.f32).
    const int quads = (ex + 3 + 3) / 4;  // enough 4-cell groups to cover a row from any alignment
    for (int r = threadIdx.x; r < ey * ez * quads; r += kThreads) {
        const int q = r % quads, row = r / quads;
        const int y = row % ey, z = row / ey;
        const size_t rowbase = (static_cast<size_t>(wrapm(oz + z, mesh)) * M + wrapm(oy + y, mesh)) * M;
        // group q covers mesh x in [xa, xa + 4) with xa 4-aligned relative to the unwrapped origin
        const int xa = ((ox >> 2) << 2) + 4 * q;
        float v[4];
        bool any = false;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int tx = xa + j - ox;
            v[j] = (tx >= 0 && tx < ex) ? static_cast<float>(tile[(z * ey + y) * ex + tx]) * unscale : 0.0f;
            any = any || v[j] != 0.0f;
        }
        if (!any)
            continue;
        const int gx = wrapm(xa, mesh);
        if (gx + 3 < mesh && (mesh & 3) == 0) {
            float* dst = rho + rowbase + gx;
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(v[0]), "f"(v[1]),
                         "f"(v[2]), "f"(v[3])
                         : "memory");
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (v[j] != 0.0f)
                    atomicAdd(&rho[rowbase + wrapm(xa + j, mesh)], v[j]);
        }
    }
}

__device__ __forceinline__ double sinc_d(double v) { return fabs(v) < 1.0e-5 ? 1.0 : sin(v) / v; }

// Green x window deconvolution x 1/M^3, once per plan.
__global__ void k_green_table(int mesh, double box, double rsplit, int order, double floor_w,
                              float* green)
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
            green[idx] = 0.0f;
            continue;
        }
        const double s3 = sinc_d(0.5 * kx * h) * sinc_d(0.5 * ky * h) * sinc_d(0.5 * kz * h);
        double W = 1.0;
        for (int i = 0; i < 2 * order; ++i)
            W *= s3;
        if (W < floor_w)
            W = floor_w;
        green[idx] = static_cast<float>(4.0 * 3.14159265358979323846 * exp(-k2 * rsplit * rsplit) / (k2 * W) * norm);
    }
}

// Isolated mesh: the Green x window deconvolution x 1/M^3 of k_green_table, evaluated per
// mode in FP64 from the device-held grid of this evaluation (its cell and split scale change
// with the particles' extent).  gradient 1 writes the three spectral gradients as
// k_green_gradient does; otherwise the potential spectrum is scaled in place.
__global__ void __launch_bounds__(kThreads) k_green_iso(cufftComplex* __restrict__ spec, int mesh,
                                                         int order, double floor_w, const IsoGrid* iso,
                                                         int gradient, cufftComplex* __restrict__ out3)
{
    const int hx = mesh / 2 + 1;
    const size_t total = static_cast<size_t>(mesh) * mesh * hx;
    const double h = iso->h, rs = iso->rsplit;
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
        float g = 0.0f;
        if (k2 > 1.0e-12) {
            const double s3 = sinc_d(0.5 * kx * h) * sinc_d(0.5 * ky * h) * sinc_d(0.5 * kz * h);
            double W = 1.0;
            for (int i = 0; i < 2 * order; ++i)
                W *= s3;
            if (W < floor_w)
                W = floor_w;
            g = static_cast<float>(4.0 * 3.14159265358979323846 * exp(-k2 * rs * rs) / (k2 * W) * norm);
        }
        const cufftComplex c = spec[idx];
        const float pr = c.x * g, pi = c.y * g;
        if (gradient == 1) {
            const int tx = x == mesh / 2 ? 0 : x;
            const int ty = y == mesh / 2 ? 0 : sy;
            const int tz = z == mesh / 2 ? 0 : sz;
            const float k[3] = {static_cast<float>(tx * ks), static_cast<float>(ty * ks),
                                static_cast<float>(tz * ks)};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                cufftComplex o;
                o.x = -k[a] * pi;
                o.y = k[a] * pr;
                out3[a * total + idx] = o;
            }
        } else {
            spec[idx] = make_cuFloatComplex(pr, pi);
        }
    }
}

// Grid of an isolated mesh from the FP64 bounds of the positions (one thread).  The formulas
// and their FP32 rounding are the reference's (TpmGridBuild.inl:98-171): FP32 bounds, extent =
// max(span x, y, z, softening), cell = max(cell_floor, extent / (G - 2)), the 2G mesh centred
// on the bounds.
__global__ void k_iso_grid(const BoxF64* box, int grid_half, float cell_floor, float softening,
                           float r_split_cells, float r_cut_factor, float node_size_factor, IsoGrid* out)
{
    float mn[3], mx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = static_cast<float>(double_from_ordered(box->mn[a]));
        mx[a] = static_cast<float>(double_from_ordered(box->mx[a]));
    }
    const float extent = fmaxf(fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]), softening);
    const float h = fmaxf(cell_floor, extent / static_cast<float>(grid_half - 2));
    const float half_extent = 0.5f * static_cast<float>(2 * grid_half) * h;
    IsoGrid g;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        g.origin[a] = 0.5f * (mn[a] + mx[a]) - half_extent;
    g.h = h;
    g.inv_h = 1.0f / h;
    g.rsplit = r_split_cells * h;
    const float rc = r_cut_factor * g.rsplit;
    g.rcut2 = rc * rc;
    g.max_node_size = node_size_factor > 0.0f ? node_size_factor * g.rsplit : 0.0f;
    *out = g;
}

__global__ void __launch_bounds__(kThreads) k_apply_green(cufftComplex* __restrict__ spec,
                                                           const float* __restrict__ green,
                                                           size_t total)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * kThreads) {
        const float g = green[i];
        cufftComplex c = spec[i];
        c.x *= g;
        c.y *= g;
        spec[i] = c;
    }
}

// Fused Green x spectral gradient: F_a = i k_a G rho_k for a = x, y, z (Nyquist derivative
// terms set to zero).
__global__ void __launch_bounds__(kThreads) k_green_gradient(const cufftComplex* __restrict__ spec,
                                                              const float* __restrict__ green,
                                                              int mesh, double box,
                                                              cufftComplex* __restrict__ out3)
{
    const int hx = mesh / 2 + 1;
    const size_t total = static_cast<size_t>(mesh) * mesh * hx;
    const float ks = static_cast<float>(2.0 * 3.14159265358979323846 / box);
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * kThreads) {
        const int x = static_cast<int>(i % hx);
        const size_t pl = i / hx;
        const int y = static_cast<int>(pl % mesh);
        const int z = static_cast<int>(pl / mesh);
        const int sx = x == mesh / 2 ? 0 : x;
        const int sy = y == mesh / 2 ? 0 : (y < mesh / 2 ? y : y - mesh);
        const int sz = z == mesh / 2 ? 0 : (z < mesh / 2 ? z : z - mesh);
        const float g = green[i];
        const cufftComplex c = spec[i];
        const float pr = c.x * g, pi = c.y * g;
        const float k[3] = {sx * ks, sy * ks, sz * ks};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            cufftComplex o;
            o.x = -k[a] * pi;  // i k (pr + i pi) = -k pi + i k pr
            o.y = k[a] * pr;
            out3[a * total + i] = o;
        }
    }
}

// Centred-difference gradient of phi into the interleaved force mesh (reference mode).  An
// isolated mesh (iso != NULL) takes its cell from the device-held grid and, as the reference's
// non-periodic gradient does (TpmFft.inl:108-141), leaves its outer layer of cells at zero.
__global__ void __launch_bounds__(kThreads) k_fd_gradient(const float* __restrict__ phi, int mesh,
                                                           float half_inv_h_fixed, const IsoGrid* iso,
                                                           float4* __restrict__ force)
{
    const size_t M = static_cast<size_t>(mesh), total = M * M * M;
    const float half_inv_h = iso ? 0.5f * iso->inv_h : half_inv_h_fixed;
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * kThreads) {
        const int x = static_cast<int>(i % M), y = static_cast<int>((i / M) % M), z = static_cast<int>(i / (M * M));
        if (iso && (x == 0 || y == 0 || z == 0 || x == mesh - 1 || y == mesh - 1 || z == mesh - 1)) {
            force[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const int xp = x + 1 == mesh ? 0 : x + 1, xm = x == 0 ? mesh - 1 : x - 1;
        const int yp = y + 1 == mesh ? 0 : y + 1, ym = y == 0 ? mesh - 1 : y - 1;
        const int zp = z + 1 == mesh ? 0 : z + 1, zm = z == 0 ? mesh - 1 : z - 1;
        const size_t row = (static_cast<size_t>(z) * M + y) * M;
        const float gx = (phi[row + xp] - phi[row + xm]) * half_inv_h;
        const float gy = (phi[(static_cast<size_t>(z) * M + yp) * M + x] - phi[(static_cast<size_t>(z) * M + ym) * M + x]) * half_inv_h;
        const float gz = (phi[(static_cast<size_t>(zp) * M + y) * M + x] - phi[(static_cast<size_t>(zm) * M + y) * M + x]) * half_inv_h;
        force[i] = make_float4(gx, gy, gz, 0.0f);
    }
}

__global__ void __launch_bounds__(kThreads) k_pack_force(const float* __restrict__ f3, size_t total,
                                                          float4* __restrict__ force)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * kThreads)
        force[i] = make_float4(f3[i], f3[total + i], f3[2 * total + i], 0.0f);
}

// Interpolation with four lanes per particle: lane q of a quad gathers stencil column
// x = bx + q of every (y, z) row of the order-p stencil from the interleaved force mesh, and the
// quad adds its partial sums.  A quad thus reads whole 64-byte rows, and the eight
// Morton-consecutive particles of a warp share most of their rows, so one load instruction
// touches a few cache lines instead of one per lane (the one-lane-per-particle form is bound
// by L1 wavefronts).
template <int P>
__global__ void __launch_bounds__(kThreads) k_interp(const float4* __restrict__ pos4, int n, int mesh,
                                                      float inv_h_fixed, const IsoGrid* iso,
                                                      const float4* __restrict__ force,
                                                      float* __restrict__ ax, float* __restrict__ ay,
                                                      float* __restrict__ az)
{
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed);
    const float inv_h = fr.inv_h;
    const size_t M = static_cast<size_t>(mesh);
    const int q = threadIdx.x & 3;
    // each block walks one contiguous (Morton-ordered) range, 64 particles at a time, so that
    // consecutive rounds reuse the stencil rows they share in L1
    constexpr int kRound = (kThreads / 32) * 8;
    const int per_block = ((n + gridDim.x - 1) / gridDim.x + kRound - 1) / kRound * kRound;
    const int start = blockIdx.x * per_block;
    const int stop = min(start + per_block, n);
    for (int i0 = start + (threadIdx.x >> 5) * 8; i0 < stop; i0 += kRound) {
        const int i = i0 + ((threadIdx.x & 31) >> 2);
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
        if (i < stop && q < P) {
            const float4 p = pos4[i];
            float wx[P], wy[P], wz[P];
            const int bx = stencil<P>(p.x - fr.ox, inv_h, mesh, wx);
            const int by = stencil<P>(p.y - fr.oy, inv_h, mesh, wy);
            const int bz = stencil<P>(p.z - fr.oz, inv_h, mesh, wz);
            const float wq = column_weight<P>(wx, q);
            const int xs = wrap1(bx + q, mesh);
#pragma unroll
            for (int c = 0; c < P; ++c) {
                const size_t zrow = static_cast<size_t>(wrap1(bz + c, mesh)) * M;
                const float wzq = wz[c] * wq;
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    const float4 f = __ldg(&force[(zrow + wrap1(by + b, mesh)) * M + xs]);
                    const float w = wzq * wy[b];
                    gx = fmaf(w, f.x, gx);
                    gy = fmaf(w, f.y, gy);
                    gz = fmaf(w, f.z, gz);
                }
            }
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            gx += __shfl_xor_sync(kFullMask, gx, o);
            gy += __shfl_xor_sync(kFullMask, gy, o);
            gz += __shfl_xor_sync(kFullMask, gz, o);
        }
        if (i < stop && q == 0) {
            ax[i] = gx;
            ay[i] = gy;
            az[i] = gz;
        }
    }
}

// Analytic differentiation with the potential staged in shared memory, the gather twin of
// k_deposit_tiled: a block takes a chunk of Morton-consecutive particles (the deposit's chunk,
// whose stencils fit one tile) and stages the box of cells their stencils cover with bulk copies
// (cp.async.bulk, global -> shared, no multicast), one per mesh row segment: rows start on a
// 16-byte boundary (x rounded down to a multiple of 4 cells; the mesh side is a multiple of 4),
// a row crossing the periodic x boundary takes two copies, and all complete on one mbarrier
// (bounded wait).  Four lanes then serve one particle, lane q reading stencil column
// x = bx + q of every (y, z) row, and the quad adds its partial sums.  The tile's row and plane
// pitches are padded by 8 and 12 cells so that the eight particles of a warp, Morton neighbours,
// read mostly distinct banks: a bank model over the 128^3 benchmark box gives about 1.5
// shared-memory wavefronts per load, against 11 for one thread per particle on an unpadded tile.
// A chunk whose box does not fit gathers from the global mesh instead.  The sum is
// a = (1/h) sum_c phi_c grad W(x - x_c), the weight of cell (a, b, c) in the x component being
// dW_x(a) W_y(b) W_z(c), and likewise for y and z.
template <int P>
__global__ void __launch_bounds__(kThreads) k_interp_ad_tiled(const float4* __restrict__ pos4, int n,
                                                               int chunk, int mesh, float inv_h_fixed,
                                                               const IsoGrid* iso,
                                                               const float* __restrict__ phi,
                                                               float* __restrict__ ax,
                                                               float* __restrict__ ay,
                                                               float* __restrict__ az, int* err)
{
    __shared__ __align__(16) float tile[kTileCells];
    __shared__ int s_lo[3], s_hi[3];
    __shared__ unsigned long long bar;
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed);
    const float inv_h = fr.inv_h;
    const int base = blockIdx.x * chunk;
    const int end = min(base + chunk, n);
    if (threadIdx.x < 3) {
        s_lo[threadIdx.x] = 1 << 30;
        s_hi[threadIdx.x] = -(1 << 30);
    }
    if (threadIdx.x == 0)
        mbar_init(&bar, 1);
    fence_mbar_init();
    __syncthreads();
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    for (int i = base + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos4[i];
        float w[P];
        const int b[3] = {stencil<P>(p.x - fr.ox, inv_h, mesh, w), stencil<P>(p.y - fr.oy, inv_h, mesh, w),
                          stencil<P>(p.z - fr.oz, inv_h, mesh, w)};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], b[a]);
            hi[a] = max(hi[a], b[a] + P - 1);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        atomicMin(&s_lo[a], lo[a]);
        atomicMax(&s_hi[a], hi[a]);
    }
    __syncthreads();
    // x rounded out to whole 16-byte groups of four cells
    const int ox = s_lo[0] - (((s_lo[0] % 4) + 4) % 4);
    const int oy = s_lo[1], oz = s_lo[2];
    const int ex = ((s_hi[0] + 1 - ox) + 3) & ~3;
    const int ey = s_hi[1] - oy + 1, ez = s_hi[2] - oz + 1;
    const int rp = ex + 8;            // padded row pitch: a multiple of 4, rows stay 16-byte aligned
    const int pp = ey * rp + 12;      // padded plane pitch, also a multiple of 4
    const bool tiled = ex > 0 && ey > 0 && ez > 0 && ex <= mesh &&
                       static_cast<long long>(pp) * ez <= kTileCells && (mesh & 3) == 0;
    const size_t M = static_cast<size_t>(mesh);
    if (tiled) {
        const int rows = ey * ez;
        if (threadIdx.x == 0)
            mbar_arrive_expect_tx(&bar, static_cast<uint32_t>(rows) * static_cast<uint32_t>(ex) * 4u);
        __syncthreads();
        for (int r = threadIdx.x; r < rows; r += kThreads) {
            const int y = r % ey, z = r / ey;
            const float* row = phi + (static_cast<size_t>(wrapm(oz + z, mesh)) * M + wrapm(oy + y, mesh)) * M;
            float* dst = tile + z * pp + y * rp;
            const int x0 = wrapm(ox, mesh);           // a multiple of four
            const int first = min(ex, mesh - x0);      // cells before the periodic x boundary
            bulk_g2s(dst, row + x0, static_cast<uint32_t>(first) * 4u, &bar);
            if (first < ex)
                bulk_g2s(dst + first, row, static_cast<uint32_t>(ex - first) * 4u, &bar);
        }
        mbar_wait_bounded(&bar, 0u, err);
    }
    // the loop bound is uniform over the block, so every lane of a quad reaches the shuffles
    const int q = threadIdx.x & 3;
    for (int i0 = base; i0 < end; i0 += kThreads / 4) {
        const int i = i0 + (threadIdx.x >> 2);
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
        if (i < end && q < P) {
            const float4 p = pos4[i];
            float wx[P], wy[P], wz[P], dx[P], dy[P], dz[P];
            const int bx = stencil_d<P>(p.x - fr.ox, inv_h, mesh, wx, dx);
            const int by = stencil_d<P>(p.y - fr.oy, inv_h, mesh, wy, dy);
            const int bz = stencil_d<P>(p.z - fr.oz, inv_h, mesh, wz, dz);
            const float wq = column_weight<P>(wx, q);
            const float dq = column_weight<P>(dx, q);
            const int xs = bx + q;
#pragma unroll
            for (int c = 0; c < P; ++c) {
                float sw = 0.0f, sd = 0.0f;  // this plane's column sums over y: W_y and dW_y weighted
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    float v;
                    if (tiled)
                        v = tile[(bz + c - oz) * pp + (by + b - oy) * rp + (xs - ox)];
                    else
                        v = __ldg(&phi[(static_cast<size_t>(wrap1(bz + c, mesh)) * M + wrap1(by + b, mesh)) * M +
                                       wrap1(xs, mesh)]);
                    sw = fmaf(v, wy[b], sw);
                    sd = fmaf(v, dy[b], sd);
                }
                gx = fmaf(sw * dq, wz[c], gx);
                gy = fmaf(sd * wq, wz[c], gy);
                gz = fmaf(sw * wq, dz[c], gz);
            }
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            gx += __shfl_xor_sync(kFullMask, gx, o);
            gy += __shfl_xor_sync(kFullMask, gy, o);
            gz += __shfl_xor_sync(kFullMask, gz, o);
        }
        if (i < end && q == 0) {
            ax[i] = gx * inv_h;
            ay[i] = gy * inv_h;
            az[i] = gz * inv_h;
        }
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

PmPlan* pm_create(int mesh, double box, double rsplit, int order, int gradient, double window_floor,
                  cudaStream_t s, int* cuda_err, const IsoGrid* iso, int* dev_err)
{
    PmPlan* p = new PmPlan();
    p->iso = iso;
    p->err = dev_err;
    p->mesh = mesh;
    p->box = box;
    p->rsplit = rsplit;
    p->order = order < 2 ? 2 : (order > 4 ? 4 : order);
    p->gradient = gradient < 0 ? 0 : (gradient > 2 ? 2 : gradient);
    p->floor = window_floor;
    const size_t cells = static_cast<size_t>(mesh) * mesh * mesh;
    const size_t half = static_cast<size_t>(mesh) * mesh * (mesh / 2 + 1);
    *cuda_err = 0;
    bool ok = cudaMalloc(&p->rho, cells * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&p->spec, half * sizeof(cufftComplex)) == cudaSuccess &&
              (iso || cudaMalloc(&p->green, half * sizeof(float)) == cudaSuccess);
    if (ok && p->gradient != 2)  // analytic differentiation needs no force mesh
        ok = cudaMalloc(&p->force, cells * sizeof(float4)) == cudaSuccess;
    if (ok && p->gradient == 1)
        ok = cudaMalloc(&p->spec3, 3 * half * sizeof(cufftComplex)) == cudaSuccess &&
             cudaMalloc(&p->field3, 3 * cells * sizeof(float)) == cudaSuccess;
    if (!ok) {
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
    p->bytes = cells * (sizeof(float) + (p->gradient != 2 ? sizeof(float4) : 0)) +
               half * (sizeof(cufftComplex) + (iso ? 0 : sizeof(float))) +
               (p->gradient == 1 ? 3 * (half * sizeof(cufftComplex) + cells * sizeof(float)) : 0) + ws1 + ws2;
    if (!iso) {
        count_launch();
        k_green_table<<<sm_count() * 4, 256, 0, s>>>(mesh, box, rsplit, p->order, window_floor, p->green);
    }
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
    cudaFree(p->spec3);
    cudaFree(p->field3);
    cudaFree(p->force);
    cudaFree(p->green);
    delete p;
}

size_t pm_bytes(const PmPlan* p) { return p ? p->bytes : 0; }
float* pm_mesh(PmPlan* p) { return p->rho; }
const float4* pm_force_mesh(PmPlan* p) { return p->force; }

void pm_deposit(PmPlan* p, const float4* pos4, int n, cudaStream_t s)
{
    const int M = p->mesh;
    const size_t cells = static_cast<size_t>(M) * M * M;
    const double h = p->iso ? 1.0 : p->box / M;  // isolated: the kernels read the cell
    const float inv_h = static_cast<float>(1.0 / h);
    const float inv_h3 = static_cast<float>(1.0 / (h * h * h));
    cudaMemsetAsync(p->rho, 0, cells * sizeof(float), s);
    const int chunk = pm_deposit_chunk(p, n);
    const int b = (n + chunk - 1) / chunk;
    count_launch();
    if (p->order == 2)
        k_deposit_tiled<2><<<b, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, inv_h3, p->iso, p->rho);
    else if (p->order == 3)
        k_deposit_tiled<3><<<b, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, inv_h3, p->iso, p->rho);
    else
        k_deposit_tiled<4><<<b, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, inv_h3, p->iso, p->rho);
}

int pm_deposit_chunk(const PmPlan* p, int n)
{
    // A chunk of c Morton-consecutive particles spans about c / (n / M^3) cells of a roughly
    // uniform distribution; keep (cbrt(cells) + p)^3 within the tile with margin.
    const double cells_per_particle = static_cast<double>(p->mesh) * p->mesh * p->mesh / (n > 0 ? n : 1);
    int chunk = 512;  // also bounds the fixed-point unit of the tile (see k_deposit_tiled)
    while (chunk > 128) {
        const double side = std::cbrt(chunk * cells_per_particle) + p->order + 1.0;
        if (side * side * side <= 0.6 * kTileCells)
            break;
        chunk >>= 1;
    }
    return chunk;
}

int pm_solve(PmPlan* p, cudaStream_t s)
{
    const int M = p->mesh;
    const size_t half = static_cast<size_t>(M) * M * (M / 2 + 1);
    const int sms = sm_count();
    // the transforms run on the caller's stream (the force pass may run the mesh leg on a
    // second stream, concurrently with the tree build and walk)
    cufftSetStream(p->r2c, s);
    cufftSetStream(p->c2r, s);
    if (cufftExecR2C(p->r2c, p->rho, p->spec) != CUFFT_SUCCESS)
        return 1;
    if (p->iso) {
        count_launch();
        k_green_iso<<<sms * 4, kThreads, 0, s>>>(p->spec, M, p->order, p->floor, p->iso, p->gradient,
                                                 p->spec3);
        const size_t cells = static_cast<size_t>(M) * M * M;
        if (p->gradient == 1) {
            for (int a = 0; a < 3; ++a)
                if (cufftExecC2R(p->c2r, p->spec3 + a * half, p->field3 + a * cells) != CUFFT_SUCCESS)
                    return 2;
            count_launch();
            k_pack_force<<<sms * 4, kThreads, 0, s>>>(p->field3, cells, p->force);
            return 0;
        }
        if (cufftExecC2R(p->c2r, p->spec, p->rho) != CUFFT_SUCCESS)
            return 2;
        if (p->gradient == 0) {
            count_launch();
            k_fd_gradient<<<sms * 4, kThreads, 0, s>>>(p->rho, M, 0.0f, p->iso, p->force);
        }
        return 0;
    }
    if (p->gradient == 1) {
        count_launch();
        k_green_gradient<<<sms * 4, kThreads, 0, s>>>(p->spec, p->green, M, p->box, p->spec3);
        const size_t cells = static_cast<size_t>(M) * M * M;
        for (int a = 0; a < 3; ++a)
            if (cufftExecC2R(p->c2r, p->spec3 + a * half, p->field3 + a * cells) != CUFFT_SUCCESS)
                return 2;
        count_launch();
        k_pack_force<<<sms * 4, kThreads, 0, s>>>(p->field3, cells, p->force);
    } else {
        count_launch();
        k_apply_green<<<sms * 4, kThreads, 0, s>>>(p->spec, p->green, half);
        if (cufftExecC2R(p->c2r, p->spec, p->rho) != CUFFT_SUCCESS)
            return 2;
        if (p->gradient == 0) {
            count_launch();
            k_fd_gradient<<<sms * 4, kThreads, 0, s>>>(p->rho, M, static_cast<float>(0.5 * M / p->box),
                                                       nullptr, p->force);
        }
    }
    return 0;
}

void pm_interp(PmPlan* p, const float4* pos4, int n, float* ax, float* ay, float* az,
               cudaStream_t s)
{
    const int M = p->mesh;
    const float inv_h = p->iso ? 1.0f : static_cast<float>(M / p->box);  // isolated: read on the device
    int b = (n + kThreads / 4 - 1) / (kThreads / 4);  // four lanes per particle
    b = b < sm_count() * 8 ? b : sm_count() * 8;
    count_launch();
    if (p->gradient == 2) {
        // the potential staged in shared memory per chunk of particles (the deposit's chunks)
        const int chunk = pm_deposit_chunk(p, n);
        const int blocks = (n + chunk - 1) / chunk;
        if (p->order == 2)
            k_interp_ad_tiled<2><<<blocks, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, p->iso, p->rho, ax, ay, az,
                                                                   p->err);
        else if (p->order == 3)
            k_interp_ad_tiled<3><<<blocks, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, p->iso, p->rho, ax, ay, az,
                                                                   p->err);
        else
            k_interp_ad_tiled<4><<<blocks, kThreads, 0, s>>>(pos4, n, chunk, M, inv_h, p->iso, p->rho, ax, ay, az,
                                                                   p->err);
        return;
    }
    if (p->order == 2)
        k_interp<2><<<b, kThreads, 0, s>>>(pos4, n, M, inv_h, p->iso, p->force, ax, ay, az);
    else if (p->order == 3)
        k_interp<3><<<b, kThreads, 0, s>>>(pos4, n, M, inv_h, p->iso, p->force, ax, ay, az);
    else
        k_interp<4><<<b, kThreads, 0, s>>>(pos4, n, M, inv_h, p->iso, p->force, ax, ay, az);
}

void launch_iso_grid(const BoxF64* box, int grid_half, float cell_floor, float softening,
                     float r_split_cells, float r_cut_factor, float node_size_factor, IsoGrid* out,
                     cudaStream_t s)
{
    count_launch();
    k_iso_grid<<<1, 1, 0, s>>>(box, grid_half, cell_floor, softening, r_split_cells, r_cut_factor,
                               node_size_factor, out);
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
