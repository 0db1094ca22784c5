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

// Mesh frame of a plan: periodic meshes start at 0 with a fixed cell; an isolated mesh reads
// its origin and cell from the device-held grid of the current force evaluation.
struct MeshFrame {
    float ox, oy, oz, inv_h;
    float inv_m;  // 1 / mesh side, for the periodic fold (one division per thread)
};
__device__ __forceinline__ MeshFrame mesh_frame(const IsoGrid* iso, float inv_h, int mesh)
{
    const float inv_m = 1.0f / static_cast<float>(mesh);
    if (iso)
        return MeshFrame{iso->origin[0], iso->origin[1], iso->origin[2], iso->inv_h, inv_m};
    return MeshFrame{0.0f, 0.0f, 0.0f, inv_h, inv_m};
}

// Stencil of order P along one axis.  coord is the position relative to the mesh origin; for an
// isolated mesh the particles lie in its central half, so the periodic fold below never applies
// there.  stencil_base returns the first (unwrapped) node index and the particle's offset t in
// its stencil: the particle lies at base + t for CIC and at base + 1 + t for TSC and PCS, with t
// in [0, 1) for CIC and PCS and in [-1/2, 1/2) for TSC (the offset from the nearest node).
template <int P>
__device__ __forceinline__ int stencil_base(float coord, float inv_h, int mesh, float inv_m, float& t)
{
    const float raw = coord * inv_h;
    const float m = static_cast<float>(mesh);
    // fold into [0, M): the product with 1/M may miss the exact quotient by one period at a
    // boundary, which the two compares put back
    float s = raw - floorf(raw * inv_m) * m;
    s = s < 0.0f ? s + m : s;
    s = s >= m ? s - m : s;
    if (P == 3) {
        const float c = floorf(s + 0.5f);
        t = s - c;
        return static_cast<int>(c) - 1;
    }
    const float fl = floorf(s);
    t = s - fl;
    return static_cast<int>(fl) - (P == 4 ? 1 : 0);
}

// The assignment weights W(d) of the P nodes, d = particle - node in cells, written per node
// for the offset t of stencil_base (no branches on |d|):
//   CIC  W = 1 - |d|;
//   TSC  W = 3/4 - d^2 (|d| < 1/2), (3/2 - |d|)^2 / 2 (|d| < 3/2);
//   PCS  W = 2/3 - d^2 + |d|^3 / 2 (|d| < 1), (2 - |d|)^3 / 6 (|d| < 2).
// dw holds dW/dd, the derivative with respect to the particle coordinate in cells.
template <int P>
__device__ __forceinline__ void stencil_weights(float t, float* w)
{
    if (P == 2) {
        w[0] = 1.0f - t;
        w[1] = t;
    } else if (P == 3) {
        const float a = 0.5f - t, b = 0.5f + t;
        w[0] = 0.5f * a * a;
        w[1] = 0.75f - t * t;
        w[2] = 0.5f * b * b;
    } else {
        const float u = 1.0f - t;
        const float t2 = t * t, u2 = u * u;
        w[0] = (1.0f / 6.0f) * u2 * u;
        w[1] = (2.0f / 3.0f) - t2 * fmaf(-0.5f, t, 1.0f);
        w[2] = (2.0f / 3.0f) - u2 * fmaf(-0.5f, u, 1.0f);
        w[3] = (1.0f / 6.0f) * t2 * t;
    }
}
template <int P>
__device__ __forceinline__ void stencil_weights_d(float t, float* w, float* dw)
{
    stencil_weights<P>(t, w);
    if (P == 2) {
        dw[0] = -1.0f;
        dw[1] = 1.0f;
    } else if (P == 3) {
        dw[0] = t - 0.5f;
        dw[1] = -2.0f * t;
        dw[2] = t + 0.5f;
    } else {
        const float u = 1.0f - t;
        dw[0] = -0.5f * u * u;
        dw[1] = t * fmaf(1.5f, t, -2.0f);
        dw[2] = u * fmaf(-1.5f, u, 2.0f);
        dw[3] = 0.5f * t * t;
    }
}

template <int P>
__device__ __forceinline__ int stencil(float coord, float inv_h, int mesh, float inv_m, float* w)
{
    float t;
    const int base = stencil_base<P>(coord, inv_h, mesh, inv_m, t);
    stencil_weights<P>(t, w);
    return base;
}

// As stencil<P>, with the derivatives dw of the weights (per cell of coordinate).
template <int P>
__device__ __forceinline__ int stencil_d(float coord, float inv_h, int mesh, float inv_m, float* w, float* dw)
{
    float t;
    const int base = stencil_base<P>(coord, inv_h, mesh, inv_m, t);
    stencil_weights_d<P>(t, w, dw);
    return base;
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

// Tile pitches of the staged interpolation and deposit boxes, padded so that the particles of a
// warp, Morton neighbours, touch mostly distinct banks.  The interpolation serves a particle
// with four lanes (eight particles a warp), the deposit with one thread, each lane of a warp
// visiting its stencil in its own order: a bank model over the 128^3 benchmark box gives about
// 1.5 and 2.1 shared-memory wavefronts per access with these pads (2.7 measured for the
// deposit), against 3.4 and 11.5 unpadded.  All are multiples of 4 cells, so rows start on a
// 16-byte boundary.
constexpr int kRowPad = 8;
constexpr int kPlanePad = 12;
constexpr int kDepositRowPad = 12;
constexpr int kDepositPlanePad = 4;
// Fixed pitches for the interpolation's boxes of the usual chunks (a chunk of 256 Morton-
// consecutive particles at 8 cells per particle spans about 20 x 20 x 12 cells); boxes that do
// not fit use the padded pitches above.  (The deposit measured no faster with fixed pitches.)
constexpr int kInterpRp = 28, kInterpPp = 572;  // rows of up to 28 cells, up to 20 rows a plane

// The scatter of k_deposit_tiled, one thread per particle: all threads of a warp add the same
// stencil offset together, so two of them meet on one cell only when their particles share a
// stencil base (four lanes per particle, one x column each, would collide whenever neighbours'
// bases differ by under four cells along x).  Fixed point into the block's tile (TILED, with
// red.shared on shared-window addresses), or floating point into the global mesh.
// w[k] <- w[k ^ s] for s in 0..3 (two conditional pair swaps, no indexed register access).
__device__ __forceinline__ void xor_permute4(float (&w)[4], int s)
{
    const bool s1 = s & 1, s2 = s & 2;
    const float a0 = s1 ? w[1] : w[0], a1 = s1 ? w[0] : w[1];
    const float a2 = s1 ? w[3] : w[2], a3 = s1 ? w[2] : w[3];
    w[0] = s2 ? a2 : a0;
    w[1] = s2 ? a3 : a1;
    w[2] = s2 ? a0 : a2;
    w[3] = s2 ? a1 : a3;
}

template <int P, bool TILED>
__device__ __forceinline__ void deposit_particles(const float4* __restrict__ pos4, int base, int end,
                                                  const MeshFrame& fr, int mesh, float inv_h3, float scale,
                                                  int* tile, int ox, int oy, int oz, int rp, int pp,
                                                  float* __restrict__ rho)
{
    const size_t M = static_cast<size_t>(mesh);
    for (int i = base + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos4[i];
        float tx, ty, tz;
        const int bx = stencil_base<P>(p.x - fr.ox, fr.inv_h, mesh, fr.inv_m, tx);
        const int by = stencil_base<P>(p.y - fr.oy, fr.inv_h, mesh, fr.inv_m, ty);
        const int bz = stencil_base<P>(p.z - fr.oz, fr.inv_h, mesh, fr.inv_m, tz);
        float wx[P], wy[P], wz[P];
        stencil_weights<P>(tx, wx);
        stencil_weights<P>(ty, wy);
        stencil_weights<P>(tz, wz);
        const float m = p.w * inv_h3;
        if (TILED) {
            const uint32_t corner = smem_u32(tile + (bz - oz) * pp + (by - oy) * rp + (bx - ox));
            // the fixed-point scale is a power of two: folding it into the x weights rounds
            // exactly as applying it to each product
            float wxs[P];
#pragma unroll
            for (int a = 0; a < P; ++a)
                wxs[a] = wx[a] * scale;
            if constexpr (P == 4) {
                // Each lane visits its 64 stencil cells in its own order: stencil offset k of
                // an axis is taken at step k ^ s, with s = lane bits (y: 0-1, z: 2-3, x: 4).
                // The warp's lanes are Morton neighbours whose bases lie about two cells apart,
                // so in one common order they hit the same banks; the staggered orders spread a
                // reduction over about half the shared-memory wavefronts (a bank model over the
                // benchmark box: 2.1 against 4.0).  Integer sums do not depend on the order.
                const int lane = threadIdx.x & 31;
                const int sy = lane & 3, sz = (lane >> 2) & 3, sx = (lane >> 4) & 1;
                xor_permute4(wy, sy);
                xor_permute4(wz, sz);
                xor_permute4(wxs, sx);
                uint32_t yoff[4], zoff[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    yoff[k] = 4u * static_cast<uint32_t>((k ^ sy) * rp);
                    zoff[k] = 4u * static_cast<uint32_t>((k ^ sz) * pp);
                }
                // x offsets a ^ sx: a = 0, 2 from the even base, a = 1, 3 from the odd one
                const uint32_t ce = corner + 4u * sx, co = corner + 4u - 4u * sx;
#pragma unroll
                for (int c = 0; c < 4; ++c)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const float wzy = m * wz[c] * wy[b];
                        const uint32_t ro = zoff[c] + yoff[b];
                        const uint32_t re = ce + ro, rd = co + ro;
                        asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(re),
                                     "r"(__float2int_rn(wzy * wxs[0])) : "memory");
                        asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(rd),
                                     "r"(__float2int_rn(wzy * wxs[1])) : "memory");
                        asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(re + 8u),
                                     "r"(__float2int_rn(wzy * wxs[2])) : "memory");
                        asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(rd + 8u),
                                     "r"(__float2int_rn(wzy * wxs[3])) : "memory");
                    }
            } else {
#pragma unroll
                for (int c = 0; c < P; ++c)
#pragma unroll
                    for (int b = 0; b < P; ++b) {
                        const float wzy = m * wz[c] * wy[b];
                        const uint32_t row = corner + 4u * static_cast<uint32_t>(c * pp + b * rp);
#pragma unroll
                        for (int a = 0; a < P; ++a)
                            asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(row + 4u * a),
                                         "r"(__float2int_rn(wzy * wxs[a]))
                                         : "memory");
                    }
            }
        } else {
#pragma unroll
            for (int c = 0; c < P; ++c) {
                const size_t zrow = static_cast<size_t>(wrap1(bz + c, mesh)) * M;
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    const float wzy = m * wz[c] * wy[b];
                    const size_t row = (zrow + wrap1(by + b, mesh)) * M;
#pragma unroll
                    for (int a = 0; a < P; ++a)
                        atomicAdd(&rho[row + wrap1(bx + a, mesh)], wzy * wx[a]);
                }
            }
        }
    }
}

// Adds four tile cells (fixed point, times unscale) into the mesh at linear cell index g with
// one vector reduction.
__device__ __forceinline__ void flush_quad(const int4 c4, float unscale, float* dst)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst),
                 "f"(static_cast<float>(c4.x) * unscale), "f"(static_cast<float>(c4.y) * unscale),
                 "f"(static_cast<float>(c4.z) * unscale), "f"(static_cast<float>(c4.w) * unscale)
                 : "memory");
}

// Flush of k_deposit_tiled's tile in groups of four cells: thread t takes groups t,
// t + kThreads, ... of the (z, y, group) range, its indices advanced by constant steps.  A box
// inside the mesh (no periodic wrap on any axis; almost every box) adds each group with one
// vector reduction at a 32-bit cell index; a box that wraps folds each index and adds a group
// that straddles the x boundary cell by cell.
__device__ __forceinline__ void flush_tile(const int* tile, int ox, int oy, int oz, int ex, int ey,
                                           int ez, int rp, int pp, int mesh, float unscale,
                                           float* __restrict__ rho)
{
    const int quads = ex / 4;
    const int items = ey * ez * quads;
    int row = threadIdx.x / quads, qd = threadIdx.x - row * quads;
    int z = row / ey, y = row - z * ey;
    const int dq = kThreads % quads, drow = kThreads / quads;
    const int dz = drow / ey, dy = drow - dz * ey;
    // 32-bit cell indices need mesh^3 < 2^31; the mesh side is a multiple of 4 for the vector
    // reductions
    const bool inside = ox >= 0 && oy >= 0 && oz >= 0 && ox + ex <= mesh && oy + ey <= mesh &&
                        oz + ez <= mesh && mesh <= 1024 && (mesh & 3) == 0;
    const size_t M = static_cast<size_t>(mesh);
    for (int f = threadIdx.x; f < items; f += kThreads) {
        const int4 c4 = *reinterpret_cast<const int4*>(tile + z * pp + y * rp + 4 * qd);
        if ((c4.x | c4.y | c4.z | c4.w) != 0) {
            if (inside) {
                const unsigned g = (static_cast<unsigned>(oz + z) * static_cast<unsigned>(mesh) +
                                    static_cast<unsigned>(oy + y)) * static_cast<unsigned>(mesh) +
                                   static_cast<unsigned>(ox + 4 * qd);
                flush_quad(c4, unscale, rho + g);
            } else {
                const size_t rowbase =
                    (static_cast<size_t>(wrap1(oz + z, mesh)) * M + wrap1(oy + y, mesh)) * M;
                const int gx = wrap1(ox + 4 * qd, mesh);
                if (gx + 3 < mesh && (mesh & 3) == 0) {
                    flush_quad(c4, unscale, rho + rowbase + gx);
                } else {
                    const float v[4] = {static_cast<float>(c4.x) * unscale, static_cast<float>(c4.y) * unscale,
                                        static_cast<float>(c4.z) * unscale, static_cast<float>(c4.w) * unscale};
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (v[j] != 0.0f)
                            atomicAdd(&rho[rowbase + wrap1(gx + j, mesh)], v[j]);
                }
            }
        }
        qd += dq;
        const int carry = qd >= quads ? 1 : 0;
        qd -= carry * quads;
        y += dy + carry;
        z += dz;
        if (y >= ey) {
            y -= ey;
            ++z;
        }
    }
}

template <int P>
__global__ void __launch_bounds__(kThreads) k_deposit_tiled(const float4* __restrict__ pos4, int n,
                                                             int chunk, int mesh, float inv_h_fixed,
                                                             float inv_h3_fixed, const IsoGrid* iso,
                                                             float* __restrict__ rho)
{
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed, mesh);
    const float inv_h = fr.inv_h;
    const float inv_h3 = iso ? 1.0f / (iso->h * iso->h * iso->h) : inv_h3_fixed;
    // The tile accumulates in 32-bit fixed point: integer shared-memory atomics are native and
    // about three times the rate of float ones, and integer sums are exact and independent of
    // the order of the additions.  The block's scale 2^k keeps any cell sum below 2^31 / 1.01: a
    // cell receives at most (largest 1-D weight)^3 x sum |m| / h^3 from the chunk, and the
    // rounding of at most chunk x P^3 contributions adds less than 2^15.  One unit is then
    // below 2 x 1.01 x (largest weight)^3 x sum |m| / h^3 / 2^31: with at most 512 particles a
    // chunk, a few 1e-7 of a mean cell.
    __shared__ __align__(16) int tile[kTileCells];
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
        float t;
        const int b[3] = {stencil_base<P>(p.x - fr.ox, inv_h, mesh, fr.inv_m, t), stencil_base<P>(p.y - fr.oy, inv_h, mesh, fr.inv_m, t),
                          stencil_base<P>(p.z - fr.oz, inv_h, mesh, fr.inv_m, t)};
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], b[a]);
            hi[a] = max(hi[a], b[a] + P - 1);
        }
        msum += fabsf(p.w);
    }
    for (int a = 0; a < 3; ++a) {
        const int wl = __reduce_min_sync(kFullMask, lo[a]), wh = __reduce_max_sync(kFullMask, hi[a]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo[a], wl);
            atomicMax(&s_hi[a], wh);
        }
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
    // x rounded out to whole groups of four cells, so that the flush reads the tile in int4 and
    // adds four cells at a time
    const int ox = s_lo[0] - (((s_lo[0] % 4) + 4) % 4);
    const int oy = s_lo[1], oz = s_lo[2];
    const int ex = ((s_hi[0] + 1 - ox) + 3) & ~3;
    const int ey = s_hi[1] - oy + 1, ez = s_hi[2] - oz + 1;
    const int rp = ex + kDepositRowPad, pp = ey * rp + kDepositPlanePad;  // padded pitches
    const bool tiled = ex > 0 && ey > 0 && ez > 0 && static_cast<long long>(pp) * ez <= kTileCells;
    if (tiled)
        for (int c = threadIdx.x; c < pp * ez / 4; c += kThreads)
            reinterpret_cast<int4*>(tile)[c] = make_int4(0, 0, 0, 0);
    __syncthreads();
    const float scale = s_scale, unscale = s_unscale;
    if (tiled)
        deposit_particles<P, true>(pos4, base, end, fr, mesh, inv_h3, scale, tile, ox, oy, oz, rp, pp, rho);
    else
        deposit_particles<P, false>(pos4, base, end, fr, mesh, inv_h3, scale, tile, ox, oy, oz, rp, pp, rho);
    if (!tiled)
        return;
    __syncthreads();
    flush_tile(tile, ox, oy, oz, ex, ey, ez, rp, pp, mesh, unscale, rho);
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

// Four modes a thread and iteration (16-byte loads and stores) keep enough bytes in flight to
// stream at HBM rate; a remainder of total % 4 modes, if any, goes one at a time.
__global__ void __launch_bounds__(kThreads) k_apply_green(cufftComplex* __restrict__ spec,
                                                           const float* __restrict__ green,
                                                           size_t total)
{
    const size_t quads = total / 4;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    float4* s4 = reinterpret_cast<float4*>(spec);
    const float4* g4 = reinterpret_cast<const float4*>(green);
    for (size_t q = blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; q < quads; q += stride) {
        const float4 g = g4[q];
        float4 a = s4[2 * q], b = s4[2 * q + 1];
        a.x *= g.x;
        a.y *= g.x;
        a.z *= g.y;
        a.w *= g.y;
        b.x *= g.z;
        b.y *= g.z;
        b.z *= g.w;
        b.w *= g.w;
        s4[2 * q] = a;
        s4[2 * q + 1] = b;
    }
    for (size_t i = 4 * quads + blockIdx.x * static_cast<size_t>(kThreads) + threadIdx.x; i < total; i += stride) {
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
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed, mesh);
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
            const int bx = stencil<P>(p.x - fr.ox, inv_h, mesh, fr.inv_m, wx);
            const int by = stencil<P>(p.y - fr.oy, inv_h, mesh, fr.inv_m, wy);
            const int bz = stencil<P>(p.z - fr.oz, inv_h, mesh, fr.inv_m, wz);
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

// The gather of k_interp_ad_tiled: four lanes per particle, lane q taking stencil column
// x = bx + q of every (y, z) row from the staged tile (TILED) or from the global mesh.  The loop
// bound is uniform over the block, so every lane of a quad reaches the shuffles.
// Stages the box [ox, ox + ex) x [oy, oy + ey) x [oz, oz + ez) of the mesh into the tile
// (row pitch rp, plane pitch pp) with 16-byte asynchronous copies (cp.async, one per thread and
// group of four cells; the caller waits with cp.async.wait_all and a block barrier).  ox, ex,
// rp, pp and the mesh side are multiples of 4, so every group is 16-byte aligned at both ends
// and lies on one side of the periodic x boundary.  Thread t takes groups t, t + kThreads, ...
// of the (z, y, group) range, its indices advanced by constant steps; a box inside the mesh
// reads at a 32-bit cell index without folding.
__device__ __forceinline__ void stage_box(const float* __restrict__ phi, int mesh, int ox, int oy, int oz,
                                          int ex, int ey, int ez, int rp, int pp, float* tile)
{
    const int quads = ex / 4;
    const int items = ey * ez * quads;
    int row = threadIdx.x / quads, qd = threadIdx.x - row * quads;
    int z = row / ey, y = row - z * ey;
    const int dq = kThreads % quads, drow = kThreads / quads;
    const int dz = drow / ey, dy = drow - dz * ey;
    const bool inside = ox >= 0 && oy >= 0 && oz >= 0 && ox + ex <= mesh && oy + ey <= mesh &&
                        oz + ez <= mesh && mesh <= 1024;
    const size_t M = static_cast<size_t>(mesh);
    for (int f = threadIdx.x; f < items; f += kThreads) {
        const float* src;
        if (inside)
            src = phi + ((static_cast<unsigned>(oz + z) * static_cast<unsigned>(mesh) +
                          static_cast<unsigned>(oy + y)) * static_cast<unsigned>(mesh) +
                         static_cast<unsigned>(ox + 4 * qd));
        else
            src = phi + (static_cast<size_t>(wrap1(oz + z, mesh)) * M + wrap1(oy + y, mesh)) * M +
                  wrap1(ox + 4 * qd, mesh);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(tile + z * pp + y * rp + 4 * qd)),
                     "l"(src)
                     : "memory");
        qd += dq;
        const int carry = qd >= quads ? 1 : 0;
        qd -= carry * quads;
        y += dy + carry;
        z += dz;
        if (y >= ey) {
            y -= ey;
            ++z;
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Analytic differentiation from the staged tile, one thread per particle, in two parts so
// that a particle's bases and weights are computed while the tile is still being staged:
// AdStencil holds them, ad_stencil computes them (the tile offset of the stencil's first cell
// and the W and dW weights of each axis), ad_gather reads the particle's 64 tile values once
// and forms per stencil row the W_x- and dW_x-weighted sums before the y and z weights.
template <int P>
struct AdStencil {
    int corner;  // tile offset of the stencil's first cell
    float wx[P], dx[P], wy[P], dy[P], wz[P], dz[P];
};

template <int P>
__device__ __forceinline__ AdStencil<P> ad_stencil(const float4 p, const MeshFrame& fr, int mesh, int ox,
                                                   int oy, int oz, int rp, int pp)
{
    AdStencil<P> st;
    float tx, ty, tz;
    const int bx = stencil_base<P>(p.x - fr.ox, fr.inv_h, mesh, fr.inv_m, tx);
    const int by = stencil_base<P>(p.y - fr.oy, fr.inv_h, mesh, fr.inv_m, ty);
    const int bz = stencil_base<P>(p.z - fr.oz, fr.inv_h, mesh, fr.inv_m, tz);
    stencil_weights_d<P>(tx, st.wx, st.dx);
    stencil_weights_d<P>(ty, st.wy, st.dy);
    stencil_weights_d<P>(tz, st.wz, st.dz);
    st.corner = (bz - oz) * pp + (by - oy) * rp + (bx - ox);
    return st;
}

// Returns the acceleration of the stencil's particle in mesh units (times 1/h afterwards).
template <int P>
__device__ __forceinline__ float3 ad_gather(AdStencil<P> st, const float* tile, int rp, int pp)
{
    const float* corner = tile + st.corner;
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
    if constexpr (P == 4) {
        // Each lane visits the rows and columns in its own order (offset k of an axis at step
        // k ^ s, s from lane bits, as the deposit does): a warp's particles are Morton
        // neighbours about two cells apart, and the staggered orders spread a warp's loads
        // over more banks (1.73 wavefronts a load measured, about 4 in one common order).
        const int lane = threadIdx.x & 31;
        const int sy = lane & 3, sz = (lane >> 2) & 3, sx = (lane >> 4) & 1;
        xor_permute4(st.wx, sx);
        xor_permute4(st.dx, sx);
        xor_permute4(st.wy, sy);
        xor_permute4(st.dy, sy);
        xor_permute4(st.wz, sz);
        xor_permute4(st.dz, sz);
        int yoff[4], zoff[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            yoff[k] = (k ^ sy) * rp;
            zoff[k] = (k ^ sz) * pp;
        }
        // x offsets a ^ sx: a = 0, 2 from the even base, a = 1, 3 from the odd one
        const float* ce = corner + sx;
        const float* co = corner + 1 - sx;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float sw = 0.0f, sd = 0.0f, sg = 0.0f;  // plane sums: W_y W_x, dW_y W_x, W_y dW_x
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = zoff[c] + yoff[b];
                const float v0 = ce[r], v1 = co[r], v2 = ce[r + 2], v3 = co[r + 2];
                const float rw = fmaf(st.wx[3], v3, fmaf(st.wx[2], v2, fmaf(st.wx[1], v1, st.wx[0] * v0)));
                const float rd = fmaf(st.dx[3], v3, fmaf(st.dx[2], v2, fmaf(st.dx[1], v1, st.dx[0] * v0)));
                sw = fmaf(st.wy[b], rw, sw);
                sd = fmaf(st.dy[b], rw, sd);
                sg = fmaf(st.wy[b], rd, sg);
            }
            gx = fmaf(st.wz[c], sg, gx);
            gy = fmaf(st.wz[c], sd, gy);
            gz = fmaf(st.dz[c], sw, gz);
        }
    } else {
#pragma unroll
        for (int c = 0; c < P; ++c) {
            float sw = 0.0f, sd = 0.0f, sg = 0.0f;
#pragma unroll
            for (int b = 0; b < P; ++b) {
                const float* row = corner + c * pp + b * rp;
                float rw = 0.0f, rd = 0.0f;
#pragma unroll
                for (int a = 0; a < P; ++a) {
                    rw = fmaf(st.wx[a], row[a], rw);
                    rd = fmaf(st.dx[a], row[a], rd);
                }
                sw = fmaf(st.wy[b], rw, sw);
                sd = fmaf(st.dy[b], rw, sd);
                sg = fmaf(st.wy[b], rd, sg);
            }
            gx = fmaf(st.wz[c], sg, gx);
            gy = fmaf(st.wz[c], sd, gy);
            gz = fmaf(st.dz[c], sw, gz);
        }
    }
    return make_float3(gx, gy, gz);
}

template <int P, bool TILED, int RP = 0, int PP = 0>
__device__ __forceinline__ void interp_ad_quads(const float4* __restrict__ pos4, int base, int end,
                                                const MeshFrame& fr, int mesh, const float* tile,
                                                int ox, int oy, int oz, int rp_dyn, int pp_dyn,
                                                const float* __restrict__ phi, float* __restrict__ ax,
                                                float* __restrict__ ay, float* __restrict__ az)
{
    const size_t M = static_cast<size_t>(mesh);
    const int rp = RP ? RP : rp_dyn, pp = PP ? PP : pp_dyn;  // RP, PP: pitches known at compile time
    const int q = threadIdx.x & 3;
    for (int i0 = base; i0 < end; i0 += kThreads / 4) {
        const int i = i0 + (threadIdx.x >> 2);
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
        if (i < end && q < P) {
            const float4 p = pos4[i];
            float tx, ty, tz;
            const int bx = stencil_base<P>(p.x - fr.ox, fr.inv_h, mesh, fr.inv_m, tx);
            const int by = stencil_base<P>(p.y - fr.oy, fr.inv_h, mesh, fr.inv_m, ty);
            const int bz = stencil_base<P>(p.z - fr.oz, fr.inv_h, mesh, fr.inv_m, tz);
            float wx[P], dx[P], wy[P], dy[P], wz[P], dz[P];
            stencil_weights_d<P>(tx, wx, dx);
            stencil_weights_d<P>(ty, wy, dy);
            stencil_weights_d<P>(tz, wz, dz);
            const float wq = column_weight<P>(wx, q);
            const float dq = column_weight<P>(dx, q);
            const int xs = bx + q;
            const float* col = nullptr;
            int xw = 0;
            if (TILED)
                col = tile + (bz - oz) * pp + (by - oy) * rp + (xs - ox);
            else
                xw = wrap1(xs, mesh);
#pragma unroll
            for (int c = 0; c < P; ++c) {
                float sw = 0.0f, sd = 0.0f;  // this plane's column sums over y: W_y and dW_y weighted
                const size_t zrow = TILED ? 0 : static_cast<size_t>(wrap1(bz + c, mesh)) * M;
#pragma unroll
                for (int b = 0; b < P; ++b) {
                    const float v = TILED ? col[c * pp + b * rp]
                                          : __ldg(&phi[(zrow + wrap1(by + b, mesh)) * M + xw]);
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
            ax[i] = gx * fr.inv_h;
            ay[i] = gy * fr.inv_h;
            az[i] = gz * fr.inv_h;
        }
    }
}

// Analytic differentiation with the potential staged in shared memory, the gather twin of
// k_deposit_tiled: a block takes a chunk of Morton-consecutive particles (the deposit's chunk,
// whose stencils fit one tile) and stages the box of cells their stencils cover with bulk copies
// (cp.async.bulk, global -> shared, into this CTA only), one per mesh row segment: rows start on a
// 16-byte boundary (x rounded down to a multiple of 4 cells; the mesh side is a multiple of 4),
// a row crossing the periodic x boundary takes two copies, and all complete on one mbarrier
// (bounded wait).  One thread then serves one particle (ad_stencil, ad_gather) over a tile with
// fixed or padded pitches (the padding spreads a warp's loads over the banks: 11 shared-memory
// wavefronts a load on an unpadded tile).  A chunk whose box does not fit gathers from the
// global mesh instead, four lanes a particle (interp_ad_quads), lane q reading stencil column
// x = bx + q.  The sum is
// a = (1/h) sum_c phi_c grad W(x - x_c), the weight of cell (a, b, c) in the x component being
// dW_x(a) W_y(b) W_z(c), and likewise for y and z.
template <int P>
__global__ void __launch_bounds__(kThreads, 4) k_interp_ad_tiled(const float4* __restrict__ pos4, int n,
                                                               int chunk, int mesh, float inv_h_fixed,
                                                               const IsoGrid* iso,
                                                               const float* __restrict__ phi,
                                                               float* __restrict__ ax,
                                                               float* __restrict__ ay,
                                                               float* __restrict__ az, int* err)
{
    __shared__ __align__(16) float tile[kTileCells];
    __shared__ int s_lo[3], s_hi[3];
    const MeshFrame fr = mesh_frame(iso, inv_h_fixed, mesh);
    const float inv_h = fr.inv_h;
    const int base = blockIdx.x * chunk;
    const int end = min(base + chunk, n);
    if (threadIdx.x < 3) {
        s_lo[threadIdx.x] = 1 << 30;
        s_hi[threadIdx.x] = -(1 << 30);
    }
    __syncthreads();
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    for (int i = base + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos4[i];
        float t;
        const int b[3] = {stencil_base<P>(p.x - fr.ox, inv_h, mesh, fr.inv_m, t), stencil_base<P>(p.y - fr.oy, inv_h, mesh, fr.inv_m, t),
                          stencil_base<P>(p.z - fr.oz, inv_h, mesh, fr.inv_m, t)};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = min(lo[a], b[a]);
            hi[a] = max(hi[a], b[a] + P - 1);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int wl = __reduce_min_sync(kFullMask, lo[a]), wh = __reduce_max_sync(kFullMask, hi[a]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo[a], wl);
            atomicMax(&s_hi[a], wh);
        }
    }
    __syncthreads();
    // x rounded out to whole 16-byte groups of four cells
    const int ox = s_lo[0] - (((s_lo[0] % 4) + 4) % 4);
    const int oy = s_lo[1], oz = s_lo[2];
    const int ex = ((s_hi[0] + 1 - ox) + 3) & ~3;
    const int ey = s_hi[1] - oy + 1, ez = s_hi[2] - oz + 1;
    const bool fixed = ex > 0 && ey > 0 && ez > 0 && ex <= kInterpRp && ey * kInterpRp <= kInterpPp &&
                       ez * kInterpPp <= kTileCells;
    const int rp = fixed ? kInterpRp : ex + kRowPad;
    const int pp = fixed ? kInterpPp : ey * rp + kPlanePad;
    const bool tiled = ex > 0 && ey > 0 && ez > 0 && ex <= mesh &&
                       static_cast<long long>(pp) * ez <= kTileCells && (mesh & 3) == 0;
    (void)err;  // the staging has no wait of its own to bound (cp.async.wait_all)
    if (tiled) {
        stage_box(phi, mesh, ox, oy, oz, ex, ey, ez, rp, pp, tile);
        // the first particle's stencil is prepared while the copies land
        const int i0 = base + threadIdx.x;
        AdStencil<P> st = {};
        if (i0 < end)
            st = ad_stencil<P>(pos4[i0], fr, mesh, ox, oy, oz, rp, pp);
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        for (int i = i0; i < end; i += kThreads) {
            if (i != i0)
                st = ad_stencil<P>(pos4[i], fr, mesh, ox, oy, oz, rp, pp);
            const float3 g = ad_gather<P>(st, tile, rp, pp);
            ax[i] = g.x * inv_h;
            ay[i] = g.y * inv_h;
            az[i] = g.z * inv_h;
        }
    } else
        interp_ad_quads<P, false>(pos4, base, end, fr, mesh, tile, ox, oy, oz, rp, pp, phi, ax, ay, az);
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
        k_apply_green<<<sms * 8, kThreads, 0, s>>>(p->spec, p->green, half);
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
