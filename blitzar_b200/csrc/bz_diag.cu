// FP64 reference accelerations on a subsample of targets, used to state every result's force
// error on the GPU itself: a direct sum for open boundaries (the softened law of
// engine/physics/treepm/model/TpmCpu.cpp:78-116 in FP64) and an Ewald sum for the periodic
// box (the reference has none).  One block per target, FP64 block reductions.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.14159265358979323846;

__device__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFullMask, v, o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kThreads / 32; ++i)
            t += sh[i];
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kThreads) k_direct_f64(const float4* __restrict__ pos4, int n,
                                                          const int* __restrict__ targets,
                                                          const int* __restrict__ src_lo,
                                                          const int* __restrict__ src_hi,
                                                          double eps2, double* acc3)
{
    __shared__ double sh[kThreads / 32];
    const int i = targets[blockIdx.x];
    const float4 me = pos4[i];
    double a[3] = {0, 0, 0};
    const int j0 = src_lo ? src_lo[blockIdx.x] : 0;
    const int j1 = src_hi ? src_hi[blockIdx.x] : n;
    for (int j = j0 + threadIdx.x; j < j1; j += kThreads) {
        if (j == i)
            continue;
        const float4 s = pos4[j];
        const double dx = (double)s.x - me.x, dy = (double)s.y - me.y, dz = (double)s.z - me.z;
        const double r2 = dx * dx + dy * dy + dz * dz + eps2;
        const double ri = 1.0 / sqrt(r2);
        const double f = (double)s.w * ri * ri * ri;
        a[0] += f * dx;
        a[1] += f * dy;
        a[2] += f * dz;
    }
    for (int c = 0; c < 3; ++c) {
        const double t = block_sum(a[c], sh);
        if (threadIdx.x == 0)
            acc3[3 * blockIdx.x + c] = t;
    }
}

// Structure factors S(k) = sum_j m_j e^{i k.x_j} for the half-space integer vectors.
__global__ void __launch_bounds__(kThreads) k_ewald_sk(const float4* __restrict__ pos4, int n,
                                                        int kmax, double kf, double* sk)
{
    __shared__ double sh[kThreads / 32];
    const int side = 2 * kmax + 1;
    int q = blockIdx.x, found = -1, idx = 0;
    int va = 0, vb = 0, vc = 0;
    for (int a = 0; a <= kmax && found < 0; ++a)
        for (int b = -kmax; b <= kmax && found < 0; ++b)
            for (int c = -kmax; c <= kmax; ++c) {
                if (a == 0 && (b < 0 || (b == 0 && c <= 0)))
                    continue;
                if (idx == q) {
                    found = idx;
                    va = a;
                    vb = b;
                    vc = c;
                    break;
                }
                ++idx;
            }
    (void)side;
    const double kx = kf * va, ky = kf * vb, kz = kf * vc;
    double re = 0.0, im = 0.0;
    for (int j = threadIdx.x; j < n; j += kThreads) {
        const float4 p = pos4[j];
        double s, c;
        sincos(kx * p.x + ky * p.y + kz * p.z, &s, &c);
        re += p.w * c;
        im += p.w * s;
    }
    re = block_sum(re, sh);
    im = block_sum(im, sh);
    if (threadIdx.x == 0) {
        sk[5 * q + 0] = kx;
        sk[5 * q + 1] = ky;
        sk[5 * q + 2] = kz;
        sk[5 * q + 3] = re;
        sk[5 * q + 4] = im;
    }
}

__global__ void __launch_bounds__(kThreads) k_ewald_target(const float4* __restrict__ pos4, int n,
                                                            const int* __restrict__ targets,
                                                            double eps2, double box,
                                                            double alpha, int nk,
                                                            const double* __restrict__ sk,
                                                            double* acc3)
{
    __shared__ double sh[kThreads / 32];
    const int i = targets[blockIdx.x];
    const float4 me = pos4[i];
    const double c2 = 2.0 * alpha / sqrt(kPi);
    const double inv_box = 1.0 / box;
    double a[3] = {0, 0, 0};
    for (int j = threadIdx.x; j < n; j += kThreads) {
        if (j == i)
            continue;
        const float4 s = pos4[j];
        double d[3] = {(double)s.x - me.x, (double)s.y - me.y, (double)s.z - me.z};
        for (int c = 0; c < 3; ++c)
            d[c] -= box * rint(d[c] * inv_box);
        const double s2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
        const double sr = sqrt(s2);
        const double w = erfc(alpha * sr) + c2 * sr * exp(-alpha * alpha * s2);
        const double f = (double)s.w * w / (s2 * sr);
        a[0] += f * d[0];
        a[1] += f * d[1];
        a[2] += f * d[2];
    }
    const double V = box * box * box;
    for (int q = threadIdx.x; q < nk; q += kThreads) {
        const double kx = sk[5 * q], ky = sk[5 * q + 1], kz = sk[5 * q + 2];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double coef = 2.0 * (4.0 * kPi / V) * exp(-k2 / (4.0 * alpha * alpha)) / k2;
        double sn, cs;
        sincos(kx * me.x + ky * me.y + kz * me.z, &sn, &cs);
        const double im = cs * sk[5 * q + 4] - sn * sk[5 * q + 3];
        a[0] += coef * im * kx;
        a[1] += coef * im * ky;
        a[2] += coef * im * kz;
    }
    for (int c = 0; c < 3; ++c) {
        const double t = block_sum(a[c], sh);
        if (threadIdx.x == 0)
            acc3[3 * blockIdx.x + c] = t;
    }
}

// Ideal long-range (Gaussian-split) force of a periodic set of sources at one target: the
// Ewald sum with the split's short-range part sum m w_split(r) r^-3 d removed, which leaves
// the real-space weight w_alpha(r) - w_split(r) (both of the form erfc(r/2s) + r/(s sqrt(pi))
// e^{-r^2/4s^2}).  Minimum image; the sources are the first n_src particles.
__global__ void __launch_bounds__(kThreads) k_lr_ideal_target(const float4* __restrict__ pos4,
                                                               int n_src,
                                                               const int* __restrict__ targets,
                                                               double box, double alpha,
                                                               double rsplit, int nk,
                                                               const double* __restrict__ sk,
                                                               double* acc3)
{
    __shared__ double sh[kThreads / 32];
    const int i = targets[blockIdx.x];
    const float4 me = pos4[i];
    const double c2 = 2.0 * alpha / sqrt(kPi);
    const double u2 = 0.5 / rsplit, cs2 = 1.0 / (rsplit * sqrt(kPi));
    const double inv_box = 1.0 / box;
    double a[3] = {0, 0, 0};
    for (int j = threadIdx.x; j < n_src; j += kThreads) {
        if (j == i)
            continue;
        const float4 s = pos4[j];
        double d[3] = {(double)s.x - me.x, (double)s.y - me.y, (double)s.z - me.z};
        for (int c = 0; c < 3; ++c)
            d[c] -= box * rint(d[c] * inv_box);
        const double s2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (s2 <= 0.0)
            continue;
        const double sr = sqrt(s2);
        const double wa = erfc(alpha * sr) + c2 * sr * exp(-alpha * alpha * s2);
        const double ws = erfc(u2 * sr) + cs2 * sr * exp(-u2 * u2 * s2);
        const double f = (double)s.w * (wa - ws) / (s2 * sr);
        a[0] += f * d[0];
        a[1] += f * d[1];
        a[2] += f * d[2];
    }
    const double V = box * box * box;
    for (int q = threadIdx.x; q < nk; q += kThreads) {
        const double kx = sk[5 * q], ky = sk[5 * q + 1], kz = sk[5 * q + 2];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double coef = 2.0 * (4.0 * kPi / V) * exp(-k2 / (4.0 * alpha * alpha)) / k2;
        double sn, cs;
        sincos(kx * me.x + ky * me.y + kz * me.z, &sn, &cs);
        const double im = cs * sk[5 * q + 4] - sn * sk[5 * q + 3];
        a[0] += coef * im * kx;
        a[1] += coef * im * ky;
        a[2] += coef * im * kz;
    }
    for (int c = 0; c < 3; ++c) {
        const double t = block_sum(a[c], sh);
        if (threadIdx.x == 0)
            acc3[3 * blockIdx.x + c] = t;
    }
}

} // namespace

void launch_lr_ideal_f64(const float4* pos4, int n_src, const int* targets, int nt, double box,
                         double alpha, int kmax, double rsplit, double* sk_scratch, double* acc3,
                         cudaStream_t s)
{
    const int nk = ewald_num_k(kmax);
    count_launch();
    k_ewald_sk<<<nk, kThreads, 0, s>>>(pos4, n_src, kmax, 2.0 * kPi / box, sk_scratch);
    if (nt > 0) {
        count_launch();
        k_lr_ideal_target<<<nt, kThreads, 0, s>>>(pos4, n_src, targets, box, alpha, rsplit, nk,
                                                   sk_scratch, acc3);
    }
}

int ewald_num_k(int kmax)
{
    const int side = 2 * kmax + 1;
    return (side * side * side - 1) / 2;
}

void launch_direct_f64(const float4* pos4, int n, const int* targets, int nt, double eps,
                       double* acc3, cudaStream_t s, const int* src_lo, const int* src_hi)
{
    if (nt > 0) {
        count_launch();
        k_direct_f64<<<nt, kThreads, 0, s>>>(pos4, n, targets, src_lo, src_hi, eps * eps, acc3);
    }
}

void launch_ewald_f64(const float4* pos4, int n, const int* targets, int nt, double eps,
                      double box, double alpha, int kmax, double* sk_scratch, double* acc3,
                      cudaStream_t s)
{
    const int nk = ewald_num_k(kmax);
    count_launch();
    k_ewald_sk<<<nk, kThreads, 0, s>>>(pos4, n, kmax, 2.0 * kPi / box, sk_scratch);
    if (nt > 0) {
        count_launch();
        k_ewald_target<<<nt, kThreads, 0, s>>>(pos4, n, targets, eps * eps, box, alpha, nk,
                                               sk_scratch, acc3);
    }
}

} // namespace bz
