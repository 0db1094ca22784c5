// Learned TreePM pair correction: a 6 -> 32 -> 32 -> 3 MLP (SiLU, BF16 weights and
// activations, FP32 accumulation) on the 5th-generation tensor cores.
//
// The network maps a pair's separation (target - source, in mesh cells) and the source's
// sub-cell offset to the residual of the mesh force of that pair against the ideal Gaussian
// long-range force, per unit source mass, scaled by h^2.  Inside the kernels the 6 inputs are
// expanded to 16 features: the separation, sin and cos of 2 pi x the source offset and of
// 2 pi x the target offset (= source offset + separation), and a constant 1 that carries the
// first layer's bias.  The mesh error is periodic in both offsets, which these features
// express directly.
//
// Every GEMM is a tcgen05.mma (kind::f16, BF16 x BF16 -> FP32 in tensor memory) with M = 128
// samples, operands in shared memory in the canonical K-major layout without swizzle (core
// matrices of 8 rows x 16 bytes; LBO = stride between the two 8-element halves of a K = 16
// step, SBO = stride between 8-row groups), issued by one thread and completed through
// tcgen05.commit on an mbarrier whose waits are bounded.  Training runs forward, backward and
// the weight-gradient GEMM in one kernel per 128-sample tile; the weight gradient reduces
// over samples, so the activations and the back-propagated errors are written transposed
// (samples along K) and stacked into one 128 x 80 product:
//   rows  0..31 dZ2^T, 32..63 dZ1^T, 64..66 dOut^T;  columns 0..31 H1, 32..47 X, 48..79 H2
// whose diagonal blocks are dW2, dW1 (with b1 in X's constant column), dW3, and whose
// X-constant column also yields db2 and db3.
#include "bz_common.cuh"
#include "bz_kernels.h"

#include <cuda_bf16.h>

namespace bz {

namespace {

constexpr int kRows = 128;
constexpr int kThreadsMlp = 128;
constexpr int kFeat = 16;
constexpr int kHid = 32;
constexpr int kOutPad = 16;
constexpr int kWgN = 80;

// TMEM columns
constexpr uint32_t kColD1 = 0, kColD2 = 32, kColD3 = 64, kColDH2 = 80, kColDH1 = 112, kColDW = 144;
constexpr uint32_t kTmemCols = 256;

struct __align__(1024) MlpSmem {
    __nv_bfloat16 x[kRows * kFeat];      // A  X       LBO 128 SBO 256
    __nv_bfloat16 h1[kRows * kHid];      // A  H1      LBO 128 SBO 512
    __nv_bfloat16 h2[kRows * kHid];      // A  H2
    __nv_bfloat16 dout[kRows * kOutPad]; // A  dOut    LBO 128 SBO 256
    __nv_bfloat16 dz2[kRows * kHid];     // A  dZ2
    __nv_bfloat16 awg[kRows * kRows];    // A  stacked errors^T, K = samples: LBO 128 SBO 2048
    __nv_bfloat16 bwg[kWgN * kRows];     // B  stacked activations^T
    __nv_bfloat16 w1[kHid * kFeat];      // B  W1      LBO 128 SBO 256
    __nv_bfloat16 w2[kHid * kHid];       // B  W2      LBO 128 SBO 512
    __nv_bfloat16 w3[kOutPad * kHid];    // B  W3 (rows 3..15 zero)
    __nv_bfloat16 w2t[kHid * kHid];      // B  W2^T
    __nv_bfloat16 w3t[kHid * kOutPad];   // B  W3^T (columns 3..15 zero) LBO 128 SBO 256
    float b2[kHid];
    float b3[4];
    float red[2][3];
    unsigned long long bar;
    uint32_t tmem;
};

// Inference needs only the forward operands: one hidden buffer serves both layers (H2 is
// written after the second product has consumed H1), and tensor memory holds D1 / D3 in
// columns 0.. and D2 in 32.. (D3 is written after D1 has been read out).  17 KB of shared
// memory and 64 TMEM columns a block, so eight blocks share an SM (512 columns).
constexpr uint32_t kInferCols = 64;
constexpr uint32_t kInferD1 = 0, kInferD2 = 32, kInferD3 = 0;
constexpr int kInferBlocksPerSm = 8;

struct __align__(1024) MlpInferSmem {
    __nv_bfloat16 x[kRows * kFeat];      // A  X       LBO 128 SBO 256
    __nv_bfloat16 h1[kRows * kHid];      // A  H1, then H2
    __nv_bfloat16 w1[kHid * kFeat];      // B  W1
    __nv_bfloat16 w2[kHid * kHid];       // B  W2
    __nv_bfloat16 w3[kOutPad * kHid];    // B  W3 (rows 3..15 zero)
    float b2[kHid];
    float b3[4];
    float red[2][3];
    unsigned long long bar;
    uint32_t tmem;
};

template <class S> struct MlpCols;
template <> struct MlpCols<MlpSmem> {
    static constexpr uint32_t d1 = kColD1, d2 = kColD2, d3 = kColD3, alloc = kTmemCols;
    __device__ static __nv_bfloat16* h2(MlpSmem& sm) { return sm.h2; }
};
template <> struct MlpCols<MlpInferSmem> {
    static constexpr uint32_t d1 = kInferD1, d2 = kInferD2, d3 = kInferD3, alloc = kInferCols;
    __device__ static __nv_bfloat16* h2(MlpInferSmem& sm) { return sm.h1; }
};

__device__ __forceinline__ uint32_t kmaj(int row, int k, int lbo, int sbo)
{
    return static_cast<uint32_t>((row & 7) * 16 + (k & 7) * 2 + (k >> 3) * lbo + (row >> 3) * sbo);
}

__device__ __forceinline__ uint64_t sdesc(const void* p, uint32_t lbo, uint32_t sbo)
{
    const uint32_t a = smem_u32(p);
    return static_cast<uint64_t>((a >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                 "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
                 "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
                 "%26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                   "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                   "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
                 "%10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i)
        v[i] = __uint_as_float(r[i]);
}

// one K-major row of `k` values (k a multiple of 8), 16-byte stores
__device__ __forceinline__ void put_row(__nv_bfloat16* base, int row, const float* v, int k, int lbo,
                                        int sbo)
{
    unsigned char* b = reinterpret_cast<unsigned char*>(base);
    for (int g = 0; g < k; g += 8) {
        __align__(16) __nv_bfloat162 q[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            q[i] = __floats2bfloat162_rn(v[g + 2 * i], v[g + 2 * i + 1]);
        *reinterpret_cast<uint4*>(b + kmaj(row, g, lbo, sbo)) = *reinterpret_cast<uint4*>(q);
    }
}

// values v[0..count) into rows row0.. of column `col` of a K-major operand (transposed write)
__device__ __forceinline__ void put_col(__nv_bfloat16* base, int row0, int col, const float* v,
                                        int count, int lbo, int sbo)
{
    unsigned char* b = reinterpret_cast<unsigned char*>(base);
    for (int r = 0; r < count; ++r)
        *reinterpret_cast<__nv_bfloat16*>(b + kmaj(row0 + r, col, lbo, sbo)) = __float2bfloat16_rn(v[r]);
}

// Fast reciprocal: the activations are rounded to BF16 right after (__fdividef returns 0 for a
// denominator above 2^126, where the sigmoid is 0 to BF16 precision anyway).
__device__ __forceinline__ float sigmoidf_(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }

__device__ __forceinline__ void features(const float* in6, float* f)
{
    f[0] = in6[0];
    f[1] = in6[1];
    f[2] = in6[2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float s, c;
        sincospif(2.0f * in6[3 + a], &s, &c);
        f[3 + a] = s;
        f[6 + a] = c;
        sincospif(2.0f * (in6[3 + a] + in6[a]), &s, &c);
        f[9 + a] = s;
        f[12 + a] = c;
    }
    f[15] = 1.0f;
}

template <class S>
__device__ void load_forward_weights(S& sm, const float* __restrict__ p)
{
    const float* W1 = p + kMlpOffW1;
    const float* W2 = p + kMlpOffW2;
    const float* W3 = p + kMlpOffW3;
    unsigned char* w1 = reinterpret_cast<unsigned char*>(sm.w1);
    unsigned char* w2 = reinterpret_cast<unsigned char*>(sm.w2);
    unsigned char* w3 = reinterpret_cast<unsigned char*>(sm.w3);
    for (int i = threadIdx.x; i < kHid * kFeat; i += blockDim.x) {
        const int n = i / kFeat, k = i % kFeat;
        *reinterpret_cast<__nv_bfloat16*>(w1 + kmaj(n, k, 128, 256)) = __float2bfloat16_rn(W1[i]);
    }
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int n = i / kHid, k = i % kHid;
        *reinterpret_cast<__nv_bfloat16*>(w2 + kmaj(n, k, 128, 512)) = __float2bfloat16_rn(W2[n * kHid + k]);
    }
    for (int i = threadIdx.x; i < kOutPad * kHid; i += blockDim.x) {
        const int n = i / kHid, k = i % kHid;
        *reinterpret_cast<__nv_bfloat16*>(w3 + kmaj(n, k, 128, 512)) =
            __float2bfloat16_rn(n < 3 ? W3[n * kHid + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kHid; i += blockDim.x)
        sm.b2[i] = p[kMlpOffB2 + i];
    if (threadIdx.x < 4)
        sm.b3[threadIdx.x] = threadIdx.x < 3 ? p[kMlpOffB3 + threadIdx.x] : 0.0f;
}

// Training also needs the transposed W2 and W3 for back-propagation.
__device__ void load_weights(MlpSmem& sm, const float* __restrict__ p)
{
    load_forward_weights(sm, p);
    const float* W2 = p + kMlpOffW2;
    const float* W3 = p + kMlpOffW3;
    unsigned char* w2t = reinterpret_cast<unsigned char*>(sm.w2t);
    unsigned char* w3t = reinterpret_cast<unsigned char*>(sm.w3t);
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int n = i / kHid, k = i % kHid;
        *reinterpret_cast<__nv_bfloat16*>(w2t + kmaj(n, k, 128, 512)) = __float2bfloat16_rn(W2[k * kHid + n]);
    }
    for (int i = threadIdx.x; i < kHid * kOutPad; i += blockDim.x) {
        const int n = i / kOutPad, k = i % kOutPad;
        *reinterpret_cast<__nv_bfloat16*>(w3t + kmaj(n, k, 128, 256)) =
            __float2bfloat16_rn(k < 3 ? W3[k * kHid + n] : 0.0f);
    }
}

template <class S>
__device__ __forceinline__ void tmem_setup(S& sm)
{
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sm.tmem)),
                     "r"(MlpCols<S>::alloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0)
        mbar_init(&sm.bar, 1);
    fence_mbar_init();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

template <class S>
__device__ __forceinline__ void tmem_release(S& sm)
{
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem),
                     "r"(MlpCols<S>::alloc));
}

// Make the operands written by all threads visible to the tensor core, issue `body` from one
// thread, and wait (bounded) for the products to land in tensor memory.
template <class S, class F>
__device__ __forceinline__ void mma_step(S& sm, uint32_t& phase, int* err, F body)
{
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        body();
        umma_commit(&sm.bar);
    }
    mbar_wait_bounded(&sm.bar, phase, err);
    phase ^= 1u;
    tc_fence_after();
}

// Forward pass of the tile already in sm.x: leaves Z1 (D1), Z2 (D2) and the network output
// (D3) in tensor memory and returns this row's pre-activations and output.  KEEP_BWG (training)
// also stores the activations transposed for the weight-gradient product.
template <bool KEEP_BWG, class S>
__device__ void forward(S& sm, uint32_t tm, uint32_t& phase, int* err, float* z1, float* z2,
                        float* out)
{
    using C = MlpCols<S>;
    const int r = threadIdx.x;
    const uint32_t lane = static_cast<uint32_t>((r & ~31)) << 16;
    mma_step(sm, phase, err, [&] {
        umma(tm + C::d1, sdesc(sm.x, 128, 256), sdesc(sm.w1, 128, 256), idesc_bf16(128, 32), 0);
    });
    float h[32];
    tmem_ld32(tm + lane + C::d1, z1);
#pragma unroll
    for (int i = 0; i < 32; ++i)
        h[i] = z1[i] * sigmoidf_(z1[i]);
    put_row(sm.h1, r, h, 32, 128, 512);
    if constexpr (KEEP_BWG)
        put_col(sm.bwg, 0, r, h, 32, 128, 2048);
    mma_step(sm, phase, err, [&] {
        for (int j = 0; j < 2; ++j)
            umma(tm + C::d2, sdesc(reinterpret_cast<unsigned char*>(sm.h1) + 256 * j, 128, 512),
                 sdesc(reinterpret_cast<unsigned char*>(sm.w2) + 256 * j, 128, 512),
                 idesc_bf16(128, 32), j);
    });
    tmem_ld32(tm + lane + C::d2, z2);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        z2[i] += sm.b2[i];
        h[i] = z2[i] * sigmoidf_(z2[i]);
    }
    __nv_bfloat16* h2 = C::h2(sm);
    put_row(h2, r, h, 32, 128, 512);
    if constexpr (KEEP_BWG)
        put_col(sm.bwg, 48, r, h, 32, 128, 2048);
    mma_step(sm, phase, err, [&] {
        for (int j = 0; j < 2; ++j)
            umma(tm + C::d3, sdesc(reinterpret_cast<unsigned char*>(h2) + 256 * j, 128, 512),
                 sdesc(reinterpret_cast<unsigned char*>(sm.w3) + 256 * j, 128, 512),
                 idesc_bf16(128, 16), j);
    });
    float o[16];
    tmem_ld16(tm + lane + C::d3, o);
    out[0] = o[0] + sm.b3[0];
    out[1] = o[1] + sm.b3[1];
    out[2] = o[2] + sm.b3[2];
}

// One training step over `n` samples: gradients of the mean squared error (targets already
// divided by their scale) accumulated into grad[kMlpParams]; loss sum into loss[0].
__global__ void __launch_bounds__(kThreadsMlp) k_mlp_train(const float* __restrict__ params,
                                                            const float* __restrict__ in6,
                                                            const float* __restrict__ y3,
                                                            const int* __restrict__ index, int n,
                                                            float inv_batch, float* __restrict__ grad,
                                                            float* __restrict__ loss, int* err)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    MlpSmem& sm = *reinterpret_cast<MlpSmem*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int r = threadIdx.x;
    load_weights(sm, params);
    for (int i = r; i < kRows * kRows / 8; i += kThreadsMlp)
        reinterpret_cast<uint4*>(sm.awg)[i] = make_uint4(0, 0, 0, 0);
    tmem_setup(sm);
    const uint32_t tm = sm.tmem;
    const uint32_t lane = static_cast<uint32_t>((r & ~31)) << 16;
    uint32_t phase = 0;

    const int s = blockIdx.x * kRows + r;
    const bool valid = s < n;
    const int src = valid ? (index ? index[s] : s) : 0;
    float in[6], f[16], tgt[3] = {0.0f, 0.0f, 0.0f};
    for (int i = 0; i < 6; ++i)
        in[i] = valid ? in6[6 * static_cast<size_t>(src) + i] : 0.0f;
    if (valid)
        for (int i = 0; i < 3; ++i)
            tgt[i] = y3[3 * static_cast<size_t>(src) + i];
    features(in, f);
    if (!valid)
        for (int i = 0; i < 16; ++i)
            f[i] = 0.0f;
    put_row(sm.x, r, f, 16, 128, 256);
    put_col(sm.bwg, 32, r, f, 16, 128, 2048);

    float z1[32], z2[32], out[3];
    forward<true>(sm, tm, phase, err, z1, z2, out);

    // dL/dout for L = sum (out - y)^2 / batch
    float d[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
        d[i] = 0.0f;
    float l = 0.0f;
    if (valid)
        for (int i = 0; i < 3; ++i) {
            const float e = out[i] - tgt[i];
            l += e * e;
            d[i] = 2.0f * e * inv_batch;
        }
    put_row(sm.dout, r, d, 16, 128, 256);
    put_col(sm.awg, 64, r, d, 3, 128, 2048);
    for (int o = 16; o > 0; o >>= 1)
        l += __shfl_xor_sync(kFullMask, l, o);
    if ((r & 31) == 0)
        atomicAdd(loss, l);

    // dH2 = dOut W3 ; dZ2 = dH2 * silu'(Z2)
    mma_step(sm, phase, err, [&] {
        umma(tm + kColDH2, sdesc(sm.dout, 128, 256), sdesc(sm.w3t, 128, 256), idesc_bf16(128, 32), 0);
    });
    float g[32];
    tmem_ld32(tm + lane + kColDH2, g);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const float sg = sigmoidf_(z2[i]);
        g[i] *= sg * (1.0f + z2[i] * (1.0f - sg));
    }
    put_row(sm.dz2, r, g, 32, 128, 512);
    put_col(sm.awg, 0, r, g, 32, 128, 2048);
    // dH1 = dZ2 W2 ; dZ1 = dH1 * silu'(Z1)
    mma_step(sm, phase, err, [&] {
        for (int j = 0; j < 2; ++j)
            umma(tm + kColDH1, sdesc(reinterpret_cast<unsigned char*>(sm.dz2) + 256 * j, 128, 512),
                 sdesc(reinterpret_cast<unsigned char*>(sm.w2t) + 256 * j, 128, 512),
                 idesc_bf16(128, 32), j);
    });
    tmem_ld32(tm + lane + kColDH1, g);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const float sg = sigmoidf_(z1[i]);
        g[i] *= sg * (1.0f + z1[i] * (1.0f - sg));
    }
    put_col(sm.awg, 32, r, g, 32, 128, 2048);
    // stacked weight gradient: [dZ2; dZ1; dOut]^T (128 x samples) x [H1 | X | H2] (80 x samples)
    mma_step(sm, phase, err, [&] {
        for (int j = 0; j < kRows / 16; ++j)
            umma(tm + kColDW, sdesc(reinterpret_cast<unsigned char*>(sm.awg) + 256 * j, 128, 2048),
                 sdesc(reinterpret_cast<unsigned char*>(sm.bwg) + 256 * j, 128, 2048),
                 idesc_bf16(128, kWgN), j);
    });
    float gw[80];
    tmem_ld32(tm + lane + kColDW, gw);
    tmem_ld32(tm + lane + kColDW + 32, gw + 32);
    tmem_ld16(tm + lane + kColDW + 64, gw + 64);
    if (r < 32) {
        for (int k = 0; k < 32; ++k)
            atomicAdd(&grad[kMlpOffW2 + r * kHid + k], gw[k]);
        atomicAdd(&grad[kMlpOffB2 + r], gw[32 + 15]);
    } else if (r < 64) {
        for (int k = 0; k < 16; ++k)
            atomicAdd(&grad[kMlpOffW1 + (r - 32) * kFeat + k], gw[32 + k]);
    } else if (r < 67) {
        for (int k = 0; k < 32; ++k)
            atomicAdd(&grad[kMlpOffW3 + (r - 64) * kHid + k], gw[48 + k]);
        atomicAdd(&grad[kMlpOffB3 + (r - 64)], gw[32 + 15]);
    }
    tmem_release(sm);
}

// Batch inference: out3 = scale * network(in6) (per sample).
__global__ void __launch_bounds__(kThreadsMlp, kInferBlocksPerSm) k_mlp_forward(
    const float* __restrict__ params, const float* __restrict__ in6, int n, float scale,
    float* __restrict__ out3, int* err)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    MlpInferSmem& sm = *reinterpret_cast<MlpInferSmem*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int r = threadIdx.x;
    load_forward_weights(sm, params);
    tmem_setup(sm);
    const uint32_t tm = sm.tmem;
    uint32_t phase = 0;
    const int tiles = (n + kRows - 1) / kRows;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int s = t * kRows + r;
        const bool valid = s < n;
        float in[6], f[16];
        for (int i = 0; i < 6; ++i)
            in[i] = valid ? in6[6 * static_cast<size_t>(s) + i] : 0.0f;
        features(in, f);
        put_row(sm.x, r, f, 16, 128, 256);
        float z1[32], z2[32], out[3];
        forward<false>(sm, tm, phase, err, z1, z2, out);
        if (valid)
            for (int i = 0; i < 3; ++i)
                out3[3 * static_cast<size_t>(s) + i] = scale * out[i];
    }
    tmem_release(sm);
}

// Pair correction: rows of a tile are (target, pair slot) for 2 targets x kPairSlots slots.
// Each listed pair subtracts m_source / h^2 * scale * network(separation, source offset)
// from its target's acceleration.
__global__ void __launch_bounds__(kThreadsMlp, kInferBlocksPerSm) k_mlp_pairs(
    const float* __restrict__ params, const float4* __restrict__ pos4, int n,
    const int* __restrict__ pair_src, const int* __restrict__ pair_cnt, float inv_h, float box,
    float coef, float* __restrict__ ax, float* __restrict__ ay, float* __restrict__ az, int* err)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    MlpInferSmem& sm = *reinterpret_cast<MlpInferSmem*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int r = threadIdx.x;
    load_forward_weights(sm, params);
    tmem_setup(sm);
    const uint32_t tm = sm.tmem;
    uint32_t phase = 0;
    const int tiles = (n + 1) / 2;
    const float inv_box = 1.0f / box;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int tgt = 2 * t + r / kPairSlots;
        const int slot = r % kPairSlots;
        bool valid = tgt < n;
        float in[6] = {0, 0, 0, 0, 0, 0};
        float ms = 0.0f;
        if (valid) {
            const int cnt = min(pair_cnt[tgt], kPairSlots);
            valid = slot < cnt;
            if (valid) {
                const float4 pt = pos4[tgt];
                const float4 ps = pos4[pair_src[static_cast<size_t>(tgt) * kPairSlots + slot]];
                float dx = pt.x - ps.x, dy = pt.y - ps.y, dz = pt.z - ps.z;
                dx -= box * rintf(dx * inv_box);
                dy -= box * rintf(dy * inv_box);
                dz -= box * rintf(dz * inv_box);
                in[0] = dx * inv_h;
                in[1] = dy * inv_h;
                in[2] = dz * inv_h;
                const float ox = ps.x * inv_h, oy = ps.y * inv_h, oz = ps.z * inv_h;
                in[3] = ox - floorf(ox);
                in[4] = oy - floorf(oy);
                in[5] = oz - floorf(oz);
                ms = ps.w;
            }
        }
        float f[16];
        features(in, f);
        put_row(sm.x, r, f, 16, 128, 256);
        float z1[32], z2[32], out[3];
        forward<false>(sm, tm, phase, err, z1, z2, out);
        float c[3];
        for (int i = 0; i < 3; ++i) {
            c[i] = valid ? coef * ms * out[i] : 0.0f;
            for (int o = 16; o > 0; o >>= 1)
                c[i] += __shfl_xor_sync(kFullMask, c[i], o);
        }
        // two warps per target: combine their sums
        if ((r & 31) == 0 && (r & 32))
            for (int i = 0; i < 3; ++i)
                sm.red[r / 64][i] = c[i];
        __syncthreads();
        if ((r & 63) == 0 && tgt < n) {
            ax[tgt] -= c[0] + sm.red[r / 64][0];
            ay[tgt] -= c[1] + sm.red[r / 64][1];
            az[tgt] -= c[2] + sm.red[r / 64][2];
        }
        __syncthreads();
    }
    tmem_release(sm);
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int count, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    g[i] = 0.0f;
}

size_t mlp_smem() { return sizeof(MlpSmem) + 1024; }
// Inference blocks request at least 1/7 of an SM's shared memory so that no more than
// kInferBlocksPerSm of them (whose TMEM columns add up to the SM's 512) are ever co-resident:
// a ninth block's tcgen05.alloc would otherwise wait for a column range to be freed.
size_t mlp_infer_smem()
{
    const size_t need = sizeof(MlpInferSmem) + 1024;
    const size_t floor = 228 * 1024 / (kInferBlocksPerSm + 1) + 1024;
    return need > floor ? need : floor;
}

void set_mlp_attrs()
{
    static bool done[kMaxDevices] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < kMaxDevices && done[dev])
        return;
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(mlp_smem()));
    cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(mlp_infer_smem()));
    cudaFuncSetAttribute(k_mlp_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(mlp_infer_smem()));
    if (dev >= 0 && dev < kMaxDevices)
        done[dev] = true;
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

} // namespace

void launch_mlp_train_step(const float* params, const float* in6, const float* y3, const int* index,
                           int n, float* grad, float* loss, int* err, cudaStream_t s)
{
    set_mlp_attrs();
    const int blocks = (n + kRows - 1) / kRows;
    count_launch();
    k_mlp_train<<<blocks, kThreadsMlp, mlp_smem(), s>>>(params, in6, y3, index, n,
                                                        1.0f / static_cast<float>(n), grad, loss, err);
}

void launch_mlp_adam(float* params, float* grad, float* m, float* v, int step, float lr, cudaStream_t s)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, static_cast<float>(step)));
    const float c2 = 1.0f / (1.0f - powf(b2, static_cast<float>(step)));
    count_launch();
    k_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_mlp_forward(const float* params, const float* in6, int n, float scale, float* out3,
                        int* err, cudaStream_t s)
{
    set_mlp_attrs();
    int blocks = (n + kRows - 1) / kRows;
    const int cap = kInferBlocksPerSm * sm_count();
    blocks = blocks < cap ? blocks : cap;
    count_launch();
    k_mlp_forward<<<blocks > 0 ? blocks : 1, kThreadsMlp, mlp_infer_smem(), s>>>(params, in6, n, scale,
                                                                                 out3, err);
}

void launch_mlp_pairs(const float* params, const float4* pos4, int n, const int* pair_src,
                      const int* pair_cnt, float h, float box, float scale, float* ax, float* ay,
                      float* az, int* err, cudaStream_t s)
{
    set_mlp_attrs();
    int blocks = (n + 1) / 2;
    const int cap = kInferBlocksPerSm * sm_count();
    blocks = blocks < cap ? blocks : cap;
    count_launch();
    k_mlp_pairs<<<blocks > 0 ? blocks : 1, kThreadsMlp, mlp_infer_smem(), s>>>(
        params, pos4, n, pair_src, pair_cnt, 1.0f / h, box, scale / (h * h), ax, ay, az, err);
}

} // namespace bz
