// Warp-cooperative group tree walk (the force hot path).
//
// One warp owns a group of at most 32 consecutive Morton-sorted targets (a run of sibling
// subtrees cut from the octree, bz_groups.cu).  It walks the tree once for the whole group: each step pops up to 32 nodes (one per lane), tests them against the
// group's bounding box, and sorts them with warp votes into
//   - pruned (beyond the short-range cutoff),
//   - accepted multipoles  -> appended to a shared-memory node list,
//   - leaves to sum directly -> appended to a shared-memory leaf list,
//   - opened internal nodes -> children pushed on a shared-memory stack (shuffle scan).
// Full lists are flushed: every lane evaluates its own target against each listed node, and
// leaf particles are pulled into a shared-memory tile with cp.async.bulk (global -> shared,
// completing on an mbarrier, into this CTA only) and summed with FP32 pair arithmetic.
// Per-flush partial sums are folded into the running force with a two-sum (compensated
// accumulation).
//
// Decisions are computed with round-to-nearest intrinsics (no contraction) so that the set
// of accepted nodes and direct leaves is bit-identical to the oracle's; the reference's
// per-particle stackless walk is engine/physics/octree/cuda/force/OctGpu.inl:100-228 and the
// TreePM pair law with the Gaussian split is engine/physics/core/cuda/prelude/
// CudForceKernels.inl:62-89.
#include "bz_common.cuh"
#include "bz_kernels.h"

namespace bz {

namespace {

constexpr int kWarps = 4;
constexpr int kStack = 512;       // shared-memory part of the traversal stack
constexpr int kSpill = 8192;      // per-warp global spill area (oldest entries)
constexpr int kList = 64;
constexpr int kTile = 128;
constexpr int kFlushParticles = 256;  // listed leaf particles that trigger a flush
constexpr int kIndexBits = 26;
constexpr int kIndexMask = (1 << kIndexBits) - 1;
constexpr int kPerPairImage = 64;  // leaf code: periodic image chosen per pair

constexpr int kNoShift = 21;       // shift code of the central image on all three axes

struct __align__(16) WarpSmem {
    float4 tile[kTile];
    union {
        struct {
            float4 nd_mono[32];
            float4 nd_qa[32];
        };
        unsigned mask[kTile / 32][32];  // leaf flush: per-lane in-cutoff bits of the tile
    };
    float2 nd_qb[32];
    float nd_tr[32];  // -tr(Q) eps^2 / 3 of each node (traceless Newtonian form only)
    int tidx[kTile];  // sorted index of each tile source (only when pairs are recorded)
    int stack[kStack];
    int nlist[kList];
    int lstart[kList];
    int lcount[kList];
    int lcode[kList];
    int lnode[kList];
    int lpre[kList];
    unsigned long long bar;
};

// erfc(u) ~= t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) e^{-u^2},  t = 1/(1 + p u)
// (Abramowitz & Stegun 7.1.26, |error| <= 1.5e-7).
__device__ __forceinline__ float erfc_as(float u, float e)
{
    const float t = rcp_approx(fmaf(0.3275911f, u, 1.0f));
    float p = 1.061405429f;
    p = fmaf(p, t, -1.453152027f);
    p = fmaf(p, t, 1.421413741f);
    p = fmaf(p, t, -0.284496736f);
    p = fmaf(p, t, 0.254829592f);
    return t * p * e;
}

constexpr float kTwoOverSqrtPi = 1.1283791670955126f;
constexpr float kFourOverSqrtPi = 2.2567583341910252f;
constexpr float kEightOverSqrtPi = 4.5135166683820503f;

struct SplitK {
    float inv2rs;  // 1 / (2 r_s)
    float cexp;    // -log2(e) / (4 r_s^2): e^{-u^2} = 2^{s^2 cexp}
    float pk;      // 0.3275911 / (2 r_s): A&S t = 1 / (1 + p u)
    float c2;      // (2/sqrt(pi)) / (2 r_s): 2u/sqrt(pi) = s c2
};

__device__ __forceinline__ float ex2_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <bool SPLIT, bool POT>
__device__ __forceinline__ void pair_pp(const float4 s, float tx, float ty, float tz,
                                        const WalkParams& p, float inv2rs, bool cut, bool self,
                                        float& fx, float& fy, float& fz, float& fp)
{
    const float dx = s.x - tx, dy = s.y - ty, dz = s.z - tz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float s2 = r2 + p.eps2;
    float m = s.w;
    if (cut && r2 > p.rcut2)
        m = 0.0f;
    float rinv = rsqrt_approx(s2);
    if (s2 <= p.min_dist2) {
        m = 0.0f;
        rinv = 0.0f;
    }
    const float rinv2 = rinv * rinv;
    float f = m * rinv * rinv2;
    if (SPLIT) {
        const float u = s2 * rinv * inv2rs;
        const float e = __expf(-u * u);
        const float ec = erfc_as(u, e);
        const float w = fmaf(kTwoOverSqrtPi * u, e, ec);
        f *= w;
        if (POT && !self)
            fp = fmaf(-m * ec, rinv, fp);
    } else {
        if (POT && !self)
            fp = fmaf(-m, rinv, fp);
    }
    fx = fmaf(f, dx, fx);
    fy = fmaf(f, dy, fy);
    fz = fmaf(f, dz, fz);
}

// Force-only pair for softening above the minimum-distance floor (no zero-distance guard
// needed): the split weight w = e^{-u^2} (t P(t) + 2u/sqrt(pi)) with the A&S 7.1.26 erfc and
// all scale factors folded into precomputed constants.
// Returns 1 when the pair lies inside the cutoff (or no cutoff is applied), else 0.
template <bool SPLIT>
__device__ __forceinline__ unsigned pair_fast(const float4 s, float tx, float ty, float tz, float eps2,
                                              float rcut2, bool cut, const SplitK& k, float& fx,
                                              float& fy, float& fz)
{
    const float dx = s.x - tx, dy = s.y - ty, dz = s.z - tz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float s2 = r2 + eps2;
    const bool outside = cut && r2 > rcut2;
    const float m = outside ? 0.0f : s.w;
    const float rinv = rsqrt_approx(s2);
    float mw = m;
    if (SPLIT) {
        const float sd = s2 * rinv;
        const float e = ex2_approx(s2 * k.cexp);
        const float t = rcp_approx(fmaf(sd, k.pk, 1.0f));
        float q = 1.061405429f;
        q = fmaf(q, t, -1.453152027f);
        q = fmaf(q, t, 1.421413741f);
        q = fmaf(q, t, -0.284496736f);
        q = fmaf(q, t, 0.254829592f);
        mw = m * (e * fmaf(t, q, sd * k.c2));
    }
    const float f = mw * (rinv * rinv * rinv);
    fx = fmaf(f, dx, fx);
    fy = fmaf(f, dy, fy);
    fz = fmaf(f, dz, fz);
    return outside ? 0u : 1u;
}

template <bool SPLIT, bool QUAD, bool POT>
__device__ __forceinline__ void pair_pn(const float4 mo, const float4 qa, const float2 qb,
                                        float tx, float ty, float tz, const WalkParams& p,
                                        float inv2rs, float& fx, float& fy, float& fz, float& fp)
{
    const float dx = mo.x - tx, dy = mo.y - ty, dz = mo.z - tz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float s2 = r2 + p.eps2;
    float rinv = rsqrt_approx(s2);
    float m = mo.w;
    if (s2 <= p.min_dist2) {
        rinv = 0.0f;
        m = 0.0f;
    }
    const float rinv2 = rinv * rinv;
    float D0, D1, D2 = 0.0f, D3 = 0.0f;
    if (SPLIT) {
        const float u = s2 * rinv * inv2rs;
        const float e = __expf(-u * u);
        const float ec = erfc_as(u, e);
        const float h = fmaf(kTwoOverSqrtPi * u, e, ec);
        D0 = ec * rinv;
        D1 = h * rinv * rinv2;
        if (QUAD) {
            const float u2 = u * u;
            const float k = fmaf(kFourOverSqrtPi * u2 * u, e, 3.0f * h);
            const float l = fmaf(kEightOverSqrtPi * u2 * u2 * u, e, 5.0f * k);
            D2 = k * rinv2 * rinv2 * rinv;
            D3 = l * rinv2 * rinv2 * rinv2 * rinv;
        }
    } else {
        D0 = rinv;
        D1 = rinv * rinv2;
        if (QUAD) {
            D2 = 3.0f * D1 * rinv2;
            D3 = 5.0f * D2 * rinv2;
        }
    }
    float c0 = m * D1;
    if (QUAD) {
        const float qdx = fmaf(qa.x, dx, fmaf(qa.y, dy, qa.z * dz));
        const float qdy = fmaf(qa.y, dx, fmaf(qa.w, dy, qb.x * dz));
        const float qdz = fmaf(qa.z, dx, fmaf(qb.x, dy, qb.y * dz));
        const float dqd = fmaf(dx, qdx, fmaf(dy, qdy, dz * qdz));
        const float tr = qa.x + qa.w + qb.y;
        if (m == 0.0f) {
            D1 = D2 = D3 = 0.0f;
        }
        c0 = fmaf(0.5f * D3, dqd, fmaf(-0.5f * D2, tr, c0));
        fx = fmaf(c0, dx, fmaf(-D2, qdx, fx));
        fy = fmaf(c0, dy, fmaf(-D2, qdy, fy));
        fz = fmaf(c0, dz, fmaf(-D2, qdz, fz));
        if (POT)
            fp += fmaf(-m, D0, fmaf(0.5f * D1, tr, -0.5f * D2 * dqd));
    } else {
        fx = fmaf(c0, dx, fx);
        fy = fmaf(c0, dy, fy);
        fz = fmaf(c0, dz, fz);
        if (POT)
            fp = fmaf(-m, D0, fp);
    }
}

// Force-only Newtonian quadrupole interaction with the traceless second moment
// Q' = Q - tr(Q)/3 I.  With softening the trace does not drop out of the expansion; written with
// Q' the acceleration is (m/s^3 + 15/2 (dQ'd + trm)/s^7) d - 3 Q'd/s^5 with s^2 = r^2 + eps^2 and
// trm = -tr(Q) eps^2/3, algebraically the same as the traceful form (the m/s^3 + (15/2 dQd/s^7 -
// 3/2 tr/s^5)) d - 3 Qd/s^5 of pair_pn).  Used only when eps^2 exceeds the minimum distance^2,
// so the minimum-distance guard of pair_pn can never trigger.
__device__ __forceinline__ void pair_pn_newton(const float4 mo, const float4 qa, const float2 qb,
                                               float trm, float tx, float ty, float tz, float eps2,
                                               float& fx, float& fy, float& fz)
{
    const float dx = mo.x - tx, dy = mo.y - ty, dz = mo.z - tz;
    const float s2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    const float rinv = rsqrt_approx(s2);
    const float a = rinv * rinv;       // 1/r^2
    const float b = rinv * a;          // 1/r^3
    const float t5 = b * a;            // 1/r^5
    const float qdx = fmaf(qa.x, dx, fmaf(qa.y, dy, qa.z * dz));
    const float qdy = fmaf(qa.y, dx, fmaf(qa.w, dy, qb.x * dz));
    const float qdz = fmaf(qa.z, dx, fmaf(qb.x, dy, qb.y * dz));
    const float dqd = fmaf(dx, qdx, fmaf(dy, qdy, fmaf(dz, qdz, trm)));
    const float c0 = fmaf(7.5f * t5, a * dqd, mo.w * b);
    const float n2 = -3.0f * t5;
    fx = fmaf(c0, dx, fmaf(n2, qdx, fx));
    fy = fmaf(c0, dy, fmaf(n2, qdy, fy));
    fz = fmaf(c0, dz, fmaf(n2, qdz, fz));
}

struct Acc {
    float s[4];
    float e[4];
    __device__ void zero()
    {
        for (int i = 0; i < 4; ++i)
            s[i] = e[i] = 0.0f;
    }
    __device__ void add(int i, float v)
    {
        float ss, ee;
        two_sum(s[i], v, ss, ee);
        s[i] = ss;
        e[i] += ee;
    }
    __device__ float total(int i) const { return s[i] + e[i]; }
};

__device__ __forceinline__ float shift_of(int code, int axis, float box)
{
    return box * static_cast<float>(((code >> (2 * axis)) & 3) - 1);
}

template <bool PERIODIC, bool SPLIT, bool QUAD, bool POT>
__device__ __forceinline__ void flush_nodes(WarpSmem& w, int nn, const TreeArrays& t,
                                            const WalkParams& p, float inv2rs, float tx,
                                            float ty, float tz, Acc& acc)
{
    const int lane = threadIdx.x & 31;
    // Newtonian force-only quadrupoles take the traceless form; it needs eps^2 > min distance^2
    const bool newton = !SPLIT && QUAD && !POT && p.eps2 > p.min_dist2;
    for (int base = 0; base < nn; base += 32) {
        const int m = min(32, nn - base);
        if (lane < m) {
            const int e = w.nlist[base + lane];
            const int k = e & kIndexMask;
            float4 mo = t.mono[k];
            if (PERIODIC) {
                const int code = static_cast<int>(static_cast<unsigned>(e) >> kIndexBits);
                mo.x -= shift_of(code, 0, p.box);
                mo.y -= shift_of(code, 1, p.box);
                mo.z -= shift_of(code, 2, p.box);
            }
            w.nd_mono[lane] = mo;
            if (QUAD) {
                float4 qa = t.quadA[k];
                float2 qb = t.quadB[k];
                if (newton) {
                    const float tr = qa.x + qa.w + qb.y;
                    const float tr3 = tr * (1.0f / 3.0f);
                    qa.x -= tr3;
                    qa.w -= tr3;
                    qb.y -= tr3;
                    w.nd_tr[lane] = -tr3 * p.eps2;
                }
                w.nd_qa[lane] = qa;
                w.nd_qb[lane] = qb;
            }
        }
        __syncwarp();
        float fx = 0.0f, fy = 0.0f, fz = 0.0f, fp = 0.0f;
        if (newton) {
            int j = 0;
            for (; j + 1 < m; j += 2) {
                pair_pn_newton(w.nd_mono[j], w.nd_qa[j], w.nd_qb[j], w.nd_tr[j], tx, ty, tz, p.eps2,
                               fx, fy, fz);
                pair_pn_newton(w.nd_mono[j + 1], w.nd_qa[j + 1], w.nd_qb[j + 1], w.nd_tr[j + 1], tx,
                               ty, tz, p.eps2, fx, fy, fz);
            }
            if (j < m)
                pair_pn_newton(w.nd_mono[j], w.nd_qa[j], w.nd_qb[j], w.nd_tr[j], tx, ty, tz, p.eps2,
                               fx, fy, fz);
        } else {
            for (int j = 0; j < m; ++j) {
                const float4 qa = QUAD ? w.nd_qa[j] : make_float4(0, 0, 0, 0);
                const float2 qb = QUAD ? w.nd_qb[j] : make_float2(0, 0);
                pair_pn<SPLIT, QUAD, POT>(w.nd_mono[j], qa, qb, tx, ty, tz, p, inv2rs, fx, fy, fz, fp);
            }
        }
        acc.add(0, fx);
        acc.add(1, fy);
        acc.add(2, fz);
        if (POT)
            acc.add(3, fp);
        __syncwarp();
    }
}

template <bool PERIODIC, bool SPLIT, bool POT>
__device__ __forceinline__ void flush_leaves(WarpSmem& w, int nl, const float4* __restrict__ pos4,
                                             const TreeArrays& t, const WalkParams& p,
                                             float inv2rs, bool cut, float tx, float ty, float tz,
                                             int self_index, Acc& acc, uint32_t& phase, int* err,
                                             const WalkOutputs& o, int pair_row, int& npair,
                                             unsigned& evald)
{
    // pairs closer than rcorr are recorded for the learned correction (pair_row < 0: a lane
    // without a target records nothing)
    const bool rec = o.pair_src != nullptr && p.rcorr2 > 0.0f;
    auto record = [&](float4 s4, int gidx) {
        const float dx = s4.x - tx, dy = s4.y - ty, dz = s4.z - tz;
        if (pair_row >= 0 && fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= p.rcorr2) {
            if (npair < kPairSlots)
                o.pair_src[static_cast<size_t>(pair_row) * kPairSlots + npair] = gidx;
            ++npair;
        }
    };
    const int lane = threadIdx.x & 31;
    // Force-only evaluation above the minimum-distance floor runs the per-lane cutoff filter
    const bool fast = !POT && p.eps2 > p.min_dist2;
    if (cut && !fast) {
        // Drop leaves that no target of this warp can reach: a leaf whose (shifted) box is
        // farther than the cutoff from every lane's target holds no pair inside the cutoff.
        // (With the per-lane filter this costs more than it saves: the filter drops the same
        // sources exactly.)
        // Lane j loads the boxes of list entries j and j + 32 in one round (no serial chain
        // of loads); each box is then broadcast by shuffle and tested against every target.
        float4 lo[2], hi[2];
        bool ppi[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = lane + 32 * h;
            lo[h] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            hi[h] = lo[h];
            ppi[h] = false;
            if (j < nl) {
                const int code = w.lcode[j];
                ppi[h] = PERIODIC && code == kPerPairImage;
                const int k = w.lnode[j];
                const float4 b0 = t.box0[k];
                const float4 b1 = t.box1[k];
                float sxo = 0.0f, syo = 0.0f, szo = 0.0f;
                if (PERIODIC && !ppi[h]) {
                    sxo = shift_of(code, 0, p.box);
                    syo = shift_of(code, 1, p.box);
                    szo = shift_of(code, 2, p.box);
                }
                lo[h] = make_float4(b0.x - sxo, b0.y - syo, b0.z - szo, 0.0f);
                hi[h] = make_float4(b1.x - sxo, b1.y - syo, b1.z - szo, 0.0f);
            }
        }
        const float lim2 = p.rcut2 * 1.0001f;
        int keep = 0;
        for (int j = 0; j < nl; ++j) {
            const int h = j >> 5, src = j & 31;
            const float bx0 = __shfl_sync(kFullMask, h ? lo[1].x : lo[0].x, src);
            const float by0 = __shfl_sync(kFullMask, h ? lo[1].y : lo[0].y, src);
            const float bz0 = __shfl_sync(kFullMask, h ? lo[1].z : lo[0].z, src);
            const float bx1 = __shfl_sync(kFullMask, h ? hi[1].x : hi[0].x, src);
            const float by1 = __shfl_sync(kFullMask, h ? hi[1].y : hi[0].y, src);
            const float bz1 = __shfl_sync(kFullMask, h ? hi[1].z : hi[0].z, src);
            const bool pp = __shfl_sync(kFullMask, h ? ppi[1] : ppi[0], src);
            bool need = true;
            if (!pp) {
                const float ddx = fmaxf(fmaxf(bx0 - tx, tx - bx1), 0.0f);
                const float ddy = fmaxf(fmaxf(by0 - ty, ty - by1), 0.0f);
                const float ddz = fmaxf(fmaxf(bz0 - tz, tz - bz1), 0.0f);
                need = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz)) <= lim2;
            }
            if (__any_sync(kFullMask, need)) {
                if (lane == 0 && keep != j) {
                    w.lstart[keep] = w.lstart[j];
                    w.lcount[keep] = w.lcount[j];
                    w.lcode[keep] = w.lcode[j];
                    w.lnode[keep] = w.lnode[j];
                }
                ++keep;
            }
        }
        __syncwarp();
        nl = keep;
        if (nl == 0)
            return;
    }
    // exclusive prefix of the leaf sizes (list holds at most 64 entries)
    const int c0 = lane < nl ? w.lcount[lane] : 0;
    const int c1 = lane + 32 < nl ? w.lcount[lane + 32] : 0;
    const int i0 = warp_incl_scan(c0);
    const int t0 = __shfl_sync(kFullMask, i0, 31);
    const int i1 = warp_incl_scan(c1) + t0;
    const int total = __shfl_sync(kFullMask, i1, 31);
    if (lane < nl)
        w.lpre[lane] = i0 - c0;
    if (lane + 32 < nl)
        w.lpre[lane + 32] = i1 - c1;
    __syncwarp();
    SplitK sk;
    sk.inv2rs = inv2rs;
    sk.cexp = -1.4426950408889634f * inv2rs * inv2rs;
    sk.pk = 0.3275911f * inv2rs;
    sk.c2 = kTwoOverSqrtPi * inv2rs;
    int jfirst = 0;
    for (int cbase = 0; cbase < total; cbase += kTile) {
        const int cend = min(cbase + kTile, total);
        // make earlier generic-proxy reads of the tile visible before the async writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            mbar_arrive_expect_tx(&w.bar, static_cast<uint32_t>(cend - cbase) * 16u);
        __syncwarp();
        // each lane copies the tile parts of its leaves and notes whether they need a periodic
        // image shift or per-pair images
        bool shifted = false, pairimg = false;
        for (int j = lane; j < nl; j += 32) {
            const int lo = max(w.lpre[j], cbase);
            const int hi = min(w.lpre[j] + w.lcount[j], cend);
            if (hi > lo) {
                bulk_g2s(&w.tile[lo - cbase], pos4 + (w.lstart[j] + (lo - w.lpre[j])),
                         static_cast<uint32_t>(hi - lo) * 16u, &w.bar);
                if (PERIODIC) {
                    const int code = w.lcode[j];
                    pairimg = pairimg || code == kPerPairImage;
                    shifted = shifted || (code != kNoShift && code != kPerPairImage);
                }
                if (rec)
                    for (int q = lo; q < hi; ++q)
                        w.tidx[q - cbase] = w.lstart[j] + (q - w.lpre[j]);
            }
        }
        const bool any_shift = PERIODIC && __any_sync(kFullMask, shifted);
        const bool per_pair = PERIODIC && __any_sync(kFullMask, pairimg);
        if (rec)
            __syncwarp();
        mbar_wait_bounded(&w.bar, phase, err);
        phase ^= 1u;
        // Periodic images: the lane that copied a shifted leaf moves its sources into the
        // group's image in place (leaves summed with per-pair images keep their stored
        // positions).  Tiles without shifted leaves, most of them, skip this.
        if (any_shift) {
            for (int j = lane; j < nl; j += 32) {
                const int lo = max(w.lpre[j], cbase);
                const int hi = min(w.lpre[j] + w.lcount[j], cend);
                const int code = w.lcode[j];
                if (hi <= lo || code == kNoShift || code == kPerPairImage)
                    continue;
                const float shx = shift_of(code, 0, p.box), shy = shift_of(code, 1, p.box),
                            shz = shift_of(code, 2, p.box);
                for (int q = lo; q < hi; ++q) {
                    float4& s4 = w.tile[q - cbase];
                    s4.x = __fsub_rn(s4.x, shx);
                    s4.y = __fsub_rn(s4.y, shy);
                    s4.z = __fsub_rn(s4.z, shz);
                }
            }
            __syncwarp();
        }
        float fx = 0.0f, fy = 0.0f, fz = 0.0f, fp = 0.0f;
        if (fast && cut && !per_pair) {
            // Cutoff filter: each lane marks the tile sources inside its own cutoff sphere
            // (the same r^2 expression as the pair law, so the set is exact), then sums only
            // those.  Skipped pairs contribute exactly zero in the unfiltered sum, so the
            // result is bit-identical to summing every listed source in tile order.
            const int nb = cend - cbase;
            const int nw = (nb + 31) >> 5;
            // r2 <= rcut2 exactly when r2 - next_float(rcut2) is negative (a float difference
            // has the exact sign), so the sign bit is the mask bit: one funnel shift appends it
            const float rc2n = __uint_as_float(__float_as_uint(p.rcut2) + 1u);
            for (int wd = 0; wd < nw; ++wd) {
                const int qb = wd << 5;
                unsigned m = 0u;
                if (qb + 32 <= nb) {
                    // highest source first, shifting the mask left (short loop body)
#pragma unroll 8
                    for (int b = 31; b >= 0; --b) {
                        const float4 s4 = w.tile[qb + b];
                        const float dx = s4.x - tx, dy = s4.y - ty, dz = s4.z - tz;
                        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        m = __funnelshift_l(__float_as_uint(__fsub_rn(r2, rc2n)), m, 1);
                    }
                } else {
                    for (int b = 0; qb + b < nb; ++b) {
                        const float4 s4 = w.tile[qb + b];
                        const float dx = s4.x - tx, dy = s4.y - ty, dz = s4.z - tz;
                        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        if (r2 <= p.rcut2)
                            m |= 1u << b;
                    }
                }
                w.mask[wd][lane] = m;
                evald += __popc(m);
            }
            int wd = 0;
            unsigned m = w.mask[0][lane];
            for (;;) {
                while (m == 0u && ++wd < nw)
                    m = w.mask[wd][lane];
                if (m == 0u)
                    break;
                const int b = __ffs(m) - 1;
                m &= m - 1u;
                const float4 s4 = w.tile[(wd << 5) + b];
                pair_fast<SPLIT>(s4, tx, ty, tz, p.eps2, p.rcut2, false, sk, fx, fy, fz);
                if (rec)
                    record(s4, w.tidx[(wd << 5) + b]);
            }
            __syncwarp();
            // (jfirst, the first leaf the unfiltered path below must look at, is left behind
            // here: that path skips the leaves that end before its tile)
        } else {
            for (int j = jfirst; j < nl; ++j) {
                const int pre = w.lpre[j];
                if (pre >= cend)
                    break;
                const int lo = max(pre, cbase);
                const int hi = min(pre + w.lcount[j], cend);
                if (hi <= lo)
                    continue;
                const int gsrc0 = w.lstart[j] + (lo - pre);
                const int off = lo - cbase;
                const int cntp = hi - lo;
                evald += cntp;  // every listed source goes through the pair law here
                if (PERIODIC && w.lcode[j] == kPerPairImage) {
                    // rare slow path: nearest image chosen per pair
                    const float inv_box = 1.0f / p.box;
                    for (int q = 0; q < cntp; ++q) {
                        float4 s4 = w.tile[off + q];
                        s4.x = tx + (s4.x - tx - p.box * rintf((s4.x - tx) * inv_box));
                        s4.y = ty + (s4.y - ty - p.box * rintf((s4.y - ty) * inv_box));
                        s4.z = tz + (s4.z - tz - p.box * rintf((s4.z - tz) * inv_box));
                        pair_pp<SPLIT, POT>(s4, tx, ty, tz, p, inv2rs, cut,
                                            POT && gsrc0 + q == self_index, fx, fy, fz, fp);
                        if (rec)
                            record(s4, gsrc0 + q);
                    }
                    if (pre + w.lcount[j] <= cend)
                        jfirst = j + 1;
                    continue;
                }
                int q = 0;
                if (fast) {
                    for (; q + 1 < cntp; q += 2) {
                        pair_fast<SPLIT>(w.tile[off + q], tx, ty, tz, p.eps2, p.rcut2, cut, sk, fx, fy, fz);
                        pair_fast<SPLIT>(w.tile[off + q + 1], tx, ty, tz, p.eps2, p.rcut2, cut, sk, fx, fy, fz);
                    }
                    if (q < cntp)
                        pair_fast<SPLIT>(w.tile[off + q], tx, ty, tz, p.eps2, p.rcut2, cut, sk, fx, fy, fz);
                } else {
                    for (; q + 1 < cntp; q += 2) {
                        pair_pp<SPLIT, POT>(w.tile[off + q], tx, ty, tz, p, inv2rs, cut,
                                            POT && gsrc0 + q == self_index, fx, fy, fz, fp);
                        pair_pp<SPLIT, POT>(w.tile[off + q + 1], tx, ty, tz, p, inv2rs, cut,
                                            POT && gsrc0 + q + 1 == self_index, fx, fy, fz, fp);
                    }
                    for (; q < cntp; ++q)
                        pair_pp<SPLIT, POT>(w.tile[off + q], tx, ty, tz, p, inv2rs, cut,
                                            POT && gsrc0 + q == self_index, fx, fy, fz, fp);
                }
                if (rec)
                    for (int q2 = 0; q2 < cntp; ++q2)
                        record(w.tile[off + q2], gsrc0 + q2);
                if (pre + w.lcount[j] <= cend)
                    jfirst = j + 1;
            }
        }
        acc.add(0, fx);
        acc.add(1, fy);
        acc.add(2, fz);
        if (POT)
            acc.add(3, fp);
        __syncwarp();
    }
}

// Persistent kernel: each warp takes groups from a global queue until none are left.  The
// traversal stack lives in shared memory; when it would overflow, its oldest half is spilled
// to a per-warp-slot global area and refilled when the shared part runs dry.
template <bool PERIODIC, bool SPLIT, bool QUAD, bool POT>
__global__ void __launch_bounds__(kWarps * 32) k_walk(const float4* __restrict__ pos4, int n,
                                                       TreeArrays t, const int* __restrict__ gstart,
                                                       const int* __restrict__ groot,
                                                       const int* __restrict__ ngroups_ptr,
                                                       WalkParams p_in, float inv_box,
                                                       WalkOutputs o, unsigned* queue,
                                                       int* spill_base, int* err)
{
    // The isolated TreePM's split scale and cutoff follow its mesh cell, which the device
    // recomputes from the particles' bounds for every evaluation: read them here.
    WalkParams p = p_in;
    if (!PERIODIC && SPLIT && p_in.iso != nullptr) {
        p.rsplit = p_in.iso->rsplit;
        p.rcut2 = p_in.iso->rcut2;
        p.max_node_size = p_in.iso->max_node_size;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpSmem& w = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
    int* spill = spill_base + static_cast<size_t>(blockIdx.x * kWarps + warp) * kSpill;
    const int ngroups = *ngroups_ptr;
    if (lane == 0)
        mbar_init(&w.bar, 1);
    fence_mbar_init();
    __syncwarp();
    const bool cut = p.rcut2 > 0.0f;
    const float inv2rs = SPLIT ? 0.5f / p.rsplit : 0.0f;
    const float rcut = __fsqrt_rn(p.rcut2);
    const float half_box = __fmul_rn(0.5f, p.box);
    const unsigned lt = lanemask_lt();
    uint32_t phase = 0;

    for (;;) {
        int g = 0;
        if (lane == 0)
            g = static_cast<int>(atomicAdd(queue, 1u));
        g = __shfl_sync(kFullMask, g, 0);
        if (g >= ngroups)
            break;
        const int g0 = gstart[g];
        const int gn = gstart[g + 1] - g0;
        const int ti = g0 + lane;
        const bool valid = lane < gn;
        const float4 me = pos4[valid ? ti : g0];
        // adaptive steps: only groups holding a target that closes its step are walked
        if (p.active != nullptr && !__any_sync(kFullMask, valid && p.active[ti] != 0))
            continue;
        float gmin[3] = {me.x, me.y, me.z}, gmax[3] = {me.x, me.y, me.z};
#pragma unroll
        for (int a = 0; a < 3; ++a)
            for (int off = 16; off > 0; off >>= 1) {
                gmin[a] = fminf(gmin[a], __shfl_xor_sync(kFullMask, gmin[a], off));
                gmax[a] = fmaxf(gmax[a], __shfl_xor_sync(kFullMask, gmax[a], off));
            }
        float gc[3], ghalf[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gc[a] = __fmul_rn(0.5f, __fadd_rn(gmin[a], gmax[a]));
            ghalf[a] = __fmul_rn(0.5f, __fsub_rn(gmax[a], gmin[a]));
        }

        if (lane == 0)
            w.stack[0] = groot[g];  // the group's system root (node 0 for a single system)
        __syncwarp();
        int top = 1, gtop = 0, nn = 0, nl = 0, lp = 0;
        unsigned long long cnt_pp = 0, cnt_pn = 0;
        Acc acc;
        acc.zero();
        int npair = 0;
        unsigned evald = 0;  // pairs this lane's target took through the pair law
        bool bail = false;
        while (top > 0 || gtop > 0) {
            if (top == 0) {  // refill from the spill area (uniform branch)
                const int m = min(gtop, kStack / 2);
                for (int i = lane; i < m; i += 32)
                    w.stack[i] = spill[gtop - m + i];
                gtop -= m;
                top = m;
                __syncwarp();
            }
            const int take = min(top, 32);
            const int k = lane < take ? w.stack[top - take + lane] : -1;
            top -= take;
            __syncwarp();
            bool accept = false, leaf = false;
            int nch = 0, link = 0, info = 0, code = 0;
            if (k >= 0) {
                const float4 b0 = t.box0[k];
                const float4 b1 = t.box1[k];
                // the centre of mass matters only to a node that may be accepted; with a node
                // size cap (TreePM) most nodes are too large, and skip the load
                const bool capped = SPLIT && p.max_node_size > 0.0f;  // the cap is a TreePM setting
                float4 mo = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (!capped)
                    mo = t.mono[k];
                link = __float_as_int(b0.w);
                info = __float_as_int(b1.w);
                const float bmin[3] = {b0.x, b0.y, b0.z}, bmax[3] = {b1.x, b1.y, b1.z};
                float sh[3] = {0.0f, 0.0f, 0.0f};
                bool amb = false;
                if (PERIODIC) {
                    // Image-ambiguous node (its extent + the group's + the cutoff reaches half
                    // the box): always opened; a leaf is summed with per-pair minimum images.
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float nh = __fmul_rn(0.5f, __fsub_rn(bmax[a], bmin[a]));
                        if (__fadd_rn(__fadd_rn(ghalf[a], nh), rcut) > half_box)
                            amb = true;
                    }
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float cn = __fmul_rn(0.5f, __fadd_rn(bmin[a], bmax[a]));
                        const float r = rintf(__fmul_rn(__fsub_rn(cn, gc[a]), inv_box));
                        sh[a] = __fmul_rn(p.box, r);
                        code |= (static_cast<int>(r) + 1) << (2 * a);
                    }
                    if (amb)
                        code = kPerPairImage;
                }
                bool pruned = false;
                if (PERIODIC && amb) {
                    if (info < 0)
                        leaf = true;
                    else
                        nch = info;
                } else if (cut) {
                    float d2 = 0.0f;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float lo = __fsub_rn(bmin[a], sh[a]), hi = __fsub_rn(bmax[a], sh[a]);
                        const float d = fmaxf(fmaxf(__fsub_rn(lo, gmax[a]), __fsub_rn(gmin[a], hi)), 0.0f);
                        d2 = __fadd_rn(d2, __fmul_rn(d, d));
                    }
                    pruned = d2 > p.rcut2;
                }
                if (!pruned && !(PERIODIC && amb)) {
                    float l = 0.0f;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        l = fmaxf(l, __fsub_rn(bmax[a], bmin[a]));
                    // The split kernel varies on the scale r_s, so its expansion error depends on
                    // the node size itself, not only on l/d: nodes at least max_node_size large
                    // are never accepted.
                    const bool small = !capped || l < p.max_node_size;
                    if (small) {
                        if (capped)
                            mo = t.mono[k];
                        const float com[3] = {mo.x, mo.y, mo.z};
                        float e2 = 0.0f;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const float c = __fsub_rn(com[a], sh[a]);
                            const float e = fmaxf(fmaxf(__fsub_rn(gmin[a], c), __fsub_rn(c, gmax[a])), 0.0f);
                            e2 = __fadd_rn(e2, __fmul_rn(e, e));
                        }
                        accept = __fmul_rn(l, l) < __fmul_rn(p.theta2, e2);
                    }
                    if (!accept) {
                        if (info < 0)
                            leaf = true;
                        else
                            nch = info;
                    }
                }
            }
            const unsigned am = __ballot_sync(kFullMask, accept);
            const unsigned lm = __ballot_sync(kFullMask, leaf);
            if (accept)
                w.nlist[nn + __popc(am & lt)] = k | (code << kIndexBits);
            if (leaf) {
                const int pos = nl + __popc(lm & lt);
                w.lstart[pos] = link;
                w.lnode[pos] = k;
                w.lcount[pos] = -info;
                w.lcode[pos] = code;
            }
            nn += __popc(am);
            nl += __popc(lm);
            int lsum = leaf ? -info : 0;
            for (int off = 16; off > 0; off >>= 1)
                lsum += __shfl_xor_sync(kFullMask, lsum, off);
            lp += lsum;
            cnt_pp += static_cast<unsigned long long>(lsum);
            cnt_pn += static_cast<unsigned long long>(__popc(am));
            const int incl = warp_incl_scan(nch);
            const int tot = __shfl_sync(kFullMask, incl, 31);
            if (top + tot > kStack) {  // spill the oldest half (uniform branch)
                const int half = kStack / 2;
                if (gtop + half > kSpill) {
                    if (lane == 0)
                        raise_error(err, kErrWalkStack);
                    bail = true;
                    break;
                }
                for (int i = lane; i < half; i += 32)
                    spill[gtop + i] = w.stack[i];
                __syncwarp();
                for (int i = lane; i < top - half; i += 32)
                    w.stack[i] = w.stack[i + half];
                __syncwarp();
                gtop += half;
                top -= half;
            }
            for (int c = 0; c < nch; ++c)
                w.stack[top + incl - nch + c] = link + c;
            top += tot;
            __syncwarp();
            if (nn >= 32) {
                flush_nodes<PERIODIC, SPLIT, QUAD, POT>(w, nn, t, p, inv2rs, me.x, me.y, me.z, acc);
                nn = 0;
            }
            if (nl >= 32 || lp >= kFlushParticles) {
                flush_leaves<PERIODIC, SPLIT, POT>(w, nl, pos4, t, p, inv2rs, cut, me.x, me.y, me.z,
                                                   ti, acc, phase, err, o, valid ? ti : -1, npair,
                                                   evald);
                nl = 0;
                lp = 0;
            }
        }
        if (!bail) {
            if (nn > 0)
                flush_nodes<PERIODIC, SPLIT, QUAD, POT>(w, nn, t, p, inv2rs, me.x, me.y, me.z, acc);
            if (nl > 0)
                flush_leaves<PERIODIC, SPLIT, POT>(w, nl, pos4, t, p, inv2rs, cut, me.x, me.y, me.z,
                                                   ti, acc, phase, err, o, valid ? ti : -1, npair,
                                                   evald);
        }
        if (valid) {
            // the walk's sum is clamped, and so is its sum with a mesh force already in the
            // output (treePmComputeAcceleration, TpmTreeForce.inl:9-25; OctGpu.inl:227)
            float fx = acc.total(0), fy = acc.total(1), fz = acc.total(2);
            clamp_acceleration(fx, fy, fz, p.max_acc);
            fx += o.ax[ti];
            fy += o.ay[ti];
            fz += o.az[ti];
            if (p.clamp_total)
                clamp_acceleration(fx, fy, fz, p.max_acc);
            o.ax[ti] = fx;
            o.ay[ti] = fy;
            o.az[ti] = fz;
            if (POT && o.pot)
                o.pot[ti] += acc.total(3);
            if (o.pair_cnt) {
                o.pair_cnt[ti] = min(npair, kPairSlots);
                if (npair > kPairSlots)
                    raise_error(err, kErrListCapacity);
            }
        }
        const unsigned long long ev = __reduce_add_sync(kFullMask, valid ? evald : 0u);
        if (lane == 0) {
            if (o.n_pp)
                o.n_pp[g] = cnt_pp;
            if (o.n_pn)
                o.n_pn[g] = cnt_pn;
            if (o.totals) {
                const unsigned long long ng = static_cast<unsigned long long>(gn);
                atomicAdd(&o.totals[0], cnt_pp * ng);
                atomicAdd(&o.totals[1], cnt_pn * ng);
                atomicAdd(&o.totals[2], ev);
            }
        }
        __syncwarp();
    }
}

__global__ void k_zero_u32(unsigned* p) { *p = 0u; }

struct WalkLaunch {
    int blocks = 0;
    int sms = 0;
    size_t smem = 0;
};

template <bool PERIODIC, bool SPLIT, bool QUAD, bool POT>
WalkLaunch walk_shape(int n, int blocks_per_sm)
{
    // function attributes and occupancy belong to the device: one cached shape per device
    static WalkLaunch cached[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    WalkLaunch local;
    WalkLaunch& c = (dev >= 0 && dev < kMaxDevices) ? cached[dev] : local;
    if (c.blocks == 0) {
        const size_t smem = sizeof(WarpSmem) * kWarps;
        cudaFuncSetAttribute(k_walk<PERIODIC, SPLIT, QUAD, POT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        int sms = 148, per_sm = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk<PERIODIC, SPLIT, QUAD, POT>,
                                                      kWarps * 32, smem);
        c.smem = smem;
        c.sms = sms;
        c.blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    WalkLaunch l = c;
    if (blocks_per_sm > 0 && l.sms * blocks_per_sm < l.blocks)
        l.blocks = l.sms * blocks_per_sm;
    const int need = (n + kWarps - 1) / kWarps;  // groups <= n
    if (l.blocks > need)
        l.blocks = need < 1 ? 1 : need;
    return l;
}

template <bool PERIODIC, bool SPLIT, bool QUAD, bool POT>
void launch_variant(const float4* pos4, int n, const TreeArrays& t, const GroupTable& g,
                    const WalkParams& p, const WalkOutputs& o, unsigned* queue, int* spill,
                    int* err, cudaStream_t s)
{
    const WalkLaunch l = walk_shape<PERIODIC, SPLIT, QUAD, POT>(n, p.blocks_per_sm);
    const float inv_box = p.box > 0.0f ? 1.0f / p.box : 0.0f;
    count_launch();
    k_zero_u32<<<1, 1, 0, s>>>(queue);
    count_launch();
    k_walk<PERIODIC, SPLIT, QUAD, POT><<<l.blocks, kWarps * 32, l.smem, s>>>(
        pos4, n, t, g.gstart, g.groot, g.ngroups, p, inv_box, o, queue, spill, err);
}

template <bool PERIODIC, bool SPLIT>
void dispatch_qp(const float4* pos4, int n, const TreeArrays& t, const GroupTable& g,
                 const WalkParams& p, const WalkOutputs& o, unsigned* queue, int* spill, int* err,
                 cudaStream_t s)
{
    if (p.quadrupole) {
        if (p.want_pot)
            launch_variant<PERIODIC, SPLIT, true, true>(pos4, n, t, g, p, o, queue, spill, err, s);
        else
            launch_variant<PERIODIC, SPLIT, true, false>(pos4, n, t, g, p, o, queue, spill, err, s);
    } else {
        if (p.want_pot)
            launch_variant<PERIODIC, SPLIT, false, true>(pos4, n, t, g, p, o, queue, spill, err, s);
        else
            launch_variant<PERIODIC, SPLIT, false, false>(pos4, n, t, g, p, o, queue, spill, err, s);
    }
}

// ---- reference formulation: the reference's walk on its one-leaf tree, i.e. a direct sum
// over the Morton-sorted order with the reference pair law (rsqrtf, erfcf, expf), FP32
// accumulation in leaf order, then the acceleration clamp (OctGpu.inl:138-227,
// CudForceKernels.inl:7-89).  One thread per particle in original order.
constexpr int kRefThreads = 256;
__global__ void __launch_bounds__(kRefThreads) k_reference_walk(
    const float4* __restrict__ orig, const float4* __restrict__ sorted,
    const uint32_t* __restrict__ sorted_index, int n, float softening, float min_distance2,
    float split_scale, float cutoff2, float max_acc, float* ax, float* ay, float* az)
{
    __shared__ float4 tile[kRefThreads];
    __shared__ int tile_id[kRefThreads];
    const int i = blockIdx.x * kRefThreads + threadIdx.x;
    const float4 self = i < n ? orig[i] : make_float4(0, 0, 0, 0);
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    const bool cutoff = cutoff2 > 0.0f;
    for (int base = 0; base < n; base += kRefThreads) {
        const int j = base + threadIdx.x;
        if (j < n) {
            tile[threadIdx.x] = sorted[j];
            tile_id[threadIdx.x] = static_cast<int>(sorted_index[j]);
        }
        __syncthreads();
        const int m = min(kRefThreads, n - base);
        if (i < n) {
            for (int q = 0; q < m; ++q) {
                if (tile_id[q] == i)
                    continue;
                const float4 s = tile[q];
                if (cutoff) {
                    const float ddx = self.x - s.x, ddy = self.y - s.y, ddz = self.z - s.z;
                    if (ddx * ddx + ddy * ddy + ddz * ddz > cutoff2)
                        continue;
                }
                const float dx = s.x - self.x, dy = s.y - self.y, dz = s.z - self.z;
                const float d2 = dx * dx + dy * dy + dz * dz + softening * softening;
                if (d2 <= min_distance2)
                    continue;
                const float inv = rsqrtf(d2);
                const float inv3 = inv * inv * inv;
                float wgt = 1.0f;
                if (split_scale > 0.0f) {
                    const float dist = 1.0f / inv;
                    const float arg = 0.5f * dist / split_scale;
                    wgt = erfcf(arg) + dist * 0.5641895835477563f / split_scale * expf(-arg * arg);
                }
                const float f = s.w * inv3 * wgt;
                fx += dx * f;
                fy += dy * f;
                fz += dz * f;
            }
        }
        __syncthreads();
    }
    if (i < n) {
        const float norm = sqrtf(fx * fx + fy * fy + fz * fz);
        if (norm > max_acc && norm > 1e-12f) {
            const float sc = max_acc / norm;
            fx *= sc;
            fy *= sc;
            fz *= sc;
        }
        ax[i] = fx;
        ay[i] = fy;
        az[i] = fz;
    }
}

} // namespace

int walk_spill_slots()
{
    // upper bound on concurrently resident warps of any walk variant
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * (2048 / 32);
}
size_t walk_spill_entries() { return static_cast<size_t>(kSpill); }

void launch_walk(const float4* pos4, int n, const TreeArrays& t, const GroupTable& g,
                 const WalkParams& p, const WalkOutputs& o, unsigned* queue, int* spill, int* err,
                 cudaStream_t s)
{
    const bool periodic = p.box > 0.0f;
    const bool split = p.rsplit > 0.0f;
    if (periodic) {
        if (split)
            dispatch_qp<true, true>(pos4, n, t, g, p, o, queue, spill, err, s);
        else
            dispatch_qp<true, false>(pos4, n, t, g, p, o, queue, spill, err, s);
    } else {
        if (split)
            dispatch_qp<false, true>(pos4, n, t, g, p, o, queue, spill, err, s);
        else
            dispatch_qp<false, false>(pos4, n, t, g, p, o, queue, spill, err, s);
    }
}

void launch_reference_walk(const float4* pos_orig, const float4* pos_sorted,
                           const uint32_t* sorted_index, int n, float softening,
                           float min_distance2, float split_scale, float cutoff2,
                           float max_acceleration, float* ax, float* ay, float* az,
                           cudaStream_t s)
{
    const int blocks = (n + kRefThreads - 1) / kRefThreads;
    count_launch();
    k_reference_walk<<<blocks, kRefThreads, 0, s>>>(pos_orig, pos_sorted, sorted_index, n,
                                                    softening, min_distance2, split_scale,
                                                    cutoff2, max_acceleration, ax, ay, az);
}

} // namespace bz
