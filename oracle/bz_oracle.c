/* oracle/bz_oracle.c -- TEST INFRASTRUCTURE ONLY (see bz_oracle.h).
 *
 * Plain C restatement of the gravity path.  Built with -ffp-contract=off so FP32 and FP64
 * expressions round exactly as written, which the bit-exact gates (keys, topology, walk
 * decisions, node moments) rely on.  Citations are paths inside the reference project.
 */
#include "bz_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static inline float fminf_(float a, float b) { return a < b ? a : b; }
static inline float fmaxf_(float a, float b) { return a > b ? a : b; }

/* ======================================================================================
 * Morton keys
 * ====================================================================================== */

/* FP32 AABB; min/max reductions are order-free, matching the thrust::transform_reduce of
 * engine/physics/octree/cuda/linear/OctBuild.inl:64-72. */
void or_bbox_f32(const float* x, const float* y, const float* z, int64_t n, float out6[6])
{
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i) {
        mn[0] = fminf(mn[0], x[i]);
        mn[1] = fminf(mn[1], y[i]);
        mn[2] = fminf(mn[2], z[i]);
        mx[0] = fmaxf(mx[0], x[i]);
        mx[1] = fmaxf(mx[1], y[i]);
        mx[2] = fmaxf(mx[2], z[i]);
    }
    for (int a = 0; a < 3; ++a) {
        out6[a] = mn[a];
        out6[3 + a] = mx[a];
    }
}

/* The reference's bit spread (engine/physics/octree/morton/OctMortonCodes.inl:7-14): the
 * masks are those of a 10-bit spread applied to a 32-bit word, so only bits 0..9 of the
 * 21-bit coordinate survive and every key fits in 30 bits. */
static uint64_t ref_spread(uint32_t v)
{
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return (uint64_t)v;
}

/* Reference-compatible key: OctKeyKernels.inl:31-45 (FP32 quantisation, round-half-up,
 * clamp to 2^21-1) + mortonEncode63 (OctMortonCodes.inl:16-22, x<<2 | y<<1 | z).
 * fused = 1 evaluates `n * 2097151.0f + 0.5f` as one fused multiply-add, which is how the
 * reference's CUDA kernel executes it under nvcc's default contraction; fused = 0 is the
 * plain host evaluation (the reference's sources compiled for the host). */
void or_morton_ref(const float* x, const float* y, const float* z, int64_t n,
                   const float bbox6[6], int fused, uint64_t* keys)
{
    const float invX = 1.0f / fmaxf(bbox6[3] - bbox6[0], 1.0e-12f);
    const float invY = 1.0f / fmaxf(bbox6[4] - bbox6[1], 1.0e-12f);
    const float invZ = 1.0f / fmaxf(bbox6[5] - bbox6[2], 1.0e-12f);
    for (int64_t i = 0; i < n; ++i) {
        const float nx = fminf(fmaxf((x[i] - bbox6[0]) * invX, 0.0f), 1.0f);
        const float ny = fminf(fmaxf((y[i] - bbox6[1]) * invY, 0.0f), 1.0f);
        const float nz = fminf(fmaxf((z[i] - bbox6[2]) * invZ, 0.0f), 1.0f);
        uint32_t qx = (uint32_t)(fused ? fmaf(nx, 2097151.0f, 0.5f) : nx * 2097151.0f + 0.5f);
        uint32_t qy = (uint32_t)(fused ? fmaf(ny, 2097151.0f, 0.5f) : ny * 2097151.0f + 0.5f);
        uint32_t qz = (uint32_t)(fused ? fmaf(nz, 2097151.0f, 0.5f) : nz * 2097151.0f + 0.5f);
        qx = qx < 2097151u ? qx : 2097151u;
        qy = qy < 2097151u ? qy : 2097151u;
        qz = qz < 2097151u ? qz : 2097151u;
        keys[i] = (ref_spread(qx) << 2) | (ref_spread(qy) << 1) | ref_spread(qz);
    }
}

/* Full 21-bit spread (every third bit of a 63-bit word). */
static uint64_t spread21(uint64_t v)
{
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

/* Production key: FP64 quantisation of the cube [origin, origin+size)^3 into 2^21 cells per
 * axis, floor rounding so that every key prefix is an exact geometric sub-cube, clamped to
 * the cube; interleave x<<2 | y<<1 | z as the reference does. */
void or_morton63(const double* x, const double* y, const double* z, int64_t n,
                 const double origin3[3], double size, uint64_t* keys)
{
    const double scale = 2097152.0 / size;
    for (int64_t i = 0; i < n; ++i) {
        const double p[3] = {x[i], y[i], z[i]};
        uint64_t q[3];
        for (int a = 0; a < 3; ++a) {
            double t = floor((p[a] - origin3[a]) * scale);
            if (!(t >= 0.0))
                t = 0.0;
            if (t > 2097151.0)
                t = 2097151.0;
            q[a] = (uint64_t)t;
        }
        keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    }
}

/* Stable sort permutation by key (LSD radix, 8 bits per pass): the order thrust's
 * sort_by_key / CUB produces for (key, 0..n-1) in OctBuild.inl:96. */
void or_stable_sort_u64(const uint64_t* keys, int64_t n, int32_t* perm)
{
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i)
        perm[i] = (int32_t)i;
    int32_t* src = perm;
    int32_t* dst = tmp;
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = 8 * pass;
        int64_t hist[257];
        memset(hist, 0, sizeof(hist));
        for (int64_t i = 0; i < n; ++i)
            hist[((keys[src[i]] >> shift) & 255u) + 1]++;
        for (int d = 0; d < 256; ++d)
            hist[d + 1] += hist[d];
        for (int64_t i = 0; i < n; ++i) {
            const int d = (int)((keys[src[i]] >> shift) & 255u);
            dst[hist[d]++] = src[i];
        }
        int32_t* t = src;
        src = dst;
        dst = t;
    }
    /* 8 passes: result is back in perm */
    free(tmp);
}

/* ======================================================================================
 * Reference linear octree (engine/physics/octree/cuda/linear/OctBuild.inl:14-248 and the
 * node kernels in OctLeafKernels.inl, OctParentKernels.inl, OctLinkKernels.inl).
 * ====================================================================================== */
typedef struct {
    float cx, cy, cz, half, mass, comx, comy, comz;
    int32_t children[8];
    int32_t leafStart, leafCount, parent, next;
    uint32_t mask;
} ref_node;

static int64_t run_length(const uint64_t* in, int64_t count, uint64_t* outKeys, int32_t* outCounts)
{
    int64_t m = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (i == 0 || in[i] != in[i - 1]) {
            outKeys[m] = in[i];
            outCounts[m] = 0;
            ++m;
        }
        outCounts[m - 1] += 1;
    }
    return m;
}

int64_t or_ref_linear_octree(const float* x, const float* y, const float* z, const float* m,
                             int64_t n, int leaf_capacity, int fused, int64_t node_cap,
                             float* hot8, int32_t* next, int32_t* child_mask,
                             int32_t* first_child, int32_t* leaf_start, int32_t* leaf_count,
                             uint64_t* sorted_keys, int32_t* sorted_index,
                             int32_t* leaf_depth_out)
{
    if (n <= 0)
        return -1;
    const int cap = leaf_capacity > 16 ? leaf_capacity : 16; /* OctBuild.inl:28 */
    int leafDepth = 1;                                       /* OctBuild.inl:30-38 */
    while (leafDepth < 21) {
        const double avg = (double)n / (double)(1ull << (3 * leafDepth));
        if (avg <= (double)cap)
            break;
        ++leafDepth;
    }
    const int shift = 3 * (21 - leafDepth); /* OctBuild.inl:39 */
    if (leaf_depth_out)
        *leaf_depth_out = leafDepth;

    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    float bb[6];
    or_bbox_f32(x, y, z, n, bb);
    or_morton_ref(x, y, z, n, bb, fused, keys);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    or_stable_sort_u64(keys, n, perm);
    for (int64_t i = 0; i < n; ++i) {
        sorted_keys[i] = keys[perm[i]];
        sorted_index[i] = perm[i];
    }

    uint64_t* prefA = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t* prefB = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* levA = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* levB = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i)
        prefA[i] = sorted_keys[i] >> shift; /* OctKeyKernels.inl:57-65 */
    const int64_t leafCount = run_length(prefA, n, prefB, counts);
    int64_t acc = 0;
    for (int64_t i = 0; i < leafCount; ++i) {
        offsets[i] = (int32_t)acc;
        acc += counts[i];
    }
    const int64_t needCap = leafCount * (leafDepth + 1) + 8; /* OctBuild.inl:128 */
    ref_node* nodes = (ref_node*)calloc((size_t)(needCap > 2 ? needCap : 2), sizeof(ref_node));

    /* leaf nodes: tight AABB, FP64 mass/COM (OctLeafKernels.inl:7-81) */
    for (int64_t L = 0; L < leafCount; ++L) {
        float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
        for (int64_t j = offsets[L]; j < offsets[L] + counts[L]; ++j) {
            const int32_t p = sorted_index[j];
            mn[0] = fminf(mn[0], x[p]);
            mn[1] = fminf(mn[1], y[p]);
            mn[2] = fminf(mn[2], z[p]);
            mx[0] = fmaxf(mx[0], x[p]);
            mx[1] = fmaxf(mx[1], y[p]);
            mx[2] = fmaxf(mx[2], z[p]);
            tm += (double)m[p];
            if (fused) {
                wx = fma((double)x[p], (double)m[p], wx);
                wy = fma((double)y[p], (double)m[p], wy);
                wz = fma((double)z[p], (double)m[p], wz);
            } else {
                wx += (double)x[p] * (double)m[p];
                wy += (double)y[p] * (double)m[p];
                wz += (double)z[p] * (double)m[p];
            }
        }
        ref_node* nd = &nodes[L];
        for (int c = 0; c < 8; ++c)
            nd->children[c] = -1;
        nd->cx = 0.5f * (mn[0] + mx[0]);
        nd->cy = 0.5f * (mn[1] + mx[1]);
        nd->cz = 0.5f * (mn[2] + mx[2]);
        {
            const float ext = fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
            nd->half = fused ? fmaf(0.5f, ext, 1.0e-6f) : 0.5f * ext + 1.0e-6f;
        }
        nd->mass = (float)tm;
        if (tm > 0.0) {
            nd->comx = (float)(wx / tm);
            nd->comy = (float)(wy / tm);
            nd->comz = (float)(wz / tm);
        } else {
            nd->comx = nd->cx;
            nd->comy = nd->cy;
            nd->comz = nd->cz;
        }
        nd->leafStart = offsets[L];
        nd->leafCount = counts[L];
        nd->parent = -1;
        nd->next = -1;
        nd->mask = 0;
        levA[L] = (int32_t)L;
    }

    /* level loop (OctBuild.inl:156-199).  As written there, the parent kernel reads the
     * prefixes through `currentPrefixes`, which aliases the buffer reduce_by_key has just
     * refilled with the PARENT prefixes; octant collisions then fall back to the first free
     * slot (OctParentKernels.inl:41-52).  Restated as is. */
    int64_t currentCount = leafCount, nextBase = leafCount, total = leafCount;
    int32_t* cur = levA;
    int32_t* nxt = levB;
    int overflow = 0;
    while (currentCount > 1) {
        for (int64_t i = 0; i < currentCount; ++i)
            prefA[i] = prefB[i] >> 3;
        const int64_t parentCount = run_length(prefA, currentCount, prefB, counts);
        if (nextBase + parentCount > needCap) {
            overflow = 1;
            break;
        }
        acc = 0;
        for (int64_t i = 0; i < parentCount; ++i) {
            offsets[i] = (int32_t)acc;
            acc += counts[i];
        }
        for (int64_t P = 0; P < parentCount; ++P) {
            ref_node nd;
            memset(&nd, 0, sizeof(nd));
            for (int c = 0; c < 8; ++c)
                nd.children[c] = -1;
            nd.parent = -1;
            nd.next = -1;
            float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
            const int32_t nodeIndex = (int32_t)(nextBase + P);
            for (int k = 0; k < counts[P]; ++k) {
                const int32_t slot = offsets[P] + k;
                const int32_t ci = cur[slot];
                int oct = (int)(prefB[slot] & 7u);
                if (nd.children[oct] >= 0) {
                    oct = 0;
                    while (oct < 8 && nd.children[oct] >= 0)
                        ++oct;
                    if (oct >= 8)
                        continue;
                }
                nd.children[oct] = ci;
                nd.mask |= 1u << oct;
                nodes[ci].parent = nodeIndex;
                const ref_node* ch = &nodes[ci];
                mn[0] = fminf(mn[0], ch->cx - ch->half);
                mn[1] = fminf(mn[1], ch->cy - ch->half);
                mn[2] = fminf(mn[2], ch->cz - ch->half);
                mx[0] = fmaxf(mx[0], ch->cx + ch->half);
                mx[1] = fmaxf(mx[1], ch->cy + ch->half);
                mx[2] = fmaxf(mx[2], ch->cz + ch->half);
                tm += (double)ch->mass;
                if (fused) {
                    wx = fma((double)ch->comx, (double)ch->mass, wx);
                    wy = fma((double)ch->comy, (double)ch->mass, wy);
                    wz = fma((double)ch->comz, (double)ch->mass, wz);
                } else {
                    wx += (double)ch->comx * (double)ch->mass;
                    wy += (double)ch->comy * (double)ch->mass;
                    wz += (double)ch->comz * (double)ch->mass;
                }
            }
            if (nd.mask == 0u) {
                mn[0] = mn[1] = mn[2] = mx[0] = mx[1] = mx[2] = 0.0f;
            }
            nd.cx = 0.5f * (mn[0] + mx[0]);
            nd.cy = 0.5f * (mn[1] + mx[1]);
            nd.cz = 0.5f * (mn[2] + mx[2]);
            {
                const float ext = fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
                nd.half = fused ? fmaf(0.5f, ext, 1.0e-6f) : 0.5f * ext + 1.0e-6f;
            }
            nd.mass = (float)tm;
            nd.comx = tm > 0.0 ? (float)(wx / tm) : nd.cx;
            nd.comy = tm > 0.0 ? (float)(wy / tm) : nd.cy;
            nd.comz = tm > 0.0 ? (float)(wz / tm) : nd.cz;
            nd.leafStart = 0;
            nd.leafCount = 0;
            nodes[nodeIndex] = nd;
            nxt[P] = nodeIndex;
        }
        total = nextBase + parentCount;
        nextBase += parentCount;
        currentCount = parentCount;
        int32_t* t = cur;
        cur = nxt;
        nxt = t;
    }
    int64_t result = -1;
    if (!overflow && total <= node_cap) {
        const int32_t root = (int32_t)(total - 1);
        nodes[root].parent = -1;
        nodes[root].next = -1;
        /* next links (OctLinkKernels.inl:7-48) */
        for (int64_t k = 0; k < total; ++k) {
            if (k == root) {
                nodes[k].next = -1;
                continue;
            }
            int32_t nx = -1, c = (int32_t)k, p = nodes[k].parent;
            while (p >= 0) {
                int slot = -1;
                for (int s = 0; s < 8; ++s)
                    if (nodes[p].children[s] == c) {
                        slot = s;
                        break;
                    }
                if (slot >= 0)
                    for (int s = slot + 1; s < 8; ++s)
                        if (nodes[p].children[s] >= 0) {
                            nx = nodes[p].children[s];
                            break;
                        }
                if (nx >= 0)
                    break;
                c = p;
                p = nodes[c].parent;
            }
            nodes[k].next = nx;
        }
        /* pack (OctLinkKernels.inl:61-113) */
        for (int64_t k = 0; k < total; ++k) {
            const ref_node* nd = &nodes[k];
            const float v[8] = {nd->cx, nd->cy, nd->cz, nd->half, nd->mass, nd->comx, nd->comy, nd->comz};
            memcpy(hot8 + 8 * k, v, sizeof(v));
            next[k] = nd->next;
            child_mask[k] = (int32_t)(nd->mask & 0xFFu);
            int32_t fc = -1;
            for (int c = 0; c < 8; ++c)
                if (nd->children[c] >= 0) {
                    fc = nd->children[c];
                    break;
                }
            first_child[k] = fc;
            leaf_start[k] = nd->leafStart;
            leaf_count[k] = nd->leafCount;
        }
        result = total;
    }
    free(keys);
    free(perm);
    free(prefA);
    free(prefB);
    free(counts);
    free(offsets);
    free(levA);
    free(levB);
    free(nodes);
    return result;
}

/* Reference pair law (engine/physics/core/cuda/prelude/CudForceKernels.inl:62-89) in FP64:
 * r^2 = |d|^2 + eps^2, skipped if <= minDistance2, weight erfc(u) + r/(r_s sqrt(pi)) e^{-u^2}
 * with u = r/(2 r_s) when r_s > 0. */
static void ref_pair(const double self[3], const double src[3], double m, double eps2,
                     double min_d2, double rs, double out[3])
{
    const double d[3] = {src[0] - self[0], src[1] - self[1], src[2] - self[2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
    if (r2 <= min_d2) {
        out[0] = out[1] = out[2] = 0.0;
        return;
    }
    const double r = sqrt(r2);
    double w = 1.0;
    if (rs > 0.0) {
        const double u = 0.5 * r / rs;
        w = erfc(u) + r / (rs * sqrt(M_PI)) * exp(-u * u);
    }
    const double s = m * w / (r2 * r);
    out[0] = d[0] * s;
    out[1] = d[1] * s;
    out[2] = d[2] * s;
}

/* Stackless reference walk (engine/physics/octree/cuda/force/OctGpu.inl:100-228) in FP64
 * arithmetic for the pair law; decisions in FP32 as written there. */
void or_ref_walk(const float* x, const float* y, const float* z, const float* m, int64_t n,
                 const float* hot8, const int32_t* next, const int32_t* child_mask,
                 const int32_t* first_child, const int32_t* leaf_start,
                 const int32_t* leaf_count, const int32_t* sorted_index, int32_t root,
                 float theta, float softening, float min_distance2, float max_acceleration,
                 int criterion, float split_scale, float cutoff2, double* acc3)
{
    const double eps2 = (double)softening * (double)softening;
    const int cut = cutoff2 > 0.0f;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        const float sx = x[i], sy = y[i], sz = z[i];
        const double self[3] = {sx, sy, sz};
        double f[3] = {0, 0, 0};
        int iters = 0;
        int32_t node = root;
        while (node >= 0) {
            if (++iters > 8192)
                break;
            const float* h = hot8 + 8 * (int64_t)node;
            const float cx = h[0], cy = h[1], cz = h[2], half = h[3], mass = h[4];
            if (mass <= 0.0f) {
                node = next[node];
                continue;
            }
            const float bdx = fmaxf(fabsf(sx - cx) - half, 0.0f);
            const float bdy = fmaxf(fabsf(sy - cy) - half, 0.0f);
            const float bdz = fmaxf(fabsf(sz - cz) - half, 0.0f);
            const float bd2 = bdx * bdx + bdy * bdy + bdz * bdz;
            const int contains = fabsf(sx - cx) <= half && fabsf(sy - cy) <= half && fabsf(sz - cz) <= half;
            if (cut && bd2 > cutoff2 && !contains) {
                node = next[node];
                continue;
            }
            if (child_mask[node] == 0) {
                for (int32_t k = 0; k < leaf_count[node]; ++k) {
                    const int32_t o = sorted_index[leaf_start[node] + k];
                    if (o == i)
                        continue;
                    if (cut) {
                        const float dx = sx - x[o], dy = sy - y[o], dz = sz - z[o];
                        if (dx * dx + dy * dy + dz * dz > cutoff2)
                            continue;
                    }
                    const double src[3] = {x[o], y[o], z[o]};
                    double a[3];
                    ref_pair(self, src, m[o], eps2, min_distance2, split_scale, a);
                    f[0] += a[0];
                    f[1] += a[1];
                    f[2] += a[2];
                }
                node = next[node];
                continue;
            }
            const float dx = h[5] - sx, dy = h[6] - sy, dz = h[7] - sz;
            const float dist2 = dx * dx + dy * dy + dz * dz + softening * softening;
            const float size = half * 2.0f;
            const float t2 = theta * theta;
            int accept = 0;
            if (!contains) {
                if (criterion == 1) {
                    const float b = fmaxf(bd2, 1.0e-12f);
                    accept = size * size < t2 * b;
                } else {
                    accept = size * size < t2 * dist2;
                }
            }
            if (accept) {
                if (cut && bd2 > cutoff2 && !contains) {
                    node = next[node];
                    continue;
                }
                const double src[3] = {h[5], h[6], h[7]};
                double a[3];
                ref_pair(self, src, mass, eps2, min_distance2, split_scale, a);
                f[0] += a[0];
                f[1] += a[1];
                f[2] += a[2];
                node = next[node];
                continue;
            }
            const int32_t fc = first_child[node];
            node = fc >= 0 ? fc : next[node];
        }
        const double norm = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        if (norm > max_acceleration && norm > 1e-12) {
            const double s = max_acceleration / norm;
            f[0] *= s;
            f[1] *= s;
            f[2] *= s;
        }
        acc3[3 * i] = f[0];
        acc3[3 * i + 1] = f[1];
        acc3[3 * i + 2] = f[2];
    }
}

/* ======================================================================================
 * Production adaptive octree.
 *
 * Nodes in breadth-first order, node 0 = root holding [0, n).  A node with more than
 * leaf_cap particles below max_level is split into its non-empty octant cells (key digit
 * at the next level), appended in parent order then octant order; otherwise it is a leaf.
 * Moments are accumulated in FP64 bottom-up in fixed order (particles of a leaf in sorted
 * order; children in octant order) and rounded once to FP32:
 *   mono4 = {com.x, com.y, com.z, mass}; tight box bmin3/bmax3 (FP32 min/max);
 *   quad6 = sum m (x-com)(x-com)^T about the node's COM {xx, xy, xz, yy, yz, zz}.
 * This is the BFS linear octree the reference builds level by level (OctBuild.inl:156-199)
 * but adaptive (leaf = cell with <= leaf_cap particles, as the CPU octree's kLeafCapacity
 * rule in engine/physics/octree/build/OctreeBuild.cpp:99-104) and top-down.
 * ====================================================================================== */
int64_t or_build_tree(const uint64_t* skeys, const float* pos4, int64_t n, int leaf_cap,
                      int max_level, int64_t node_cap, int32_t* start, int32_t* count,
                      int32_t* child, int32_t* nchild, int32_t* parent, int32_t* level,
                      float* mono4, float* bmin3, float* bmax3, float* quad6)
{
    if (n <= 0 || node_cap < 1)
        return -1;
    int64_t nn = 1;
    start[0] = 0;
    count[0] = (int32_t)n;
    parent[0] = -1;
    level[0] = 0;
    int64_t lb = 0, le = 1;
    for (int l = 0; lb < le; ++l) {
        for (int64_t k = lb; k < le; ++k) {
            child[k] = -1;
            nchild[k] = 0;
            if (count[k] <= leaf_cap || l >= max_level)
                continue;
            const int shift = 3 * (max_level - l - 1);
            const int64_t s = start[k], e = start[k] + count[k];
            child[k] = (int32_t)nn;
            int64_t runStart = s;
            for (int64_t i = s + 1; i <= e; ++i) {
                if (i == e || ((skeys[i] >> shift) & 7u) != ((skeys[i - 1] >> shift) & 7u)) {
                    if (nn >= node_cap)
                        return -1;
                    start[nn] = (int32_t)runStart;
                    count[nn] = (int32_t)(i - runStart);
                    parent[nn] = (int32_t)k;
                    level[nn] = l + 1;
                    ++nn;
                    nchild[k]++;
                    runStart = i;
                }
            }
        }
        lb = le;
        le = nn;
    }
    double* M = (double*)malloc(sizeof(double) * (size_t)nn);
    double* S = (double*)malloc(sizeof(double) * 3 * (size_t)nn);
    double* C = (double*)malloc(sizeof(double) * 3 * (size_t)nn);
    double* Q = (double*)malloc(sizeof(double) * 6 * (size_t)nn);
    for (int64_t k = nn - 1; k >= 0; --k) {
        float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        double tm = 0.0, s[3] = {0, 0, 0}, q[6] = {0, 0, 0, 0, 0, 0}, com[3];
        if (nchild[k] == 0) {
            for (int64_t i = start[k]; i < start[k] + count[k]; ++i) {
                const float* p = pos4 + 4 * i;
                for (int a = 0; a < 3; ++a) {
                    mn[a] = fminf_(mn[a], p[a]);
                    mx[a] = fmaxf_(mx[a], p[a]);
                }
                tm += (double)p[3];
                s[0] += (double)p[3] * (double)p[0];
                s[1] += (double)p[3] * (double)p[1];
                s[2] += (double)p[3] * (double)p[2];
            }
            for (int a = 0; a < 3; ++a)
                com[a] = tm > 0.0 ? s[a] / tm : 0.5 * ((double)mn[a] + (double)mx[a]);
            for (int64_t i = start[k]; i < start[k] + count[k]; ++i) {
                const float* p = pos4 + 4 * i;
                const double dx = (double)p[0] - com[0], dy = (double)p[1] - com[1],
                             dz = (double)p[2] - com[2], w = (double)p[3];
                q[0] += w * dx * dx;
                q[1] += w * dx * dy;
                q[2] += w * dx * dz;
                q[3] += w * dy * dy;
                q[4] += w * dy * dz;
                q[5] += w * dz * dz;
            }
        } else {
            for (int c = child[k]; c < child[k] + nchild[k]; ++c) {
                for (int a = 0; a < 3; ++a) {
                    mn[a] = fminf_(mn[a], bmin3[3 * c + a]);
                    mx[a] = fmaxf_(mx[a], bmax3[3 * c + a]);
                }
                tm += M[c];
                s[0] += S[3 * c];
                s[1] += S[3 * c + 1];
                s[2] += S[3 * c + 2];
            }
            for (int a = 0; a < 3; ++a)
                com[a] = tm > 0.0 ? s[a] / tm : 0.5 * ((double)mn[a] + (double)mx[a]);
            for (int c = child[k]; c < child[k] + nchild[k]; ++c) {
                const double dx = C[3 * c] - com[0], dy = C[3 * c + 1] - com[1],
                             dz = C[3 * c + 2] - com[2], w = M[c];
                q[0] += Q[6 * c] + w * dx * dx;
                q[1] += Q[6 * c + 1] + w * dx * dy;
                q[2] += Q[6 * c + 2] + w * dx * dz;
                q[3] += Q[6 * c + 3] + w * dy * dy;
                q[4] += Q[6 * c + 4] + w * dy * dz;
                q[5] += Q[6 * c + 5] + w * dz * dz;
            }
        }
        M[k] = tm;
        for (int a = 0; a < 3; ++a) {
            S[3 * k + a] = s[a];
            C[3 * k + a] = com[a];
            bmin3[3 * k + a] = mn[a];
            bmax3[3 * k + a] = mx[a];
            mono4[4 * k + a] = (float)com[a];
        }
        mono4[4 * k + 3] = (float)tm;
        for (int j = 0; j < 6; ++j) {
            Q[6 * k + j] = q[j];
            quad6[6 * k + j] = (float)q[j];
        }
    }
    free(M);
    free(S);
    free(C);
    free(Q);
    return nn;
}

/* ======================================================================================
 * Group walk.
 *
 * Targets are processed in groups of prm->group consecutive sorted particles.  For each
 * (group, node) the decisions are evaluated in FP32 exactly as the CUDA walk evaluates them
 * (same operations, same order, no contraction):
 *   shift_a  = box * rintf((0.5*(bmin_a+bmax_a) - 0.5*(gmin_a+gmax_a)) * (1/box))  [periodic]
 *   box distance^2 between the shifted node box and the group box  > rcut2  -> prune
 *   l = max_a(bmax_a - bmin_a); e_a = max(gmin_a - c_a, c_a - gmax_a, 0) for the shifted
 *   COM c; accept as multipole iff l*l < theta2 * |e|^2
 *   otherwise a leaf interacts particle by particle, an internal node is opened.
 * The pair law is the reference's (CudForceKernels.inl:62-89), the multipole adds the
 * quadrupole term of the same softened (and split) kernel.  Accumulation in FP64.
 * ====================================================================================== */
typedef struct {
    const float *pos4, *mono4, *bmin3, *bmax3, *quad6;
    const int32_t *start, *count, *child, *nchild;
    const or_walk_params* prm;
    float gmin[3], gmax[3];
    int64_t g0, g1;
    double* acc; /* per target in group */
    double* pot;
    double* asum; /* optional: per target, sum of |a| over its pair and node terms */
    int64_t pp, pn;
} walk_ctx;

static inline float rn_mul(float a, float b) { return a * b; }

/* Reduced derivatives D1..D3 of the (split) softened kernel at softened distance s. */
static void kernel_derivs(double s2, double rs, double* D0, double* D1, double* D2, double* D3)
{
    const double s = sqrt(s2);
    if (rs <= 0.0) {
        const double ri = 1.0 / s, ri2 = ri * ri;
        *D0 = ri;
        *D1 = ri * ri2;
        *D2 = 3.0 * (*D1) * ri2;
        *D3 = 5.0 * (*D2) * ri2;
        return;
    }
    const double u = 0.5 * s / rs;
    const double e = exp(-u * u);
    const double sp = sqrt(M_PI);
    const double h = erfc(u) + s / (rs * sp) * e;
    const double k = 3.0 * h + s * s * s * e / (2.0 * rs * rs * rs * sp);
    const double l = 5.0 * k + s * s * s * s * s * e / (4.0 * rs * rs * rs * rs * rs * sp);
    *D0 = erfc(u) / s;
    *D1 = h / (s2 * s);
    *D2 = k / (s2 * s2 * s);
    *D3 = l / (s2 * s2 * s2 * s);
}

double or_split_weight(double s, double rsplit)
{
    if (rsplit <= 0.0)
        return 1.0;
    const double u = 0.5 * s / rsplit;
    return erfc(u) + s / (rsplit * sqrt(M_PI)) * exp(-u * u);
}

static void direct_leaf(walk_ctx* w, int32_t k, const float sh[3], int per_pair_image)
{
    const or_walk_params* p = w->prm;
    const int64_t s = w->start[k], e = s + w->count[k];
    w->pp += e - s;
    for (int64_t t = w->g0; t < w->g1; ++t) {
        const float* tp = w->pos4 + 4 * t;
        double* acc = w->acc + 3 * (t - w->g0);
        for (int64_t j = s; j < e; ++j) {
            const float* sp = w->pos4 + 4 * j;
            double d[3];
            for (int a = 0; a < 3; ++a) {
                if (per_pair_image) {
                    d[a] = (double)sp[a] - tp[a];
                    d[a] -= (double)p->box * rint(d[a] / (double)p->box);
                } else {
                    d[a] = (double)sp[a] - sh[a] - tp[a];
                }
            }
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (p->rcut2 > 0.0f && r2 > (double)p->rcut2)
                continue;
            const double s2 = r2 + (double)p->eps2;
            if (s2 <= (double)p->min_dist2)
                continue;
            const double s1 = sqrt(s2);
            const double wgt = or_split_weight(s1, p->rsplit);
            const double f = (double)sp[3] * wgt / (s2 * s1);
            acc[0] += f * d[0];
            acc[1] += f * d[1];
            acc[2] += f * d[2];
            if (w->asum)
                w->asum[t - w->g0] += fabs(f) * sqrt(r2);
            if (w->pot && j != t) {
                const double f0 = p->rsplit > 0.0f ? erfc(0.5 * s1 / p->rsplit) / s1 : 1.0 / s1;
                w->pot[t - w->g0] -= (double)sp[3] * f0;
            }
        }
    }
}

static void walk_node(walk_ctx* w, int32_t k)
{
    const or_walk_params* p = w->prm;
    const float* bmin = w->bmin3 + 3 * (int64_t)k;
    const float* bmax = w->bmax3 + 3 * (int64_t)k;
    const float* mono = w->mono4 + 4 * (int64_t)k;
    float sh[3] = {0.0f, 0.0f, 0.0f};
    if (p->box > 0.0f) {
        /* A node whose extent plus the group's plus the cutoff reaches half the box may hold
         * sources whose nearest image differs across the group: open it, or (leaf) sum it with
         * a per-pair minimum image. */
        const float rc = sqrtf(p->rcut2);
        int amb = 0;
        for (int a = 0; a < 3; ++a) {
            const float gh = 0.5f * (w->gmax[a] - w->gmin[a]);
            const float nh = 0.5f * (bmax[a] - bmin[a]);
            if ((gh + nh) + rc > 0.5f * p->box)
                amb = 1;
        }
        if (amb) {
            if (w->nchild[k] == 0) {
                direct_leaf(w, k, sh, 1);
            } else {
                for (int32_t c = w->child[k]; c < w->child[k] + w->nchild[k]; ++c)
                    walk_node(w, c);
            }
            return;
        }
        const float inv = 1.0f / p->box;
        for (int a = 0; a < 3; ++a) {
            const float cn = 0.5f * (bmin[a] + bmax[a]);
            const float cg = 0.5f * (w->gmin[a] + w->gmax[a]);
            sh[a] = p->box * rintf((cn - cg) * inv);
        }
    }
    if (p->rcut2 > 0.0f) {
        float d2 = 0.0f;
        for (int a = 0; a < 3; ++a) {
            const float lo = bmin[a] - sh[a], hi = bmax[a] - sh[a];
            const float d = fmaxf_(fmaxf_(lo - w->gmax[a], w->gmin[a] - hi), 0.0f);
            d2 = d2 + rn_mul(d, d);
        }
        if (d2 > p->rcut2)
            return;
    }
    float e2 = 0.0f, l = 0.0f;
    for (int a = 0; a < 3; ++a) {
        const float c = mono[a] - sh[a];
        const float e = fmaxf_(fmaxf_(w->gmin[a] - c, c - w->gmax[a]), 0.0f);
        e2 = e2 + rn_mul(e, e);
        l = fmaxf_(l, bmax[a] - bmin[a]);
    }
    /* split kernel: its multipole expansion is governed by the node size relative to r_s as
     * well as by l/d, so nodes larger than max_node_size are never accepted */
    const int accept = rn_mul(l, l) < rn_mul(p->theta2, e2) && (p->max_node_size <= 0.0f || l < p->max_node_size);
    if (accept) {
        w->pn++;
        const double m = mono[3];
        const float* q = w->quad6 + 6 * (int64_t)k;
        for (int64_t t = w->g0; t < w->g1; ++t) {
            const float* tp = w->pos4 + 4 * t;
            const double d[3] = {(double)mono[0] - sh[0] - tp[0], (double)mono[1] - sh[1] - tp[1],
                                 (double)mono[2] - sh[2] - tp[2]};
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const double s2 = r2 + (double)p->eps2;
            if (s2 <= (double)p->min_dist2)
                continue;
            double D0, D1, D2, D3;
            kernel_derivs(s2, p->rsplit, &D0, &D1, &D2, &D3);
            double a[3] = {m * D1 * d[0], m * D1 * d[1], m * D1 * d[2]};
            double phi = -m * D0;
            if (p->quadrupole) {
                const double Qd[3] = {q[0] * d[0] + q[1] * d[1] + q[2] * d[2],
                                      q[1] * d[0] + q[3] * d[1] + q[4] * d[2],
                                      q[2] * d[0] + q[4] * d[1] + q[5] * d[2]};
                const double dQd = d[0] * Qd[0] + d[1] * Qd[1] + d[2] * Qd[2];
                const double tr = (double)q[0] + (double)q[3] + (double)q[5];
                const double c0 = -0.5 * D2 * tr + 0.5 * D3 * dQd;
                for (int ax = 0; ax < 3; ++ax)
                    a[ax] += c0 * d[ax] - D2 * Qd[ax];
                phi += 0.5 * D1 * tr - 0.5 * D2 * dQd;
            }
            double* acc = w->acc + 3 * (t - w->g0);
            acc[0] += a[0];
            acc[1] += a[1];
            acc[2] += a[2];
            if (w->pot)
                w->pot[t - w->g0] += phi;
            if (w->asum)
                w->asum[t - w->g0] += sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        }
        return;
    }
    if (w->nchild[k] == 0) {
        direct_leaf(w, k, sh, 0);
        return;
    }
    for (int32_t c = w->child[k]; c < w->child[k] + w->nchild[k]; ++c)
        walk_node(w, c);
}

/* Target groups cut from the tree (the CUDA rule of blitzar_b200/csrc/bz_groups.cu): a split
 * node packs its children, in order, into runs of at most gmax particles; a child above gmax,
 * or a "sparse" child, is split in turn; a split leaf is cut into chunks of gmax (above gmax)
 * or single particles (sparse).  A node of at most gmax particles is sparse when its tight box
 * is wider than 0.5 x its distance from the root centre of mass (the root never is).  A root
 * with at most gmax particles is one group.  Writes the group starts in sorted order followed
 * by the end sentinel; returns the group count. */
typedef struct {
    const int32_t *start, *count, *child, *nchild;
    const float *bmin3, *bmax3;
    float com[3];
    int32_t gmax;
    int64_t* gstart;
    int64_t ng;
} group_ctx;

static int node_sparse(const group_ctx* g, int32_t k)
{
    if (k == 0)
        return 0;
    const float* lo = g->bmin3 + 3 * (int64_t)k;
    const float* hi = g->bmax3 + 3 * (int64_t)k;
    float e = 0.0f, d2 = 0.0f;
    for (int a = 0; a < 3; ++a) {
        const float ex = hi[a] - lo[a];
        e = ex > e ? ex : e;
    }
    float dd[3];
    for (int a = 0; a < 3; ++a) {
        float v = lo[a] - g->com[a];
        const float w = g->com[a] - hi[a];
        v = w > v ? w : v;
        dd[a] = v > 0.0f ? v : 0.0f;
    }
    d2 = (dd[0] * dd[0] + dd[1] * dd[1]) + dd[2] * dd[2];
    return e > 0.5f * sqrtf(d2);
}

static void groups_visit(group_ctx* g, int32_t k)
{
    if (g->nchild[k] == 0) {
        const int32_t step = g->count[k] > g->gmax ? g->gmax : 1;
        for (int32_t i = 0; i < g->count[k]; i += step)
            g->gstart[g->ng++] = g->start[k] + i;
        return;
    }
    int32_t run = 0;
    for (int32_t c = g->child[k]; c < g->child[k] + g->nchild[k]; ++c) {
        if (g->count[c] > g->gmax || node_sparse(g, c)) {
            run = 0;
            groups_visit(g, c);
            continue;
        }
        if (run == 0 || run + g->count[c] > g->gmax) {
            g->gstart[g->ng++] = g->start[c];
            run = 0;
        }
        run += g->count[c];
    }
}

int64_t or_tree_groups(const int32_t* start, const int32_t* count, const int32_t* child,
                       const int32_t* nchild, const float* bmin3, const float* bmax3,
                       const float* mono4, int32_t gmax, int64_t* gstart)
{
    group_ctx g = {start, count, child, nchild, bmin3, bmax3, {mono4[0], mono4[1], mono4[2]},
                   gmax, gstart, 0};
    if (count[0] <= gmax)
        gstart[g.ng++] = start[0];
    else
        groups_visit(&g, 0);
    gstart[g.ng] = start[0] + count[0];
    return g.ng;
}

/* Group walk.  only (may be NULL): walk just the groups only[0..n_only) (their targets' rows
 * of acc3/pot/asum are written, the others are left untouched); asum (may be NULL): per
 * target, the sum of the magnitudes of its pair and node terms (the scale of the rounding
 * error of an FP32 sum of them). */
void or_walk_ex(const float* pos4, int64_t n, const int32_t* start, const int32_t* count,
                const int32_t* child, const int32_t* nchild, const float* mono4,
                const float* bmin3, const float* bmax3, const float* quad6,
                const or_walk_params* prm, const int64_t* gstart, int64_t ngroups, double* acc3,
                double* pot, int64_t* n_pp, int64_t* n_pn, const int64_t* only, int64_t n_only,
                double* asum)
{
    const int G = prm->group > 0 ? prm->group : 32;
    const int64_t ng = gstart ? ngroups : (n + G - 1) / G;
    const int64_t nw = only ? n_only : ng;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t q = 0; q < nw; ++q) {
        const int64_t g = only ? only[q] : q;
        walk_ctx w;
        memset(&w, 0, sizeof(w));
        w.pos4 = pos4;
        w.mono4 = mono4;
        w.bmin3 = bmin3;
        w.bmax3 = bmax3;
        w.quad6 = quad6;
        w.start = start;
        w.count = count;
        w.child = child;
        w.nchild = nchild;
        w.prm = prm;
        if (gstart) {
            w.g0 = gstart[g];
            w.g1 = gstart[g + 1];
        } else {
            w.g0 = g * G;
            w.g1 = w.g0 + G < n ? w.g0 + G : n;
        }
        for (int a = 0; a < 3; ++a) {
            w.gmin[a] = FLT_MAX;
            w.gmax[a] = -FLT_MAX;
        }
        for (int64_t t = w.g0; t < w.g1; ++t)
            for (int a = 0; a < 3; ++a) {
                w.gmin[a] = fminf_(w.gmin[a], pos4[4 * t + a]);
                w.gmax[a] = fmaxf_(w.gmax[a], pos4[4 * t + a]);
            }
        w.acc = acc3 + 3 * w.g0;
        for (int64_t t = 0; t < 3 * (w.g1 - w.g0); ++t)
            w.acc[t] = 0.0;
        w.pot = pot ? pot + w.g0 : NULL;
        if (w.pot)
            for (int64_t t = 0; t < w.g1 - w.g0; ++t)
                w.pot[t] = 0.0;
        w.asum = asum ? asum + w.g0 : NULL;
        if (w.asum)
            for (int64_t t = 0; t < w.g1 - w.g0; ++t)
                w.asum[t] = 0.0;
        walk_node(&w, 0);
        if (n_pp)
            n_pp[g] = w.pp;
        if (n_pn)
            n_pn[g] = w.pn;
    }
}

void or_walk(const float* pos4, int64_t n, const int32_t* start, const int32_t* count,
             const int32_t* child, const int32_t* nchild, const float* mono4,
             const float* bmin3, const float* bmax3, const float* quad6,
             const or_walk_params* prm, const int64_t* gstart, int64_t ngroups, double* acc3,
             double* pot, int64_t* n_pp, int64_t* n_pn)
{
    or_walk_ex(pos4, n, start, count, child, nchild, mono4, bmin3, bmax3, quad6, prm, gstart,
               ngroups, acc3, pot, n_pp, n_pn, NULL, 0, NULL);
}

/* ======================================================================================
 * Direct sums.
 * ====================================================================================== */

/* FP64 direct sum over all sources for the listed targets (FP32 inputs promoted), the
 * softened law of engine/physics/treepm/model/TpmCpu.cpp:78-116.  box > 0: minimum image;
 * rsplit > 0: short-range split weight; rcut > 0: pairs beyond rcut (unsoftened) skipped.
 * pot (optional): softened potential -sum m f(s), self excluded. */
void or_direct_f64(const float* pos4, int64_t n, const int64_t* targets, int64_t nt,
                   double eps, double box, double rsplit, double rcut, double* acc3,
                   double* pot)
{
    const double eps2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t i = targets ? targets[t] : t;
        const double xi[3] = {pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]};
        double a[3] = {0, 0, 0}, ph = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i)
                continue;
            double d[3];
            for (int c = 0; c < 3; ++c) {
                d[c] = (double)pos4[4 * j + c] - xi[c];
                if (box > 0.0)
                    d[c] -= box * rint(d[c] / box);
            }
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (rcut > 0.0 && r2 > rcut * rcut)
                continue;
            const double s2 = r2 + eps2;
            if (s2 <= 1e-300)
                continue;
            const double s = sqrt(s2);
            const double w = or_split_weight(s, rsplit);
            const double f = (double)pos4[4 * j + 3] * w / (s2 * s);
            a[0] += f * d[0];
            a[1] += f * d[1];
            a[2] += f * d[2];
            ph -= (double)pos4[4 * j + 3] * (rsplit > 0.0 ? erfc(0.5 * s / rsplit) : 1.0) / s;
        }
        acc3[3 * t] = a[0];
        acc3[3 * t + 1] = a[1];
        acc3[3 * t + 2] = a[2];
        if (pot)
            pot[t] = ph;
    }
}

/* Ewald-summed periodic FP64 acceleration (cubic box, G = 1, neutralising background):
 * real space over the minimum image with erfc(alpha r) screening, softened as the engine
 * softens (weight evaluated at s = sqrt(r^2 + eps^2)); reciprocal space over integer
 * vectors |n_i| <= kmax with k = 2 pi n / box:
 *   a_i = sum_j m_j d_ij [erfc(alpha s) + 2 alpha s/sqrt(pi) e^{-alpha^2 s^2}] / s^3
 *       + (4 pi / V) sum_{k != 0} k/k^2 e^{-k^2/(4 alpha^2)} Im[ e^{-i k.x_i} S(k) ],
 *   S(k) = sum_j m_j e^{i k.x_j}. */
void or_ewald_f64(const float* pos4, int64_t n, const int64_t* targets, int64_t nt, double eps,
                  double box, double alpha, int kmax, double* acc3)
{
    const double eps2 = eps * eps;
    const double V = box * box * box;
    const double kf = 2.0 * M_PI / box;
    int nk = 0;
    const int side = 2 * kmax + 1;
    double* kv = (double*)malloc(sizeof(double) * 4 * (size_t)side * side * side);
    for (int a = -kmax; a <= kmax; ++a)
        for (int b = -kmax; b <= kmax; ++b)
            for (int c = -kmax; c <= kmax; ++c) {
                /* half space: one of each +/- pair */
                if (a < 0 || (a == 0 && (b < 0 || (b == 0 && c <= 0))))
                    continue;
                const double k[3] = {kf * a, kf * b, kf * c};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                kv[4 * nk] = k[0];
                kv[4 * nk + 1] = k[1];
                kv[4 * nk + 2] = k[2];
                kv[4 * nk + 3] = 2.0 * (4.0 * M_PI / V) * exp(-k2 / (4.0 * alpha * alpha)) / k2;
                ++nk;
            }
    double* Sre = (double*)calloc((size_t)nk, sizeof(double));
    double* Sim = (double*)calloc((size_t)nk, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int q = 0; q < nk; ++q) {
        double re = 0.0, im = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double ph = kv[4 * q] * pos4[4 * j] + kv[4 * q + 1] * pos4[4 * j + 1] +
                              kv[4 * q + 2] * pos4[4 * j + 2];
            re += pos4[4 * j + 3] * cos(ph);
            im += pos4[4 * j + 3] * sin(ph);
        }
        Sre[q] = re;
        Sim[q] = im;
    }
    const double c2 = 2.0 * alpha / sqrt(M_PI);
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t i = targets ? targets[t] : t;
        const double xi[3] = {pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]};
        double a[3] = {0, 0, 0};
        for (int64_t j = 0; j < n; ++j) {
            if (j == i)
                continue;
            double d[3];
            for (int c = 0; c < 3; ++c) {
                d[c] = (double)pos4[4 * j + c] - xi[c];
                d[c] -= box * rint(d[c] / box);
            }
            const double s2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
            const double s = sqrt(s2);
            const double w = erfc(alpha * s) + c2 * s * exp(-alpha * alpha * s2);
            const double f = (double)pos4[4 * j + 3] * w / (s2 * s);
            a[0] += f * d[0];
            a[1] += f * d[1];
            a[2] += f * d[2];
        }
        for (int q = 0; q < nk; ++q) {
            const double ph = kv[4 * q] * xi[0] + kv[4 * q + 1] * xi[1] + kv[4 * q + 2] * xi[2];
            /* Im[e^{-i k.x} S] = cos(ph) Sim - sin(ph) Sre */
            const double im = cos(ph) * Sim[q] - sin(ph) * Sre[q];
            const double f = kv[4 * q + 3] * im;
            a[0] += f * kv[4 * q];
            a[1] += f * kv[4 * q + 1];
            a[2] += f * kv[4 * q + 2];
        }
        acc3[3 * t] = a[0];
        acc3[3 * t + 1] = a[1];
        acc3[3 * t + 2] = a[2];
    }
    free(kv);
    free(Sre);
    free(Sim);
}

/* ======================================================================================
 * Periodic particle-mesh leg, FP64 (engine/physics/treepm/deposit/TpmAssignment.inl and
 * engine/physics/treepm/field/TpmField.inl driven with a periodic grid of `mesh` cells,
 * origin 0, cell = box/mesh, CIC assignment).
 * ====================================================================================== */
static void fft1d(double* re, double* im, int64_t stride, int size, int inverse)
{
    for (int i = 1, j = 0; i < size; ++i) {
        int bit = size >> 1;
        for (; j & bit; bit >>= 1)
            j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i * stride];
            re[i * stride] = re[j * stride];
            re[j * stride] = t;
            t = im[i * stride];
            im[i * stride] = im[j * stride];
            im[j * stride] = t;
        }
    }
    for (int len = 2; len <= size; len <<= 1) {
        const double ang = (inverse ? 2.0 : -2.0) * M_PI / len;
        for (int off = 0; off < size; off += len)
            for (int i = 0; i < len / 2; ++i) {
                const double wr = cos(ang * i), wi = sin(ang * i);
                const int64_t e = (int64_t)(off + i) * stride, o = (int64_t)(off + i + len / 2) * stride;
                const double orr = re[o] * wr - im[o] * wi, oi = re[o] * wi + im[o] * wr;
                re[o] = re[e] - orr;
                im[o] = im[e] - oi;
                re[e] += orr;
                im[e] += oi;
            }
    }
}

/* 3-D complex FFT over an interleaved (re, im) cube indexed (z*size + y)*size + x, with
 * 1/size^3 on the inverse (the convention of TpmMath.inl:53-118). */
void or_fft3d(double* re_im, int size, int inverse)
{
    const int64_t cells = (int64_t)size * size * size;
    double* re = (double*)malloc(sizeof(double) * (size_t)cells);
    double* im = (double*)malloc(sizeof(double) * (size_t)cells);
    for (int64_t c = 0; c < cells; ++c) {
        re[c] = re_im[2 * c];
        im[c] = re_im[2 * c + 1];
    }
    const int64_t S = size;
#pragma omp parallel for schedule(static)
    for (int64_t zy = 0; zy < S * S; ++zy)
        fft1d(re + zy * S, im + zy * S, 1, size, inverse);
#pragma omp parallel for schedule(static)
    for (int64_t zx = 0; zx < S * S; ++zx) {
        const int64_t z = zx / S, x = zx % S;
        fft1d(re + z * S * S + x, im + z * S * S + x, S, size, inverse);
    }
#pragma omp parallel for schedule(static)
    for (int64_t yx = 0; yx < S * S; ++yx)
        fft1d(re + yx, im + yx, S * S, size, inverse);
    const double sc = inverse ? 1.0 / (double)cells : 1.0;
    for (int64_t c = 0; c < cells; ++c) {
        re_im[2 * c] = re[c] * sc;
        re_im[2 * c + 1] = im[c] * sc;
    }
    free(re);
    free(im);
}

static inline int wrapi(int v, int m)
{
    const int w = v % m;
    return w < 0 ? w + m : w;
}

/* Assignment stencil of order p (2 CIC, 3 TSC, 4 PCS) along one axis: first node index
 * (wrapped) and p weights.  CIC and TSC are the reference's stencils
 * (TpmAssignment.inl:64-117); PCS uses the full support floor(s)-1 .. floor(s)+2 (the
 * reference starts at floor(s+0.5)-1, which drops a node when frac(s) >= 0.5). */
static double tsc_w(double d)
{
    const double a = fabs(d);
    if (a < 0.5)
        return 0.75 - a * a;
    if (a < 1.5)
        return 0.5 * (1.5 - a) * (1.5 - a);
    return 0.0;
}
static double pcs_w(double d)
{
    const double a = fabs(d);
    if (a < 1.0)
        return (4.0 - 6.0 * a * a + 3.0 * a * a * a) / 6.0;
    if (a < 2.0)
        return (2.0 - a) * (2.0 - a) * (2.0 - a) / 6.0;
    return 0.0;
}
/* Derivatives of the assignment kernels with respect to the particle coordinate (cells). */
static double cic_dw(double d) { return fabs(d) < 1.0 ? (d > 0.0 ? -1.0 : 1.0) : 0.0; }
static double tsc_dw(double d)
{
    const double a = fabs(d), sg = d > 0.0 ? 1.0 : -1.0;
    if (a < 0.5)
        return -2.0 * d;
    if (a < 1.5)
        return -sg * (1.5 - a);
    return 0.0;
}
static double pcs_dw(double d)
{
    const double a = fabs(d), sg = d > 0.0 ? 1.0 : -1.0;
    if (a < 1.0)
        return -2.0 * d + 1.5 * d * a;
    if (a < 2.0)
        return -sg * 0.5 * (2.0 - a) * (2.0 - a);
    return 0.0;
}
/* Stencil weights and their derivatives d w / d s (s = coordinate in cells). */
static void stencil_dp(double coord01, double inv_cell, int mesh, int order, int idx[4], double w[4],
                       double dw[4])
{
    const double raw = coord01 * inv_cell;
    const double s = raw - floor(raw / (double)mesh) * (double)mesh;
    if (order == 2) {
        const double fl = floor(s);
        for (int k = 0; k < 2; ++k) {
            idx[k] = wrapi((int)fl + k, mesh);
            const double d = s - (fl + k);
            w[k] = 1.0 - fabs(d);
            dw[k] = cic_dw(d);
        }
    } else if (order == 3) {
        const double c = floor(s + 0.5);
        for (int k = 0; k < 3; ++k) {
            idx[k] = wrapi((int)c - 1 + k, mesh);
            const double d = s - (c - 1.0 + k);
            w[k] = tsc_w(d);
            dw[k] = tsc_dw(d);
        }
    } else {
        const double fl = floor(s);
        for (int k = 0; k < 4; ++k) {
            idx[k] = wrapi((int)fl - 1 + k, mesh);
            const double d = s - (fl - 1.0 + k);
            w[k] = pcs_w(d);
            dw[k] = pcs_dw(d);
        }
    }
}

static void stencil_p(double coord01, double inv_cell, int mesh, int order, int idx[4], double w[4])
{
    const double raw = coord01 * inv_cell;
    const double s = raw - floor(raw / (double)mesh) * (double)mesh;
    if (order == 2) {
        const double fl = floor(s);
        idx[0] = wrapi((int)fl, mesh);
        idx[1] = wrapi((int)fl + 1, mesh);
        w[1] = s - fl;
        w[0] = 1.0 - w[1];
    } else if (order == 3) {
        const double c = floor(s + 0.5);
        for (int k = 0; k < 3; ++k) {
            idx[k] = wrapi((int)c - 1 + k, mesh);
            w[k] = tsc_w(s - (c - 1.0 + k));
        }
    } else {
        const double fl = floor(s);
        for (int k = 0; k < 4; ++k) {
            idx[k] = wrapi((int)fl - 1 + k, mesh);
            w[k] = pcs_w(s - (fl - 1.0 + k));
        }
    }
}

static inline double sinc(double v) { return fabs(v) < 1.0e-5 ? 1.0 : sin(v) / v; }

/* Periodic PM accelerations.  order: 2/3/4; gradient: 0 centred differences of the potential
 * (TpmField.inl:48-89), 1 spectral i k (Nyquist derivative terms zero), 2 analytic
 * differentiation (the potential interpolated with the gradient of the assignment weights;
 * Hockney & Eastwood's "ad" scheme); floor_w: lower bound
 * of the deconvolution window.  density/phi (optional) receive the deposited density and
 * (centred-difference mode) the potential. */
int or_pm_periodic(const float* pos4, int64_t n, int mesh, double box, double rsplit, int order,
                   int gradient, double floor_w, double* acc3, double* density, double* phi)
{
    return or_pm_periodic_at(pos4, n, mesh, box, rsplit, order, gradient, floor_w, NULL, n, acc3,
                             density, phi);
}

/* As or_pm_periodic, interpolating the mesh force only at targets[0..nt) (all particles when
 * targets is NULL); acc3 holds 3 nt values in target order. */
int or_pm_periodic_at(const float* pos4, int64_t n, int mesh, double box, double rsplit,
                      int order, int gradient, double floor_w, const int64_t* targets, int64_t nt,
                      double* acc3, double* density, double* phi)
{
    const int64_t M = mesh, cells = M * M * M;
    const double h = box / (double)mesh, inv = 1.0 / h;
    double* rho = (double*)calloc((size_t)cells, sizeof(double));
    for (int64_t i = 0; i < n; ++i) {
        int ix[4], iy[4], iz[4];
        double wx[4], wy[4], wz[4];
        stencil_p(pos4[4 * i], inv, mesh, order, ix, wx);
        stencil_p(pos4[4 * i + 1], inv, mesh, order, iy, wy);
        stencil_p(pos4[4 * i + 2], inv, mesh, order, iz, wz);
        const double sc = (double)pos4[4 * i + 3] / (h * h * h);
        for (int c = 0; c < order; ++c)
            for (int b = 0; b < order; ++b)
                for (int a = 0; a < order; ++a)
                    rho[(iz[c] * M + iy[b]) * M + ix[a]] += sc * wx[a] * wy[b] * wz[c];
    }
    if (density)
        memcpy(density, rho, sizeof(double) * (size_t)cells);
    double* sp = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
    for (int64_t c = 0; c < cells; ++c) {
        sp[2 * c] = rho[c];
        sp[2 * c + 1] = 0.0;
    }
    or_fft3d(sp, mesh, 0);
    const double ks = 2.0 * M_PI / ((double)M * h);
    for (int64_t z = 0; z < M; ++z)
        for (int64_t y = 0; y < M; ++y)
            for (int64_t x = 0; x < M; ++x) {
                const int64_t sx = x <= M / 2 ? x : x - M, sy = y <= M / 2 ? y : y - M,
                              sz = z <= M / 2 ? z : z - M;
                const double kx = sx * ks, ky = sy * ks, kz = sz * ks;
                const double k2 = kx * kx + ky * ky + kz * kz;
                const int64_t c = (z * M + y) * M + x;
                if (k2 <= 1.0e-12) {
                    sp[2 * c] = sp[2 * c + 1] = 0.0;
                    continue;
                }
                const double s3 = sinc(0.5 * kx * h) * sinc(0.5 * ky * h) * sinc(0.5 * kz * h);
                double W = 1.0;
                for (int i = 0; i < 2 * order; ++i)
                    W *= s3;
                if (W < floor_w)
                    W = floor_w;
                const double f = 4.0 * M_PI * exp(-k2 * rsplit * rsplit) / (k2 * W);
                sp[2 * c] *= f;
                sp[2 * c + 1] *= f;
            }
    double* field[3] = {NULL, NULL, NULL};
    for (int a = 0; a < 3; ++a)
        field[a] = (double*)malloc(sizeof(double) * (size_t)cells);
    if (gradient == 2) {
        /* analytic differentiation: the force is the gradient of the interpolated potential,
         * a = sum_c psi_c grad W(x - x_c), with psi the inverse transform of the (negated)
         * potential spectrum; one inverse transform instead of three */
        double* q = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
        memcpy(q, sp, sizeof(double) * 2 * (size_t)cells);
        or_fft3d(q, mesh, 1);
        double* psi = (double*)malloc(sizeof(double) * (size_t)cells);
        for (int64_t c = 0; c < cells; ++c)
            psi[c] = q[2 * c];
        free(q);
        const int64_t nout = targets ? nt : n;
#pragma omp parallel for schedule(static)
        for (int64_t o = 0; o < nout; ++o) {
            const int64_t i = targets ? targets[o] : o;
            int ix[4], iy[4], iz[4];
            double wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
            stencil_dp(pos4[4 * i], inv, mesh, order, ix, wx, dx);
            stencil_dp(pos4[4 * i + 1], inv, mesh, order, iy, wy, dy);
            stencil_dp(pos4[4 * i + 2], inv, mesh, order, iz, wz, dz);
            double acc[3] = {0, 0, 0};
            for (int c = 0; c < order; ++c)
                for (int b = 0; b < order; ++b)
                    for (int a2 = 0; a2 < order; ++a2) {
                        const double v = psi[(iz[c] * M + iy[b]) * M + ix[a2]];
                        acc[0] += v * dx[a2] * wy[b] * wz[c];
                        acc[1] += v * wx[a2] * dy[b] * wz[c];
                        acc[2] += v * wx[a2] * wy[b] * dz[c];
                    }
            for (int a = 0; a < 3; ++a)
                acc3[3 * o + a] = acc[a] * inv;
        }
        free(psi);
        for (int a = 0; a < 3; ++a)
            free(field[a]);
        free(rho);
        free(sp);
        return 0;
    }
    if (gradient == 0) {
        double* q = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
        memcpy(q, sp, sizeof(double) * 2 * (size_t)cells);
        or_fft3d(q, mesh, 1);
        double* p = (double*)malloc(sizeof(double) * (size_t)cells);
        for (int64_t c = 0; c < cells; ++c)
            p[c] = q[2 * c];
        if (phi)
            memcpy(phi, p, sizeof(double) * (size_t)cells);
        for (int64_t Z = 0; Z < M; ++Z)
            for (int64_t Y = 0; Y < M; ++Y)
                for (int64_t X = 0; X < M; ++X) {
                    const int64_t c = (Z * M + Y) * M + X;
                    field[0][c] = (p[(Z * M + Y) * M + wrapi((int)X + 1, mesh)] - p[(Z * M + Y) * M + wrapi((int)X - 1, mesh)]) * 0.5 * inv;
                    field[1][c] = (p[(Z * M + wrapi((int)Y + 1, mesh)) * M + X] - p[(Z * M + wrapi((int)Y - 1, mesh)) * M + X]) * 0.5 * inv;
                    field[2][c] = (p[(wrapi((int)Z + 1, mesh) * M + Y) * M + X] - p[(wrapi((int)Z - 1, mesh) * M + Y) * M + X]) * 0.5 * inv;
                }
        free(q);
        free(p);
    } else {
        double* q = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
        for (int a = 0; a < 3; ++a) {
            for (int64_t z = 0; z < M; ++z)
                for (int64_t y = 0; y < M; ++y)
                    for (int64_t x = 0; x < M; ++x) {
                        const int64_t idx3[3] = {x, y, z};
                        const int64_t v = idx3[a];
                        const int64_t sv = v == M / 2 ? 0 : (v < M / 2 ? v : v - M);
                        const double k = sv * ks;
                        const int64_t c = (z * M + y) * M + x;
                        q[2 * c] = -k * sp[2 * c + 1];
                        q[2 * c + 1] = k * sp[2 * c];
                    }
            or_fft3d(q, mesh, 1);
            for (int64_t c = 0; c < cells; ++c)
                field[a][c] = q[2 * c];
        }
        free(q);
    }
    const int64_t nout = targets ? nt : n;
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < nout; ++o) {
        const int64_t i = targets ? targets[o] : o;
        int ix[4], iy[4], iz[4];
        double wx[4], wy[4], wz[4];
        stencil_p(pos4[4 * i], inv, mesh, order, ix, wx);
        stencil_p(pos4[4 * i + 1], inv, mesh, order, iy, wy);
        stencil_p(pos4[4 * i + 2], inv, mesh, order, iz, wz);
        double acc[3] = {0, 0, 0};
        for (int c = 0; c < order; ++c)
            for (int b = 0; b < order; ++b)
                for (int q2 = 0; q2 < order; ++q2) {
                    const int64_t cell = (iz[c] * M + iy[b]) * M + ix[q2];
                    const double w = wx[q2] * wy[b] * wz[c];
                    for (int a = 0; a < 3; ++a)
                        acc[a] += w * field[a][cell];
                }
        for (int a = 0; a < 3; ++a)
            acc3[3 * o + a] = acc[a];
    }
    for (int a = 0; a < 3; ++a)
        free(field[a]);
    free(rho);
    free(sp);
    return 0;
}

/* ======================================================================================
 * Isolated (open-boundary) PM of the reference's GPU TreePM: a cubic mesh of 2G cells, the
 * periodic convolution isolated by the empty half of the doubled domain.
 *   grid   : engine/physics/treepm/cuda/deposit/TpmGridBuild.inl:98-171 (FP32 bounds, cell =
 *            max(cell_floor, extent / (G - 2)), extent = max(span x, y, z, softening), origin
 *            centring the mesh on the bounds);
 *   deposit: TpmDeposit.inl:9-61 (scaled coordinate clamped to [0, 2G - 1], nodes
 *            floor(s + 0.5) - 2 .. + 2 clamped, kernel weights of TpmMath.inl:84-108);
 *   solve  : TpmFft.inl:9-54 (phi_k = -4 pi e^{-k^2 r_s^2} rho_k / (k^2 max(W, floor)), W =
 *            prod sinc^{2p}(k h / 2)), TpmFftRuntime.inl (C2R, / cells);
 *   gradient 0: TpmFft.inl:108-141 (a = -(phi[i+1] - phi[i-1]) / 2h, outer cells zero);
 *            1 spectral i k, 2 analytic differentiation (the engine's production options);
 *   sample : TpmMath.inl:110-158 (the deposit's stencil).
 * params8 (may be NULL) receives {cell, origin x, y, z, mesh, r_s (given), extent, 0}. */
static double iso_w(double d, int order)
{
    return order == 2 ? (fabs(d) < 1.0 ? 1.0 - fabs(d) : 0.0) : (order == 3 ? tsc_w(d) : pcs_w(d));
}
static double iso_dw(double d, int order)
{
    return order == 2 ? cic_dw(d) : (order == 3 ? tsc_dw(d) : pcs_dw(d));
}

int or_pm_isolated(const float* pos4, int64_t n, int grid_half, float cell_floor, float softening,
                   double rsplit_cells, int order, int gradient, double floor_w,
                   const int64_t* targets, int64_t nt, double* acc3, double* params8,
                   double* density, double* phi_out)
{
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            mn[a] = fminf_(mn[a], pos4[4 * i + a]);
            mx[a] = fmaxf_(mx[a], pos4[4 * i + a]);
        }
    float extent = softening;
    for (int a = 0; a < 3; ++a)
        extent = fmaxf_(extent, mx[a] - mn[a]);
    const float cell = fmaxf_(cell_floor, extent / (float)(grid_half - 2));
    const int M = 2 * grid_half;
    const float inv = 1.0f / cell;
    const float half_ext = 0.5f * (float)M * cell;
    float origin[3];
    for (int a = 0; a < 3; ++a)
        origin[a] = 0.5f * (mn[a] + mx[a]) - half_ext;
    const double h = cell, rs = rsplit_cells * (double)cell;
    if (params8) {
        params8[0] = cell;
        for (int a = 0; a < 3; ++a)
            params8[1 + a] = origin[a];
        params8[4] = M;
        params8[5] = rs;
        params8[6] = extent;
        params8[7] = 0.0;
    }
    const int64_t MM = M, cells = MM * MM * MM;
    double* rho = (double*)calloc((size_t)cells, sizeof(double));
    const double vinv = 1.0 / (h * h * h);
    for (int64_t i = 0; i < n; ++i) {
        float sc[3];
        int c0[3];
        for (int a = 0; a < 3; ++a) {
            const float s0 = (pos4[4 * i + a] - origin[a]) * inv;
            sc[a] = fminf_(fmaxf_(s0, 0.0f), (float)M - 1.0f);
            int c = (int)floorf(sc[a] + 0.5f);
            c0[a] = c < 0 ? 0 : (c > M - 1 ? M - 1 : c);
        }
        const double md = (double)pos4[4 * i + 3] * vinv;
        for (int dz = -2; dz <= 2; ++dz) {
            const int z = c0[2] + dz < 0 ? 0 : (c0[2] + dz > M - 1 ? M - 1 : c0[2] + dz);
            const double wz = iso_w((double)sc[2] - (double)(c0[2] + dz), order);
            for (int dy = -2; dy <= 2; ++dy) {
                const int y = c0[1] + dy < 0 ? 0 : (c0[1] + dy > M - 1 ? M - 1 : c0[1] + dy);
                const double wy = iso_w((double)sc[1] - (double)(c0[1] + dy), order);
                for (int dx = -2; dx <= 2; ++dx) {
                    const int x = c0[0] + dx < 0 ? 0 : (c0[0] + dx > M - 1 ? M - 1 : c0[0] + dx);
                    const double wx = iso_w((double)sc[0] - (double)(c0[0] + dx), order);
                    rho[(z * MM + y) * MM + x] += md * wx * wy * wz;
                }
            }
        }
    }
    if (density)
        memcpy(density, rho, sizeof(double) * (size_t)cells);
    double* sp = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
    for (int64_t c = 0; c < cells; ++c) {
        sp[2 * c] = rho[c];
        sp[2 * c + 1] = 0.0;
    }
    or_fft3d(sp, M, 0);
    const double ks = 2.0 * M_PI / ((double)M * h);
    for (int64_t z = 0; z < MM; ++z)
        for (int64_t y = 0; y < MM; ++y)
            for (int64_t x = 0; x < MM; ++x) {
                const int64_t sx = x <= MM / 2 ? x : x - MM, sy = y <= MM / 2 ? y : y - MM,
                              sz = z <= MM / 2 ? z : z - MM;
                const double kx = sx * ks, ky = sy * ks, kz = sz * ks;
                const double k2 = kx * kx + ky * ky + kz * kz;
                const int64_t c = (z * MM + y) * MM + x;
                if (k2 <= 1.0e-12) {
                    sp[2 * c] = sp[2 * c + 1] = 0.0;
                    continue;
                }
                const double s3 = sinc(0.5 * kx * h) * sinc(0.5 * ky * h) * sinc(0.5 * kz * h);
                double W = 1.0;
                for (int i = 0; i < 2 * order; ++i)
                    W *= s3;
                if (W < floor_w)
                    W = floor_w;
                /* the physical potential (negative Green function): acceleration = -grad phi */
                const double f = -4.0 * M_PI * exp(-k2 * rs * rs) / (k2 * W);
                sp[2 * c] *= f;
                sp[2 * c + 1] *= f;
            }
    double* phi = (double*)malloc(sizeof(double) * (size_t)cells);
    double* field[3] = {NULL, NULL, NULL};
    {
        double* q = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
        memcpy(q, sp, sizeof(double) * 2 * (size_t)cells);
        or_fft3d(q, M, 1); /* the inverse transform includes the 1/cells */
        for (int64_t c = 0; c < cells; ++c)
            phi[c] = q[2 * c];
        free(q);
    }
    if (phi_out)
        memcpy(phi_out, phi, sizeof(double) * (size_t)cells);
    if (gradient != 2)
        for (int a = 0; a < 3; ++a)
            field[a] = (double*)calloc((size_t)cells, sizeof(double));
    if (gradient == 0) {
        for (int64_t Z = 1; Z < MM - 1; ++Z)
            for (int64_t Y = 1; Y < MM - 1; ++Y)
                for (int64_t X = 1; X < MM - 1; ++X) {
                    const int64_t c = (Z * MM + Y) * MM + X;
                    field[0][c] = -(phi[c + 1] - phi[c - 1]) * 0.5 / h;
                    field[1][c] = -(phi[c + MM] - phi[c - MM]) * 0.5 / h;
                    field[2][c] = -(phi[c + MM * MM] - phi[c - MM * MM]) * 0.5 / h;
                }
    } else if (gradient == 1) {
        double* q = (double*)malloc(sizeof(double) * 2 * (size_t)cells);
        for (int a = 0; a < 3; ++a) {
            for (int64_t z = 0; z < MM; ++z)
                for (int64_t y = 0; y < MM; ++y)
                    for (int64_t x = 0; x < MM; ++x) {
                        const int64_t idx3[3] = {x, y, z};
                        const int64_t v = idx3[a];
                        const int64_t sv = v == MM / 2 ? 0 : (v < MM / 2 ? v : v - MM);
                        const double k = sv * ks;
                        const int64_t c = (z * MM + y) * MM + x;
                        /* a = -i k phi_k */
                        q[2 * c] = k * sp[2 * c + 1];
                        q[2 * c + 1] = -k * sp[2 * c];
                    }
            or_fft3d(q, M, 1);
            for (int64_t c = 0; c < cells; ++c)
                field[a][c] = q[2 * c];
        }
        free(q);
    }
    const int64_t nout = targets ? nt : n;
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < nout; ++o) {
        const int64_t i = targets ? targets[o] : o;
        float sc[3];
        int c0[3];
        for (int a = 0; a < 3; ++a) {
            const float s0 = (pos4[4 * i + a] - origin[a]) * inv;
            sc[a] = fminf_(fmaxf_(s0, 0.0f), (float)M - 1.0f);
            int c = (int)floorf(sc[a] + 0.5f);
            c0[a] = c < 0 ? 0 : (c > M - 1 ? M - 1 : c);
        }
        double acc[3] = {0, 0, 0};
        for (int dz = -2; dz <= 2; ++dz) {
            const int z = c0[2] + dz < 0 ? 0 : (c0[2] + dz > M - 1 ? M - 1 : c0[2] + dz);
            const double dzd = (double)sc[2] - (double)(c0[2] + dz);
            const double wz = iso_w(dzd, order), gz = iso_dw(dzd, order);
            for (int dy = -2; dy <= 2; ++dy) {
                const int y = c0[1] + dy < 0 ? 0 : (c0[1] + dy > M - 1 ? M - 1 : c0[1] + dy);
                const double dyd = (double)sc[1] - (double)(c0[1] + dy);
                const double wy = iso_w(dyd, order), gy = iso_dw(dyd, order);
                for (int dx = -2; dx <= 2; ++dx) {
                    const int x = c0[0] + dx < 0 ? 0 : (c0[0] + dx > M - 1 ? M - 1 : c0[0] + dx);
                    const double dxd = (double)sc[0] - (double)(c0[0] + dx);
                    const double wx = iso_w(dxd, order), gx = iso_dw(dxd, order);
                    const int64_t cc = (z * MM + y) * MM + x;
                    if (gradient == 2) {
                        /* a = -grad phi(x) = -(1/h) sum_c phi_c grad_s W */
                        acc[0] -= phi[cc] * gx * wy * wz / h;
                        acc[1] -= phi[cc] * wx * gy * wz / h;
                        acc[2] -= phi[cc] * wx * wy * gz / h;
                    } else {
                        const double w = wx * wy * wz;
                        for (int a = 0; a < 3; ++a)
                            acc[a] += field[a][cc] * w;
                    }
                }
            }
        }
        for (int a = 0; a < 3; ++a)
            acc3[3 * o + a] = acc[a];
    }
    for (int a = 0; a < 3; ++a)
        free(field[a]);
    free(phi);
    free(rho);
    free(sp);
    return 0;
}

/* ======================================================================================
 * Learned pair correction: the MLP of blitzar_b200/csrc/bz_mlp.cu restated on the CPU with
 * the same BF16 rounding points (features, weights, hidden activations and back-propagated
 * errors are rounded to BF16 before each product; products accumulate in FP64 here, FP32 on
 * the tensor cores).  Parameter block: W1[32][16] (column 15 = b1), W2[32][32], b2[32],
 * W3[3][32], b3[3].
 * ====================================================================================== */

static float bf16_round(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u)
        return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

static void mlp_features(const float* in6, float* f)
{
    f[0] = in6[0];
    f[1] = in6[1];
    f[2] = in6[2];
    for (int a = 0; a < 3; ++a) {
        const double ps = 2.0 * M_PI * (double)in6[3 + a];
        const double pt = 2.0 * M_PI * ((double)in6[3 + a] + (double)in6[a]);
        f[3 + a] = (float)sin(ps);
        f[6 + a] = (float)cos(ps);
        f[9 + a] = (float)sin(pt);
        f[12 + a] = (float)cos(pt);
    }
    f[15] = 1.0f;
    for (int i = 0; i < 16; ++i)
        f[i] = bf16_round(f[i]);
}

static double sigm(double z) { return 1.0 / (1.0 + exp(-z)); }

/* forward of one sample; keeps the intermediate values for the backward pass */
static void mlp_fwd1(const float* p, const float* in6, float* f, double* z1, float* h1, double* z2,
                     float* h2, double* out)
{
    mlp_features(in6, f);
    for (int n = 0; n < 32; ++n) {
        double a = 0.0;
        for (int k = 0; k < 16; ++k)
            a += (double)bf16_round(p[n * 16 + k]) * f[k];
        z1[n] = (float)a;
        h1[n] = bf16_round((float)(z1[n] * sigm(z1[n])));
    }
    for (int n = 0; n < 32; ++n) {
        double a = 0.0;
        for (int k = 0; k < 32; ++k)
            a += (double)bf16_round(p[512 + n * 32 + k]) * h1[k];
        z2[n] = (float)a + p[1536 + n];
        h2[n] = bf16_round((float)(z2[n] * sigm(z2[n])));
    }
    for (int o = 0; o < 3; ++o) {
        double a = 0.0;
        for (int k = 0; k < 32; ++k)
            a += (double)bf16_round(p[1568 + o * 32 + k]) * h2[k];
        out[o] = (float)a + p[1664 + o];
    }
}

void or_mlp_forward(const float* params, const float* x6, int64_t n, float scale, float* out3)
{
    for (int64_t i = 0; i < n; ++i) {
        float f[16], h1[32], h2[32];
        double z1[32], z2[32], out[3];
        mlp_fwd1(params, x6 + 6 * i, f, z1, h1, z2, h2, out);
        for (int o = 0; o < 3; ++o)
            out3[3 * i + o] = (float)(scale * out[o]);
    }
}

/* gradient of (1/n) sum_i |out_i - y_i|^2 with respect to the parameter block */
void or_mlp_grad(const float* params, const float* x6, const float* y3, int64_t n, double* grad,
                 double* loss)
{
    const int np = 1667;
    for (int i = 0; i < np; ++i)
        grad[i] = 0.0;
    double L = 0.0;
    for (int64_t s = 0; s < n; ++s) {
        float f[16], h1[32], h2[32];
        double z1[32], z2[32], out[3];
        mlp_fwd1(params, x6 + 6 * s, f, z1, h1, z2, h2, out);
        float dout[3];
        for (int o = 0; o < 3; ++o) {
            const double e = (float)out[o] - y3[3 * s + o];
            L += e * e;
            dout[o] = bf16_round((float)(2.0 * e / (double)n));
        }
        float dz2[32], dz1[32];
        for (int j = 0; j < 32; ++j) {
            double a = 0.0;
            for (int o = 0; o < 3; ++o)
                a += (double)dout[o] * bf16_round(params[1568 + o * 32 + j]);
            const double sg = sigm(z2[j]);
            dz2[j] = bf16_round((float)((float)a * sg * (1.0 + z2[j] * (1.0 - sg))));
        }
        for (int j = 0; j < 32; ++j) {
            double a = 0.0;
            for (int k = 0; k < 32; ++k)
                a += (double)dz2[k] * bf16_round(params[512 + k * 32 + j]);
            const double sg = sigm(z1[j]);
            dz1[j] = bf16_round((float)((float)a * sg * (1.0 + z1[j] * (1.0 - sg))));
        }
        for (int r = 0; r < 32; ++r) {
            for (int k = 0; k < 16; ++k)
                grad[r * 16 + k] += (double)dz1[r] * f[k];
            for (int k = 0; k < 32; ++k)
                grad[512 + r * 32 + k] += (double)dz2[r] * h1[k];
            grad[1536 + r] += dz2[r];
        }
        for (int o = 0; o < 3; ++o) {
            for (int k = 0; k < 32; ++k)
                grad[1568 + o * 32 + k] += (double)dout[o] * h2[k];
            grad[1664 + o] += dout[o];
        }
    }
    *loss = L / (double)n;
}
