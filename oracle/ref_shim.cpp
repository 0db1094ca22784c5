// oracle/ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (the oracle's "reference" arm).
//
// This translation unit compiles the reference's own source files where they lie
// (include path = the reference's `engine/` directory, passed by oracle/Makefile) and
// exposes them through a small C ABI so that tests, golden-fixture generation and the
// CPU baseline of bench.py can run the reference's arithmetic on the host.  Nothing in
// the product (blitzar_b200/, include/) links or loads this library.
//
// Two kinds of reference code are wired here:
//  * host C++ that the reference compiles for its CPU solvers (octree_cpu: Octree build,
//    traversal and pair force; TreePM CPU templates; FP64 pairwise) -- used unchanged;
//  * CUDA kernel fragments of the reference's GPU linear octree (Morton keys, leaf,
//    parent and link kernels, the stackless walk).  These are plain SIMT code with no
//    warp intrinsics, so they are compiled as host C++ with the CUDA keywords defined
//    away and each "launch" run as a loop that sets threadIdx/blockIdx.  The host-side
//    orchestration of those kernels (engine/physics/octree/cuda/linear/OctBuild.inl:14-248,
//    which uses thrust) is restated below with std:: algorithms, line by line.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <numeric>
#include <optional>
#include <string>
#include <vector>
#include <omp.h>

// ---------------------------------------------------------------- CUDA keyword shims
#define __global__ static inline
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__ __restrict
struct ShimDim3 {
    unsigned x, y, z;
};
static thread_local ShimDim3 blockIdx{0, 0, 0}, threadIdx{0, 0, 0};
static const ShimDim3 blockDim{256, 1, 1};
template <class T> static inline T __ldg(const T* p) { return *p; }
static inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }

// Run a 1-D "launch" of the given body over n threads (blockDim 256, as the reference).
template <class F> static void shimLaunch(int n, F&& body)
{
    for (int i = 0; i < n; ++i) {
        blockIdx.x = static_cast<unsigned>(i / 256);
        threadIdx.x = static_cast<unsigned>(i % 256);
        body();
    }
}
template <class F> static void shimLaunchParallel(int n, F&& body)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        blockIdx.x = static_cast<unsigned>(i / 256);
        threadIdx.x = static_cast<unsigned>(i % 256);
        body();
    }
}

// ---------------------------------------------------------------- reference headers
#include "physics/core/force/PhyForceLawPolicy.hpp"
#include "physics/core/particle/PhyParticle.hpp"
#include "physics/core/particle/PhyParticleHotData.hpp"
#include "physics/core/particle/PhyParticleSoAView.hpp"
#include "physics/core/vector/PhyVector.hpp"
#include "physics/octree/model/Octree.hpp"
#include "physics/treepm/model/TpmCpu.hpp"

// Handle typedefs of engine/physics/core/cuda/prelude/CudConfiguration.inl:73-76.
typedef GpuOctreeNode* OctreeNodeHandle;
typedef const int* IndexConstHandle;
typedef int* IndexHandle;
typedef Vector3* Vector3Handle;

#include "physics/octree/morton/OctMortonCodes.inl"

namespace refgpu {
// The GPU pair law and clamp (engine/physics/core/cuda/prelude/CudForceKernels.inl:7-89),
// host branch (1/sqrtf where the device uses rsqrtf).
#include "physics/core/cuda/prelude/CudForceKernels.inl"
#include "physics/octree/cuda/linear/OctKeyKernels.inl"
#include "physics/octree/cuda/linear/OctLeafKernels.inl"
#include "physics/octree/cuda/linear/OctParentKernels.inl"
#include "physics/octree/cuda/linear/OctLinkKernels.inl"
#include "physics/octree/cuda/force/OctGpu.inl"

// The GPU TreePM's isolated-mesh kernels (deposit, Green, gradient, sampling), run on the host:
// cuFFT's types stand in as plain structs, atomics as plain updates (the shim runs the
// deposit serially), and the transforms are done around the kernels below.
typedef int cufftResult;
constexpr int CUFFT_SUCCESS = 0;
struct cufftComplex {
    float x, y;
};
static inline cufftComplex make_cuFloatComplex(float r, float i) { return cufftComplex{r, i}; }
static inline float atomicAdd(float* p, float v)
{
    const float o = *p;
    *p = o + v;
    return o;
}
static inline unsigned atomicOr(unsigned* p, unsigned v)
{
    const unsigned o = *p;
    *p = o | v;
    return o;
}
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
// The grid parameter block the TreePM kernels take (field list of
// engine/physics/core/cuda/prelude/CudConfiguration.inl:42-60).
struct TreePmGridParams {
    int gridSize;
    int totalCells;
    int assignment;
    int periodic;
    float cellSize;
    float invCellSize;
    float originX;
    float originY;
    float originZ;
    float boundaryMass;
    float boundaryCenterX;
    float boundaryCenterY;
    float boundaryCenterZ;
    float boundarySoftening;
    float shortRangeScale;
    float densityScale;
    float poissonCoefficient;
};
#include "physics/treepm/cuda/field/TpmMath.inl"
#include "physics/treepm/cuda/fft/TpmFft.inl"
#include "physics/treepm/cuda/deposit/TpmDeposit.inl"
} // namespace refgpu

extern "C" {

// ---------------------------------------------------------------- Morton keys
// Reference: bbox = float min/max over positions (OctBuild.inl:64-72, order-free), then
// buildMortonCodesKernel (OctKeyKernels.inl:22-46) with mortonEncode63 (OctMortonCodes.inl).
void ref_morton_keys(const float* px, const float* py, const float* pz, int n,
                     unsigned long long* keys, int* indices, float* bboxOut6)
{
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < n; ++i) {
        mn[0] = fminf(mn[0], px[i]);
        mn[1] = fminf(mn[1], py[i]);
        mn[2] = fminf(mn[2], pz[i]);
        mx[0] = fmaxf(mx[0], px[i]);
        mx[1] = fmaxf(mx[1], py[i]);
        mx[2] = fmaxf(mx[2], pz[i]);
    }
    ParticleSoAView view{};
    view.posX = const_cast<float*>(px);
    view.posY = const_cast<float*>(py);
    view.posZ = const_cast<float*>(pz);
    view.count = n;
    shimLaunch(n, [&] {
        refgpu::buildMortonCodesKernel(view, n, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], keys,
                                       indices);
    });
    for (int a = 0; a < 3; ++a) {
        bboxOut6[a] = mn[a];
        bboxOut6[3 + a] = mx[a];
    }
}

// ---------------------------------------------------------------- linear octree
// Host orchestration of engine/physics/octree/cuda/linear/OctBuild.inl:14-248 restated with
// std:: algorithms (thrust::sort_by_key -> std::stable_sort on (key, index); reduce_by_key
// -> run-length encode; exclusive_scan -> std::exclusive_scan).  Node kernels are the
// reference's own, run on the host.
//
// Outputs (caller-allocated, capacity nodeCap): hot[8*k] = {cx,cy,cz,half,mass,comx,comy,comz},
// next[k], childMask[k], firstChild[k], leafStart[k], leafCount[k]; sortedKeys[n],
// sortedIndex[n].  Returns node count (root = count-1), or -1 on capacity overflow.
int ref_linear_octree(const float* px, const float* py, const float* pz, const float* mass, int n,
                      int leafCapacityIn, int nodeCap, float* hot, int* next, int* childMask,
                      int* firstChild, int* leafStart, int* leafCount,
                      unsigned long long* sortedKeys, int* sortedIndex, int* leafDepthOut)
{
    if (n <= 0)
        return -1;
    std::vector<float> vx(px, px + n), vy(py, py + n), vz(pz, pz + n), vm(mass, mass + n);
    std::vector<float> zeros(n, 0.0f);
    ParticleSoAView view{};
    view.posX = vx.data();
    view.posY = vy.data();
    view.posZ = vz.data();
    view.mass = vm.data();
    view.velX = zeros.data();
    view.velY = zeros.data();
    view.velZ = zeros.data();
    view.count = n;

    const int leafCapacity = std::max(16, leafCapacityIn);  // OctBuild.inl:28
    int leafDepth = 1;                                      // OctBuild.inl:30-38
    while (leafDepth < 21) {
        const double avg = static_cast<double>(n) / static_cast<double>(1ull << (3 * leafDepth));
        if (avg <= static_cast<double>(leafCapacity))
            break;
        ++leafDepth;
    }
    const int leafShiftBits = 3 * (21 - leafDepth);  // OctBuild.inl:39
    if (leafDepthOut)
        *leafDepthOut = leafDepth;

    std::vector<unsigned long long> keys(n);
    std::vector<int> idx(n);
    float bbox[6];
    ref_morton_keys(px, py, pz, n, keys.data(), idx.data(), bbox);

    // thrust::sort_by_key (OctBuild.inl:96); CUB radix sort is stable.
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return keys[a] < keys[b]; });
    std::vector<unsigned long long> sk(n);
    std::vector<int> si(n);
    for (int i = 0; i < n; ++i) {
        sk[i] = keys[order[i]];
        si[i] = idx[order[i]];
    }
    for (int i = 0; i < n; ++i) {
        sortedKeys[i] = sk[i];
        sortedIndex[i] = si[i];
    }

    // Leaf prefixes + reduce_by_key + exclusive_scan (OctBuild.inl:109-124).
    std::vector<unsigned long long> prefA(n), prefB(n);
    shimLaunch(n, [&] { refgpu::buildLeafPrefixesKernel(sk.data(), n, leafShiftBits, prefA.data()); });
    auto reduceByKey = [](const std::vector<unsigned long long>& in, int count,
                          std::vector<unsigned long long>& outKeys, std::vector<int>& outCounts) {
        int m = 0;
        for (int i = 0; i < count; ++i) {
            if (i == 0 || in[i] != in[i - 1]) {
                outKeys[m] = in[i];
                outCounts[m] = 0;
                ++m;
            }
            outCounts[m - 1] += 1;
        }
        return m;
    };
    std::vector<int> counts(n), offsets(n);
    const int leafCount0 = reduceByKey(prefA, n, prefB, counts);
    std::exclusive_scan(counts.begin(), counts.begin() + leafCount0, offsets.begin(), 0);

    const int requiredNodeCapacity = std::max(2, leafCount0 * (leafDepth + 1) + 8);  // :128
    std::vector<GpuOctreeNode> nodes(static_cast<size_t>(requiredNodeCapacity));
    shimLaunch(leafCount0, [&] {
        refgpu::buildLinearOctreeLeafNodesKernel(nodes.data(), si.data(), offsets.data(),
                                                 counts.data(), view, leafCount0);
    });
    std::vector<int> levelA(n), levelB(n);
    shimLaunch(leafCount0, [&] { refgpu::initLevelIndicesKernel(levelA.data(), leafCount0); });

    // Level loop (OctBuild.inl:156-199).  currentPrefixes aliases prefixesB, exactly as there.
    int currentCount = leafCount0;
    int nextNodeBase = leafCount0;
    int totalNodeCount = leafCount0;
    std::vector<int>* cur = &levelA;
    std::vector<int>* nxt = &levelB;
    while (currentCount > 1) {
        shimLaunch(currentCount, [&] {
            refgpu::buildParentPrefixesKernel(prefB.data(), currentCount, prefA.data());
        });
        const int parentCount = reduceByKey(prefA, currentCount, prefB, counts);
        if (nextNodeBase + parentCount > requiredNodeCapacity)
            return -1;
        std::exclusive_scan(counts.begin(), counts.begin() + parentCount, offsets.begin(), 0);
        // prefB now holds the parent prefixes, but the parent kernel reads the *child*
        // prefixes: OctBuild.inl passes currentPrefixes (== prefixesB) which reduce_by_key has
        // just overwritten with parent prefixes -- reproduced as written.
        shimLaunch(parentCount, [&] {
            refgpu::buildLinearOctreeParentNodesKernel8(nodes.data(), cur->data(), prefB.data(),
                                                        offsets.data(), counts.data(), parentCount,
                                                        nextNodeBase, nxt->data());
        });
        totalNodeCount = nextNodeBase + parentCount;
        nextNodeBase += parentCount;
        currentCount = parentCount;
        std::swap(cur, nxt);
    }
    const int root = totalNodeCount - 1;
    shimLaunch(1, [&] { refgpu::setLinearOctreeRootLinksKernel(nodes.data(), root); });
    shimLaunch(totalNodeCount, [&] {
        refgpu::buildLinearOctreeNextLinksKernel(nodes.data(), totalNodeCount, root);
    });
    if (totalNodeCount > nodeCap)
        return -1;
    std::vector<GpuOctreeNodeHotData> h(totalNodeCount);
    std::vector<GpuOctreeNodeNavData> nv(totalNodeCount);
    shimLaunch(totalNodeCount, [&] {
        refgpu::packLinearOctreeCompactKernel(nodes.data(), totalNodeCount, h.data(), nv.data(),
                                              firstChild, leafStart, leafCount);
    });
    for (int k = 0; k < totalNodeCount; ++k) {
        const float v[8] = {h[k].centerX, h[k].centerY, h[k].centerZ, h[k].halfSize,
                            h[k].mass,    h[k].comX,    h[k].comY,    h[k].comZ};
        std::memcpy(hot + 8 * k, v, sizeof(v));
        next[k] = nv[k].nextIndex;
        childMask[k] = nv[k].childMask;
    }
    return totalNodeCount;
}

// The reference GPU walk (OctGpu.inl:100-245) on the tree above, all particles, original
// order.  treePmShortRangeScale / cutoffSquared select the TreePM short-range variant.
// Returns 0, or -1 when the tree capacity is exceeded.
int ref_octree_gpu_accel(const float* px, const float* py, const float* pz, const float* mass,
                         int n, int leafCapacity, float theta, float softening,
                         float minDistance2, float maxAcceleration, int openingCriterion,
                         float shortRangeScale, float cutoffSquared, float* ax, float* ay,
                         float* az, int* nodeCountOut)
{
    const int cap = std::max(64, 8 * n + 64);
    std::vector<float> hot(8 * static_cast<size_t>(cap));
    std::vector<int> next(cap), mask(cap), first(cap), lstart(cap), lcount(cap);
    std::vector<unsigned long long> sk(n);
    std::vector<int> si(n);
    int depth = 0;
    const int nodes = ref_linear_octree(px, py, pz, mass, n, leafCapacity, cap, hot.data(),
                                        next.data(), mask.data(), first.data(), lstart.data(),
                                        lcount.data(), sk.data(), si.data(), &depth);
    if (nodes <= 0)
        return -1;
    if (nodeCountOut)
        *nodeCountOut = nodes;
    std::vector<GpuOctreeNodeHotData> h(nodes);
    std::vector<GpuOctreeNodeNavData> nv(nodes);
    for (int k = 0; k < nodes; ++k) {
        std::memcpy(&h[k], &hot[8 * static_cast<size_t>(k)], 8 * sizeof(float));
        nv[k].nextIndex = next[k];
        nv[k].childMask = static_cast<std::uint8_t>(mask[k]);
    }
    std::vector<float> vx(px, px + n), vy(py, py + n), vz(pz, pz + n), vm(mass, mass + n);
    ParticleSoAView view{};
    view.posX = vx.data();
    view.posY = vy.data();
    view.posZ = vz.data();
    view.mass = vm.data();
    view.count = n;
    ForceLawPolicy law = resolveForceLawPolicy(theta, softening, 0.0f, minDistance2, 0.0f);
    law.treePmShortRangeScale = shortRangeScale;
    std::vector<Vector3> out(n);
    shimLaunchParallel(n, [&] {
        refgpu::computeOctreeAccelerationKernel(view, out.data(), n, h.data(), nv.data(),
                                                first.data(), lstart.data(), lcount.data(),
                                                nodes - 1, si.data(), law, maxAcceleration,
                                                openingCriterion, cutoffSquared);
    });
    for (int i = 0; i < n; ++i) {
        ax[i] = out[i].x;
        ay[i] = out[i].y;
        az[i] = out[i].z;
    }
    return 0;
}

// ---------------------------------------------------------------- octree_cpu
// The CPU-only build's octree_cpu force evaluation: Octree::build on ParticleHotData
// (octree/build/OctreeBuild.cpp) + Octree::computeForceOn per particle, OpenMP over
// targets (octree/force/OctForces.cpp dispatch), clamp by maxAcceleration.
// cutoffSquared/shortRangeScale > 0 select the TreePM short-range variant.
// Returns the node count.
// A built octree_cpu tree kept between calls, so that a caller can time the build once and
// the walk over many target chunks (the bench's CPU baseline).
struct RefOctreeCpu {
    std::vector<ParticleHotData> hot;
    Octree tree;
    ForceLawPolicy law;
    OctreeOpeningCriterion crit;
    float maxAcceleration;
    float cutoffSquared;
};

void* ref_octree_cpu_build(const float* px, const float* py, const float* pz, const float* mass,
                           int n, float theta, float softening, float minDistance2,
                           float maxAcceleration, int boundsCriterion, float shortRangeScale,
                           float cutoffSquared)
{
    auto* t = new RefOctreeCpu();
    t->hot.resize(n);
    for (int i = 0; i < n; ++i)
        t->hot[i] = ParticleHotData(px[i], py[i], pz[i], mass[i]);
    t->tree.build(t->hot);
    t->law = resolveForceLawPolicy(theta, softening, 0.0f, minDistance2, 0.0f);
    t->law.treePmShortRangeScale = shortRangeScale;
    t->crit = boundsCriterion ? OctreeOpeningCriterion::Bounds : OctreeOpeningCriterion::CenterOfMass;
    t->maxAcceleration = maxAcceleration;
    t->cutoffSquared = cutoffSquared;
    return t;
}

// Forces on the listed targets (all particles when targets is NULL), clamped by
// maxAcceleration as OctForces.cpp:128-132 does.
void ref_octree_cpu_walk(void* handle, const int* targets, int nTargets, float* ax, float* ay,
                         float* az)
{
    auto* t = static_cast<RefOctreeCpu*>(handle);
    const int count = targets ? nTargets : static_cast<int>(t->hot.size());
#pragma omp parallel for schedule(dynamic, 64)
    for (int k = 0; k < count; ++k) {
        const int i = targets ? targets[k] : k;
        Vector3 a = t->tree.computeForceOn(t->hot, static_cast<size_t>(i), t->law, t->crit,
                                           t->cutoffSquared);
        const float norm = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        if (norm > t->maxAcceleration && norm > 1e-12f)
            a = a * (t->maxAcceleration / norm);
        ax[k] = a.x;
        ay[k] = a.y;
        az[k] = a.z;
    }
}

int ref_octree_cpu_nodes(void* handle)
{
    return static_cast<int>(static_cast<RefOctreeCpu*>(handle)->tree.getNodeCount());
}

void ref_octree_cpu_free(void* handle) { delete static_cast<RefOctreeCpu*>(handle); }

int ref_octree_cpu_accel(const float* px, const float* py, const float* pz, const float* mass,
                         int n, float theta, float softening, float minDistance2,
                         float maxAcceleration, int boundsCriterion, float shortRangeScale,
                         float cutoffSquared, const int* targets, int nTargets, float* ax,
                         float* ay, float* az)
{
    void* t = ref_octree_cpu_build(px, py, pz, mass, n, theta, softening, minDistance2,
                                   maxAcceleration, boundsCriterion, shortRangeScale, cutoffSquared);
    ref_octree_cpu_walk(t, targets, nTargets, ax, ay, az);
    const int nodes = ref_octree_cpu_nodes(t);
    ref_octree_cpu_free(t);
    return nodes;
}

// ---------------------------------------------------------------- TreePM CPU templates
// computeCpuFp64PairwiseForces (treepm/model/TpmCpu.cpp:78-116).
int ref_fp64_pairwise(const float* px, const float* py, const float* pz, const float* mass, int n,
                      float softening, float minDistance2, float* ax, float* ay, float* az)
{
    std::vector<Particle> ps(n);
    for (int i = 0; i < n; ++i) {
        ps[i].setPosition(Vector3(px[i], py[i], pz[i]));
        ps[i].setMass(mass[i]);
    }
    ForceLawPolicy law = resolveForceLawPolicy(0.5f, softening, 0.0f, minDistance2, 0.0f);
    std::vector<Vector3> f;
    if (!computeCpuFp64PairwiseForces(ps, law, f))
        return -1;
    for (int i = 0; i < n; ++i) {
        ax[i] = f[i].x;
        ay[i] = f[i].y;
        az[i] = f[i].z;
    }
    return 0;
}

} // extern "C"

// The CPU TreePM field templates compiled the way TpmCpu.cpp:14-28 compiles them.
namespace refpm {
#include "physics/treepm/field/TpmMath.inl"
#include "physics/treepm/deposit/TpmAssignment.inl"
#include "physics/treepm/field/TpmField.inl"
#include "physics/treepm/short_range/TpmShortRange.inl"

template <typename Scalar>
static int meshForces(const float* px, const float* py, const float* pz, const float* mass, int n,
                      int gridSize, Scalar boxLength, Scalar shortRangeScale, const char* assign,
                      float* ax, float* ay, float* az, Scalar* densityOut, Scalar* fieldOut)
{
    Grid<Scalar> grid;
    grid.size = gridSize;
    grid.periodic = true;
    grid.cellSize = boxLength / static_cast<Scalar>(gridSize);
    grid.inverseCellSize = static_cast<Scalar>(1.0) / grid.cellSize;
    CpuTreePmWorkspaceT<Scalar> ws;
    const size_t cells = static_cast<size_t>(gridSize) * gridSize * gridSize;
    ws.density.assign(cells, static_cast<Scalar>(0.0));
    const std::string_view assignment(assign);
    for (int i = 0; i < n; ++i) {
        Particle p;
        p.setPosition(Vector3(px[i], py[i], pz[i]));
        p.setMass(mass[i]);
        depositParticle(p, grid, ws.density, assignment);
    }
    if (densityOut)
        std::copy(ws.density.begin(), ws.density.end(), densityOut);
    buildFftFields<Scalar>(grid, shortRangeScale, kFourPi<Scalar>, assignment, ws);
    if (fieldOut) {
        for (size_t c = 0; c < cells; ++c) {
            fieldOut[3 * c + 0] = ws.fieldX[c];
            fieldOut[3 * c + 1] = ws.fieldY[c];
            fieldOut[3 * c + 2] = ws.fieldZ[c];
        }
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const Vector3 pos(px[i], py[i], pz[i]);
        ax[i] = static_cast<float>(sample(ws.fieldX, grid, pos, assignment));
        ay[i] = static_cast<float>(sample(ws.fieldY, grid, pos, assignment));
        az[i] = static_cast<float>(sample(ws.fieldZ, grid, pos, assignment));
    }
    return 0;
}
} // namespace refpm

extern "C" {
// Periodic mesh (long-range) accelerations from the reference CPU TreePM templates driven
// with explicit parameters (deposit TpmAssignment.inl:160-199, Green/FFT/gradient
// TpmField.inl:6-89, sample TpmAssignment.inl:120-158).  fp64 selects the double template.
int ref_pm_periodic(const float* px, const float* py, const float* pz, const float* mass, int n,
                    int gridSize, double boxLength, double shortRangeScale, int fp64,
                    const char* assignment, float* ax, float* ay, float* az, double* densityOut,
                    double* fieldOut)
{
    if (fp64)
        return refpm::meshForces<double>(px, py, pz, mass, n, gridSize, boxLength,
                                         shortRangeScale, assignment, ax, ay, az, densityOut,
                                         fieldOut);
    const size_t cells = static_cast<size_t>(gridSize) * gridSize * gridSize;
    std::vector<float> d(densityOut ? cells : 0), f(fieldOut ? 3 * cells : 0);
    const int rc = refpm::meshForces<float>(px, py, pz, mass, n, gridSize,
                                            static_cast<float>(boxLength),
                                            static_cast<float>(shortRangeScale), assignment, ax,
                                            ay, az, densityOut ? d.data() : nullptr,
                                            fieldOut ? f.data() : nullptr);
    if (densityOut)
        std::copy(d.begin(), d.end(), densityOut);
    if (fieldOut)
        std::copy(f.begin(), f.end(), fieldOut);
    return rc;
}

// The reference CPU FFT (TpmMath.inl:53-118) on a complex cube, for pinning the oracle's FFT.
void ref_fft3d(double* reIm, int size, int inverse)
{
    const size_t cells = static_cast<size_t>(size) * size * size;
    std::vector<std::complex<double>> v(cells);
    for (size_t c = 0; c < cells; ++c)
        v[c] = std::complex<double>(reIm[2 * c], reIm[2 * c + 1]);
    refpm::fft3d<double>(v, size, inverse != 0);
    for (size_t c = 0; c < cells; ++c) {
        reIm[2 * c] = v[c].real();
        reIm[2 * c + 1] = v[c].imag();
    }
}

// TreePM short-range pair law of the CPU templates (TpmShortRange.inl:6-33), FP64 Scalar.
void ref_short_range_pair(const float* self3, const float* src3, float srcMass, float softening,
                          float minDistance2, float shortRangeScale, float* out3)
{
    Particle src;
    src.setPosition(Vector3(src3[0], src3[1], src3[2]));
    src.setMass(srcMass);
    ForceLawPolicy law = resolveForceLawPolicy(0.5f, softening, 0.0f, minDistance2, 0.0f);
    law.treePmShortRangeScale = shortRangeScale;
    const Vector3 a =
        refpm::sourceAcceleration<double>(Vector3(self3[0], self3[1], self3[2]), src, law);
    out3[0] = a.x;
    out3[1] = a.y;
    out3[2] = a.z;
}

int ref_omp_threads(void) { return omp_get_max_threads(); }
} // extern "C"

// ---------------------------------------------------------------- isolated GPU TreePM mesh
// The reference's isolated TreePM mesh (octree_gpu with treepm enabled), its kernels run on
// the host.  Grid set-up restated from engine/physics/treepm/cuda/deposit/TpmGridBuild.inl:98-171
// (FP32 bounds, cell = max(0.25, extent / (G - 2)), doubled mesh centred on the bounds,
// r_s = clamp(cutoffFactor, 1, 2) x cell / 4.5); deposit treePmDepositMassKernel; transforms
// as buildTreePmFftField (TpmFftRuntime.inl): R2C, treePmApplyFftKernel, C2R and the division
// by the cell count (here: the reference CPU fft3d on the Hermitian-completed spectrum, whose
// inverse divides by the cell count); treePmPotentialGradientKernel; treePmSampleAcceleration.
// params8 = {cell, origin x, y, z, mesh, r_s, cutoff, extent}.
extern "C" int ref_treepm_isolated(const float* px, const float* py, const float* pz,
                                   const float* mass, int n, int gridSize, float softening,
                                   float cutoffFactor, int assignment, double* params8,
                                   float* densityOut, float* potentialOut, float* ax, float* ay,
                                   float* az)
{
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < n; ++i) {
        const float q[3] = {px[i], py[i], pz[i]};
        for (int a = 0; a < 3; ++a) {
            mn[a] = fminf(mn[a], q[a]);
            mx[a] = fmaxf(mx[a], q[a]);
        }
    }
    const int requested = std::clamp(gridSize, 32, 128);
    const float extent = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2], softening});
    const float cellSize = std::max(0.25f, extent / static_cast<float>(requested - 2));
    const int G = requested * 2;
    const int total = G * G * G;
    refgpu::TreePmGridParams grid{};
    grid.gridSize = G;
    grid.totalCells = total;
    grid.assignment = assignment;
    grid.periodic = 0;
    grid.cellSize = cellSize;
    grid.invCellSize = 1.0f / cellSize;
    const float halfGridExtent = 0.5f * static_cast<float>(G) * cellSize;
    grid.originX = 0.5f * (mn[0] + mx[0]) - halfGridExtent;
    grid.originY = 0.5f * (mn[1] + mx[1]) - halfGridExtent;
    grid.originZ = 0.5f * (mn[2] + mx[2]) - halfGridExtent;
    const float cutoff = std::clamp(cutoffFactor, 1.0f, 2.0f) * cellSize;
    grid.shortRangeScale = cutoff / 4.5f;
    grid.densityScale = 1.0f;
    grid.poissonCoefficient = 0.0f;
    if (params8) {
        params8[0] = cellSize;
        params8[1] = grid.originX;
        params8[2] = grid.originY;
        params8[3] = grid.originZ;
        params8[4] = G;
        params8[5] = grid.shortRangeScale;
        params8[6] = cutoff;
        params8[7] = extent;
    }
    ParticleSoAView view{};
    view.posX = const_cast<float*>(px);
    view.posY = const_cast<float*>(py);
    view.posZ = const_cast<float*>(pz);
    view.mass = const_cast<float*>(mass);
    view.count = n;
    std::vector<float> density(total, 0.0f);
    std::vector<unsigned> mask((total + 31) / 32, 0u);
    shimLaunch(n, [&] {
        refgpu::blitzar_cuda_tree_pm_gpu::treePmDepositMassKernel(view, n, n, grid, density.data(),
                                                                  mask.data());
    });
    if (densityOut)
        std::copy(density.begin(), density.end(), densityOut);
    // R2C: forward transform, keep x <= G / 2
    std::vector<std::complex<float>> full(total);
    for (int c = 0; c < total; ++c)
        full[c] = std::complex<float>(density[c], 0.0f);
    refpm::fft3d<float>(full, G, false);
    const int hx = G / 2 + 1;
    const int spectrumCells = G * G * hx;
    std::vector<refgpu::cufftComplex> spec(spectrumCells), pot(spectrumCells);
    for (int z = 0; z < G; ++z)
        for (int y = 0; y < G; ++y)
            for (int x = 0; x < hx; ++x) {
                const std::complex<float> v = full[(z * G + y) * G + x];
                spec[(z * G + y) * hx + x] = refgpu::cufftComplex{v.real(), v.imag()};
            }
    shimLaunch(spectrumCells, [&] {
        refgpu::blitzar_cuda_tree_pm_gpu::treePmApplyFftKernel(spec.data(), pot.data(), grid,
                                                               softening);
    });
    // C2R + normalisation: the Hermitian completion, then the inverse transform (which
    // divides by the cell count, as treePmNormalizeFftFieldKernel does after cuFFT)
    for (int z = 0; z < G; ++z)
        for (int y = 0; y < G; ++y)
            for (int x = 0; x < G; ++x) {
                std::complex<float> v;
                if (x < hx) {
                    const refgpu::cufftComplex c = pot[(z * G + y) * hx + x];
                    v = std::complex<float>(c.x, c.y);
                } else {
                    const int xs = G - x, ys = (G - y) % G, zs = (G - z) % G;
                    const refgpu::cufftComplex c = pot[(zs * G + ys) * hx + xs];
                    v = std::complex<float>(c.x, -c.y);
                }
                full[(z * G + y) * G + x] = v;
            }
    refpm::fft3d<float>(full, G, true);
    std::vector<float> potential(total);
    for (int c = 0; c < total; ++c)
        potential[c] = full[c].real();
    if (potentialOut)
        std::copy(potential.begin(), potential.end(), potentialOut);
    std::vector<float> gx(total), gy(total), gz(total);
    shimLaunch(total, [&] {
        refgpu::blitzar_cuda_tree_pm_gpu::treePmPotentialGradientKernel(potential.data(), gx.data(),
                                                                        gy.data(), gz.data(), grid);
    });
    for (int i = 0; i < n; ++i) {
        const Vector3 a = refgpu::blitzar_cuda_tree_pm_gpu::treePmSampleAcceleration(
            grid, Vector3(px[i], py[i], pz[i]), gx.data(), gy.data(), gz.data());
        ax[i] = a.x;
        ay[i] = a.y;
        az[i] = a.z;
    }
    return 0;
}
