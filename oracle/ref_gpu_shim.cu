// oracle/ref_gpu_shim.cu -- TEST AND BENCHMARK INFRASTRUCTURE ONLY (the reference's own GPU
// octree, run on the GPU as the comparator of the reference arm).
//
// This translation unit compiles the reference's GPU linear-octree kernels where they lie
// (include path = the reference's `engine/` directory, passed by oracle/Makefile) as real CUDA
// for sm_100a: the Morton key, leaf, parent and link kernels
// (engine/physics/octree/cuda/linear/Oct{Key,Leaf,Parent,Link}Kernels.inl), the stackless walk
// and its symplectic-Euler update kernel (engine/physics/octree/cuda/force/OctGpu.inl), the GPU
// pair law (engine/physics/core/cuda/prelude/CudForceKernels.inl) and the pooled thrust
// allocator (engine/physics/octree/cuda/linear/OctAllocator.inl over
// engine/physics/core/cuda/buffer/CudMemoryPool.cu, linked in by the Makefile).
//
// The host side restates the reference's orchestration with the same thrust calls in the same
// order:
//  * scratch sized as engine/physics/core/cuda/buffer/CudOctreeScratch.inl does (per-particle
//    arrays of n entries; node arrays of expectedLeaves * (leafDepth + 1) * 4 + 8 entries);
//  * buildLinearOctreeGpu (engine/physics/octree/cuda/linear/OctBuild.inl:14-248): thrust AABB,
//    keys, thrust::sort_by_key, leaf prefixes, reduce_by_key + exclusive_scan, leaf nodes, the
//    level loop, root and next links, compact pack -- on the legacy default stream, with the
//    same capacity checks;
//  * the octree_gpu Euler step (engine/physics/core/cuda/integration/CudOctreeGpuRegular.inl:44
//    then CudOctreeGpuIntegrators.inl:257-267): updateParticlesOctree into the next state,
//    cudaDeviceSynchronize, swap of the position and velocity buffers.
//
// The reference's ParticleSystem translation unit (CudParticleSystem.cu) is not built: it
// needs the reference's own build system and does not compile unmodified with nvcc 12.9 on
// Linux (uint64_t passed where unsigned long long* is declared). Nothing in the product
// (blitzar_b200/, include/) links or loads this library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>

#include "physics/core/cuda/buffer/CudMemoryPool.hpp"
#include "physics/core/force/PhyForceLawPolicy.hpp"
#include "physics/core/particle/PhyParticle.hpp"
#include "physics/core/particle/PhyParticleSoAView.hpp"
#include "physics/core/vector/PhyVector.hpp"
#include "physics/octree/model/Octree.hpp"

// Handle typedefs of engine/physics/core/cuda/prelude/CudConfiguration.inl:73-76.
typedef GpuOctreeNode* OctreeNodeHandle;
typedef const int* IndexConstHandle;
typedef int* IndexHandle;
typedef Vector3* Vector3Handle;

#include "physics/octree/morton/OctMortonCodes.inl"
#include "physics/core/cuda/prelude/CudForceKernels.inl"
#include "physics/octree/cuda/linear/OctAllocator.inl"
#include "physics/octree/cuda/linear/OctKeyKernels.inl"
#include "physics/octree/cuda/linear/OctLeafKernels.inl"
#include "physics/octree/cuda/linear/OctParentKernels.inl"
#include "physics/octree/cuda/linear/OctLinkKernels.inl"
#include "physics/octree/cuda/force/OctGpu.inl"

namespace {

constexpr int kThreads = 256;  // Particle::kDefaultCudaBlockSize

// Error codes of this shim (0 = success).
constexpr int kErrArgs = -1;
constexpr int kErrCuda = -2;
constexpr int kErrCapacity = -3;
constexpr int kErrTree = -4;

enum Field { PX, PY, PZ, VX, VY, VZ, PRX, PRY, PRZ, MASS, TEMP, DENS, kFields };

struct RefGpu {
    int n = 0;
    int leafCapacity = 0;
    int leafDepth = 1;
    float* cur[kFields] = {};
    float* nxt[kFields] = {};
    int* leafIndices = nullptr;
    unsigned long long* keys = nullptr;
    unsigned long long* prefA = nullptr;
    unsigned long long* prefB = nullptr;
    int* levelA = nullptr;
    int* levelB = nullptr;
    int* parentCounts = nullptr;
    int* parentOffsets = nullptr;
    int nodeCap = 0;
    GpuOctreeNode* nodes = nullptr;
    GpuOctreeNodeHotData* hot = nullptr;
    GpuOctreeNodeNavData* nav = nullptr;
    int* firstChild = nullptr;
    int* leafStarts = nullptr;
    int* leafCounts = nullptr;
    Vector3* acc = nullptr;
    int root = -1;
    int nodeCount = 0;
    int leafCount = 0;
};

ParticleSoAView view_of(float* const* f, int n)
{
    ParticleSoAView v{};
    v.posX = f[PX];
    v.posY = f[PY];
    v.posZ = f[PZ];
    v.velX = f[VX];
    v.velY = f[VY];
    v.velZ = f[VZ];
    v.pressX = f[PRX];
    v.pressY = f[PRY];
    v.pressZ = f[PRZ];
    v.mass = f[MASS];
    v.temp = f[TEMP];
    v.dens = f[DENS];
    v.count = n;
    return v;
}

template <class T> bool dev_alloc(T** p, size_t count)
{
    *p = nullptr;
    return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(1, count) * sizeof(T)) ==
           cudaSuccess;
}

void release(RefGpu* h)
{
    for (int f = 0; f < kFields; ++f) {
        cudaFree(h->cur[f]);
        cudaFree(h->nxt[f]);
    }
    void* ptrs[] = {h->leafIndices, h->keys,       h->prefA,      h->prefB,      h->levelA,
                    h->levelB,      h->parentCounts, h->parentOffsets, h->nodes, h->hot,
                    h->nav,         h->firstChild, h->leafStarts, h->leafCounts, h->acc};
    for (void* p : ptrs)
        cudaFree(p);
    delete h;
}

// buildLinearOctreeGpu (OctBuild.inl:14-248) on the current state.  Returns 0 or an error code.
int build_tree(RefGpu* h)
{
    cudaStream_t stream = 0;
    const int n = h->n;
    const int blocks = (n + kThreads - 1) / kThreads;
    const int leafShiftBits = 3 * (21 - h->leafDepth);
    const ParticleSoAView view = view_of(h->cur, n);

    ThrustPoolAllocator thrustAllocator;
    auto exec = thrust::cuda::par(thrustAllocator).on(stream);

    thrust::device_ptr<float> posX(view.posX);
    thrust::device_ptr<float> posY(view.posY);
    thrust::device_ptr<float> posZ(view.posZ);
    const auto zipBegin = thrust::make_zip_iterator(thrust::make_tuple(posX, posY, posZ));
    OctreeAabb init{};
    init.minX = init.minY = init.minZ = FLT_MAX;
    init.maxX = init.maxY = init.maxZ = -FLT_MAX;
    const OctreeAabb bbox = thrust::transform_reduce(exec, zipBegin, zipBegin + n,
                                                     OctreeAabbFromTuple{}, init, OctreeAabbMerge{});

    buildMortonCodesKernel<<<blocks, kThreads, 0, stream>>>(view, n, bbox.minX, bbox.minY,
                                                            bbox.minZ, bbox.maxX, bbox.maxY,
                                                            bbox.maxZ, h->keys, h->leafIndices);
    if (cudaGetLastError() != cudaSuccess)
        return kErrCuda;

    thrust::device_ptr<unsigned long long> sortedKeys(h->keys);
    thrust::device_ptr<int> sortedIndices(h->leafIndices);
    thrust::device_ptr<unsigned long long> prefixesA(h->prefA);
    thrust::device_ptr<unsigned long long> prefixesB(h->prefB);
    thrust::device_ptr<int> levelIndicesA(h->levelA);
    thrust::device_ptr<int> levelIndicesB(h->levelB);
    thrust::device_ptr<int> parentCounts(h->parentCounts);
    thrust::device_ptr<int> parentOffsets(h->parentOffsets);

    thrust::sort_by_key(exec, sortedKeys, sortedKeys + n, sortedIndices);
    buildLeafPrefixesKernel<<<blocks, kThreads, 0, stream>>>(h->keys, n, leafShiftBits, h->prefA);
    if (cudaGetLastError() != cudaSuccess)
        return kErrCuda;
    const auto leafEnd = thrust::reduce_by_key(exec, prefixesA, prefixesA + n,
                                               thrust::make_constant_iterator<int>(1), prefixesB,
                                               parentCounts);
    const int leafCount = static_cast<int>(leafEnd.first - prefixesB);
    if (leafCount <= 0)
        return kErrTree;
    thrust::exclusive_scan(exec, parentCounts, parentCounts + leafCount, parentOffsets);

    const int requiredNodeCapacity = std::max(2, leafCount * (h->leafDepth + 1) + 8);
    if (requiredNodeCapacity > h->nodeCap)
        return kErrCapacity;

    const int leafBlocks = (leafCount + kThreads - 1) / kThreads;
    buildLinearOctreeLeafNodesKernel<<<leafBlocks, kThreads, 0, stream>>>(
        h->nodes, h->leafIndices, h->parentOffsets, h->parentCounts, view, leafCount);
    initLevelIndicesKernel<<<leafBlocks, kThreads, 0, stream>>>(h->levelA, leafCount);
    if (cudaGetLastError() != cudaSuccess)
        return kErrCuda;

    thrust::device_ptr<unsigned long long> currentPrefixes = prefixesB;
    thrust::device_ptr<int> currentLevel = levelIndicesA;
    thrust::device_ptr<int> nextLevel = levelIndicesB;
    int currentCount = leafCount;
    int nextNodeBase = leafCount;
    int totalNodeCount = leafCount;
    while (currentCount > 1) {
        const int currentBlocks = (currentCount + kThreads - 1) / kThreads;
        buildParentPrefixesKernel<<<currentBlocks, kThreads, 0, stream>>>(
            thrust::raw_pointer_cast(currentPrefixes), currentCount, h->prefA);
        if (cudaGetLastError() != cudaSuccess)
            return kErrCuda;
        const auto parentEnd = thrust::reduce_by_key(exec, prefixesA, prefixesA + currentCount,
                                                     thrust::make_constant_iterator<int>(1),
                                                     prefixesB, parentCounts);
        const int parentCount = static_cast<int>(parentEnd.first - prefixesB);
        if (parentCount <= 0)
            return kErrTree;
        if (nextNodeBase + parentCount > h->nodeCap)
            return kErrCapacity;
        thrust::exclusive_scan(exec, parentCounts, parentCounts + parentCount, parentOffsets);
        const int parentBlocks = (parentCount + kThreads - 1) / kThreads;
        buildLinearOctreeParentNodesKernel8<<<parentBlocks, kThreads, 0, stream>>>(
            h->nodes, thrust::raw_pointer_cast(currentLevel),
            thrust::raw_pointer_cast(currentPrefixes), h->parentOffsets, h->parentCounts,
            parentCount, nextNodeBase, thrust::raw_pointer_cast(nextLevel));
        if (cudaGetLastError() != cudaSuccess)
            return kErrCuda;
        totalNodeCount = nextNodeBase + parentCount;
        nextNodeBase += parentCount;
        currentCount = parentCount;
        currentPrefixes = prefixesB;
        std::swap(currentLevel, nextLevel);
    }

    h->leafCount = leafCount;
    h->nodeCount = totalNodeCount;
    h->root = totalNodeCount - 1;
    setLinearOctreeRootLinksKernel<<<1, 1, 0, stream>>>(h->nodes, h->root);
    const int linkBlocks = (totalNodeCount + kThreads - 1) / kThreads;
    buildLinearOctreeNextLinksKernel<<<linkBlocks, kThreads, 0, stream>>>(h->nodes, totalNodeCount,
                                                                         h->root);
    packLinearOctreeCompactKernel<<<linkBlocks, kThreads, 0, stream>>>(
        h->nodes, totalNodeCount, h->hot, h->nav, h->firstChild, h->leafStarts, h->leafCounts);
    return cudaGetLastError() == cudaSuccess ? 0 : kErrCuda;
}

ForceLawPolicy law_of(float theta, float softening, float minDistance2)
{
    return resolveForceLawPolicy(theta, softening, 0.0f, minDistance2, 0.0f);
}

}  // namespace

extern "C" {

// Allocates the reference's state and octree scratch for n particles on the current device and
// uploads positions, velocities and masses (temperature, density and the pressure proxy start at
// zero).  leafCapacity as the reference's linear-octree leaf capacity (its default is 256;
// values below 16 are raised to 16).  Returns a handle, or null.
void* refgpu_create(int n, int leafCapacity, const float* px, const float* py, const float* pz,
                    const float* vx, const float* vy, const float* vz, const float* mass)
{
    if (n <= 0 || !px || !py || !pz || !vx || !vy || !vz || !mass)
        return nullptr;
    RefGpu* h = new (std::nothrow) RefGpu();
    if (!h)
        return nullptr;
    h->n = n;
    h->leafCapacity = std::max(16, leafCapacity);
    while (h->leafDepth < 21) {  // CudOctreeScratch.inl / OctBuild.inl leaf-depth rule
        const double avg = static_cast<double>(n) / static_cast<double>(1ull << (3 * h->leafDepth));
        if (avg <= static_cast<double>(h->leafCapacity))
            break;
        ++h->leafDepth;
    }
    const int expectedLeaves = std::max(1, (n + h->leafCapacity - 1) / h->leafCapacity);
    h->nodeCap = std::max(2, expectedLeaves * (h->leafDepth + 1) * 4 + 8);
    bool ok = true;
    for (int f = 0; f < kFields; ++f)
        ok = ok && dev_alloc(&h->cur[f], n) && dev_alloc(&h->nxt[f], n);
    ok = ok && dev_alloc(&h->leafIndices, n) && dev_alloc(&h->keys, n) &&
         dev_alloc(&h->prefA, n) && dev_alloc(&h->prefB, n) && dev_alloc(&h->levelA, n) &&
         dev_alloc(&h->levelB, n) && dev_alloc(&h->parentCounts, n) &&
         dev_alloc(&h->parentOffsets, n) && dev_alloc(&h->nodes, h->nodeCap) &&
         dev_alloc(&h->hot, h->nodeCap) && dev_alloc(&h->nav, h->nodeCap) &&
         dev_alloc(&h->firstChild, h->nodeCap) && dev_alloc(&h->leafStarts, h->nodeCap) &&
         dev_alloc(&h->leafCounts, h->nodeCap) && dev_alloc(&h->acc, n);
    if (!ok) {
        release(h);
        return nullptr;
    }
    const float* src[] = {px, py, pz, vx, vy, vz};
    for (int f = 0; f < 6; ++f)
        ok = ok && cudaMemcpy(h->cur[f], src[f], n * sizeof(float), cudaMemcpyHostToDevice) ==
                       cudaSuccess;
    ok = ok && cudaMemcpy(h->cur[MASS], mass, n * sizeof(float), cudaMemcpyHostToDevice) ==
                   cudaSuccess;
    for (int f : {PRX, PRY, PRZ, TEMP, DENS})
        ok = ok && cudaMemset(h->cur[f], 0, n * sizeof(float)) == cudaSuccess;
    if (!ok) {
        release(h);
        return nullptr;
    }
    return h;
}

void refgpu_destroy(void* handle)
{
    if (handle)
        release(static_cast<RefGpu*>(handle));
}

// One octree_gpu symplectic-Euler step (tree build, updateParticlesOctree, synchronise, swap).
// openingCriterion 0 = centre of mass, 1 = bounds.  Returns 0 or an error code.
int refgpu_step(void* handle, float dt, float theta, float softening, float minDistance2,
                float maxAcceleration, int openingCriterion)
{
    RefGpu* h = static_cast<RefGpu*>(handle);
    if (!h)
        return kErrArgs;
    const int rc = build_tree(h);
    if (rc != 0)
        return rc;
    const int blocks = (h->n + kThreads - 1) / kThreads;
    updateParticlesOctree<<<blocks, kThreads>>>(
        view_of(h->cur, h->n), view_of(h->nxt, h->n), h->n, h->hot, h->nav, h->firstChild,
        h->leafStarts, h->leafCounts, h->root, h->leafIndices, law_of(theta, softening, minDistance2),
        dt, maxAcceleration, openingCriterion, 0.0f);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return kErrCuda;
    for (int f = 0; f < kFields; ++f)
        std::swap(h->cur[f], h->nxt[f]);
    return 0;
}

// The same steps timed with CUDA events on the legacy default stream, the one the reference
// launches on: `warmup` untimed steps, then `steps` timed ones; *msOut = mean ms per step.
int refgpu_time_steps(void* handle, int warmup, int steps, float dt, float theta, float softening,
                      float minDistance2, float maxAcceleration, int openingCriterion,
                      double* msOut)
{
    if (!handle || steps <= 0 || !msOut)
        return kErrArgs;
    for (int s = 0; s < warmup; ++s) {
        const int rc = refgpu_step(handle, dt, theta, softening, minDistance2, maxAcceleration,
                                   openingCriterion);
        if (rc != 0)
            return rc;
    }
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return kErrCuda;
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    int rc = 0;
    for (int s = 0; s < steps && rc == 0; ++s)
        rc = refgpu_step(handle, dt, theta, softening, minDistance2, maxAcceleration,
                         openingCriterion);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *msOut = static_cast<double>(ms) / steps;
    return rc;
}

// Accelerations of the current state (tree build + computeOctreeAccelerationKernel,
// OctGpu.inl:230-245), downloaded in the caller's particle order.  *nodeCountOut and
// *leafCountOut receive the tree's node and leaf counts.
int refgpu_accel(void* handle, float theta, float softening, float minDistance2,
                 float maxAcceleration, int openingCriterion, float* ax, float* ay, float* az,
                 int* nodeCountOut, int* leafCountOut)
{
    RefGpu* h = static_cast<RefGpu*>(handle);
    if (!h || !ax || !ay || !az)
        return kErrArgs;
    int rc = build_tree(h);
    if (rc != 0)
        return rc;
    const int blocks = (h->n + kThreads - 1) / kThreads;
    computeOctreeAccelerationKernel<<<blocks, kThreads>>>(
        view_of(h->cur, h->n), h->acc, h->n, h->hot, h->nav, h->firstChild, h->leafStarts,
        h->leafCounts, h->root, h->leafIndices, law_of(theta, softening, minDistance2),
        maxAcceleration, openingCriterion, 0.0f);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return kErrCuda;
    Vector3* host = new (std::nothrow) Vector3[h->n];
    if (!host)
        return kErrArgs;
    rc = cudaMemcpy(host, h->acc, h->n * sizeof(Vector3), cudaMemcpyDeviceToHost) == cudaSuccess
             ? 0
             : kErrCuda;
    for (int i = 0; rc == 0 && i < h->n; ++i) {
        ax[i] = host[i].x;
        ay[i] = host[i].y;
        az[i] = host[i].z;
    }
    delete[] host;
    if (nodeCountOut)
        *nodeCountOut = h->nodeCount;
    if (leafCountOut)
        *leafCountOut = h->leafCount;
    return rc;
}

// Downloads the current positions and velocities.
int refgpu_get_state(void* handle, float* px, float* py, float* pz, float* vx, float* vy,
                     float* vz)
{
    RefGpu* h = static_cast<RefGpu*>(handle);
    if (!h || !px || !py || !pz || !vx || !vy || !vz)
        return kErrArgs;
    float* dst[] = {px, py, pz, vx, vy, vz};
    for (int f = 0; f < 6; ++f)
        if (cudaMemcpy(dst[f], h->cur[f], h->n * sizeof(float), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return kErrCuda;
    return 0;
}

}  // extern "C"
