// C ABI of the engine (include/bzgrav.h): handle lifetime, device memory plan, the per-step
// pipeline and its CUDA graph, host <-> device transfers, parity entry points.
//
// Per step (production):
//   kick_drift (FP64, cached force) -> [bbox] -> keys63 -> radix sort -> permute state into
//   Morton order -> octree build -> [PM mesh forces] -> group walk (+=) -> closing kick.
// All of it is enqueued on the handle's stream without host synchronisation, so a whole step
// is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/bzgrav.h"
#include "bz_common.cuh"
#include "bz_kernels.h"

using namespace bz;

namespace bz {
std::atomic<unsigned long long> g_kernel_launches{0};
}

namespace {

enum Phase { kPhKeys = 0, kPhSort, kPhPermute, kPhTree, kPhMesh, kPhWalk, kPhIntegrate, kPhTotal };
constexpr int kNumPhases = 8;
constexpr int kEvStepStart = kNumPhases + 1;  // event slot before the opening kick-drift

struct DeviceBuffers {
    // state in Morton order, two copies (the permutation gathers from one into the other)
    double* st[2][6] = {};
    float* mass[2] = {};
    int* id[2] = {};
    float4* pos4 = nullptr;
    float* acc[3] = {};
    float* acc_pm[3] = {};  // mesh-leg accelerations when it runs on the second stream
    float4* pos4_drift = nullptr;  // drifted FP32 positions in the pre-sort order (mesh mode 2)
    float* pot = nullptr;
    unsigned long long* keys = nullptr;
    uint32_t* perm = nullptr;
    BoxF64* box = nullptr;
    unsigned* bbox32 = nullptr;
    int* err = nullptr;
    double* dt = nullptr;  // {dt, dt/2}
    double* energy = nullptr;  // energy/momentum reduction scratch + results
    unsigned* queue = nullptr;
    int* spill = nullptr;
    unsigned long long* counters = nullptr;  // [3] listed pp, pn, evaluated pp
    float* stage = nullptr;                  // 10n floats for host transfers
    float* ref_xyzm = nullptr;               // 4n floats, caller order, reference mode
    float4* ref_orig = nullptr;              // n float4, caller order
    float* ref_hot8 = nullptr;               // 8 floats
};

} // namespace

struct bz_handle {
    bz_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t pm_stream = nullptr;  // TreePM: the mesh leg overlaps the tree build and walk
    // TreePM mesh-leg schedule (bz_autotune decides): 0 in line on the main stream; 1 on
    // pm_stream, forked after the sort, concurrent with the tree build and walk; 2 as 1, but in a
    // step the deposit and field solve are forked right after the drift (they take the particles
    // in any order), so they also run concurrently with the keys, sort and permutation; only the
    // interpolation waits for the new order
    int mesh_overlap = 2;
    int walk_blocks_per_sm = 0;  // cap on resident walk blocks per SM (0: as many as fit)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_sorted = nullptr;
    size_t capacity = 0;
    size_t n = 0;
    int cur = 0;
    bool forces_valid = false;
    DeviceBuffers d;
    SortWorkspace sort{};
    AdaptiveSortWorkspace asort{};  // the per-step re-sort of nearly sorted keys
    TreeArrays tree{};
    GroupTable groups{};
    PmPlan* pm = nullptr;
    IsoGrid* iso = nullptr;  // isolated TreePM: grid of the current evaluation (device)
    int spill_slots = 0;
    size_t bytes = 0;
    std::vector<void*> allocations;
    std::string last_error;
    // timing
    bool timing = false;
    cudaEvent_t ev[kNumPhases + 2] = {};
    bool stepping = false;  // last timed call was bz_step (has an opening kick-drift)
    // bz_step_get_state_acc_f64: the drifted positions leave on io_stream while the step runs
    cudaStream_t io_stream = nullptr;
    cudaEvent_t ev_drift = nullptr, ev_io = nullptr;
    double* io_pos = nullptr;       // 3 x capacity doubles of caller-order positions
    double* io_host_pos = nullptr;  // set only while that call enqueues its step
    float phase_ms[kNumPhases] = {};
    // graphs (one per state-buffer parity)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_failed = false;
    double* h_dt = nullptr;  // pinned {dt, dt/2}
    unsigned long long last_pp = 0, last_pn = 0, last_eval = 0;
    bool ref_tree_valid = false;
    // adaptive block steps
    struct {
        AdaptiveState st{};
        unsigned char* active = nullptr;  // [capacity] sorted-slot flags of the current substep
        int* lmax = nullptr;
        bool ready = false;               // levels and cached accelerations match the state
    } ad;
    const unsigned char* walk_active = nullptr;  // mask handed to the walk (adaptive substeps)
    // ensembles of independent systems (0 = one system)
    int systems = 0;
    long long* sys_offsets = nullptr;  // [kMaxSystems + 1] caller-index offsets
    BoxF64* sys_boxes = nullptr;       // [kMaxSystems]
    std::vector<long long> host_offsets;
    // learned pair correction (TreePM)
    struct {
        float* params = nullptr;  // FP32 master weights [kMlpParams]
        float* grad = nullptr;
        float* adam_m = nullptr;
        float* adam_v = nullptr;
        float* loss = nullptr;
        float scale = 0.0f;       // the network predicts residual / scale
        float radius_cells = 0.0f;  // pairs closer than this (mesh cells) are corrected
        bool trained = false;
        bool enabled = false;
        int* pair_src = nullptr;  // [capacity * kPairSlots]
        int* pair_cnt = nullptr;  // [capacity]
    } learn;
};

namespace {

bz_status fail(bz_handle* h, bz_status s, const std::string& msg)
{
    if (h)
        h->last_error = msg;
    return s;
}

bz_status cuda_fail(bz_handle* h, cudaError_t e, const char* what)
{
    return fail(h, BZ_CUDA_ERROR, std::string("[cuda] ") + what + " failed: " + cudaGetErrorString(e));
}

template <class T> bool dalloc(bz_handle* h, T** p, size_t count)
{
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMalloc(&q, bytes) != cudaSuccess) {
        *p = nullptr;
        return false;
    }
    h->allocations.push_back(q);
    h->bytes += bytes;
    *p = static_cast<T*>(q);
    return true;
}

bool periodic(const bz_handle* h) { return h->cfg.solver == BZ_SOLVER_TREEPM && h->cfg.box_length > 0.0; }
// Open-boundary TreePM: the reference's GPU TreePM on a doubled, particle-centred mesh.
bool isolated(const bz_handle* h) { return h->cfg.solver == BZ_SOLVER_TREEPM && h->cfg.box_length <= 0.0; }

float rsplit_len(const bz_handle* h)
{
    return static_cast<float>(h->cfg.treepm_r_split_cells * h->cfg.box_length / h->cfg.treepm_grid_size);
}

// Correction radius in mesh cells: the short-range cutoff, capped so that the mean number of
// neighbours inside it (at the handle's mean particle density) stays at 40 % of the recorded
// pair slots per target.
float learn_radius_cells(const bz_handle* h)
{
    const double M = h->cfg.treepm_grid_size;
    const double rho = static_cast<double>(std::max<size_t>(h->n, 1)) / (M * M * M);
    const double cap = std::cbrt(0.4 * kPairSlots / (4.18879020478639 * rho));
    const double rc = h->cfg.treepm_r_cut_factor * h->cfg.treepm_r_split_cells;
    return static_cast<float>(std::min(rc, cap));
}

void record(bz_handle* h, int i)
{
    if (h->timing)
        cudaEventRecord(h->ev[i], h->stream);
}

WalkParams walk_params(const bz_handle* h, bool want_pot)
{
    WalkParams p{};
    const float th = std::max(h->cfg.octree_theta, h->cfg.physics_min_theta);
    p.theta2 = th * th;
    const float eps = std::max(h->cfg.octree_softening, h->cfg.physics_min_softening);
    p.eps2 = eps * eps;
    p.min_dist2 = h->cfg.physics_min_distance2;
    p.quadrupole = h->cfg.multipole_order >= 2 ? 1 : 0;
    p.want_pot = want_pot ? 1 : 0;
    p.max_acc = h->cfg.physics_max_acceleration;
    if (isolated(h)) {
        // split scale, cutoff and node cap follow the mesh cell of each evaluation: the walk
        // reads them from the device-held grid (the values here only select its variant)
        p.rsplit = 1.0f;
        p.rcut2 = 1.0f;
        p.box = 0.0f;
        p.iso = h->iso;
    } else if (h->cfg.solver == BZ_SOLVER_TREEPM) {
        const float rs = rsplit_len(h);
        const float rc = h->cfg.treepm_r_cut_factor * rs;
        p.rsplit = rs;
        p.rcut2 = rc * rc;
        p.max_node_size = h->cfg.treepm_node_size_factor > 0.0f ? h->cfg.treepm_node_size_factor * rs : 0.0f;
        p.box = static_cast<float>(h->cfg.box_length);
    }
    return p;
}

// Keys, sort and permutation: the state ends up in Morton order in buffer `cur`.
void enqueue_order(bz_handle* h)
{
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    record(h, kPhKeys);
    if (h->systems > 0) {
        launch_keys_ensemble(s[0], s[1], s[2], d.id[h->cur], n, h->sys_offsets, h->systems,
                             h->sys_boxes, d.keys, d.perm, h->stream);
    } else {
        if (!periodic(h))
            launch_bbox_f64(s[0], s[1], s[2], n, d.box, h->stream);
        launch_keys63(s[0], s[1], s[2], n, d.box, periodic(h) ? h->cfg.box_length : 0.0, d.keys,
                      d.perm, h->stream);
    }
    record(h, kPhSort);
    // the keys arrive in the previous sorted order (perm = identity): nearly sorted after a step
    launch_radix_sort_adaptive(d.keys, d.perm, n, 64, h->sort, h->asort, d.err, h->stream);
    record(h, kPhPermute);
    const int nxt = h->cur ^ 1;
    launch_permute(d.perm, n, d.st[h->cur], d.st[nxt], 6, d.mass[h->cur], d.mass[nxt],
                   d.id[h->cur], d.id[nxt], d.pos4, 0.0, h->stream);
    h->cur = nxt;
}

// TreePM with the mesh leg on the second stream (outside phase timing).
bool mesh_concurrent(const bz_handle* h)
{
    return h->cfg.solver == BZ_SOLVER_TREEPM && h->pm && h->pm_stream && h->mesh_overlap > 0 &&
           !h->timing;
}

// Forces of the (already ordered) state into d.acc; optional closing kick.  `mesh_forked`: the
// step already forked the deposit and field solve onto pm_stream (mesh mode 2).
void enqueue_forces(bz_handle* h, bool kick, bool want_pot, bool mesh_forked = false)
{
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    // isolated TreePM: this evaluation's mesh grid, from the bounds the ordering just reduced
    if (isolated(h))
        launch_iso_grid(d.box, h->cfg.treepm_grid_size, h->cfg.treepm_cell_floor,
                        h->cfg.octree_softening, h->cfg.treepm_r_split_cells, h->cfg.treepm_r_cut_factor,
                        h->cfg.treepm_node_size_factor, h->iso, h->stream);
    // TreePM: the mesh leg needs only the ordered positions, so it runs on a second stream
    // while this one builds the tree and walks; joined before the kick
    const bool overlap = mesh_concurrent(h);
    if (overlap) {
        if (mesh_forked) {
            // deposit and solve are under way; the interpolation needs the new order
            cudaEventRecord(h->ev_sorted, h->stream);
            cudaStreamWaitEvent(h->pm_stream, h->ev_sorted, 0);
            pm_interp(h->pm, d.pos4, n, d.acc_pm[0], d.acc_pm[1], d.acc_pm[2], h->pm_stream);
        } else {
            cudaEventRecord(h->ev_fork, h->stream);
            cudaStreamWaitEvent(h->pm_stream, h->ev_fork, 0);
            pm_forces(h->pm, d.pos4, n, d.acc_pm[0], d.acc_pm[1], d.acc_pm[2], h->pm_stream);
        }
        cudaEventRecord(h->ev_join, h->pm_stream);
    }
    record(h, kPhTree);
    const int root_level = h->systems > 0 ? kSystemLevels : 0;
    launch_tree_build(d.keys, d.pos4, n, h->cfg.leaf_capacity, kMaxLevels, h->tree, d.err,
                      h->stream, root_level, h->cfg.multipole_order >= 2);
    launch_groups(h->tree, n, h->cfg.walk_group_size, root_level, d.keys, h->groups, h->stream);
    record(h, kPhMesh);
    if (h->cfg.solver == BZ_SOLVER_TREEPM && h->pm && !overlap) {
        pm_forces(h->pm, d.pos4, n, d.acc[0], d.acc[1], d.acc[2], h->stream);
    } else {
        for (int a = 0; a < 3; ++a)
            cudaMemsetAsync(d.acc[a], 0, sizeof(float) * n, h->stream);
    }
    if (want_pot)
        cudaMemsetAsync(d.pot, 0, sizeof(float) * n, h->stream);
    record(h, kPhWalk);
    cudaMemsetAsync(d.counters, 0, 3 * sizeof(unsigned long long), h->stream);
    WalkOutputs o{};
    o.ax = d.acc[0];
    o.ay = d.acc[1];
    o.az = d.acc[2];
    o.pot = want_pot ? d.pot : nullptr;
    o.totals = d.counters;
    WalkParams wp = walk_params(h, want_pot);
    wp.active = h->walk_active;
    wp.blocks_per_sm = h->walk_blocks_per_sm;
    // the mesh force computed in line is already in d.acc: the walk clamps the sum
    wp.clamp_total = h->cfg.solver == BZ_SOLVER_TREEPM && h->pm && !overlap ? 1 : 0;
    const bool learned = h->learn.enabled && h->learn.trained && h->cfg.solver == BZ_SOLVER_TREEPM;
    if (learned) {
        o.pair_src = h->learn.pair_src;
        o.pair_cnt = h->learn.pair_cnt;
        const float rc = (h->learn.radius_cells > 0.0f ? h->learn.radius_cells : learn_radius_cells(h)) *
                         static_cast<float>(h->cfg.box_length / h->cfg.treepm_grid_size);
        wp.rcorr2 = std::min(rc * rc, wp.rcut2);
    }
    launch_walk(d.pos4, n, h->tree, h->groups, wp, o, d.queue, d.spill, d.err, h->stream);
    // the mesh leg's accelerations complete d.acc here, or inside the closing kick
    const bool add_in_kick = overlap && kick && !learned;
    if (overlap) {
        cudaStreamWaitEvent(h->stream, h->ev_join, 0);
        if (!add_in_kick)
            launch_add3(d.acc[0], d.acc[1], d.acc[2], d.acc_pm[0], d.acc_pm[1], d.acc_pm[2], n,
                        h->cfg.physics_max_acceleration, h->stream);
    }
    if (learned) {
        const float hcell = static_cast<float>(h->cfg.box_length / h->cfg.treepm_grid_size);
        launch_mlp_pairs(h->learn.params, d.pos4, n, h->learn.pair_src, h->learn.pair_cnt, hcell,
                         static_cast<float>(h->cfg.box_length), h->learn.scale, d.acc[0], d.acc[1],
                         d.acc[2], d.err, h->stream);
    }
    record(h, kPhIntegrate);
    if (kick) {
        double* const* s = d.st[h->cur];
        if (add_in_kick)
            launch_kick(s[3], s[4], s[5], d.acc[0], d.acc[1], d.acc[2], n, d.dt + 1, h->stream,
                        d.acc_pm[0], d.acc_pm[1], d.acc_pm[2], h->cfg.physics_max_acceleration);
        else
            launch_kick(s[3], s[4], s[5], d.acc[0], d.acc[1], d.acc[2], n, d.dt + 1, h->stream);
    }
}

void enqueue_io_positions(bz_handle* h);

void enqueue_step(bz_handle* h)
{
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    // (the isolated mesh's grid needs the new bounds first: no early fork there)
    const bool early = mesh_concurrent(h) && h->mesh_overlap == 2 && !isolated(h);
    // leapfrog: the opening half kick (the closing one follows the force evaluation);
    // symplectic Euler: the whole kick with the force of the step's start positions
    const bool euler = h->cfg.integrator == BZ_INTEGRATOR_EULER;
    launch_kick_drift(s[0], s[1], s[2], s[3], s[4], s[5], d.acc[0], d.acc[1], d.acc[2], n, d.dt,
                      periodic(h) ? h->cfg.box_length : 0.0, nullptr, h->stream,
                      early ? d.mass[h->cur] : nullptr, early ? d.pos4_drift : nullptr,
                      euler ? 1.0 : 0.5);
    if (h->io_host_pos)  // the step's positions are final here: send them while the step runs
        enqueue_io_positions(h);
    if (early) {
        // the mass deposit is a sum over particles in any order: start it and the field solve
        // now, concurrently with the keys, sort and permutation of this stream
        cudaEventRecord(h->ev_fork, h->stream);
        cudaStreamWaitEvent(h->pm_stream, h->ev_fork, 0);
        pm_deposit(h->pm, d.pos4_drift, n, h->pm_stream);
        pm_solve(h->pm, h->pm_stream);
    }
    enqueue_order(h);
    enqueue_forces(h, !euler, false, early);
}

bz_status check_device(bz_handle* h, const char* what)
{
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
        return cuda_fail(h, e, what);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(h, e, what);
    int err = 0;
    e = cudaMemcpy(&err, h->d.err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_fail(h, e, what);
    if (err) {
        cudaMemset(h->d.err, 0, sizeof(int));
        std::string m = std::string("[device] ") + what + ":";
        if (err & kErrWalkStack)
            m += " walk traversal stack exhausted;";
        if (err & kErrSortSpin)
            m += " radix-sort look-back wait limit reached;";
        if (err & kErrTreeCapacity)
            m += " octree node capacity exceeded;";
        if (err & kErrTreeSpin)
            m += " octree look-back wait limit reached;";
        if (err & kErrBulkWait)
            m += " bulk-copy wait limit reached;";
        if (err & kErrListCapacity)
            m += " interaction list capacity exceeded;";
        return fail(h, BZ_DEVICE_LIMIT, m);
    }
    return BZ_OK;
}

void collect_timing(bz_handle* h)
{
    if (!h->timing)
        return;
    cudaEventSynchronize(h->ev[kNumPhases]);
    float total = 0.0f;
    for (int i = 0; i < kPhTotal; ++i) {
        float ms = 0.0f;
        const int next = i + 1 <= kPhIntegrate ? i + 1 : kNumPhases;
        cudaEventElapsedTime(&ms, h->ev[i], h->ev[next]);
        h->phase_ms[i] = ms;
        total += ms;
    }
    if (h->stepping) {  // opening kick-drift of the last step
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, h->ev[kEvStepStart], h->ev[kPhKeys]);
        h->phase_ms[kPhIntegrate] += ms;
        total += ms;
    }
    h->phase_ms[kPhTotal] = total;
}

void read_counters(bz_handle* h)
{
    unsigned long long c[3] = {0, 0, 0};
    cudaMemcpy(c, h->d.counters, sizeof(c), cudaMemcpyDeviceToHost);
    h->last_pp = c[0];
    h->last_pn = c[1];
    h->last_eval = c[2];
}

bz_status ensure_forces(bz_handle* h)
{
    if (h->forces_valid)
        return BZ_OK;
    enqueue_order(h);
    enqueue_forces(h, false, false);
    bz_status s = check_device(h, "initial force evaluation");
    if (s != BZ_OK)
        return s;
    h->forces_valid = true;
    return BZ_OK;
}

// One-time capture of a step for each state-buffer parity.  Capturing records the work
// without executing it; the host-side parity is restored afterwards.
void build_graphs(bz_handle* h)
{
    if (h->graph_failed || (h->graph[0] && h->graph[1]))
        return;
    const int orig = h->cur;
    const bool saved = h->timing;
    h->timing = false;
    for (int parity = 0; parity < 2 && !h->graph_failed; ++parity) {
        if (h->graph[parity])
            continue;
        h->cur = parity;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            h->graph_failed = true;
            break;
        }
        enqueue_step(h);
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        cudaGraphExec_t ex = nullptr;
        if (e != cudaSuccess || !g || cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
            h->graph_failed = true;
            if (g)
                cudaGraphDestroy(g);
            break;
        }
        cudaGraphDestroy(g);
        h->graph[parity] = ex;
    }
    if (h->graph_failed)
        cudaGetLastError();
    h->timing = saved;
    h->cur = orig;
}

} // namespace

extern "C" {

const char* bz_version(void) { return "bzgrav 0.1 (sm_100a)"; }

uint64_t bz_kernel_launches(void) { return g_kernel_launches.load(); }

bz_status bz_launches_per_step(bz_handle* h, uint64_t* launches)
{
    if (!h || !launches || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    // count one eagerly enqueued step into a throw-away capture (nothing executes)
    cudaSetDevice(h->device);
    const unsigned long long before = g_kernel_launches.load();
    const int cur = h->cur;
    const bool timing = h->timing;
    h->timing = false;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(h, BZ_CUDA_ERROR, "capture for launch count");
    enqueue_step(h);
    cudaStreamEndCapture(h->stream, &g);
    if (g)
        cudaGraphDestroy(g);
    h->cur = cur;
    h->timing = timing;
    *launches = g_kernel_launches.load() - before;
    g_kernel_launches.fetch_sub(*launches);
    return BZ_OK;
}

const char* bz_status_string(bz_status s)
{
    switch (s) {
    case BZ_OK: return "ok";
    case BZ_INVALID_ARGUMENT: return "invalid argument";
    case BZ_NOT_READY: return "not ready";
    case BZ_TIMEOUT: return "timeout";
    case BZ_INTERNAL_ERROR: return "internal error";
    case BZ_CUDA_ERROR: return "cuda error";
    case BZ_OUT_OF_MEMORY: return "out of memory";
    case BZ_DEVICE_LIMIT: return "device limit";
    case BZ_UNSUPPORTED: return "unsupported";
    }
    return "unknown";
}

bz_status bz_config_init(bz_config* c)
{
    if (!c)
        return BZ_INVALID_ARGUMENT;
    std::memset(c, 0, sizeof(*c));
    c->struct_size = sizeof(bz_config);
    c->solver = BZ_SOLVER_OCTREE;
    c->octree_theta = 0.5f;
    c->octree_softening = 0.01f;
    c->octree_opening_criterion = 0;
    c->linear_octree_leaf_capacity = 256;
    c->leaf_capacity = 16;
    c->multipole_order = 2;
    c->physics_max_acceleration = 64.0f;  // kPhysicsMaxAccelerationDefault (FndConstants.hpp:21)
    c->physics_min_softening = 0.0f;
    c->physics_min_distance2 = 1.0e-12f;
    c->physics_min_theta = 0.05f;
    c->treepm_grid_size = 128;
    c->treepm_r_split_cells = 1.25f;
    c->treepm_r_cut_factor = 4.5f;
    c->treepm_assignment = 0;
    c->treepm_gradient = 0;
    c->treepm_window_floor = 0.08f;
    c->treepm_node_size_factor = 0.0f;
    c->treepm_cell_floor = 0.25f;  // the reference's isolated-mesh cell floor (TpmGridBuild.inl:100)
    c->box_length = 0.0;
    c->key_mode = BZ_KEYS_PRODUCTION;
    c->device = 0;
    c->stream = 0;
    c->use_graph = 1;
    c->walk_group_size = kGroupMax;
    c->adaptive_max_level = 0;
    c->adaptive_eta = 0.02f;
    c->integrator = BZ_INTEGRATOR_LEAPFROG;
    return BZ_OK;
}

size_t bz_last_error(const bz_handle* h, char* buf, size_t cap)
{
    const std::string& e = h ? h->last_error : std::string();
    if (buf && cap > 0) {
        const size_t k = std::min(cap - 1, e.size());
        std::memcpy(buf, e.data(), k);
        buf[k] = '\0';
    }
    return e.size();
}

bz_status bz_destroy(bz_handle* h)
{
    if (!h)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    for (int i = 0; i < 2; ++i)
        if (h->graph[i])
            cudaGraphExecDestroy(h->graph[i]);
    for (int i = 0; i <= kEvStepStart; ++i)
        if (h->ev[i])
            cudaEventDestroy(h->ev[i]);
    if (h->pm_stream)
        cudaStreamSynchronize(h->pm_stream);
    pm_destroy(h->pm);
    if (h->ev_fork)
        cudaEventDestroy(h->ev_fork);
    if (h->ev_join)
        cudaEventDestroy(h->ev_join);
    if (h->ev_sorted)
        cudaEventDestroy(h->ev_sorted);
    if (h->pm_stream)
        cudaStreamDestroy(h->pm_stream);
    if (h->io_stream) {
        cudaStreamSynchronize(h->io_stream);
        cudaStreamDestroy(h->io_stream);
    }
    if (h->ev_drift)
        cudaEventDestroy(h->ev_drift);
    if (h->ev_io)
        cudaEventDestroy(h->ev_io);
    for (void* p : h->allocations)
        cudaFree(p);
    if (h->h_dt)
        cudaFreeHost(h->h_dt);
    if (h->own_stream && h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
    return BZ_OK;
}

bz_status bz_create(const bz_config* cfg, size_t capacity, bz_handle** out)
{
    if (!cfg || !out || capacity == 0 || cfg->struct_size != sizeof(bz_config))
        return BZ_INVALID_ARGUMENT;
    if (capacity > (1u << 25))
        return BZ_UNSUPPORTED;  // node indices are packed in 26 bits by the walk
    *out = nullptr;
    bz_handle* h = new bz_handle();
    h->cfg = *cfg;
    h->device = cfg->device;
    h->capacity = capacity;
    if (cfg->solver == BZ_SOLVER_TREEPM && cfg->box_length <= 0.0) {
        // isolated mesh of 2G cells, G = treepm_grid_size
        if (cfg->treepm_grid_size < 8 || cfg->treepm_grid_size > 1024 || !(cfg->treepm_r_split_cells > 0.0f) ||
            !(cfg->treepm_r_cut_factor > 0.0f) || !(cfg->treepm_cell_floor > 0.0f) ||
            cfg->treepm_assignment < 0 || cfg->treepm_assignment > 2 || cfg->treepm_gradient < 0 ||
            cfg->treepm_gradient > 2 || cfg->treepm_node_size_factor < 0.0f) {
            delete h;
            return BZ_INVALID_ARGUMENT;
        }
    } else if (cfg->solver == BZ_SOLVER_TREEPM) {
        const int M = cfg->treepm_grid_size;
        if (cfg->box_length <= 0.0 || M < 8 || (M & (M - 1)) != 0 || cfg->treepm_r_split_cells <= 0.0f ||
            cfg->treepm_r_cut_factor <= 0.0f || cfg->treepm_assignment < 0 || cfg->treepm_assignment > 2 ||
            cfg->treepm_gradient < 0 || cfg->treepm_gradient > 2 ||
            cfg->treepm_r_cut_factor * cfg->treepm_r_split_cells * 2.0 >= M) {
            delete h;
            return BZ_INVALID_ARGUMENT;
        }
    }
    // physics_max_acceleration: the reference's validator rejects values <= 0
    // (engine/config/validation/physics/CfgPhysics.cpp:20-24)
    if (cfg->leaf_capacity < 1 || cfg->octree_theta <= 0.0f || cfg->walk_group_size < 1 ||
        !(cfg->physics_max_acceleration > 0.0f) ||
        cfg->walk_group_size > kGroupMax || cfg->adaptive_max_level < 0 || cfg->adaptive_max_level > 12 ||
        (cfg->adaptive_max_level > 0 && (cfg->solver != BZ_SOLVER_OCTREE || !(cfg->adaptive_eta > 0.0f))) ||
        (cfg->integrator != BZ_INTEGRATOR_LEAPFROG && cfg->integrator != BZ_INTEGRATOR_EULER)) {
        delete h;
        return BZ_INVALID_ARGUMENT;
    }
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
        delete h;
        return BZ_CUDA_ERROR;
    }
    if (cfg->stream) {
        h->stream = reinterpret_cast<cudaStream_t>(cfg->stream);
    } else {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete h;
            return BZ_CUDA_ERROR;
        }
        h->own_stream = true;
    }
    const size_t n = capacity;
    DeviceBuffers& d = h->d;
    bool ok = true;
    for (int b = 0; b < 2; ++b) {
        for (int c = 0; c < 6; ++c)
            ok = ok && dalloc(h, &d.st[b][c], n);
        ok = ok && dalloc(h, &d.mass[b], n) && dalloc(h, &d.id[b], n);
    }
    ok = ok && dalloc(h, &d.pos4, n);
    for (int a = 0; a < 3; ++a)
        ok = ok && dalloc(h, &d.acc[a], n);
    ok = ok && dalloc(h, &d.pot, n) && dalloc(h, &d.keys, n) && dalloc(h, &d.perm, n) &&
         dalloc(h, &d.box, 1) && dalloc(h, &d.bbox32, 8) && dalloc(h, &d.err, 1) &&
         dalloc(h, &d.dt, 2) && dalloc(h, &d.energy, energy_scratch_doubles()) &&
         dalloc(h, &d.queue, 1) && dalloc(h, &d.counters, 3) &&
         dalloc(h, &d.stage, 10 * n) && dalloc(h, &d.ref_xyzm, 4 * n) && dalloc(h, &d.ref_orig, n) &&
         dalloc(h, &d.ref_hot8, 8);
    // sort workspace
    SortWorkspace& sw = h->sort;
    const size_t words = sort_state_words(static_cast<int>(n));
    ok = ok && dalloc(h, &sw.keys_alt, n) && dalloc(h, &sw.vals_alt, n) && dalloc(h, &sw.hist, 8 * 256) &&
         dalloc(h, &sw.base, 8 * 256) && dalloc(h, &sw.ticket, 8) && dalloc(h, &sw.epoch, 1) &&
         dalloc(h, &sw.trivial, 8) && dalloc(h, &sw.state, words);
    sw.max_tiles = static_cast<int>(words / 256);
    AdaptiveSortWorkspace& aw = h->asort;
    aw.cap = adaptive_sort_cap(static_cast<int>(n));
    ok = ok && dalloc(h, &aw.fkeys, aw.cap) && dalloc(h, &aw.fvals, aw.cap) && dalloc(h, &aw.falt_keys, aw.cap) &&
         dalloc(h, &aw.falt_vals, aw.cap) && dalloc(h, &aw.flag, n) &&
         dalloc(h, &aw.block_sums, adaptive_sort_blocks(static_cast<int>(n))) && dalloc(h, &aw.ctl, 4) &&
         dalloc(h, &aw.job, 1);
    // tree
    TreeArrays& t = h->tree;
    t.cap = static_cast<int>(2 * n + 1024);
    const size_t cap = static_cast<size_t>(t.cap);
    ok = ok && dalloc(h, &t.start, cap) && dalloc(h, &t.count, cap) && dalloc(h, &t.child, cap) &&
         dalloc(h, &t.nchild, cap) && dalloc(h, &t.parent, cap) && dalloc(h, &t.level, cap) &&
         dalloc(h, &t.lvl_first, kMaxLevels + 2) && dalloc(h, &t.lvl_count, kMaxLevels + 2) &&
         dalloc(h, &t.lvl_split, kMaxLevels + 2) &&
         dalloc(h, &t.n_nodes, 1) && dalloc(h, &t.ticket, kMaxLevels + 2) &&
         dalloc(h, &t.lookback, tree_lookback_words(t.cap)) && dalloc(h, &t.arrive, cap) &&
         dalloc(h, &t.m64, cap) && dalloc(h, &t.s64, 3 * cap) && dalloc(h, &t.c64, 3 * cap) &&
         dalloc(h, &t.q64, 6 * cap) && dalloc(h, &t.box0, cap) && dalloc(h, &t.box1, cap) &&
         dalloc(h, &t.mono, cap) && dalloc(h, &t.quadA, cap) && dalloc(h, &t.quadB, cap);
    GroupTable& gt = h->groups;
    ok = ok && dalloc(h, &gt.flag, group_flag_bytes(static_cast<int>(n))) && dalloc(h, &gt.gstart, n + 1) && dalloc(h, &gt.ngroups, 1) &&
         dalloc(h, &gt.groot, n + 1) && dalloc(h, &gt.sysroot, kMaxSystems) &&
         (cfg->adaptive_max_level == 0 ||
          (dalloc(h, &h->ad.st.level, n) && dalloc(h, &h->ad.st.ax, n) && dalloc(h, &h->ad.st.ay, n) &&
           dalloc(h, &h->ad.st.az, n) && dalloc(h, &h->ad.st.updates, 1) && dalloc(h, &h->ad.active, n) &&
           dalloc(h, &h->ad.lmax, 1))) &&
         dalloc(h, &gt.block_sums, static_cast<size_t>(group_count_blocks(static_cast<int>(n))));
    // walk spill area: one slot per warp the persistent walk grid can hold
    h->spill_slots = walk_spill_slots();
    ok = ok && dalloc(h, &d.spill, static_cast<size_t>(h->spill_slots) * walk_spill_entries());
    if (!ok) {
        bz_destroy(h);
        return BZ_OUT_OF_MEMORY;
    }
    cudaMemsetAsync(sw.state, 0, words * sizeof(unsigned long long), h->stream);
    cudaMemsetAsync(sw.epoch, 0, sizeof(uint32_t), h->stream);
    cudaMemsetAsync(d.err, 0, sizeof(int), h->stream);
    if (cfg->solver == BZ_SOLVER_TREEPM) {
        int perr = 0;
        if (isolated(h)) {
            void* g = nullptr;
            if (cudaMalloc(&g, sizeof(IsoGrid)) != cudaSuccess) {
                bz_destroy(h);
                return BZ_OUT_OF_MEMORY;
            }
            h->allocations.push_back(g);
            h->iso = static_cast<IsoGrid*>(g);
            h->pm = pm_create(2 * cfg->treepm_grid_size, 0.0, 0.0, cfg->treepm_assignment + 2,
                              cfg->treepm_gradient, cfg->treepm_window_floor, h->stream, &perr, h->iso,
                              h->d.err);
        } else {
            h->pm = pm_create(cfg->treepm_grid_size, cfg->box_length, rsplit_len(h),
                              cfg->treepm_assignment + 2, cfg->treepm_gradient,
                              cfg->treepm_window_floor, h->stream, &perr, nullptr, h->d.err);
        }
        if (!h->pm) {
            bz_destroy(h);
            return BZ_OUT_OF_MEMORY;
        }
        h->bytes += pm_bytes(h->pm);
        // second stream and fork/join events for the concurrent mesh leg (best effort: without
        // them the mesh leg runs in line)
        if (!dalloc(h, &h->d.acc_pm[0], n) || !dalloc(h, &h->d.acc_pm[1], n) || !dalloc(h, &h->d.acc_pm[2], n) ||
            !dalloc(h, &h->d.pos4_drift, n)) {
            bz_destroy(h);
            return BZ_OUT_OF_MEMORY;
        }
        if (cudaStreamCreateWithFlags(&h->pm_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_sorted, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            if (h->pm_stream)
                cudaStreamDestroy(h->pm_stream);
            h->pm_stream = nullptr;
        }
    }
    for (int i = 0; i <= kEvStepStart; ++i)
        cudaEventCreate(&h->ev[i]);
    cudaMallocHost(&h->h_dt, 2 * sizeof(double));
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        bz_destroy(h);
        return BZ_CUDA_ERROR;
    }
    *out = h;
    return BZ_OK;
}

size_t bz_particle_count(const bz_handle* h) { return h ? h->n : 0; }
size_t bz_device_bytes(const bz_handle* h) { return h ? h->bytes : 0; }

}  // extern "C"

namespace {

__global__ void k_unpack_state(const float* __restrict__ st, int n, int have_vel, double* x,
                               double* y, double* z, double* vx, double* vy, double* vz,
                               float* m, int* id, double box)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double p[3] = {st[i], st[n + i], st[2 * n + i]};
        if (box > 0.0)
            for (int a = 0; a < 3; ++a) {
                p[a] -= box * floor(p[a] / box);
                if (p[a] >= box)
                    p[a] = 0.0;
            }
        x[i] = p[0];
        y[i] = p[1];
        z[i] = p[2];
        vx[i] = have_vel ? st[3 * n + i] : 0.0;
        vy[i] = have_vel ? st[4 * n + i] : 0.0;
        vz[i] = have_vel ? st[5 * n + i] : 0.0;
        m[i] = st[6 * n + i];
        id[i] = i;
    }
}

// As k_unpack_state, into the device's current particle order: slot i takes caller particle
// id[i] (ids kept), with the accelerations staged after the state (caller order).
__global__ void k_unpack_state_kept(const float* __restrict__ st, int n, int have_vel, double* x,
                                    double* y, double* z, double* vx, double* vy, double* vz,
                                    float* m, const int* __restrict__ id, double box,
                                    float* ax, float* ay, float* az)
{
    const float* acc = st + 7 * static_cast<size_t>(n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = id[i];
        double p[3] = {st[c], st[n + c], st[2 * n + c]};
        if (box > 0.0)
            for (int a = 0; a < 3; ++a) {
                p[a] -= box * floor(p[a] / box);
                if (p[a] >= box)
                    p[a] = 0.0;
            }
        x[i] = p[0];
        y[i] = p[1];
        z[i] = p[2];
        vx[i] = have_vel ? st[3 * n + c] : 0.0;
        vy[i] = have_vel ? st[4 * n + c] : 0.0;
        vz[i] = have_vel ? st[5 * n + c] : 0.0;
        m[i] = st[6 * n + c];
        ax[i] = acc[c];
        ay[i] = acc[n + c];
        az[i] = acc[2 * n + c];
    }
}

__global__ void k_pack_state(const double* x, const double* y, const double* z,
                             const double* vx, const double* vy, const double* vz,
                             const int* __restrict__ id, int n, float* out, int want_vel)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = id[i];
        out[o] = static_cast<float>(x[i]);
        out[n + o] = static_cast<float>(y[i]);
        out[2 * n + o] = static_cast<float>(z[i]);
        if (want_vel) {
            out[3 * n + o] = static_cast<float>(vx[i]);
            out[4 * n + o] = static_cast<float>(vy[i]);
            out[5 * n + o] = static_cast<float>(vz[i]);
        }
    }
}

__global__ void k_gather_f64(const double* const* __restrict__ src_unused, const double* x,
                             const double* y, const double* z, const double* vx,
                             const double* vy, const double* vz, const int* __restrict__ id,
                             int n, double* out, int want_vel)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = id[i];
        out[o] = x[i];
        out[n + o] = y[i];
        out[2 * n + o] = z[i];
        if (want_vel) {
            out[3 * n + o] = vx[i];
            out[4 * n + o] = vy[i];
            out[5 * n + o] = vz[i];
        }
    }
}

// Six FP64 arrays (x, y, z, vx, vy, vz) by value.
struct Soa6 {
    double* a[6];
};

// FP64 state into caller order, one output array per component (the alternate state buffers
// serve as the staging area between steps: nothing reads them until the next permutation).
__global__ void k_gather_f64_soa(const double* x, const double* y, const double* z,
                                 const double* vx, const double* vy, const double* vz,
                                 const int* __restrict__ id, int n, Soa6 out, int want_vel)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = id[i];
        out.a[0][o] = x[i];
        out.a[1][o] = y[i];
        out.a[2][o] = z[i];
        if (want_vel) {
            out.a[3][o] = vx[i];
            out.a[4][o] = vy[i];
            out.a[5][o] = vz[i];
        }
    }
}

// As k_unpack_state_kept for an FP64 state staged in caller order in `in` (slot i takes caller
// particle id[i]); masses and accelerations staged as FP32 in st (mass at 6n, acc at 7n).
__global__ void k_unpack_state_kept_f64(Soa6 in, const float* __restrict__ st, int n, int have_vel,
                                        double* x, double* y, double* z, double* vx, double* vy,
                                        double* vz, float* m, const int* __restrict__ id,
                                        double box, float* ax, float* ay, float* az)
{
    const float* acc = st + 7 * static_cast<size_t>(n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = id[i];
        double p[3] = {in.a[0][c], in.a[1][c], in.a[2][c]};
        if (box > 0.0)
            for (int a = 0; a < 3; ++a) {
                p[a] -= box * floor(p[a] / box);
                if (p[a] >= box)
                    p[a] = 0.0;
            }
        x[i] = p[0];
        y[i] = p[1];
        z[i] = p[2];
        vx[i] = have_vel ? in.a[3][c] : 0.0;
        vy[i] = have_vel ? in.a[4][c] : 0.0;
        vz[i] = have_vel ? in.a[5][c] : 0.0;
        m[i] = st[6 * n + c];
        ax[i] = acc[c];
        ay[i] = acc[n + c];
        az[i] = acc[2 * n + c];
    }
}

// caller-order FP32 positions + mass (reference mode / key parity)
__global__ void k_caller_xyzm(const double* x, const double* y, const double* z,
                              const float* m, const int* __restrict__ id, int n, float* xyzm,
                              float4* orig)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = id[i];
        const float px = static_cast<float>(x[i]), py = static_cast<float>(y[i]),
                    pz = static_cast<float>(z[i]);
        xyzm[o] = px;
        xyzm[n + o] = py;
        xyzm[2 * n + o] = pz;
        xyzm[3 * n + o] = m[i];
        orig[o] = make_float4(px, py, pz, m[i]);
    }
}

__global__ void k_gather_pos4(const float4* __restrict__ orig, const uint32_t* __restrict__ perm,
                              int n, float4* sorted)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        sorted[i] = orig[perm[i]];
}

__global__ void k_f64_from_f64soa(const double* src, double* dst, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[i];
}

int blocks_for(size_t n) { return static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 8)); }

void drop_graphs(bz_handle* h);

bz_status upload_common(bz_handle* h, size_t n)
{
    if (h->systems > 0) {  // back to a single system: the captured step differs
        h->systems = 0;
        drop_graphs(h);
    }
    h->n = n;
    h->cur = 0;
    h->forces_valid = false;
    h->ad.ready = false;
    h->ref_tree_valid = false;
    return BZ_OK;
}

// Reference mode: caller-order FP32 copy, reference keys + stable sort, one-leaf tree.
void enqueue_reference_order(bz_handle* h)
{
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    count_launch();
    k_caller_xyzm<<<blocks_for(n), 256, 0, h->stream>>>(s[0], s[1], s[2], d.mass[h->cur], d.id[h->cur],
                                                        n, d.ref_xyzm, d.ref_orig);
    launch_keys_reference(d.ref_xyzm, d.ref_xyzm + n, d.ref_xyzm + 2 * n, n, d.bbox32, d.keys,
                          d.perm, h->stream);
    launch_radix_sort(d.keys, d.perm, n, 32, h->sort, d.err, h->stream);
    count_launch();
    k_gather_pos4<<<blocks_for(n), 256, 0, h->stream>>>(d.ref_orig, d.perm, n, d.pos4);
    launch_reference_leaf(d.ref_xyzm, d.ref_xyzm + n, d.ref_xyzm + 2 * n, d.ref_xyzm + 3 * n,
                          d.perm, n, d.ref_hot8, h->stream);
}

} // namespace

extern "C" {

// Downloads the FP64 state in caller order through the alternate state buffers.
static void enqueue_get_f64(bz_handle* h, double* pos, double* vel)
{
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    double* const* alt = d.st[h->cur ^ 1];
    Soa6 out;
    for (int a = 0; a < 6; ++a)
        out.a[a] = alt[a];
    count_launch();
    k_gather_f64_soa<<<blocks_for(n), 256, 0, h->stream>>>(s[0], s[1], s[2], s[3], s[4], s[5],
                                                           d.id[h->cur], static_cast<int>(n), out,
                                                           vel ? 1 : 0);
    for (int a = 0; a < 3; ++a)
        cudaMemcpyAsync(pos + a * n, alt[a], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (vel)
        for (int a = 0; a < 3; ++a)
            cudaMemcpyAsync(vel + a * n, alt[3 + a], n * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream);
}

}  // extern "C"

namespace {

// The drifted positions of the step being enqueued, gathered into caller order and copied to
// the host on io_stream (they stay untouched in buffer `cur` for the rest of the step: the
// permutation writes the other buffer); ev_io marks the copies done.
void enqueue_io_positions(bz_handle* h)
{
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    Soa6 out{};
    for (int a = 0; a < 3; ++a)
        out.a[a] = h->io_pos + a * n;
    cudaEventRecord(h->ev_drift, h->stream);
    cudaStreamWaitEvent(h->io_stream, h->ev_drift, 0);
    count_launch();
    k_gather_f64_soa<<<blocks_for(n), 256, 0, h->io_stream>>>(s[0], s[1], s[2], s[3], s[4], s[5],
                                                              d.id[h->cur], static_cast<int>(n), out, 0);
    for (int a = 0; a < 3; ++a)
        cudaMemcpyAsync(h->io_host_pos + a * n, out.a[a], n * sizeof(double), cudaMemcpyDeviceToHost,
                        h->io_stream);
    cudaEventRecord(h->ev_io, h->io_stream);
}

} // namespace

extern "C" {

// Uploads and unpacks an FP32 state (caller order, buffer 0) on the handle's stream.
static void enqueue_set_state(bz_handle* h, const float* pos, const float* vel, const float* mass,
                              size_t n)
{
    DeviceBuffers& d = h->d;
    cudaMemcpyAsync(d.stage, pos, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (vel)
        cudaMemcpyAsync(d.stage + 3 * n, vel, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(d.stage + 6 * n, mass, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    upload_common(h, n);
    double* const* s = d.st[0];
    count_launch();
    k_unpack_state<<<blocks_for(n), 256, 0, h->stream>>>(d.stage, static_cast<int>(n), vel ? 1 : 0,
                                                         s[0], s[1], s[2], s[3], s[4], s[5],
                                                         d.mass[0], d.id[0],
                                                         periodic(h) ? h->cfg.box_length : 0.0);
}

bz_status bz_set_state(bz_handle* h, const float* pos, const float* vel, const float* mass,
                       size_t n)
{
    if (!h || !pos || !mass || n == 0 || n > h->capacity)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    enqueue_set_state(h, pos, vel, mass, n);
    return check_device(h, "bz_set_state");
}

bz_status bz_set_state_acc(bz_handle* h, const float* pos, const float* vel, const float* mass,
                           const float* acc, size_t n)
{
    if (!h || !pos || !mass || !acc || n == 0 || n > h->capacity)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.adaptive_max_level > 0)
        return fail(h, BZ_UNSUPPORTED, "adaptive steps keep per-particle accelerations of their own");
    cudaSetDevice(h->device);
    DeviceBuffers& d = h->d;
    if (h->n == n && h->systems == 0) {
        // A state of the same size replaces the held one in the device's current particle order
        // (the last sort's): a host round trip of the state then leaves it nearly sorted, and
        // the next step's re-sort and mesh deposit stay on their fast paths.  The result is
        // that of a caller-order upload (the step sorts either way), up to the order of
        // particles with equal keys.
        cudaMemcpyAsync(d.stage, pos, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        if (vel)
            cudaMemcpyAsync(d.stage + 3 * n, vel, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(d.stage + 6 * n, mass, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(d.stage + 7 * n, acc, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        h->ad.ready = false;
        h->ref_tree_valid = false;
        double* const* s = d.st[h->cur];
        count_launch();
        k_unpack_state_kept<<<blocks_for(n), 256, 0, h->stream>>>(
            d.stage, static_cast<int>(n), vel ? 1 : 0, s[0], s[1], s[2], s[3], s[4], s[5],
            d.mass[h->cur], d.id[h->cur], periodic(h) ? h->cfg.box_length : 0.0, d.acc[0], d.acc[1],
            d.acc[2]);
    } else {
        enqueue_set_state(h, pos, vel, mass, n);
        // the state sits in caller order now (buffer 0, identity ids): so do the accelerations
        for (int a = 0; a < 3; ++a)
            cudaMemcpyAsync(d.acc[a], acc + a * n, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    }
    const bz_status st = check_device(h, "bz_set_state_acc");
    if (st == BZ_OK)
        h->forces_valid = true;
    return st;
}

bz_status bz_set_state_f64(bz_handle* h, const double* pos, const double* vel, const float* mass,
                           size_t n)
{
    if (!h || !pos || !mass || n == 0 || n > h->capacity)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    DeviceBuffers& d = h->d;
    double* const* s = d.st[0];
    for (int a = 0; a < 3; ++a) {
        cudaMemcpyAsync(s[a], pos + a * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        if (vel)
            cudaMemcpyAsync(s[3 + a], vel + a * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        else
            cudaMemsetAsync(s[3 + a], 0, n * sizeof(double), h->stream);
    }
    cudaMemcpyAsync(d.stage + 6 * n, mass, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(d.mass[0], mass, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    upload_common(h, n);
    std::vector<int> ids(n);
    for (size_t i = 0; i < n; ++i)
        ids[i] = static_cast<int>(i);
    cudaMemcpyAsync(d.id[0], ids.data(), n * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    return check_device(h, "bz_set_state_f64");
}

bz_status bz_set_ensemble(bz_handle* h, const double* pos, const double* vel, const float* mass,
                          const int64_t* offsets, int32_t systems)
{
    if (!h || !pos || !mass || !offsets || systems < 1 || systems > kMaxSystems)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver != BZ_SOLVER_OCTREE)
        return fail(h, BZ_UNSUPPORTED, "bz_set_ensemble: ensembles run on the octree solver");
    if (offsets[0] != 0)
        return fail(h, BZ_INVALID_ARGUMENT, "bz_set_ensemble: offsets[0] must be 0");
    for (int s = 0; s < systems; ++s)
        if (offsets[s + 1] <= offsets[s])
            return fail(h, BZ_INVALID_ARGUMENT, "bz_set_ensemble: every system needs a particle");
    const size_t n = static_cast<size_t>(offsets[systems]);
    if (n > h->capacity || n > static_cast<size_t>(INT32_MAX))
        return BZ_INVALID_ARGUMENT;
    bz_status st = bz_set_state_f64(h, pos, vel, mass, n);
    if (st != BZ_OK)
        return st;
    if (!h->sys_offsets && (!dalloc(h, &h->sys_offsets, kMaxSystems + 1) ||
                            !dalloc(h, &h->sys_boxes, kMaxSystems)))
        return fail(h, BZ_OUT_OF_MEMORY, "bz_set_ensemble");
    h->host_offsets.assign(offsets, offsets + systems + 1);
    cudaMemcpyAsync(h->sys_offsets, h->host_offsets.data(), sizeof(long long) * (systems + 1),
                    cudaMemcpyHostToDevice, h->stream);
    h->systems = systems;
    drop_graphs(h);
    return check_device(h, "bz_set_ensemble");
}

bz_status bz_get_state(bz_handle* h, float* pos, float* vel)
{
    if (!h || !pos || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    count_launch();
    k_pack_state<<<blocks_for(n), 256, 0, h->stream>>>(s[0], s[1], s[2], s[3], s[4], s[5], d.id[h->cur],
                                                       static_cast<int>(n), d.stage, vel ? 1 : 0);
    cudaMemcpyAsync(pos, d.stage, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (vel)
        cudaMemcpyAsync(vel, d.stage + 3 * n, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_get_state");
}

bz_status bz_get_state_acc(bz_handle* h, float* pos, float* vel, float* acc)
{
    if (!h || !pos || !acc || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    if (h->cfg.adaptive_max_level > 0)
        return fail(h, BZ_UNSUPPORTED, "adaptive steps keep per-particle accelerations of their own");
    bz_status st = ensure_forces(h);
    if (st != BZ_OK)
        return st;
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    double* const* s = d.st[h->cur];
    count_launch();
    k_pack_state<<<blocks_for(n), 256, 0, h->stream>>>(s[0], s[1], s[2], s[3], s[4], s[5], d.id[h->cur],
                                                       static_cast<int>(n), d.stage, vel ? 1 : 0);
    launch_scatter3(d.acc[0], d.acc[1], d.acc[2], d.id[h->cur], static_cast<int>(n), d.stage + 6 * n,
                    h->stream);
    // the three copies follow each other without a kernel between them
    cudaMemcpyAsync(pos, d.stage, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (vel)
        cudaMemcpyAsync(vel, d.stage + 3 * n, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(acc, d.stage + 6 * n, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_get_state_acc");
}

bz_status bz_get_state_f64(bz_handle* h, double* pos, double* vel)
{
    if (!h || !pos || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    enqueue_get_f64(h, pos, vel);
    return check_device(h, "bz_get_state_f64");
}

bz_status bz_get_state_acc_f64(bz_handle* h, double* pos, double* vel, float* acc)
{
    if (!h || !pos || !acc || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    if (h->cfg.adaptive_max_level > 0)
        return fail(h, BZ_UNSUPPORTED, "adaptive steps keep per-particle accelerations of their own");
    bz_status st = ensure_forces(h);
    if (st != BZ_OK)
        return st;
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    launch_scatter3(d.acc[0], d.acc[1], d.acc[2], d.id[h->cur], static_cast<int>(n), d.stage + 6 * n,
                    h->stream);
    enqueue_get_f64(h, pos, vel);
    cudaMemcpyAsync(acc, d.stage + 6 * n, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_get_state_acc_f64");
}

bz_status bz_step_get_state_acc_f64(bz_handle* h, double dt, double* pos, double* vel, float* acc)
{
    if (!h || !pos || !vel || !acc || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE)
        return fail(h, BZ_UNSUPPORTED, "the reference formulation is a parity mode; step with BZ_SOLVER_OCTREE");
    if (h->cfg.adaptive_max_level > 0)
        return fail(h, BZ_UNSUPPORTED, "adaptive steps keep per-particle accelerations of their own");
    cudaSetDevice(h->device);
    if (!h->io_stream) {
        if (cudaStreamCreateWithFlags(&h->io_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_drift, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_io, cudaEventDisableTiming) != cudaSuccess)
            return fail(h, BZ_CUDA_ERROR, "bz_step_get_state_acc_f64: stream or events");
        if (!dalloc(h, &h->io_pos, 3 * h->capacity))
            return fail(h, BZ_OUT_OF_MEMORY, "bz_step_get_state_acc_f64: position staging");
    }
    h->h_dt[0] = dt;
    h->h_dt[1] = 0.5 * dt;
    cudaMemcpyAsync(h->d.dt, h->h_dt, 2 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    bz_status s = ensure_forces(h);
    if (s != BZ_OK)
        return s;
    h->stepping = true;
    // one step enqueued eagerly, so that the position download can start inside it
    const bool timing = h->timing;
    h->timing = false;
    h->io_host_pos = pos;
    enqueue_step(h);
    h->io_host_pos = nullptr;
    h->timing = timing;
    // velocities and accelerations of the step's end; the alternate state buffer that stages
    // the velocities is the one io_stream reads positions from, so wait for it first
    cudaStreamWaitEvent(h->stream, h->ev_io, 0);
    const size_t n = h->n;
    DeviceBuffers& d = h->d;
    launch_scatter3(d.acc[0], d.acc[1], d.acc[2], d.id[h->cur], static_cast<int>(n), d.stage + 6 * n,
                    h->stream);
    double* const* st = d.st[h->cur];
    double* const* alt = d.st[h->cur ^ 1];
    Soa6 out{};
    for (int a = 0; a < 3; ++a)
        out.a[a] = alt[3 + a];
    count_launch();
    k_gather_f64_soa<<<blocks_for(n), 256, 0, h->stream>>>(st[3], st[4], st[5], st[3], st[4], st[5],
                                                           d.id[h->cur], static_cast<int>(n), out, 0);
    for (int a = 0; a < 3; ++a)
        cudaMemcpyAsync(vel + a * n, alt[3 + a], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(acc, d.stage + 6 * n, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    s = check_device(h, "bz_step_get_state_acc_f64");
    if (s != BZ_OK)
        return s;
    read_counters(h);
    return BZ_OK;
}

bz_status bz_set_state_acc_f64(bz_handle* h, const double* pos, const double* vel, const float* mass,
                               const float* acc, size_t n)
{
    if (!h || !pos || !mass || !acc || n == 0 || n > h->capacity)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.adaptive_max_level > 0)
        return fail(h, BZ_UNSUPPORTED, "adaptive steps keep per-particle accelerations of their own");
    cudaSetDevice(h->device);
    DeviceBuffers& d = h->d;
    if (h->n == n && h->systems == 0) {
        // as bz_set_state_acc: a state of the same size keeps the device's particle order; the
        // FP64 arrays are staged in caller order in the alternate state buffers
        double* const* alt = d.st[h->cur ^ 1];
        Soa6 in;
        for (int a = 0; a < 3; ++a) {
            in.a[a] = alt[a];
            in.a[3 + a] = alt[3 + a];
            cudaMemcpyAsync(alt[a], pos + a * n, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
            if (vel)
                cudaMemcpyAsync(alt[3 + a], vel + a * n, n * sizeof(double), cudaMemcpyHostToDevice,
                                h->stream);
        }
        cudaMemcpyAsync(d.stage + 6 * n, mass, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(d.stage + 7 * n, acc, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
        h->ad.ready = false;
        h->ref_tree_valid = false;
        double* const* s = d.st[h->cur];
        count_launch();
        k_unpack_state_kept_f64<<<blocks_for(n), 256, 0, h->stream>>>(
            in, d.stage, static_cast<int>(n), vel ? 1 : 0, s[0], s[1], s[2], s[3], s[4], s[5],
            d.mass[h->cur], d.id[h->cur], periodic(h) ? h->cfg.box_length : 0.0, d.acc[0], d.acc[1],
            d.acc[2]);
    } else {
        const bz_status st0 = bz_set_state_f64(h, pos, vel, mass, n);
        if (st0 != BZ_OK)
            return st0;
        // caller order now (buffer 0, identity ids): so are the accelerations
        for (int a = 0; a < 3; ++a)
            cudaMemcpyAsync(d.acc[a], acc + a * n, n * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    }
    const bz_status st = check_device(h, "bz_set_state_acc_f64");
    if (st == BZ_OK)
        h->forces_valid = true;
    return st;
}

bz_status bz_enable_phase_timing(bz_handle* h, int enable)
{
    if (!h)
        return BZ_INVALID_ARGUMENT;
    h->timing = enable != 0;
    return BZ_OK;
}

bz_status bz_phase_times(bz_handle* h, float* ms, int n)
{
    if (!h || !ms)
        return BZ_INVALID_ARGUMENT;
    for (int i = 0; i < n && i < kNumPhases; ++i)
        ms[i] = h->phase_ms[i];
    return BZ_OK;
}

bz_status bz_interaction_counts(bz_handle* h, uint64_t* n_pp, uint64_t* n_pn)
{
    if (!h)
        return BZ_INVALID_ARGUMENT;
    if (n_pp)
        *n_pp = h->last_pp;
    if (n_pn)
        *n_pn = h->last_pn;
    return BZ_OK;
}

bz_status bz_walk_counts(bz_handle* h, uint64_t* listed_pairs, uint64_t* evaluated_pairs,
                         uint64_t* node_terms)
{
    if (!h)
        return BZ_INVALID_ARGUMENT;
    if (listed_pairs)
        *listed_pairs = h->last_pp;
    if (evaluated_pairs)
        *evaluated_pairs = h->last_eval;
    if (node_terms)
        *node_terms = h->last_pn;
    return BZ_OK;
}

bz_status bz_accelerations(bz_handle* h, float* acc, float* pot)
{
    if (!h || !acc || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE) {
        if (pot)
            return fail(h, BZ_UNSUPPORTED, "potentials are not part of the reference formulation");
        enqueue_reference_order(h);
        const float eps = std::max(h->cfg.octree_softening, h->cfg.physics_min_softening);
        launch_reference_walk(d.ref_orig, d.pos4, d.perm, n, eps, h->cfg.physics_min_distance2, 0.0f,
                              0.0f, h->cfg.physics_max_acceleration, d.stage, d.stage + n,
                              d.stage + 2 * n, h->stream);
        cudaMemcpyAsync(acc, d.stage, 3 * static_cast<size_t>(n) * sizeof(float),
                        cudaMemcpyDeviceToHost, h->stream);
        bz_status s = check_device(h, "bz_accelerations (reference)");
        if (s == BZ_OK)
            h->ref_tree_valid = true;
        return s;
    }
    h->stepping = false;
    enqueue_order(h);
    enqueue_forces(h, false, pot != nullptr);
    record(h, kNumPhases);
    launch_scatter3(d.acc[0], d.acc[1], d.acc[2], d.id[h->cur], n, d.stage, h->stream);
    cudaMemcpyAsync(acc, d.stage, 3 * static_cast<size_t>(n) * sizeof(float), cudaMemcpyDeviceToHost,
                    h->stream);
    if (pot) {
        launch_scatter3(d.pot, d.pot, d.pot, d.id[h->cur], n, d.stage + 3 * n, h->stream);
        cudaMemcpyAsync(pot, d.stage + 3 * n, static_cast<size_t>(n) * sizeof(float),
                        cudaMemcpyDeviceToHost, h->stream);
    }
    bz_status s = check_device(h, "bz_accelerations");
    if (s != BZ_OK)
        return s;
    collect_timing(h);
    read_counters(h);
    h->forces_valid = true;
    return BZ_OK;
}

bz_status bz_energy(bz_handle* h, double* kinetic, double* potential, double* momentum3)
{
    if (!h || h->n == 0 || (!kinetic && !potential && !momentum3))
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE)
        return fail(h, BZ_UNSUPPORTED, "energies are not part of the reference formulation");
    if (potential && h->cfg.solver == BZ_SOLVER_TREEPM)
        return fail(h, BZ_UNSUPPORTED, "bz_energy: the TreePM mesh leg has no potential output");
    cudaSetDevice(h->device);
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    h->stepping = false;
    if (potential) {
        enqueue_order(h);
        enqueue_forces(h, false, true);
    }
    double* const* st = d.st[h->cur];
    launch_energy(st[3], st[4], st[5], d.mass[h->cur], potential ? d.pot : nullptr, n, d.energy,
                  h->stream);
    double out[5] = {};
    cudaMemcpyAsync(out, d.energy + energy_scratch_doubles() - 8, 5 * sizeof(double),
                    cudaMemcpyDeviceToHost, h->stream);
    const bz_status s = check_device(h, "bz_energy");
    if (s != BZ_OK)
        return s;
    if (potential)
        h->forces_valid = true;
    if (kinetic)
        *kinetic = out[0];
    if (potential)
        *potential = out[1];
    if (momentum3) {
        momentum3[0] = out[2];
        momentum3[1] = out[3];
        momentum3[2] = out[4];
    }
    return BZ_OK;
}

} // extern "C"

namespace {

AdaptiveParams adaptive_params(const bz_handle* h, double dt)
{
    AdaptiveParams p{};
    p.dt_max = dt;
    p.eta = h->cfg.adaptive_eta;
    p.eps = std::max(h->cfg.octree_softening, h->cfg.physics_min_softening);
    p.max_level = h->cfg.adaptive_max_level;
    return p;
}

// Block steps with power-of-two levels (the kernels in bz_adaptive.cu describe the scheme).
// The forces of the current state are valid on entry (ensure_forces).
bz_status adaptive_steps(bz_handle* h, double dt, uint32_t nsteps)
{
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    const AdaptiveParams p = adaptive_params(h, dt);
    if (!h->ad.ready) {
        double* const* st = d.st[h->cur];
        cudaMemsetAsync(h->ad.st.updates, 0, sizeof(unsigned long long), h->stream);
        launch_adaptive_init(d.acc[0], d.acc[1], d.acc[2], st[3], st[4], st[5], d.id[h->cur], n, p,
                             h->ad.st, h->stream);
        h->ad.ready = true;
    }
    for (uint32_t b = 0; b < nsteps; ++b) {
        launch_level_max(h->ad.st.level, n, h->ad.lmax, h->stream);
        int L = 0;
        cudaMemcpyAsync(&L, h->ad.lmax, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
            return check_device(h, "bz_step (adaptive)");
        L = std::min(std::max(L, 0), h->cfg.adaptive_max_level);
        // The first substep of a block drifts, sorts and builds the tree as a plain step does;
        // later substeps keep that topology, drift the particles inside it and refit every
        // node's box and moments bottom-up (the walk needs correct ranges, boxes and moments,
        // not Morton-consistent cells).
        const int root_level = h->systems > 0 ? kSystemLevels : 0;
        for (int sub = 0; sub < (1 << L); ++sub) {
            record(h, kEvStepStart);
            {
                double* const* st = d.st[h->cur];
                launch_adaptive_open_drift(st[0], st[1], st[2], st[3], st[4], st[5], d.id[h->cur], n,
                                           p, h->ad.st, sub, L, h->stream);
            }
            if (sub == 0) {
                enqueue_order(h);
                record(h, kPhTree);
                launch_tree_build(d.keys, d.pos4, n, h->cfg.leaf_capacity, kMaxLevels, h->tree, d.err,
                                  h->stream, root_level, h->cfg.multipole_order >= 2);
                launch_groups(h->tree, n, h->cfg.walk_group_size, root_level, d.keys, h->groups,
                              h->stream);
            } else {
                double* const* st = d.st[h->cur];
                record(h, kPhKeys);
                record(h, kPhSort);
                record(h, kPhPermute);
                launch_refresh_pos4(st[0], st[1], st[2], d.mass[h->cur], n, d.pos4, h->stream);
                record(h, kPhTree);
                launch_tree_refit(d.pos4, h->tree, h->stream, h->cfg.multipole_order >= 2);
            }
            double* const* st = d.st[h->cur];
            launch_adaptive_active(d.id[h->cur], n, h->ad.st, sub, L, h->ad.active, h->stream);
            record(h, kPhMesh);
            for (int a = 0; a < 3; ++a)
                cudaMemsetAsync(d.acc[a], 0, sizeof(float) * n, h->stream);
            record(h, kPhWalk);
            cudaMemsetAsync(d.counters, 0, 3 * sizeof(unsigned long long), h->stream);
            WalkOutputs o{};
            o.ax = d.acc[0];
            o.ay = d.acc[1];
            o.az = d.acc[2];
            o.totals = d.counters;
            WalkParams wp = walk_params(h, false);
            wp.active = h->ad.active;
            launch_walk(d.pos4, n, h->tree, h->groups, wp, o, d.queue, d.spill, d.err, h->stream);
            record(h, kPhIntegrate);
            launch_adaptive_close(d.acc[0], d.acc[1], d.acc[2], st[3], st[4], st[5], d.id[h->cur],
                                  h->ad.active, n, p, h->ad.st, sub, L, h->stream);
        }
    }
    // d.acc holds only the closing particles of the last substep: re-evaluate before a plain step
    h->forces_valid = false;
    if (h->timing)
        record(h, kNumPhases);
    const bz_status s = check_device(h, "bz_step (adaptive)");
    if (s != BZ_OK)
        return s;
    collect_timing(h);  // phases of the last substep
    read_counters(h);
    return BZ_OK;
}

} // namespace

extern "C" {

bz_status bz_adaptive_levels(bz_handle* h, uint8_t* levels)
{
    if (!h || !levels || h->cfg.adaptive_max_level <= 0 || !h->ad.ready)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    cudaMemcpyAsync(levels, h->ad.st.level, h->n, cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_adaptive_levels");
}

bz_status bz_adaptive_updates(bz_handle* h, uint64_t* updates)
{
    if (!h || !updates || h->cfg.adaptive_max_level <= 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    unsigned long long u = 0;
    if (h->ad.ready)
        cudaMemcpyAsync(&u, h->ad.st.updates, sizeof(u), cudaMemcpyDeviceToHost, h->stream);
    const bz_status s = check_device(h, "bz_adaptive_updates");
    *updates = u;
    return s;
}

bz_status bz_step(bz_handle* h, double dt, uint32_t nsteps)
{
    if (!h || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE)
        return fail(h, BZ_UNSUPPORTED, "the reference formulation is a parity mode; step with BZ_SOLVER_OCTREE");
    if (nsteps == 0)
        return BZ_OK;
    cudaSetDevice(h->device);
    h->h_dt[0] = dt;
    h->h_dt[1] = 0.5 * dt;
    cudaMemcpyAsync(h->d.dt, h->h_dt, 2 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    // adaptive block steps carry their own cached accelerations once started
    bz_status s = (h->cfg.adaptive_max_level > 0 && h->ad.ready) ? BZ_OK : ensure_forces(h);
    if (s != BZ_OK)
        return s;
    h->stepping = true;
    if (h->cfg.adaptive_max_level > 0)
        return adaptive_steps(h, dt, nsteps);
    uint32_t done = 0;
    if (h->cfg.use_graph && !h->timing) {
        build_graphs(h);
        if (!h->graph_failed)
            for (; done < nsteps; ++done) {
                cudaGraphLaunch(h->graph[h->cur], h->stream);
                h->cur ^= 1;
            }
    }
    for (; done < nsteps; ++done) {
        record(h, kEvStepStart);
        enqueue_step(h);
    }
    if (h->timing)
        record(h, kNumPhases);
    s = check_device(h, "bz_step");
    if (s != BZ_OK)
        return s;
    collect_timing(h);
    read_counters(h);
    return BZ_OK;
}

bz_status bz_walk_blocks_per_sm(bz_handle* h, int32_t set_value, int32_t* current)
{
    if (!h || set_value > 64)
        return BZ_INVALID_ARGUMENT;
    if (set_value >= 0 && set_value != h->walk_blocks_per_sm) {
        h->walk_blocks_per_sm = set_value;
        for (int i = 0; i < 2; ++i) {  // captured steps hold the old grid
            if (h->graph[i])
                cudaGraphExecDestroy(h->graph[i]);
            h->graph[i] = nullptr;
        }
    }
    if (current)
        *current = h->walk_blocks_per_sm;
    return BZ_OK;
}

bz_status bz_set_mesh_schedule(bz_handle* h, int32_t schedule)
{
    if (!h || schedule < 0 || schedule > 2)
        return BZ_INVALID_ARGUMENT;
    if (h->mesh_overlap != schedule) {
        h->mesh_overlap = schedule;
        for (int i = 0; i < 2; ++i) {  // captured steps hold the old schedule
            if (h->graph[i])
                cudaGraphExecDestroy(h->graph[i]);
            h->graph[i] = nullptr;
        }
    }
    return BZ_OK;
}

bz_status bz_autotune(bz_handle* h, int32_t trials, int32_t* leaf_capacity, int32_t* group_size,
                      float* ms_per_evaluation, int32_t* mesh_overlap)
{
    if (!h || h->n == 0 || trials < 1)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE)
        return fail(h, BZ_UNSUPPORTED, "the reference formulation has nothing to tune");
    cudaSetDevice(h->device);
    static const int kLeaf[] = {8, 12, 16, 24, 32, 48};
    static const int kGroup[] = {16, 24, 32};
    const int leaf0 = h->cfg.leaf_capacity, group0 = h->cfg.walk_group_size;
    const int overlap0 = h->mesh_overlap, bps0 = h->walk_blocks_per_sm;
    const int n_overlap = h->pm_stream ? 3 : 1;  // TreePM: the three mesh-leg schedules
    const bool timing0 = h->timing;
    h->timing = false;
    h->stepping = false;
    // The timed unit is a step of zero length (drift, order, forces, kick): it leaves positions
    // and velocities unchanged (x + 0 v, v + 0 a with finite forces of the current state), and
    // it is the unit in which the mesh schedules differ.
    bz_status st = ensure_forces(h);
    if (st != BZ_OK)
        return st;
    cudaMemsetAsync(h->d.dt, 0, 2 * sizeof(double), h->stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // ms per zero-length step with the handle's current parameters, launched the way bz_step
    // launches them: as a captured graph (two steps, so the state buffers end where they began)
    // unless the handle steps eagerly
    auto time_steps = [&](float* ms) -> bz_status {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ex = nullptr;
        bool graph = h->cfg.use_graph && !h->graph_failed;
        if (graph) {
            if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                enqueue_step(h);
                enqueue_step(h);
                if (cudaStreamEndCapture(h->stream, &g) != cudaSuccess || !g ||
                    cudaGraphInstantiate(&ex, g, 0) != cudaSuccess)
                    graph = false;
            } else {
                graph = false;
            }
            if (!graph) {
                if (g)
                    cudaGraphDestroy(g);
                g = nullptr;
                cudaGetLastError();
            }
        }
        auto run = [&]() {
            if (graph) {
                cudaGraphLaunch(ex, h->stream);
            } else {
                enqueue_step(h);
                enqueue_step(h);
            }
        };
        run();  // warm-up with these parameters
        cudaEventRecord(e0, h->stream);
        for (int r = 0; r < trials; ++r)
            run();
        cudaEventRecord(e1, h->stream);
        const bz_status rc = check_device(h, "bz_autotune");
        if (ex)
            cudaGraphExecDestroy(ex);
        if (g)
            cudaGraphDestroy(g);
        if (rc != BZ_OK)
            return rc;
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= static_cast<float>(2 * trials);
        return BZ_OK;
    };
    float best = -1.0f;
    int best_leaf = leaf0, best_group = group0;
    int best_overlap = overlap0, best_bps = bps0;
    // stage 1: leaf capacity x walk group size
    for (int leaf : kLeaf) {
        for (int group : kGroup) {
            h->cfg.leaf_capacity = leaf;
            h->cfg.walk_group_size = group;
            float ms = 0.0f;
            st = time_steps(&ms);
            if (st != BZ_OK)
                break;
            if (best < 0.0f || ms < best) {
                best = ms;
                best_leaf = leaf;
                best_group = group;
            }
        }
        if (st != BZ_OK)
            break;
    }
    // stage 2 (TreePM with the second stream): mesh schedule x cap on resident walk blocks per
    // SM (the walk holds every SM's registers; a lower cap lets the mesh kernels co-run)
    if (st == BZ_OK && n_overlap > 1) {
        static const int kBps[] = {0, 6, 5};
        h->cfg.leaf_capacity = best_leaf;
        h->cfg.walk_group_size = best_group;
        for (int ov = 0; ov < n_overlap && st == BZ_OK; ++ov) {
            for (int bps : kBps) {
                if (ov == 0 && bps != 0)
                    continue;  // in line: nothing runs beside the walk
                h->mesh_overlap = ov;
                h->walk_blocks_per_sm = bps;
                float ms = 0.0f;
                st = time_steps(&ms);
                if (st != BZ_OK)
                    break;
                if (ms < best) {
                    best = ms;
                    best_overlap = ov;
                    best_bps = bps;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->timing = timing0;
    h->cfg.leaf_capacity = st == BZ_OK ? best_leaf : leaf0;
    h->cfg.walk_group_size = st == BZ_OK ? best_group : group0;
    h->mesh_overlap = st == BZ_OK ? best_overlap : overlap0;
    h->walk_blocks_per_sm = st == BZ_OK ? best_bps : bps0;
    // the captured step holds the old parameters: capture again on the next bz_step
    for (int i = 0; i < 2; ++i) {
        if (h->graph[i])
            cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
    }
    h->forces_valid = false;
    if (st != BZ_OK)
        return st;
    if (leaf_capacity)
        *leaf_capacity = best_leaf;
    if (group_size)
        *group_size = best_group;
    if (ms_per_evaluation)
        *ms_per_evaluation = best;
    if (mesh_overlap)
        *mesh_overlap = best_overlap;
    return BZ_OK;
}

} // extern "C"

namespace {

bool learn_alloc(bz_handle* h)
{
    auto& L = h->learn;
    if (L.params)
        return true;
    return dalloc(h, &L.params, kMlpParams) && dalloc(h, &L.grad, kMlpParams) &&
           dalloc(h, &L.adam_m, kMlpParams) && dalloc(h, &L.adam_v, kMlpParams) &&
           dalloc(h, &L.loss, 1);
}

bool learn_pairs_alloc(bz_handle* h)
{
    auto& L = h->learn;
    if (L.pair_src)
        return true;
    return dalloc(h, &L.pair_src, h->capacity * static_cast<size_t>(kPairSlots)) &&
           dalloc(h, &L.pair_cnt, h->capacity);
}

void drop_graphs(bz_handle* h)
{
    for (int i = 0; i < 2; ++i) {
        if (h->graph[i])
            cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
    }
    h->forces_valid = false;
}

// Xavier-style uniform initialisation of the MLP parameters (seeded)
std::vector<float> learn_init(uint64_t seed)
{
    std::vector<float> p(kMlpParams, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols) {
        const float a = std::sqrt(6.0f / static_cast<float>(rows + cols));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < rows * cols; ++i)
            p[off + i] = u(rng);
    };
    fill(kMlpOffW1, 32, 16);
    for (int r = 0; r < 32; ++r)
        p[kMlpOffW1 + r * 16 + 15] = 0.0f;  // b1
    fill(kMlpOffW2, 32, 32);
    fill(kMlpOffW3, 3, 32);
    return p;
}

template <class T> struct DevBuf {
    T* p = nullptr;
    explicit DevBuf(size_t n) { cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
    ~DevBuf() { cudaFree(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

} // namespace

extern "C" {

bz_status bz_learn_generate(bz_handle* h, int64_t nsamples, uint64_t seed, float* x6, float* y3)
{
    if (!h || nsamples <= 0 || !x6 || !y3)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver != BZ_SOLVER_TREEPM || !h->pm || isolated(h))
        return fail(h, BZ_UNSUPPORTED, "bz_learn_generate: residuals are defined for the periodic TreePM solver");
    cudaSetDevice(h->device);
    const int M = h->cfg.treepm_grid_size;
    const double L = h->cfg.box_length, hc = L / M;
    const double rs = rsplit_len(h);
    const double R = learn_radius_cells(h);  // probe ball radius in cells
    h->learn.radius_cells = static_cast<float>(R);
    // sources on a coarse lattice, far enough apart that each probe's mesh error comes from
    // its own source; probes uniformly in the ball of radius r_cut around each source
    int sp = std::max(16, 2 * static_cast<int>(std::ceil(R)) + 8);
    int per_axis = std::max(1, M / sp);
    sp = M / per_axis;
    const int S = per_axis * per_axis * per_axis;
    const int P = static_cast<int>(std::min<int64_t>(256, (nsamples + S - 1) / S));
    const int batch = S * P;
    const int ntot = S + batch;
    DevBuf<float4> dpos(ntot);
    DevBuf<float> dacc(3 * static_cast<size_t>(ntot));
    DevBuf<int> dtg(batch);
    DevBuf<double> dlr(3 * static_cast<size_t>(batch));
    const int kmax = 8;
    DevBuf<double> dsk(5 * static_cast<size_t>(ewald_num_k(kmax)));
    if (!dpos.p || !dacc.p || !dtg.p || !dlr.p || !dsk.p)
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_generate: temporary buffers");
    std::vector<int> tg(batch);
    for (int i = 0; i < batch; ++i)
        tg[i] = S + i;
    cudaMemcpyAsync(dtg.p, tg.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, h->stream);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::normal_distribution<double> G(0.0, 1.0);
    std::vector<float4> pos(ntot);
    std::vector<double> off(3 * static_cast<size_t>(S)), sep(3 * static_cast<size_t>(batch));
    std::vector<float> acc(3 * static_cast<size_t>(ntot));
    std::vector<double> lr(3 * static_cast<size_t>(batch));
    int64_t done = 0;
    while (done < nsamples) {
        for (int a = 0; a < per_axis; ++a)
            for (int b = 0; b < per_axis; ++b)
                for (int c = 0; c < per_axis; ++c) {
                    const int sidx = (a * per_axis + b) * per_axis + c;
                    const int cell[3] = {a * sp + sp / 2, b * sp + sp / 2, c * sp + sp / 2};
                    double q[3];
                    for (int k = 0; k < 3; ++k) {
                        off[3 * sidx + k] = U(rng);
                        q[k] = (cell[k] + off[3 * sidx + k]) * hc;
                    }
                    pos[sidx] = make_float4(static_cast<float>(q[0]), static_cast<float>(q[1]),
                                            static_cast<float>(q[2]), 1.0f);
                }
        for (int sidx = 0; sidx < S; ++sidx)
            for (int j = 0; j < P; ++j) {
                double u[3], nrm = 0.0;
                for (int k = 0; k < 3; ++k) {
                    u[k] = G(rng);
                    nrm += u[k] * u[k];
                }
                nrm = std::sqrt(nrm);
                const double r = std::max(0.02, R * std::cbrt(U(rng)));
                const int pi = sidx * P + j;
                double q[3];
                const float4 sp4 = pos[sidx];
                const double sq[3] = {sp4.x, sp4.y, sp4.z};
                for (int k = 0; k < 3; ++k) {
                    double v = sq[k] + u[k] / nrm * r * hc;
                    v -= L * std::floor(v / L);
                    q[k] = v;
                }
                pos[S + pi] = make_float4(static_cast<float>(q[0]), static_cast<float>(q[1]),
                                          static_cast<float>(q[2]), 0.0f);
                for (int k = 0; k < 3; ++k) {
                    double d = static_cast<double>((k == 0 ? pos[S + pi].x : k == 1 ? pos[S + pi].y
                                                                                     : pos[S + pi].z)) - sq[k];
                    d -= L * std::nearbyint(d / L);
                    sep[3 * static_cast<size_t>(pi) + k] = d / hc;
                }
            }
        cudaMemcpyAsync(dpos.p, pos.data(), sizeof(float4) * ntot, cudaMemcpyHostToDevice, h->stream);
        pm_forces(h->pm, dpos.p, ntot, dacc.p, dacc.p + ntot, dacc.p + 2 * static_cast<size_t>(ntot), h->stream);
        launch_lr_ideal_f64(dpos.p, S, dtg.p, batch, L, 6.4 / L, kmax, rs, dsk.p, dlr.p, h->stream);
        cudaMemcpyAsync(acc.data(), dacc.p, sizeof(float) * 3 * static_cast<size_t>(ntot),
                        cudaMemcpyDeviceToHost, h->stream);
        cudaMemcpyAsync(lr.data(), dlr.p, sizeof(double) * 3 * static_cast<size_t>(batch),
                        cudaMemcpyDeviceToHost, h->stream);
        const bz_status st = check_device(h, "bz_learn_generate");
        if (st != BZ_OK)
            return st;
        const int64_t take = std::min<int64_t>(batch, nsamples - done);
        for (int64_t i = 0; i < take; ++i) {
            const int sidx = static_cast<int>(i / P);
            const int64_t o = done + i;
            for (int k = 0; k < 3; ++k) {
                x6[6 * o + k] = static_cast<float>(sep[3 * i + k]);
                x6[6 * o + 3 + k] = static_cast<float>(off[3 * sidx + k]);
                const double fpm = acc[static_cast<size_t>(k) * ntot + S + i];
                y3[3 * o + k] = static_cast<float>((fpm - lr[3 * i + k]) * hc * hc);
            }
        }
        done += take;
    }
    return BZ_OK;
}

bz_status bz_learn_set(bz_handle* h, const float* params, float scale)
{
    if (!h || !params || !(scale > 0.0f))
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    if (!learn_alloc(h) || (h->cfg.solver == BZ_SOLVER_TREEPM && !learn_pairs_alloc(h)))
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_set");
    cudaMemcpyAsync(h->learn.params, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, h->stream);
    h->learn.scale = scale;
    h->learn.trained = true;
    drop_graphs(h);
    return check_device(h, "bz_learn_set");
}

bz_status bz_learn_get(bz_handle* h, float* params, float* scale)
{
    if (!h || !params || !h->learn.trained)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    cudaMemcpyAsync(params, h->learn.params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, h->stream);
    if (scale)
        *scale = h->learn.scale;
    return check_device(h, "bz_learn_get");
}

bz_status bz_learn_enable(bz_handle* h, int32_t enable)
{
    if (!h)
        return BZ_INVALID_ARGUMENT;
    if (enable && (!h->learn.trained || h->cfg.solver != BZ_SOLVER_TREEPM))
        return fail(h, BZ_NOT_READY, "bz_learn_enable: no trained correction for a TreePM handle");
    h->learn.enabled = enable != 0;
    drop_graphs(h);
    return BZ_OK;
}

bz_status bz_learn_train(bz_handle* h, const float* x6, const float* y3, int64_t n, int32_t steps,
                         int32_t batch, float lr, uint64_t seed, float* final_loss)
{
    if (!h || !x6 || !y3 || n < batch || steps < 1 || batch < 128 || batch % 128 != 0 || !(lr > 0.0f))
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    if (!learn_alloc(h) || (h->cfg.solver == BZ_SOLVER_TREEPM && !learn_pairs_alloc(h)))
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_train");
    double ss = 0.0;
    for (int64_t i = 0; i < 3 * n; ++i)
        ss += static_cast<double>(y3[i]) * y3[i];
    const float scale = static_cast<float>(std::sqrt(ss / (3.0 * n)));
    if (!(scale > 0.0f))
        return fail(h, BZ_INVALID_ARGUMENT, "bz_learn_train: all targets are zero");
    std::vector<float> yn(3 * static_cast<size_t>(n));
    for (int64_t i = 0; i < 3 * n; ++i)
        yn[i] = y3[i] / scale;
    DevBuf<float> dx(6 * static_cast<size_t>(n)), dy(3 * static_cast<size_t>(n));
    DevBuf<int> didx(n);
    if (!dx.p || !dy.p || !didx.p)
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_train: sample buffers");
    cudaMemcpyAsync(dx.p, x6, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(dy.p, yn.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, h->stream);
    const std::vector<float> p0 = learn_init(seed);
    cudaMemcpyAsync(h->learn.params, p0.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(h->learn.grad, 0, sizeof(float) * kMlpParams, h->stream);
    cudaMemsetAsync(h->learn.adam_m, 0, sizeof(float) * kMlpParams, h->stream);
    cudaMemsetAsync(h->learn.adam_v, 0, sizeof(float) * kMlpParams, h->stream);
    std::vector<int> perm(n);
    for (int64_t i = 0; i < n; ++i)
        perm[i] = static_cast<int>(i);
    std::mt19937_64 rng(seed ^ 0x9e3779b97f4a7c15ull);
    const int64_t per_epoch = n / batch;
    const int tail = std::min(steps, 100);
    for (int st = 0; st < steps; ++st) {
        const int64_t k = st % per_epoch;
        if (k == 0) {
            std::shuffle(perm.begin(), perm.end(), rng);
            cudaMemcpyAsync(didx.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream);
            // the host vector is reshuffled next epoch: wait for the upload first
            cudaStreamSynchronize(h->stream);
        }
        if (st == steps - tail)
            cudaMemsetAsync(h->learn.loss, 0, sizeof(float), h->stream);
        launch_mlp_train_step(h->learn.params, dx.p, dy.p, didx.p + k * batch, batch, h->learn.grad,
                              h->learn.loss, h->d.err, h->stream);
        const float lr_t = 0.5f * lr * (1.0f + std::cos(3.14159265f * st / steps));
        launch_mlp_adam(h->learn.params, h->learn.grad, h->learn.adam_m, h->learn.adam_v, st + 1, lr_t,
                        h->stream);
    }
    float loss = 0.0f;
    cudaMemcpyAsync(&loss, h->learn.loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    const bz_status s = check_device(h, "bz_learn_train");
    if (s != BZ_OK)
        return s;
    h->learn.scale = scale;
    h->learn.trained = true;
    drop_graphs(h);
    if (final_loss)
        *final_loss = loss / static_cast<float>(static_cast<int64_t>(tail) * batch * 3);
    return BZ_OK;
}

bz_status bz_learn_forward(bz_handle* h, const float* x6, int64_t n, float* y3)
{
    if (!h || !x6 || !y3 || n <= 0 || !h->learn.trained)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    DevBuf<float> dx(6 * static_cast<size_t>(n)), dy(3 * static_cast<size_t>(n));
    if (!dx.p || !dy.p)
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_forward");
    cudaMemcpyAsync(dx.p, x6, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, h->stream);
    launch_mlp_forward(h->learn.params, dx.p, static_cast<int>(n), h->learn.scale, dy.p, h->d.err, h->stream);
    cudaMemcpyAsync(y3, dy.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_learn_forward");
}

bz_status bz_learn_gradient(bz_handle* h, const float* x6, const float* y3, int64_t n, float* grad,
                            float* loss)
{
    if (!h || !x6 || !y3 || !grad || n <= 0 || !h->learn.trained)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    DevBuf<float> dx(6 * static_cast<size_t>(n)), dy(3 * static_cast<size_t>(n));
    if (!dx.p || !dy.p)
        return fail(h, BZ_OUT_OF_MEMORY, "bz_learn_gradient");
    cudaMemcpyAsync(dx.p, x6, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(dy.p, y3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(h->learn.grad, 0, sizeof(float) * kMlpParams, h->stream);
    cudaMemsetAsync(h->learn.loss, 0, sizeof(float), h->stream);
    launch_mlp_train_step(h->learn.params, dx.p, dy.p, nullptr, static_cast<int>(n), h->learn.grad,
                          h->learn.loss, h->d.err, h->stream);
    cudaMemcpyAsync(grad, h->learn.grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, h->stream);
    float l = 0.0f;
    cudaMemcpyAsync(&l, h->learn.loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    const bz_status s = check_device(h, "bz_learn_gradient");
    cudaMemsetAsync(h->learn.grad, 0, sizeof(float) * kMlpParams, h->stream);
    if (loss)
        *loss = l / static_cast<float>(n);
    return s;
}

bz_status bz_morton_keys(bz_handle* h, uint64_t* sorted_keys, int32_t* perm)
{
    if (!h || h->n == 0 || !sorted_keys || !perm)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int n = static_cast<int>(h->n);
    DeviceBuffers& d = h->d;
    if (h->cfg.key_mode == BZ_KEYS_REFERENCE || h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE) {
        enqueue_reference_order(h);
        h->ref_tree_valid = true;
    } else {
        // production keys computed in the caller's order (stable ties follow caller order)
        double* const* s = d.st[h->cur];
        double* tmp = nullptr;
        if (!dalloc(h, &tmp, 3 * static_cast<size_t>(n)))
            return fail(h, BZ_OUT_OF_MEMORY, "bz_morton_keys staging");
        count_launch();
        k_gather_f64<<<blocks_for(n), 256, 0, h->stream>>>(nullptr, s[0], s[1], s[2], s[3], s[4], s[5],
                                                           d.id[h->cur], n, tmp, 0);
        if (!periodic(h))
            launch_bbox_f64(tmp, tmp + n, tmp + 2 * n, n, d.box, h->stream);
        launch_keys63(tmp, tmp + n, tmp + 2 * n, n, d.box, periodic(h) ? h->cfg.box_length : 0.0,
                      d.keys, d.perm, h->stream);
        launch_radix_sort_adaptive(d.keys, d.perm, n, 64, h->sort, h->asort, d.err, h->stream);
        cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        h->allocations.pop_back();
        h->bytes -= 3 * static_cast<size_t>(n) * sizeof(double);
        h->forces_valid = false;  // keys buffer reused
    }
    cudaMemcpyAsync(sorted_keys, d.keys, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(perm, d.perm, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream);
    return check_device(h, "bz_morton_keys");
}

bz_status bz_reference_tree(bz_handle* h, int64_t* node_count, float* hot8, int32_t* next,
                            int32_t* child_mask, int32_t* first_child, int32_t* leaf_start,
                            int32_t* leaf_count)
{
    if (!h || !node_count || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    if (!h->ref_tree_valid) {
        enqueue_reference_order(h);
        bz_status s = check_device(h, "bz_reference_tree");
        if (s != BZ_OK)
            return s;
        h->ref_tree_valid = true;
    }
    *node_count = 1;
    if (hot8) {
        cudaMemcpy(hot8, h->d.ref_hot8, 8 * sizeof(float), cudaMemcpyDeviceToHost);
    }
    if (next)
        next[0] = -1;
    if (child_mask)
        child_mask[0] = 0;
    if (first_child)
        first_child[0] = -1;
    if (leaf_start)
        leaf_start[0] = 0;
    if (leaf_count)
        leaf_count[0] = static_cast<int32_t>(h->n);
    return BZ_OK;
}

bz_status bz_tree_topology(bz_handle* h, int64_t* node_count, int32_t* start, int32_t* count,
                           int32_t* child, int32_t* nchild, float* mono4, float* bmin3,
                           float* bmax3, float* quad6)
{
    if (!h || !node_count || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    if (h->cfg.solver == BZ_SOLVER_OCTREE_REFERENCE)
        return fail(h, BZ_UNSUPPORTED, "use bz_reference_tree in reference mode");
    cudaSetDevice(h->device);
    bz_status s = ensure_forces(h);
    if (s != BZ_OK)
        return s;
    int nn = 0;
    cudaMemcpy(&nn, h->tree.n_nodes, sizeof(int), cudaMemcpyDeviceToHost);
    *node_count = nn;
    if (!start && !count && !child && !nchild && !mono4 && !bmin3 && !bmax3 && !quad6)
        return BZ_OK;
    const size_t k = static_cast<size_t>(nn);
    if (start)
        cudaMemcpy(start, h->tree.start, k * sizeof(int), cudaMemcpyDeviceToHost);
    if (count)
        cudaMemcpy(count, h->tree.count, k * sizeof(int), cudaMemcpyDeviceToHost);
    if (child)
        cudaMemcpy(child, h->tree.child, k * sizeof(int), cudaMemcpyDeviceToHost);
    if (nchild)
        cudaMemcpy(nchild, h->tree.nchild, k * sizeof(int), cudaMemcpyDeviceToHost);
    if (mono4)
        cudaMemcpy(mono4, h->tree.mono, k * sizeof(float4), cudaMemcpyDeviceToHost);
    std::vector<float4> b(k);
    if (bmin3) {
        cudaMemcpy(b.data(), h->tree.box0, k * sizeof(float4), cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < k; ++i) {
            bmin3[3 * i] = b[i].x;
            bmin3[3 * i + 1] = b[i].y;
            bmin3[3 * i + 2] = b[i].z;
        }
    }
    if (bmax3) {
        cudaMemcpy(b.data(), h->tree.box1, k * sizeof(float4), cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < k; ++i) {
            bmax3[3 * i] = b[i].x;
            bmax3[3 * i + 1] = b[i].y;
            bmax3[3 * i + 2] = b[i].z;
        }
    }
    if (quad6) {
        std::vector<float4> qa(k);
        std::vector<float2> qb(k);
        cudaMemcpy(qa.data(), h->tree.quadA, k * sizeof(float4), cudaMemcpyDeviceToHost);
        cudaMemcpy(qb.data(), h->tree.quadB, k * sizeof(float2), cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < k; ++i) {
            quad6[6 * i] = qa[i].x;
            quad6[6 * i + 1] = qa[i].y;
            quad6[6 * i + 2] = qa[i].z;
            quad6[6 * i + 3] = qa[i].w;
            quad6[6 * i + 4] = qb[i].x;
            quad6[6 * i + 5] = qb[i].y;
        }
    }
    return check_device(h, "bz_tree_topology");
}

bz_status bz_pm_mesh(bz_handle* h, int which, float* out)
{
    if (!h || !out || !h->pm || h->n == 0 || which < 0 || which > 4)
        return BZ_INVALID_ARGUMENT;
    if (which == 1 && h->cfg.treepm_gradient == 1)
        return fail(h, BZ_UNSUPPORTED, "the spectral-gradient mode keeps no potential mesh");
    if (which >= 2 && h->cfg.treepm_gradient == 2)
        return fail(h, BZ_UNSUPPORTED, "analytic differentiation keeps no force mesh");
    cudaSetDevice(h->device);
    bz_status s = ensure_forces(h);
    if (s != BZ_OK)
        return s;
    const size_t M = static_cast<size_t>(h->cfg.treepm_grid_size) * (isolated(h) ? 2 : 1);
    if (isolated(h))  // the grid of the current state (the one its forces were computed on)
        launch_iso_grid(h->d.box, h->cfg.treepm_grid_size, h->cfg.treepm_cell_floor,
                        h->cfg.octree_softening, h->cfg.treepm_r_split_cells, h->cfg.treepm_r_cut_factor,
                        h->cfg.treepm_node_size_factor, h->iso, h->stream);
    pm_deposit(h->pm, h->d.pos4, static_cast<int>(h->n), h->stream);
    if (which == 0) {
        cudaMemcpyAsync(out, pm_mesh(h->pm), M * M * M * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
        return check_device(h, "bz_pm_mesh");
    }
    if (pm_solve(h->pm, h->stream) != 0)
        return fail(h, BZ_CUDA_ERROR, "[cufft] mesh solve failed");
    if (which == 1) {
        cudaMemcpyAsync(out, pm_mesh(h->pm), M * M * M * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
        return check_device(h, "bz_pm_mesh");
    }
    std::vector<float4> f(M * M * M);
    cudaMemcpyAsync(f.data(), pm_force_mesh(h->pm), f.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                    h->stream);
    s = check_device(h, "bz_pm_mesh");
    if (s != BZ_OK)
        return s;
    for (size_t c = 0; c < f.size(); ++c)
        out[c] = which == 2 ? f[c].x : (which == 3 ? f[c].y : f[c].z);
    return BZ_OK;
}

bz_status bz_pm_grid(bz_handle* h, double* out6)
{
    if (!h || !out6 || h->cfg.solver != BZ_SOLVER_TREEPM)
        return BZ_INVALID_ARGUMENT;
    if (isolated(h)) {
        cudaSetDevice(h->device);
        IsoGrid g{};
        if (cudaMemcpy(&g, h->iso, sizeof(g), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(h, BZ_CUDA_ERROR, "bz_pm_grid");
        const float rc = std::sqrt(g.rcut2);
        const double v[6] = {g.origin[0], g.origin[1], g.origin[2], g.h, g.rsplit, rc};
        std::copy(v, v + 6, out6);
        return BZ_OK;
    }
    const double cell = h->cfg.box_length / h->cfg.treepm_grid_size;
    const float rs = rsplit_len(h);
    const double v[6] = {0.0, 0.0, 0.0, cell, rs, h->cfg.treepm_r_cut_factor * rs};
    std::copy(v, v + 6, out6);
    return BZ_OK;
}

bz_status bz_force_errors(bz_handle* h, int32_t nsample, uint64_t seed, float* errs,
                          int32_t* idx, double* median, double* p99)
{
    if (!h || nsample <= 0 || h->n == 0)
        return BZ_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    bz_status s = ensure_forces(h);
    if (s != BZ_OK)
        return s;
    const int n = static_cast<int>(h->n);
    const int ns = std::min(nsample, n);
    // sample caller indices without replacement, then map to sorted slots
    std::mt19937_64 rng(seed);
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i)
        all[i] = i;
    for (int i = 0; i < ns; ++i) {
        std::uniform_int_distribution<int> u(i, n - 1);
        std::swap(all[i], all[u(rng)]);
    }
    std::vector<int> ids(n);
    cudaMemcpy(ids.data(), h->d.id[h->cur], n * sizeof(int), cudaMemcpyDeviceToHost);
    std::vector<int> slot_of(n);
    for (int i = 0; i < n; ++i)
        slot_of[ids[i]] = i;
    std::vector<int> slots(ns);
    for (int i = 0; i < ns; ++i)
        slots[i] = slot_of[all[i]];
    int* dslots = nullptr;
    double* dref = nullptr;
    double* sk = nullptr;
    const int kmax = 8;
    const bool per = periodic(h);
    if (cudaMalloc(&dslots, ns * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&dref, 3 * ns * sizeof(double)) != cudaSuccess ||
        (per && cudaMalloc(&sk, 5 * static_cast<size_t>(ewald_num_k(kmax)) * sizeof(double)) != cudaSuccess)) {
        cudaFree(dslots);
        cudaFree(dref);
        cudaFree(sk);
        return fail(h, BZ_OUT_OF_MEMORY, "bz_force_errors scratch");
    }
    cudaMemcpy(dslots, slots.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
    const double eps = std::max(h->cfg.octree_softening, h->cfg.physics_min_softening);
    if (per)
        launch_ewald_f64(h->d.pos4, n, dslots, ns, eps, h->cfg.box_length, 6.4 / h->cfg.box_length,
                         kmax, sk, dref, h->stream);
    else if (h->systems > 0) {
        // each target sums over its own system only (systems are contiguous in sorted order)
        std::vector<int> lo(ns), hi(ns), sys_first(h->systems, n), sys_last(h->systems, 0);
        auto sys_of = [&](int caller) {
            return static_cast<int>(std::upper_bound(h->host_offsets.begin(), h->host_offsets.end(),
                                                     static_cast<long long>(caller)) -
                                    h->host_offsets.begin()) - 1;
        };
        for (int i = 0; i < n; ++i) {
            const int sy = sys_of(ids[i]);
            sys_first[sy] = std::min(sys_first[sy], i);
            sys_last[sy] = std::max(sys_last[sy], i + 1);
        }
        for (int i = 0; i < ns; ++i) {
            const int sy = sys_of(all[i]);
            lo[i] = sys_first[sy];
            hi[i] = sys_last[sy];
        }
        int* drange = nullptr;
        if (cudaMalloc(&drange, 2 * ns * sizeof(int)) != cudaSuccess) {
            cudaFree(dslots);
            cudaFree(dref);
            return fail(h, BZ_OUT_OF_MEMORY, "bz_force_errors scratch");
        }
        cudaMemcpy(drange, lo.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(drange + ns, hi.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
        launch_direct_f64(h->d.pos4, n, dslots, ns, eps, dref, h->stream, drange, drange + ns);
        cudaStreamSynchronize(h->stream);
        cudaFree(drange);
    } else
        launch_direct_f64(h->d.pos4, n, dslots, ns, eps, dref, h->stream);
    std::vector<double> ref(3 * ns);
    std::vector<float> ax(n), ay(n), az(n);
    cudaMemcpyAsync(ref.data(), dref, 3 * ns * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(ax.data(), h->d.acc[0], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(ay.data(), h->d.acc[1], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(az.data(), h->d.acc[2], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    s = check_device(h, "bz_force_errors");
    cudaFree(dslots);
    cudaFree(dref);
    cudaFree(sk);
    if (s != BZ_OK)
        return s;
    std::vector<double> e(ns);
    for (int i = 0; i < ns; ++i) {
        const int k = slots[i];
        const double dx = ax[k] - ref[3 * i], dy = ay[k] - ref[3 * i + 1], dz = az[k] - ref[3 * i + 2];
        const double rn = std::sqrt(ref[3 * i] * ref[3 * i] + ref[3 * i + 1] * ref[3 * i + 1] +
                                    ref[3 * i + 2] * ref[3 * i + 2]);
        e[i] = std::sqrt(dx * dx + dy * dy + dz * dz) / (rn > 0 ? rn : 1.0);
        if (errs)
            errs[i] = static_cast<float>(e[i]);
        if (idx)
            idx[i] = all[i];
    }
    std::vector<double> sorted = e;
    std::sort(sorted.begin(), sorted.end());
    auto pct = [&](double q) {
        const double pos = q * (ns - 1);
        const int lo = static_cast<int>(std::floor(pos));
        const int hi = std::min(lo + 1, ns - 1);
        return sorted[lo] + (sorted[hi] - sorted[lo]) * (pos - lo);
    };
    if (median)
        *median = pct(0.5);
    if (p99)
        *p99 = pct(0.99);
    return BZ_OK;
}

}  // extern "C"
