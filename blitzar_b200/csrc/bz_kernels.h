// Internal launch interface between the C-ABI layer (bz_api.cu) and the kernel files.
// Every launcher enqueues on the given stream and never synchronises.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace bz {

// Number of this library's kernel launches enqueued so far (cuFFT's own kernels are not
// counted).  Launches recorded into a CUDA graph are counted once, at capture.
extern std::atomic<unsigned long long> g_kernel_launches;
inline void count_launch(unsigned long long k = 1) { g_kernel_launches.fetch_add(k, std::memory_order_relaxed); }

// ---------------------------------------------------------------- keys (bz_keys.cu)
struct BoxF64 {
    unsigned long long mn[3];  // ordered-integer images of the FP64 minima
    unsigned long long mx[3];  // ... and maxima
};
void launch_bbox_f64(const double* x, const double* y, const double* z, int n, BoxF64* box,
                     cudaStream_t s);
// Production keys: 21 bits per axis, floor quantisation of a cube.  periodic_len > 0 uses
// the cube [0, L)^3; otherwise the cube is derived on the device from *box.
void launch_keys63(const double* x, const double* y, const double* z, int n,
                   const BoxF64* box, double periodic_len, unsigned long long* keys,
                   uint32_t* perm, cudaStream_t s);
// Ensembles: system s owns caller indices [offsets[s], offsets[s+1]); id[i] is the caller
// index of slot i.  Keys carry the system in bits 54..62 (up to kMaxSystems systems) and 18
// bits per axis of the system's own cube, so the top three octree levels split systems apart.
constexpr int kMaxSystems = 512;
constexpr int kSystemLevels = 3;
void launch_keys_ensemble(const double* x, const double* y, const double* z, const int* id, int n,
                          const long long* offsets, int systems, BoxF64* boxes,
                          unsigned long long* keys, uint32_t* perm, cudaStream_t s);
// Reference-compatible keys (FP32 bbox, the reference's quantisation and bit spread).
void launch_keys_reference(const float* x, const float* y, const float* z, int n,
                           unsigned* bbox_ordered6, unsigned long long* keys, uint32_t* perm,
                           cudaStream_t s);

// ---------------------------------------------------------------- sort (bz_sort.cu)
struct SortWorkspace {
    unsigned long long* keys_alt;
    uint32_t* vals_alt;
    uint32_t* hist;              // [8][256] digit counts
    uint32_t* base;              // [8][256] exclusive digit bases
    uint32_t* ticket;            // [8] tile tickets
    uint32_t* epoch;             // [1] sort-call counter (look-back state tag)
    int* trivial;                // [8] pass-is-identity flags
    unsigned long long* state;   // [max_tiles][256] look-back words
    int max_tiles;
};
size_t sort_state_words(int n);
int sort_tile_items();
// Stable LSD radix sort of (keys, vals) on the low `bits` key bits (multiple of 8).  The
// sorted result lands back in (keys, vals).
void launch_radix_sort(unsigned long long* keys, uint32_t* vals, int n, int bits,
                       SortWorkspace& ws, int* err, cudaStream_t s);
// Arrays and count of one radix sort, read by the sort kernels from device memory.
struct SortJob {
    unsigned long long* ka;
    uint32_t* va;
    unsigned long long* kb;  // alternate buffers
    uint32_t* vb;
    int n;
};
// Workspace of launch_radix_sort_adaptive: the locally out-of-order pairs F (at most cap of
// them) and alternate buffers to sort them, flags, compaction block sums, four control words
// (out-of-order count, in-order-part-not-sorted flag, fast-path count, full-sort count) and
// the radix sort's job.
struct AdaptiveSortWorkspace {
    unsigned long long* fkeys;      // [cap]
    uint32_t* fvals;                // [cap]
    unsigned long long* falt_keys;  // [cap]
    uint32_t* falt_vals;            // [cap]
    unsigned char* flag;            // [n] out-of-order flags
    int* block_sums;                // [adaptive_sort_blocks(n)]
    int* ctl;                       // [4]
    SortJob* job;                   // [1]
    int cap;
};
int adaptive_sort_blocks(int n);
int adaptive_sort_cap(int n);
// The same stable sort as launch_radix_sort for vals = 0..n-1 on entry (the original
// positions), fast when the keys are nearly sorted (a step's re-sort of the previous order):
// only the locally out-of-order pairs are radix-sorted and merged back; other inputs take the
// full sort, decided on the device.  Uses ws.keys_alt / ws.vals_alt for the in-order pairs.
void launch_radix_sort_adaptive(unsigned long long* keys, uint32_t* vals, int n, int bits,
                                SortWorkspace& ws, AdaptiveSortWorkspace& aws, int* err,
                                cudaStream_t s);

// ---------------------------------------------------------------- tree (bz_tree.cu)
struct TreeArrays {
    int cap;           // node capacity
    int* start;        // particle range of each node
    int* count;
    int* child;        // first child (-1 for leaves)
    int* nchild;
    int* parent;
    int* level;
    int* lvl_first;    // [kMaxLevels+2]
    int* lvl_count;    // [kMaxLevels+2]
    int* lvl_split;    // [kMaxLevels+2] 1 when some node of the level holds more than a leaf
    int* n_nodes;      // [1]
    uint32_t* ticket;  // [kMaxLevels+2]
    int* arrive;       // [cap] bottom-up arrival counters of the moments climb
    unsigned long long* lookback;  // [tree_lookback_words(cap)]
    double* m64;       // [cap] FP64 mass
    double* s64;       // [3*cap] FP64 first moments
    double* c64;       // [3*cap] FP64 centre of mass
    double* q64;       // [6*cap] FP64 second moments about the COM
    float4* box0;      // {bmin.xyz, link}
    float4* box1;      // {bmax.xyz, info}
    float4* mono;      // {com.xyz, mass}
    float4* quadA;     // {qxx, qxy, qxz, qyy}
    float2* quadB;     // {qyz, qzz}
};
constexpr int kMaxLevels = 21;
// Upper bound on device ordinals for per-device caches (function attributes, launch shapes).
constexpr int kMaxDevices = 64;
size_t tree_lookback_words(int cap);
// min_split: nodes above this level split even when small (ensembles use kSystemLevels)
// quad = false: second moments left zero (walks without quadrupoles)
void launch_tree_build(const unsigned long long* sorted_keys, const float4* pos4, int n,
                       int leaf_cap, int max_level, TreeArrays& t, int* err, cudaStream_t s,
                       int min_split = 0, bool quad = true);

// Keep the topology, recompute every node's tight box and moments from the current pos4
// (particles drifted inside their nodes: adaptive substeps).
void launch_tree_refit(const float4* pos4, TreeArrays& t, cudaStream_t s, bool quad = true);

// Reference-mode topology: the single leaf the reference builds for its own keys.
void launch_reference_leaf(const float* x, const float* y, const float* z, const float* m,
                           const uint32_t* sorted_index, int n, float* hot8, cudaStream_t s);

// ---------------------------------------------------------------- walk (bz_walk.cu)
struct IsoGrid;
struct WalkParams {
    float theta2;
    float eps2;
    float rcut2;      // 0 disables the cutoff
    float box;        // periodic length, 0 = open
    float rsplit;     // Gaussian split scale, 0 = Newtonian
    float min_dist2;
    float max_node_size;  // > 0: nodes at least this large are never accepted as multipoles
    int quadrupole;
    int want_pot;
    float rcorr2;     // > 0 with WalkOutputs.pair_src: record the pairs closer than this
    const unsigned char* active;  // optional [n]: walk only groups with an active target
    int blocks_per_sm;            // > 0: at most this many resident walk blocks per SM (room
                                  // for kernels of a concurrent stream); 0 = as many as fit
    float max_acc;                // acceleration clamp of the walk's sum (and of the total)
    int clamp_total;              // the output already holds the mesh force: clamp the sum
    const IsoGrid* iso;           // isolated TreePM: rsplit, rcut2, max_node_size read here
};
// ---------------------------------------------------------------- target groups (bz_groups.cu)
constexpr int kGroupMax = 32;  // largest walk group (one warp)
struct GroupTable {
    unsigned char* flag;  // [group_flag_bytes(n)] group-start flags (0 / 1), zero past n
    int* gstart;      // [n + 1] group start indices in sorted order, then the end sentinel
    int* ngroups;     // [1]
    int* block_sums;  // [group_count_blocks(n)]
    int* groot;       // [n]: node where each group's walk starts (its system's root)
    int* sysroot;     // [kMaxSystems]: root node of each system (ensembles)
};
int group_count_blocks(int n);
size_t group_flag_bytes(int n);
// root_level: level of the system roots (0 for one system, kSystemLevels for ensembles, whose
// system id the sorted keys carry in bits 54..62)
void launch_groups(const TreeArrays& t, int n, int gmax, int root_level,
                   const unsigned long long* keys, GroupTable& g, cudaStream_t s);

struct WalkOutputs {
    float* ax;        // accumulated into (+=)
    float* ay;
    float* az;
    float* pot;       // optional (+=)
    unsigned long long* n_pp;  // optional per-group counters
    unsigned long long* n_pn;
    unsigned long long* totals; // optional [3]: listed pairs, node terms (x targets), pairs
                                //   evaluated by the pair law (inside the cutoff)
    int* pair_src;    // optional [n * kPairSlots]: sorted source index of each recorded pair
    int* pair_cnt;    // [n]: recorded pairs per target (above kPairSlots raises kErrListCapacity)
};
void launch_walk(const float4* pos4, int n, const TreeArrays& t, const GroupTable& g,
                 const WalkParams& p, const WalkOutputs& o, unsigned* queue, int* spill, int* err,
                 cudaStream_t s);
int walk_spill_slots();       // warp slots that need a spill area
size_t walk_spill_entries();  // ints per slot

// Reference-formulation direct sum (the walk the reference runs on its one-leaf tree).
void launch_reference_walk(const float4* pos_orig, const float4* pos_sorted,
                           const uint32_t* sorted_index, int n, float softening,
                           float min_distance2, float split_scale, float cutoff2,
                           float max_acceleration, float* ax, float* ay, float* az,
                           cudaStream_t s);

// ---------------------------------------------------------------- PM (bz_pm.cu)
struct PmPlan;
// Grid of the isolated (open-boundary) mesh, recomputed on the device for every force
// evaluation from the particles' bounds (the reference's TpmGridBuild.inl:98-171): a cubic
// mesh of `mesh` = 2G cells of size h = max(cell_floor, extent / (G - 2)), centred on the
// bounds; the split scale and cutoff follow h.
struct IsoGrid {
    float origin[3];
    float h;
    float inv_h;
    float rsplit;
    float rcut2;
    float max_node_size;
};
// order: 2 CIC, 3 TSC, 4 PCS; gradient: 0 centred differences of phi, 1 spectral (i k), 2
// analytic differentiation; window_floor: lower bound of the deconvolution window (the
// reference uses 0.08).  iso != NULL: isolated mesh whose grid the device holds at iso (box
// and rsplit unused); the Green's function is then evaluated in the solve, not tabulated.
// dev_err: the handle's device error bits (a staged gather whose bulk copies time out sets
// kErrBulkWait there).
PmPlan* pm_create(int mesh, double box, double rsplit, int order, int gradient, double window_floor,
                  cudaStream_t s, int* cuda_err, const IsoGrid* iso = nullptr, int* dev_err = nullptr);
// Isolated grid from the FP64 bounding box of the positions: grid_half = G, r_split_cells and
// r_cut_factor in units of the cell, node_size_factor in units of r_s.
void launch_iso_grid(const BoxF64* box, int grid_half, float cell_floor, float softening,
                     float r_split_cells, float r_cut_factor, float node_size_factor, IsoGrid* out,
                     cudaStream_t s);
void pm_destroy(PmPlan* p);
size_t pm_bytes(const PmPlan* p);
// Deposit, FFT Poisson solve with split + deconvolution, then interpolate the centred-
// difference gradient at each particle; writes (=) ax, ay, az.
int pm_forces(PmPlan* p, const float4* pos4, int n, float* ax, float* ay, float* az,
              cudaStream_t s);
// The three stages separately (tests read the mesh between them): the mesh buffer holds the
// density after pm_deposit and, in centred-difference mode, the potential after pm_solve.
void pm_deposit(PmPlan* p, const float4* pos4, int n, cudaStream_t s);
// particles per deposit block, chosen so that a block's stencils fit a shared-memory tile
int pm_deposit_chunk(const PmPlan* p, int n);
int pm_solve(PmPlan* p, cudaStream_t s);
void pm_interp(PmPlan* p, const float4* pos4, int n, float* ax, float* ay, float* az,
               cudaStream_t s);
float* pm_mesh(PmPlan* p);
const float4* pm_force_mesh(PmPlan* p);  // interleaved {ax, ay, az, 0}

// ---------------------------------------------------------------- state (bz_state.cu)
void launch_permute(const uint32_t* perm, int n, const double* const* src, double* const* dst,
                    int ndouble, const float* msrc, float* mdst, const int* idsrc, int* iddst,
                    float4* pos4, double periodic_len, cudaStream_t s);
// Closing half kick; with b (may be NULL) the accelerations are first completed,
// a = clamp(a + b, max_acc).
void launch_kick(double* vx, double* vy, double* vz, float* ax, float* ay, float* az, int n,
                 const double* dt_half, cudaStream_t s, const float* bx = nullptr,
                 const float* by = nullptr, const float* bz = nullptr, float max_acc = 0.0f);
void launch_kick_drift(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                       const float* ax, const float* ay, const float* az, int n,
                       const double* dt, double periodic_len, BoxF64* box, cudaStream_t s,
                       const float* mass = nullptr, float4* pos4 = nullptr, double kick_frac = 0.5);
// FP64 energy/momentum sums over the sorted state (scratch: energy_scratch_doubles(); the
// five results land at scratch[5 * 1024 .. 5 * 1024 + 5)).
size_t energy_scratch_doubles();
void launch_energy(const double* vx, const double* vy, const double* vz, const float* m,
                   const float* pot, int n, double* scratch, cudaStream_t s);
void launch_scatter3(const float* ax, const float* ay, const float* az, const int* id, int n,
                     float* out_soa3, cudaStream_t s);
void launch_f64_to_f32(const double* src, float* dst, int n, cudaStream_t s);
// pos4[i] = {x, y, z, m} in FP32 from the FP64 state (same order)
void launch_refresh_pos4(const double* x, const double* y, const double* z, const float* m, int n,
                         float4* pos4, cudaStream_t s);
// a = clamp(a + b, max_acc), three components (the reference's clamp of the TreePM sum)
void launch_add3(float* ax, float* ay, float* az, const float* bx, const float* by, const float* bz,
                 int n, float max_acc, cudaStream_t s);

// ---------------------------------------------------------------- adaptive steps (bz_adaptive.cu)
struct AdaptiveParams {
    double dt_max;
    float eta;
    float eps;
    int max_level;
};
struct AdaptiveState {        // indexed by caller index
    unsigned char* level;
    float* ax;
    float* ay;
    float* az;
    unsigned long long* updates;  // [1] particle steps closed so far
};
void launch_adaptive_init(const float* ax, const float* ay, const float* az, const double* vx,
                          const double* vy, const double* vz, const int* id, int n,
                          const AdaptiveParams& p, const AdaptiveState& a, cudaStream_t s);
void launch_level_max(const unsigned char* level, int n, int* out, cudaStream_t s);
void launch_adaptive_open_drift(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                                const int* id, int n, const AdaptiveParams& p, const AdaptiveState& a,
                                int sub, int L, cudaStream_t s);
void launch_adaptive_active(const int* id, int n, const AdaptiveState& a, int sub, int L,
                            unsigned char* active, cudaStream_t s);
void launch_adaptive_close(const float* ax, const float* ay, const float* az, double* vx, double* vy,
                           double* vz, const int* id, const unsigned char* active, int n,
                           const AdaptiveParams& p, const AdaptiveState& a, int sub, int L,
                           cudaStream_t s);

// ---------------------------------------------------------------- learned correction (bz_mlp.cu)
// Parameter block of the 6 -> 32 -> 32 -> 3 MLP (16 features incl. a constant 1 that carries
// b1): W1[32][16], W2[32][32], b2[32], W3[3][32], b3[3].
constexpr int kMlpOffW1 = 0;
constexpr int kMlpOffW2 = kMlpOffW1 + 32 * 16;
constexpr int kMlpOffB2 = kMlpOffW2 + 32 * 32;
constexpr int kMlpOffW3 = kMlpOffB2 + 32;
constexpr int kMlpOffB3 = kMlpOffW3 + 3 * 32;
constexpr int kMlpParams = kMlpOffB3 + 3;
constexpr int kPairSlots = 64;  // recorded pairs per target for the correction
void launch_mlp_train_step(const float* params, const float* in6, const float* y3, const int* index,
                           int n, float* grad, float* loss, int* err, cudaStream_t s);
void launch_mlp_adam(float* params, float* grad, float* m, float* v, int step, float lr, cudaStream_t s);
void launch_mlp_forward(const float* params, const float* in6, int n, float scale, float* out3,
                        int* err, cudaStream_t s);
void launch_mlp_pairs(const float* params, const float4* pos4, int n, const int* pair_src,
                      const int* pair_cnt, float h, float box, float scale, float* ax, float* ay,
                      float* az, int* err, cudaStream_t s);

// ---------------------------------------------------------------- diagnostics (bz_diag.cu)
// FP64 reference accelerations for the listed (sorted-order) targets: direct sum (open) or
// Ewald (periodic).
// src_lo/src_hi (optional, per target): sum only sources [src_lo, src_hi) (ensembles)
void launch_direct_f64(const float4* pos4, int n, const int* targets, int nt, double eps,
                       double* acc3, cudaStream_t s, const int* src_lo = nullptr,
                       const int* src_hi = nullptr);
void launch_ewald_f64(const float4* pos4, int n, const int* targets, int nt, double eps,
                      double box, double alpha, int kmax, double* sk_scratch, double* acc3,
                      cudaStream_t s);
int ewald_num_k(int kmax);
// Ideal Gaussian long-range force (Ewald with the real-space part of the split kernel removed)
// at the listed targets from the first n_src particles, which also fill sk_scratch.
void launch_lr_ideal_f64(const float4* pos4, int n_src, const int* targets, int nt, double box,
                         double alpha, int kmax, double rsplit, double* sk_scratch, double* acc3,
                         cudaStream_t s);

} // namespace bz
