/* bzgrav.h -- C ABI of the B200 Barnes-Hut / TreePM gravity engine (libbzgrav.so).
 *
 * The library sits behind BLITZAR's solver dispatch as the engine of the `octree_gpu` /
 * TreePM path.  Plain C types only: host pointers and sizes in, status codes out.  One
 * handle owns all device memory of one particle system on one GPU and one CUDA stream;
 * handles are not thread-safe (one host thread drives a handle, as one host thread drives a
 * reference ParticleSystem).
 *
 * Reference interfaces each entry point replaces are cited as paths inside the BLITZAR
 * project.
 */
#ifndef BZGRAV_H
#define BZGRAV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; 0..4 mirror blitzar_core_result_t (runtime/ffi/core/FfiApi.hpp:15-21). */
typedef enum bz_status {
    BZ_OK = 0,
    BZ_INVALID_ARGUMENT = 1,
    BZ_NOT_READY = 2,
    BZ_TIMEOUT = 3,
    BZ_INTERNAL_ERROR = 4,
    BZ_CUDA_ERROR = 5,        /* a CUDA/cuFFT call failed (text in bz_last_error) */
    BZ_OUT_OF_MEMORY = 6,
    BZ_DEVICE_LIMIT = 7,      /* a bounded device-side loop gave up (stack, wait, capacity) */
    BZ_UNSUPPORTED = 8
} bz_status;

/* Which solver the handle runs (the `--solver` / simulation(solver=...) selection,
 * engine/config/registry/entries/CfgEntriesCore.cpp:22, mapped to ParticleSystem::SolverMode
 * by engine/server/simulation/runtime/SrvHelpers.cpp:91-102). */
typedef enum bz_solver {
    BZ_SOLVER_OCTREE = 0,           /* Barnes-Hut octree (drop-in for octree_gpu) */
    BZ_SOLVER_TREEPM = 1,           /* periodic TreePM: mesh long range + tree short range */
    BZ_SOLVER_OCTREE_REFERENCE = 2  /* the reference octree_gpu formulation: reference keys,
                                       reference topology and its walk (parity mode) */
} bz_solver;

typedef enum bz_key_mode {
    BZ_KEYS_PRODUCTION = 0, /* FP64 quantisation, 21 bits per axis (63-bit keys) */
    BZ_KEYS_REFERENCE = 1   /* bit-exact reference keys (FP32 quantisation and bit spread of
                               engine/physics/octree/cuda/linear/OctKeyKernels.inl:22-46) */
} bz_key_mode;

/* Time integrator of bz_step (simulation(integrator=...)); one force evaluation per step either
   way, the accelerations of the step's end positions kept for the next step.
   Replaces the integrator switch of ParticleSystem::updateOctreeGpuIntegrators
   (engine/physics/core/cuda/integration/CudOctreeGpuIntegrators.inl:31-296). */
typedef enum bz_integrator {
    BZ_INTEGRATOR_LEAPFROG = 0, /* kick-drift-kick: v += a dt/2, x += v dt, a = F(x), v += a dt/2
                                   (the reference's leapfrog, CudOctreeGpuIntegrators.inl:42-196) */
    BZ_INTEGRATOR_EULER = 1     /* symplectic Euler, the reference's default integrator=euler:
                                   a = F(x), v += a dt, x += v dt (updateParticlesOctree,
                                   engine/physics/octree/cuda/force/OctGpu.inl:246-275).
                                   Adaptive block steps (adaptive_max_level > 0) keep their own
                                   scheme whatever this says, as the reference's adaptive path
                                   does (CudOctreeGpuAdaptive.inl) */
} bz_integrator;

/* Configuration; field names follow the simulation.ini keys they mirror. */
typedef struct bz_config {
    uint32_t struct_size;          /* sizeof(bz_config), set by bz_config_init */
    int32_t solver;                /* bz_solver */
    float octree_theta;            /* octree_theta */
    float octree_softening;        /* octree_softening (Plummer epsilon) */
    int32_t octree_opening_criterion; /* octree_opening_criterion: 0 com, 1 bounds (reference mode) */
    int32_t linear_octree_leaf_capacity; /* reference-mode leaf rule (default 256) */
    int32_t leaf_capacity;         /* production adaptive octree: particles per leaf */
    int32_t multipole_order;       /* 1 monopole, 2 monopole + quadrupole */
    float physics_max_acceleration;/* physics_max_acceleration: every particle's acceleration is
                                      clamped to this length, the walk's sum first and then its
                                      sum with the mesh force (reference default 64; must be
                                      > 0; 1e30 leaves physical forces unclamped) */
    float physics_min_softening;   /* physics_min_softening */
    float physics_min_distance2;   /* physics_min_distance2 */
    float physics_min_theta;       /* physics_min_theta */
    int32_t treepm_grid_size;      /* treepm_grid_size: PM mesh cells per side; with box_length
                                      = 0 (isolated TreePM, the reference's GPU TreePM) the
                                      mesh has 2 x this many cells per side, of size max(
                                      treepm_cell_floor, extent / (grid - 2)), centred on the
                                      particles and recomputed for every force evaluation */
    float treepm_r_split_cells;    /* Gaussian split scale r_s in mesh cells */
    float treepm_r_cut_factor;     /* short-range cutoff r_cut = factor * r_s */
    int32_t treepm_assignment;     /* treepm_assignment: 0 cic, 1 tsc, 2 pcs */
    int32_t treepm_gradient;       /* 0 centred differences of the potential (reference),
                                      1 spectral i k gradient fused with the Green's function
                                      (three inverse transforms), 2 analytic differentiation:
                                      one inverse transform to the potential, interpolated
                                      with the gradient of the assignment weights */
    float treepm_window_floor;     /* lower bound of the deconvolution window (reference 0.08) */
    float treepm_node_size_factor; /* short range: tree nodes at least this many r_s across are
                                      never accepted as multipoles (0 = no cap) */
    double box_length;             /* periodic box length (TreePM); 0 = open boundaries (TreePM:
                                      the isolated doubled mesh) */
    int32_t key_mode;              /* bz_key_mode */
    int32_t device;                /* CUDA device ordinal */
    uint64_t stream;               /* cudaStream_t to run on, or 0 for a private stream */
    int32_t use_graph;             /* capture bz_step's per-step work in a CUDA graph */
    int32_t walk_group_size;       /* targets per walk group, 1..32 (default 32; bz_autotune) */
    int32_t adaptive_max_level;    /* adaptive(max_level): 0 = fixed steps; k > 0: power-of-two
                                      block steps dt / 2^l, l <= k (octree solver) */
    float adaptive_eta;            /* adaptive(eta): stable dt = eta * min(sqrt(eps/|a|), eps/|v|) */
    float treepm_cell_floor;       /* isolated TreePM (box_length = 0): smallest mesh cell (the
                                      reference's 0.25, TpmGridBuild.inl:100) */
    int32_t integrator;            /* bz_integrator: the time integrator of bz_step */
} bz_config;

typedef struct bz_handle bz_handle;

/* Default configuration (reference defaults: theta 0.5, softening 0.01, leaf capacity 256,
 * max acceleration 64, TreePM grid 128, split 1.25 cells, cutoff 4.5 r_s, quadrupole on). */
bz_status bz_config_init(bz_config* cfg);

/* Create an engine for up to `capacity` particles.  Replaces ParticleSystem construction +
 * runtime buffer planning (engine/physics/core/particle/PhyParticleSystem.hpp:146,
 * engine/physics/core/cuda/core/CudSolverConfiguration.inl:116-156) and the solver setters
 * setOctreeTheta/Softening/OpeningCriterion, setTreePmParameters,
 * setLinearOctreeLeafCapacity, setPhysicsStabilityConstants (PhyParticleSystem.hpp:187-252). */
bz_status bz_create(const bz_config* cfg, size_t capacity, bz_handle** out);
bz_status bz_destroy(bz_handle* h);

/* Upload particles in the reference SoA layout (engine/physics/core/particle/
 * PhyParticleSoAView.hpp:18-33): pos = x[n], y[n], z[n] back to back; vel likewise; mass[n].
 * vel may be NULL (zero velocities).  The _f64 variant keeps full FP64 state. */
bz_status bz_set_state(bz_handle* h, const float* pos_soa3, const float* vel_soa3,
                       const float* mass, size_t n);
bz_status bz_set_state_f64(bz_handle* h, const double* pos_soa3, const double* vel_soa3,
                           const float* mass, size_t n);

/* Ensembles of independent systems in one handle (no counterpart in the reference, which
 * steps one system per process): system s owns caller indices [offsets[s], offsets[s+1]),
 * offsets[0] = 0, num_systems <= 512, each with at least one particle; FP64 SoA state as in
 * bz_set_state_f64.  Systems never interact: keys carry the system in their top 9 bits, the
 * top three octree levels separate the systems, and every walk group starts at its own
 * system's root.  All systems share one launch per phase and one captured step.  Octree
 * solver only.  A later bz_set_state returns the handle to a single system. */
bz_status bz_set_ensemble(bz_handle* h, const double* pos_soa3, const double* vel_soa3,
                          const float* mass, const int64_t* offsets, int32_t num_systems);

/* Advance nsteps leapfrog (KDK) steps of size dt.  Replaces ParticleSystem::update
 * (PhyParticleSystem.hpp:163; octree_gpu leapfrog in engine/physics/core/cuda/integration/
 * CudOctreeGpuIntegrators.inl:121-195).  The force at the end of a step is reused at the
 * start of the next, so each step evaluates the force once. */
bz_status bz_step(bz_handle* h, double dt, uint32_t nsteps);

/* Adaptive block steps (adaptive_max_level > 0): each bz_step step is one block of dt split
 * into 2^L substeps (L = finest level present at its start); the per-particle level follows
 * engine/physics/core/cuda/integration/CudAdaptive.inl:42-71.  bz_adaptive_levels writes
 * each particle's level (caller order); bz_adaptive_updates the particle steps closed so far
 * (each is one force evaluation and one kick of one particle). */
bz_status bz_adaptive_levels(bz_handle* h, uint8_t* levels);
bz_status bz_adaptive_updates(bz_handle* h, uint64_t* updates);

/* Autotuner (no counterpart in the reference, whose leaf capacity and launch shapes are fixed
 * settings): times 2 x `trials` steps of zero length (drift, keys, sort, forces, kick; positions
 * and velocities come out unchanged) of the current state, launched as bz_step launches them (a
 * captured graph unless use_graph is 0), first for each leaf capacity in
 * {8, 12, 16, 24, 32, 48} x walk group size in {16, 24, 32}, then, for TreePM, with the best of
 * those, for each mesh-leg schedule x walk blocks per SM in {as many as fit, 6, 5}
 * (bz_walk_blocks_per_sm).  Schedules: *mesh_overlap = 0 in line; 1 on a second stream
 * concurrent with the tree build and walk; 2 as 1 with the deposit and field solve also
 * concurrent with the keys, sort and permutation of a step.  Keeps the fastest choice in the
 * handle and reports it, with the time of one such step in *ms_per_evaluation.  Outputs may be
 * NULL. */
bz_status bz_autotune(bz_handle* h, int32_t trials, int32_t* leaf_capacity, int32_t* group_size,
                      float* ms_per_evaluation, int32_t* mesh_overlap);

/* Pins the TreePM mesh-leg schedule (0, 1 or 2 as reported by bz_autotune; the default is 2).
 * Schedules 1 and 2 need the second stream, created with the handle; without it every schedule
 * runs in line.  The results of the schedules differ only in the order of the float mass sums. */
bz_status bz_set_mesh_schedule(bz_handle* h, int32_t schedule);

/* Cap on the resident blocks per SM of the walk kernel (0: as many as fit, the default).  The
 * walk is a persistent kernel that otherwise holds every SM's registers; a lower cap lets the
 * TreePM mesh leg's kernels co-run with it.  bz_autotune picks it with the mesh schedule.
 * set_value < 0 only queries; *current (may be NULL) receives the value in force.  Results do
 * not depend on it. */
bz_status bz_walk_blocks_per_sm(bz_handle* h, int32_t set_value, int32_t* current);

/* Accelerations (and optionally potentials) of the current state, caller's particle order,
 * SoA 3n floats.  Replaces computeOctreeAccelerationKernel (engine/physics/octree/cuda/force/
 * OctGpu.inl:230-245) / the TreePM force kernels (engine/physics/treepm/short_range/
 * TpmTreeForce.inl:142-159).  pot may be NULL. */
bz_status bz_accelerations(bz_handle* h, float* acc_soa3, float* pot);

/* FP64 diagnostics of the current state, replacing the reference's sampled energy
 * (engine/physics/thermal/energy/ThmEnergyGpu.inl:77,
 * engine/server/simulation/telemetry/SrvSnapshotAndEnergy.cpp:321-349) with
 * full sums: kinetic = sum m v^2 / 2, potential = sum m phi / 2 (runs one potential-evaluating
 * force pass; octree solver only), momentum3 = sum m v.  Any output may be NULL. */
bz_status bz_energy(bz_handle* h, double* kinetic, double* potential, double* momentum3);

/* Download the state in the caller's particle order (ParticleSystem::syncHostState /
 * getParticles, PhyParticleSystem.hpp:351,377).  vel may be NULL.  _f64 returns FP64 state. */
bz_status bz_get_state(bz_handle* h, float* pos_soa3, float* vel_soa3);
bz_status bz_get_state_f64(bz_handle* h, double* pos_soa3, double* vel_soa3);

/* Leapfrog (kick-drift-kick) state with its accelerations, for hosts that keep the state in
 * their own memory between steps (no counterpart in the reference, whose state stays on its
 * device between ParticleSystem::update calls).  bz_get_state_acc returns positions, velocities (may be
 * NULL) and the accelerations of those positions (SoA 3n floats each, caller order; computed
 * first if the handle has none).  bz_set_state_acc uploads a state together with its
 * accelerations, which must be the forces at these positions (as bz_get_state_acc or
 * bz_accelerations returned them): the next bz_step then needs no set-up force evaluation,
 * as a step of a resident state needs none.  A state of the size the handle already holds
 * replaces it in the device's current particle order, so that a round trip through the host
 * keeps the next re-sort cheap; results are those of a fresh upload up to the order of
 * particles with identical keys.  Neither applies to adaptive block steps (BZ_UNSUPPORTED). */
bz_status bz_set_state_acc(bz_handle* h, const float* pos3n, const float* vel3n, const float* mass,
                           const float* acc3n, size_t n);
bz_status bz_get_state_acc(bz_handle* h, float* pos3n, float* vel3n, float* acc3n);

/* The same with the FP64 positions and velocities the engine integrates (accelerations stay
 * FP32, the precision they are computed in), so that a state kept on the host between steps
 * loses nothing to rounding.  Neither allocates device memory. */
bz_status bz_set_state_acc_f64(bz_handle* h, const double* pos3n, const double* vel3n,
                               const float* mass, const float* acc3n, size_t n);
bz_status bz_get_state_acc_f64(bz_handle* h, double* pos3n, double* vel3n, float* acc3n);

/* One bz_step(h, dt, 1) followed by bz_get_state_acc_f64, with the download of the positions
 * overlapping the step: the positions are final after the step's drift, so they are copied to
 * the host on a second stream while the tree, mesh and walk run; velocities and accelerations
 * follow the step.  The result equals that of the two calls bit for bit (the step is launched
 * eagerly rather than as the captured graph).  The first call allocates a staging buffer of
 * 3 x capacity doubles and a stream; not with adaptive block steps.  For hosts that keep the
 * state between steps (bz_set_state_acc_f64 / this call), where each step otherwise pays both
 * transfers in full; no counterpart in the reference, whose state stays on the device. */
bz_status bz_step_get_state_acc_f64(bz_handle* h, double dt, double* pos3n, double* vel3n,
                                    float* acc3n);

/* Morton keys of the current state, sorted, with the stable sort permutation (sorted
 * position -> caller index): buildMortonCodesKernel + thrust::sort_by_key
 * (engine/physics/octree/cuda/linear/OctKeyKernels.inl:22-46, OctBuild.inl:96). */
bz_status bz_morton_keys(bz_handle* h, uint64_t* sorted_keys, int32_t* perm);

/* Tree of the current state.  First call with all arrays NULL to learn the node count.
 * Production octree (breadth-first, node 0 = root):
 *   start/count = particle range in sorted order, child = first child or -1, nchild,
 *   mono4 = {com.xyz, mass}, bmin3/bmax3 = tight box, quad6 = second moments about the COM.
 * Reference mode (BZ_SOLVER_OCTREE_REFERENCE): the reference's node arrays
 *   (engine/physics/octree/cuda/linear/OctLinkKernels.inl:61-113): mono4 <- hot {cx,cy,cz,half}
 *   and bmin3[0..2] unused; see bz_reference_tree. */
bz_status bz_tree_topology(bz_handle* h, int64_t* node_count, int32_t* start, int32_t* count,
                           int32_t* child, int32_t* nchild, float* mono4, float* bmin3,
                           float* bmax3, float* quad6);

/* Reference-mode tree in the reference's packed layout: hot8 = {cx,cy,cz,half,mass,comx,
 * comy,comz}, next, child_mask, first_child, leaf_start, leaf_count (OctLinkKernels.inl:61-113). */
bz_status bz_reference_tree(bz_handle* h, int64_t* node_count, float* hot8, int32_t* next,
                            int32_t* child_mask, int32_t* first_child, int32_t* leaf_start,
                            int32_t* leaf_count);

/* Interaction counts of the last force evaluation (particle-particle, particle-node). */
bz_status bz_interaction_counts(bz_handle* h, uint64_t* n_pp, uint64_t* n_pn);

/* Work counters of the last walk (no counterpart in the reference): listed_pairs = source
 * particles listed for the targets (each listed pair is at least a distance test),
 * evaluated_pairs = pairs taken through the pair law (with a cutoff, those inside it),
 * node_terms = multipole interactions.  Any output may be NULL. */
bz_status bz_walk_counts(bz_handle* h, uint64_t* listed_pairs, uint64_t* evaluated_pairs,
                         uint64_t* node_terms);

/* Per-phase device times of the last bz_step/bz_accelerations call, in milliseconds, from
 * CUDA events on the handle's stream: [0] keys, [1] sort, [2] permute, [3] tree, [4] mesh,
 * [5] walk, [6] integrate, [7] total.  Timing is recorded only when enabled. */
bz_status bz_enable_phase_timing(bz_handle* h, int enable);
bz_status bz_phase_times(bz_handle* h, float* ms, int n);

/* Relative force errors of the current state's accelerations against an FP64 reference on
 * `nsample` seeded targets: direct sum (open) or Ewald (periodic).  Writes the per-target
 * errors |a - a_ref| / |a_ref| (caller order of the sampled targets) if errs != NULL, and
 * the sampled caller indices if idx != NULL. */
bz_status bz_force_errors(bz_handle* h, int32_t nsample, uint64_t seed, float* errs,
                          int32_t* idx, double* median, double* p99);

/* Debug access to the PM mesh of the current state: which = 0 density after the deposit,
 * 1 potential after the solve (gradient modes 0 and 2; the negated potential, whose gradient is
 * the acceleration), 2/3/4 the x/y/z force mesh (modes 0 and 1).  Isolated meshes have 2 grid
 * cells per side.
 * out holds grid^3 floats, index (z*M + y)*M + x. */
bz_status bz_pm_mesh(bz_handle* h, int which, float* out);

/* Mesh grid of the last force evaluation (TreePM): out6 = {origin x, y, z, cell, r_s, r_cut}.
 * Periodic: origin 0, cell = box / grid.  Isolated: the doubled mesh's grid, which follows the
 * particles' bounds (TpmGridBuild.inl:98-171).  No counterpart in the reference's C ABI (its
 * grid is internal). */
bz_status bz_pm_grid(bz_handle* h, double* out6);

/* Kernel launches of this library enqueued so far (cuFFT's own kernels excluded), and the
 * number one bz_step step enqueues. */
uint64_t bz_kernel_launches(void);
bz_status bz_launches_per_step(bz_handle* h, uint64_t* launches);

size_t bz_particle_count(const bz_handle* h);
size_t bz_device_bytes(const bz_handle* h);

/* ---- learned TreePM pair correction (no counterpart in the reference) -----------------
 * A small MLP (6 -> 32 -> 32 -> 3, SiLU, BF16 weights and activations, FP32 accumulation on
 * the tensor cores) maps a close pair's separation (target - source, in mesh cells) and the
 * source's sub-cell offset to the residual of the mesh force of that pair against the ideal
 * Gaussian long-range force (per unit source mass, times h^2).  With the correction enabled,
 * every pair inside the short-range cutoff subtracts m_source / h^2 * prediction from its
 * target's acceleration, which removes most of the mesh's anisotropy error near r_split.
 *
 * bz_learn_generate: residual samples produced by the engine itself for this handle's mesh,
 *   split and assignment: sources on a coarse lattice with random sub-cell offsets, massless
 *   probes around them, PM force minus the FP64 ideal long-range force (Ewald with the split's
 *   real-space part removed).  x6 = {sep_x, sep_y, sep_z, off_x, off_y, off_z}, y3 = residual.
 * bz_learn_train: Adam on the GPU with the library's own forward and backward kernels
 *   (mean squared error of y3 / rms(y3)); keeps the weights in the handle.
 * bz_learn_set / bz_learn_get: weights as kMlpParams = 1667 floats (W1[32][16] with b1 in
 *   column 15, W2[32][32], b2[32], W3[3][32], b3[3]) and the target scale.
 * bz_learn_enable: apply the correction in bz_step / bz_accelerations (TreePM only).
 * bz_learn_forward: batch inference (scale applied); bz_learn_gradient: one backward pass
 *   of the unscaled mean squared error against y3, no update (for gradient checks). */
#define BZ_MLP_PARAMS 1667
bz_status bz_learn_generate(bz_handle* h, int64_t nsamples, uint64_t seed, float* x6, float* y3);
bz_status bz_learn_train(bz_handle* h, const float* x6, const float* y3, int64_t n, int32_t steps,
                         int32_t batch, float lr, uint64_t seed, float* final_loss);
bz_status bz_learn_set(bz_handle* h, const float* params, float scale);
bz_status bz_learn_get(bz_handle* h, float* params, float* scale);
bz_status bz_learn_enable(bz_handle* h, int32_t enable);
bz_status bz_learn_forward(bz_handle* h, const float* x6, int64_t n, float* y3);
bz_status bz_learn_gradient(bz_handle* h, const float* x6, const float* y3, int64_t n, float* grad,
                            float* loss);

/* Allocation-free stable radix sort of device-resident (key, value) pairs, in place, on the
 * calling thread's current device.  No counterpart in the reference (its sort,
 * thrust::sort_by_key, allocates temporary storage on every call).
 *
 * For callers that must not allocate device memory: a host application that reserves HBM
 * for its own pool or arena (a cudaMalloc from a plug-in would fail or escape the pool's
 * accounting), and step loops where cudaMalloc/cudaFree are too costly (cudaFree waits for
 * the whole device).  The handle-based API above allocates in bz_create; this call does
 * not: its scratch is a fixed array in device memory, sized for BZ_SORT_NOALLOC_MAX_KEYS
 * pairs (about 12.6 MiB), that every process loading this library holds on each device it
 * uses until exit.  It calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * keys/values: device (or managed) memory of the current device, n entries each; sorted by
 * the low key_bits bits (8, 16, ..., 64), ties kept in input order (the same order as
 * bz_morton_keys).  stream: a cudaStream_t as an integer (0 = the default stream).  The
 * call returns once the sort has finished on that stream.
 * Returns BZ_INVALID_ARGUMENT for n < 0 or n > BZ_SORT_NOALLOC_MAX_KEYS, key_bits not a
 * multiple of 8 in 8..64, NULL or misaligned pointers, or memory the device cannot address;
 * BZ_DEVICE_LIMIT if a look-back wait gave up; BZ_CUDA_ERROR if a CUDA call failed.
 * The first call on each device looks up the scratch's device address (this may load the
 * library's device code on that device); make that first call before any stream capture.
 * All calls on a device share the one scratch array and it keeps the last call's contents:
 * calls that overlap on the GPU (from several host threads or streams at once) race on it
 * and must be serialised by the caller. */
#define BZ_SORT_NOALLOC_MAX_KEYS 1048576
bz_status bz_sort_pairs_noalloc(uint64_t* keys, uint32_t* values, int64_t n, int key_bits,
                                uint64_t stream);

/* Last error text (blitzar_core_get_last_error, runtime/ffi/core/FfiApi.hpp:99-100).
 * Returns the full length; writes at most cap-1 bytes plus NUL. */
size_t bz_last_error(const bz_handle* h, char* buf, size_t cap);
const char* bz_status_string(bz_status s);
const char* bz_version(void);

#ifdef __cplusplus
}
#endif
#endif
