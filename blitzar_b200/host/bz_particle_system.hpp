// C++ host adapter over the libbzgrav C ABI with the calls of the reference's ParticleSystem
// (engine/physics/core/particle/PhyParticleSystem.hpp:109-718): construction from a particle
// list, the solver setters, update(dt) and the host-state export.  Header-only; links
// against libbzgrav.so.  Errors follow the reference convention: calls return false and the
// message is kept (lastError()), no exceptions on the stepping path.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "bzgrav.h"

namespace bzhost {

// One particle as the reference's Particle carries it for gravity and export
// (engine/physics/core/particle/PhyParticle.hpp:25-183: position, velocity, mass,
// temperature).
struct Particle {
    float px = 0, py = 0, pz = 0;
    float vx = 0, vy = 0, vz = 0;
    float mass = 0;
    float temperature = 0;
};

class GravitySystem {
public:
    enum class SolverMode { OctreeGpu, TreePm, OctreeReference };
    // ParticleSystem::IntegratorMode (PhyParticleSystem.hpp:131-135)
    enum class IntegratorMode { Euler, Rk4, Leapfrog };

    // The integrator starts as symplectic Euler, the reference's default (integrator=euler,
    // SrvSimulationServer.hpp:410); setIntegratorMode(Leapfrog) selects kick-drift-kick.
    explicit GravitySystem(std::vector<Particle> particles) : particles_(std::move(particles))
    {
        bz_config_init(&cfg_);
        cfg_.integrator = BZ_INTEGRATOR_EULER;
    }
    ~GravitySystem() { release(); }
    GravitySystem(const GravitySystem&) = delete;
    GravitySystem& operator=(const GravitySystem&) = delete;

    // setIntegratorMode / getIntegratorMode (PhyParticleSystem.hpp:316-324).  RK4 is not
    // provided (the reference rejects it with octree_gpu, CfgNormalize.cpp:103-106): false.
    bool setIntegratorMode(IntegratorMode m)
    {
        if (m == IntegratorMode::Rk4) {
            err_ = "integrator rk4 is not provided with the octree solvers (euler, leapfrog)";
            return false;
        }
        cfg_.integrator = m == IntegratorMode::Euler ? BZ_INTEGRATOR_EULER : BZ_INTEGRATOR_LEAPFROG;
        invalidate();
        return true;
    }
    IntegratorMode getIntegratorMode() const
    {
        return cfg_.integrator == BZ_INTEGRATOR_EULER ? IntegratorMode::Euler : IntegratorMode::Leapfrog;
    }

    // setters of PhyParticleSystem.hpp:187-252; they take effect at the next update()
    void setSolverMode(SolverMode m)
    {
        cfg_.solver = m == SolverMode::TreePm ? BZ_SOLVER_TREEPM
                      : m == SolverMode::OctreeReference ? BZ_SOLVER_OCTREE_REFERENCE
                                                          : BZ_SOLVER_OCTREE;
        invalidate();
    }
    void setOctreeTheta(float theta) { cfg_.octree_theta = theta; invalidate(); }
    void setOctreeSoftening(float eps) { cfg_.octree_softening = eps; invalidate(); }
    void setOctreeOpeningCriterion(int c) { cfg_.octree_opening_criterion = c; invalidate(); }
    void setLinearOctreeLeafCapacity(int cap) { cfg_.linear_octree_leaf_capacity = cap; invalidate(); }
    void setLeafCapacity(int cap) { cfg_.leaf_capacity = cap; invalidate(); }
    void setMultipoleOrder(int order) { cfg_.multipole_order = order; invalidate(); }
    void setPhysicsStabilityConstants(float max_acceleration, float min_softening,
                                      float min_distance2, float min_theta)
    {
        cfg_.physics_max_acceleration = max_acceleration;
        cfg_.physics_min_softening = min_softening;
        cfg_.physics_min_distance2 = min_distance2;
        cfg_.physics_min_theta = min_theta;
        invalidate();
    }
    // setTreePmParameters with the reference's signature (PhyParticleSystem.hpp:204-207) and
    // clamps (CudSolverConfiguration.inl:55-74), for the path of octree_gpu that integrates
    // leapfrog (CudOctreeGpuIntegrators.inl:75-110), the integrator of this engine:
    //   - TreePM runs when enabled and model != "exact_tree" (the reference's octree_gpu runs
    //     TreePM for every other model when it integrates leapfrog, CudOctreeGpuUpdate.inl:37;
    //     exact_tree names the CPU FP64 pairwise sum, so the octree solver stays);
    //   - it is the reference's isolated TreePM: a mesh of 2 x clamp(gridSize, 32, 128) cells of
    //     max(0.25, extent / (G - 2)) centred on the particles, cutoff clamp(cutoffFactor, 1, 2)
    //     cells, r_s = cutoff / 4.5, CIC / TSC / PCS (any other name: CIC), centred differences
    //     with the 0.08 window floor;
    //   - layout, precision, localGrid, jacobiIterations, maxLocalNeighbors, particleLimit,
    //     denseCellThreshold and gravityOnlyBuffers select the reference's memory layouts, its
    //     CPU precision, its Euler-only local-grid and hybrid kernels and its finite-difference
    //     fallback solver; the reference's leapfrog path does not read them and neither does
    //     this engine (they are kept, clamped as the reference clamps them, for the getters).
    // Returns true (every combination maps); it takes effect at the next update().
    bool setTreePmParameters(bool enabled, const std::string& model, const std::string& layout,
                             const std::string& precision, const std::string& assignment,
                             bool localGrid, int gridSize, int jacobiIterations, float cutoffFactor,
                             int maxLocalNeighbors, int particleLimit, int denseCellThreshold,
                             bool gravityOnlyBuffers)
    {
        tpm_.enabled = enabled;
        tpm_.model = model;
        tpm_.layout = layout;
        tpm_.precision = precision == "fp64" ? "fp64" : "fp32";
        tpm_.assignment = assignment == "tsc" || assignment == "pcs" ? assignment : "cic";
        tpm_.localGrid = localGrid;
        tpm_.gridSize = clampi(gridSize, 32, 128);
        tpm_.jacobiIterations = clampi(jacobiIterations, 4, 64);
        tpm_.cutoffFactor = cutoffFactor < 1.0f ? 1.0f : (cutoffFactor > 2.0f ? 2.0f : cutoffFactor);
        tpm_.maxLocalNeighbors = clampi(maxLocalNeighbors, 0, 256);
        tpm_.particleLimit = particleLimit > 0 ? particleLimit : 0;
        tpm_.denseCellThreshold = denseCellThreshold > 1 ? denseCellThreshold : 1;
        tpm_.gravityOnlyBuffers = gravityOnlyBuffers;
        if (!enabled || model == "exact_tree") {
            cfg_.solver = BZ_SOLVER_OCTREE;
        } else {
            cfg_.solver = BZ_SOLVER_TREEPM;
            cfg_.box_length = 0.0;  // isolated mesh
            cfg_.treepm_grid_size = tpm_.gridSize;
            cfg_.treepm_cell_floor = 0.25f;
            cfg_.treepm_r_split_cells = tpm_.cutoffFactor / 4.5f;
            cfg_.treepm_r_cut_factor = 4.5f;
            cfg_.treepm_assignment = tpm_.assignment == "tsc" ? 1 : (tpm_.assignment == "pcs" ? 2 : 0);
            cfg_.treepm_gradient = 0;
            cfg_.treepm_window_floor = 0.08f;
            cfg_.treepm_node_size_factor = 0.0f;
        }
        invalidate();
        return true;
    }
    // the reference's TreePM settings as last set (getters of the same fields)
    struct TreePmSettings {
        bool enabled = false;
        std::string model = "auto", layout = "auto", precision = "fp32", assignment = "cic";
        bool localGrid = true;
        int gridSize = 64, jacobiIterations = 12;
        float cutoffFactor = 1.0f;
        int maxLocalNeighbors = 64, particleLimit = 0, denseCellThreshold = 64;
        bool gravityOnlyBuffers = true;
    };
    const TreePmSettings& treePmSettings() const { return tpm_; }

    // the periodic TreePM of this engine (no counterpart in the reference's GPU solvers, whose
    // periodic PM is the comoving PM-only cosmology): grid, split and cutoff in mesh cells
    void setPeriodicTreePmParameters(int grid_size, float r_split_cells, float r_cut_factor,
                                     int assignment, int gradient, double box_length)
    {
        cfg_.treepm_grid_size = grid_size;
        cfg_.treepm_r_split_cells = r_split_cells;
        cfg_.treepm_r_cut_factor = r_cut_factor;
        cfg_.treepm_assignment = assignment;
        cfg_.treepm_gradient = gradient;
        cfg_.treepm_window_floor = gradient == 1 ? 0.0f : 0.08f;
        cfg_.box_length = box_length;
        invalidate();
    }
    void setTreePmNodeSizeFactor(float f) { cfg_.treepm_node_size_factor = f; invalidate(); }
    void setTreePmCellFloor(float f) { cfg_.treepm_cell_floor = f; invalidate(); }
    void setDevice(int device) { cfg_.device = device; invalidate(); }
    bz_config& config() { return cfg_; }

    // ParticleSystem::update(dt): one leapfrog step (PhyParticleSystem.hpp:163)
    bool update(float dt) { return step(dt, 1); }
    bool step(double dt, uint32_t nsteps)
    {
        if (!ensure())
            return false;
        return check(bz_step(h_, dt, nsteps));
    }
    // syncHostState(): copy the device state into particles() (PhyParticleSystem.hpp:351)
    bool syncHostState()
    {
        if (!h_)
            return true;  // never uploaded: the host copy is current
        const size_t n = particles_.size();
        std::vector<float> p(3 * n), v(3 * n);
        if (!check(bz_get_state(h_, p.data(), v.data())))
            return false;
        for (size_t i = 0; i < n; ++i) {
            Particle& q = particles_[i];
            q.px = p[i], q.py = p[n + i], q.pz = p[2 * n + i];
            q.vx = v[i], q.vy = v[n + i], q.vz = v[2 * n + i];
        }
        return true;
    }
    const std::vector<Particle>& getParticles() const { return particles_; }
    bool accelerations(std::vector<float>& acc_soa3)
    {
        if (!ensure())
            return false;
        acc_soa3.resize(3 * particles_.size());
        return check(bz_accelerations(h_, acc_soa3.data(), nullptr));
    }
    bool energy(double& kinetic, double& potential, double momentum[3])
    {
        if (!ensure())
            return false;
        return check(bz_energy(h_, &kinetic, &potential, momentum));
    }
    const std::string& lastError() const { return err_; }

private:
    static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
    void invalidate()
    {
        if (h_) {
            syncHostState();
            release();
        }
    }
    void release()
    {
        if (h_)
            bz_destroy(h_);
        h_ = nullptr;
    }
    bool ensure()
    {
        if (h_)
            return true;
        const size_t n = particles_.size();
        if (n == 0)
            return fail("no particles");
        if (bz_create(&cfg_, n, &h_) != BZ_OK) {
            h_ = nullptr;
            return fail("[bz] engine creation failed (configuration or device memory)");
        }
        std::vector<float> p(3 * n), v(3 * n), m(n);
        for (size_t i = 0; i < n; ++i) {
            const Particle& q = particles_[i];
            p[i] = q.px, p[n + i] = q.py, p[2 * n + i] = q.pz;
            v[i] = q.vx, v[n + i] = q.vy, v[2 * n + i] = q.vz;
            m[i] = q.mass;
        }
        return check(bz_set_state(h_, p.data(), v.data(), m.data(), n));
    }
    bool check(bz_status s)
    {
        if (s == BZ_OK)
            return true;
        char buf[1024] = {0};
        if (h_)
            bz_last_error(h_, buf, sizeof buf);
        return fail(std::string("[bz] ") + bz_status_string(s) + (buf[0] ? ": " : "") + buf);
    }
    bool fail(const std::string& m)
    {
        err_ = m;
        return false;
    }

    std::vector<Particle> particles_;
    bz_config cfg_{};
    TreePmSettings tpm_;
    bz_handle* h_ = nullptr;
    std::string err_;
};

} // namespace bzhost
