// Headless driver: the reference's `blitzar-headless` batch run on the bzgrav engine.
//
// Reads the reference configuration (the directive form `section(key=value, ...)` of
// simulation.ini, or flat `key=value` lines), loads the initial state from an NBSIMBIN `.bin`
// or `.xyz` file, advances the requested number of leapfrog steps through GravitySystem, and
// exports the final state in the reference's formats (.bin: SrvPersistenceInternal.hpp:21-39,
// writer SrvIO.cpp:139-165; .xyz: SrvIO.cpp:173-181).  Keys and flags follow the reference
// (engine/config/registry/entries/CfgEntriesCore.cpp; --config, --run, --target-steps,
// --export-on-exit, --export-format, --export-path).
//
// Modes that need no GPU: --dry-run prints the resolved engine configuration as JSON;
// --convert IN OUT rewrites a snapshot in another format.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "bz_particle_system.hpp"

namespace {

using bzhost::GravitySystem;
using bzhost::Particle;

std::string trim(const std::string& s)
{
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos)
        return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::string unquote(std::string v)
{
    v = trim(v);
    if (v.size() >= 2 && v.front() == '"' && v.back() == '"')
        v = v.substr(1, v.size() - 2);
    return v;
}

// Both forms end up as flat keys: `octree(theta=0.5)` -> "octree_theta", `theta=0.5` -> "theta".
bool parse_config(const std::string& path, std::map<std::string, std::string>& kv, std::string& err)
{
    std::ifstream f(path);
    if (!f) {
        err = "cannot open config " + path;
        return false;
    }
    std::string line;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        line = trim(line);
        if (line.empty() || line[0] == '#' || line[0] == ';' || line[0] == '[')
            continue;
        const size_t paren = line.find('(');
        const size_t eq = line.find('=');
        if (paren != std::string::npos && (eq == std::string::npos || paren < eq)) {
            const size_t close = line.rfind(')');
            if (close == std::string::npos || close < paren) {
                err = path + ":" + std::to_string(lineno) + ": unterminated directive";
                return false;
            }
            const std::string section = trim(line.substr(0, paren));
            const std::string body = line.substr(paren + 1, close - paren - 1);
            // split on commas outside quotes
            std::vector<std::string> items;
            std::string cur;
            bool q = false;
            for (char c : body) {
                if (c == '"')
                    q = !q;
                if (c == ',' && !q) {
                    items.push_back(cur);
                    cur.clear();
                } else {
                    cur += c;
                }
            }
            if (!trim(cur).empty())
                items.push_back(cur);
            for (const std::string& it : items) {
                const size_t e = it.find('=');
                if (e == std::string::npos)
                    continue;
                kv[section + "_" + trim(it.substr(0, e))] = unquote(it.substr(e + 1));
            }
        } else if (eq != std::string::npos) {
            kv[trim(line.substr(0, eq))] = unquote(line.substr(eq + 1));
        } else {
            err = path + ":" + std::to_string(lineno) + ": cannot parse '" + line + "'";
            return false;
        }
    }
    return true;
}

const std::string* lookup(const std::map<std::string, std::string>& kv,
                          std::initializer_list<const char*> names)
{
    for (const char* n : names) {
        auto it = kv.find(n);
        if (it != kv.end())
            return &it->second;
    }
    return nullptr;
}

template <class T> bool get_num(const std::map<std::string, std::string>& kv,
                                std::initializer_list<const char*> names, T& out)
{
    const std::string* v = lookup(kv, names);
    if (!v)
        return false;
    std::istringstream is(*v);
    T x{};
    if (!(is >> x))
        return false;
    out = x;
    return true;
}

bool truthy(const std::string& v) { return v == "true" || v == "1" || v == "yes" || v == "on"; }

// ---- snapshot formats
bool read_bin(const std::string& path, std::vector<Particle>& ps, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    char magic[8];
    uint32_t version = 0, count = 0;
    if (!f.read(magic, 8) || std::memcmp(magic, "NBSIMBIN", 8) != 0) {
        err = path + ": not an NBSIMBIN file";
        return false;
    }
    f.read(reinterpret_cast<char*>(&version), 4);
    f.read(reinterpret_cast<char*>(&count), 4);
    if (version != 1) {
        err = path + ": unsupported NBSIMBIN version " + std::to_string(version);
        return false;
    }
    ps.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        float r[8];
        if (!f.read(reinterpret_cast<char*>(r), sizeof r)) {
            err = path + ": truncated";
            return false;
        }
        ps[i] = Particle{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]};
    }
    return true;
}

bool write_bin(const std::string& path, const std::vector<Particle>& ps)
{
    std::ofstream f(path, std::ios::binary);
    const uint32_t version = 1, count = static_cast<uint32_t>(ps.size());
    f.write("NBSIMBIN", 8);
    f.write(reinterpret_cast<const char*>(&version), 4);
    f.write(reinterpret_cast<const char*>(&count), 4);
    for (const Particle& p : ps) {
        const float r[8] = {p.px, p.py, p.pz, p.vx, p.vy, p.vz, p.mass, p.temperature};
        f.write(reinterpret_cast<const char*>(r), sizeof r);
    }
    return static_cast<bool>(f);
}

// .xyz carries no velocities (the reference's import leaves them zero)
bool read_xyz(const std::string& path, std::vector<Particle>& ps, std::string& err)
{
    std::ifstream f(path);
    size_t n = 0;
    std::string line;
    if (!(f >> n)) {
        err = path + ": missing particle count";
        return false;
    }
    std::getline(f, line);
    std::getline(f, line);
    ps.assign(n, Particle{});
    for (size_t i = 0; i < n; ++i) {
        std::string tag;
        Particle& p = ps[i];
        if (!(f >> tag >> p.px >> p.py >> p.pz >> p.mass >> p.temperature)) {
            err = path + ": truncated";
            return false;
        }
    }
    return true;
}

bool write_xyz(const std::string& path, const std::vector<Particle>& ps, const std::string& solver,
               const std::string& integrator, uint64_t step)
{
    std::ofstream f(path);
    f << ps.size() << "\n" << "solver=" << solver << " integrator=" << integrator
      << " step=" << step << "\n";
    for (const Particle& p : ps)
        f << "P " << p.px << " " << p.py << " " << p.pz << " " << p.mass << " " << p.temperature
          << "\n";
    return static_cast<bool>(f);
}

bool ends_with(const std::string& s, const std::string& t)
{
    return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

bool load(const std::string& path, const std::string& fmt, std::vector<Particle>& ps, std::string& err)
{
    const bool xyz = fmt == "xyz" || (fmt != "bin" && ends_with(path, ".xyz"));
    return xyz ? read_xyz(path, ps, err) : read_bin(path, ps, err);
}

bool save(const std::string& path, const std::string& fmt, const std::vector<Particle>& ps,
          const std::string& solver, const std::string& integrator, uint64_t step)
{
    const bool xyz = fmt == "xyz" || (fmt != "bin" && ends_with(path, ".xyz"));
    return xyz ? write_xyz(path, ps, solver, integrator, step) : write_bin(path, ps);
}

struct RunConfig {
    std::string solver = "octree_gpu";
    std::string integrator = "euler";  // the reference's default (CfgMain.cpp)
    bool treepm = false;
    double dt = 1e-3;
    std::string input, input_format = "auto";
};

int fail(const std::string& m)
{
    std::cerr << "[headless] error: " << m << "\n";
    return 2;
}

// Resolve the engine configuration from the reference keys.
bool resolve(const std::map<std::string, std::string>& kv, GravitySystem& sys, RunConfig& rc,
             std::string& err)
{
    if (const std::string* s = lookup(kv, {"simulation_solver", "solver"}))
        rc.solver = *s;
    if (rc.solver == "octree-gpu")
        rc.solver = "octree_gpu";
    if (rc.solver != "octree_gpu" && rc.solver != "octree_reference") {
        err = "solver=" + rc.solver + " is not provided by this engine (octree_gpu, with "
              "treepm(enabled=true) for TreePM, or octree_reference)";
        return false;
    }
    if (const std::string* s = lookup(kv, {"simulation_integrator", "integrator"}))
        rc.integrator = *s;
    if (rc.integrator != "leapfrog" && rc.integrator != "euler") {
        err = "integrator=" + rc.integrator + " is not provided with octree_gpu (euler or leapfrog)";
        return false;
    }
    sys.setIntegratorMode(rc.integrator == "euler" ? GravitySystem::IntegratorMode::Euler
                                                   : GravitySystem::IntegratorMode::Leapfrog);
    if (const std::string* s = lookup(kv, {"treepm_enabled"}))
        rc.treepm = truthy(*s);
    get_num(kv, {"substep_target_dt", "simulation_dt", "dt"}, rc.dt);
    if (const std::string* s = lookup(kv, {"input_file", "scene_file"}))
        rc.input = *s;
    if (const std::string* s = lookup(kv, {"input_format", "scene_format"}))
        rc.input_format = *s;

    bz_config& c = sys.config();
    get_num(kv, {"octree_theta"}, c.octree_theta);
    get_num(kv, {"octree_softening"}, c.octree_softening);
    if (const std::string* s = lookup(kv, {"octree_criterion", "octree_opening_criterion"}))
        c.octree_opening_criterion = *s == "bounds" ? 1 : 0;
    get_num(kv, {"octree_leaf_capacity", "linear_octree_leaf_capacity"}, c.linear_octree_leaf_capacity);
    get_num(kv, {"leaf_capacity", "bz_leaf_capacity"}, c.leaf_capacity);
    get_num(kv, {"multipole_order", "octree_multipole_order"}, c.multipole_order);
    get_num(kv, {"physics_max_acceleration"}, c.physics_max_acceleration);
    get_num(kv, {"physics_min_softening"}, c.physics_min_softening);
    get_num(kv, {"physics_min_distance2"}, c.physics_min_distance2);
    get_num(kv, {"physics_min_theta"}, c.physics_min_theta);
    if (rc.solver == "octree_reference") {
        c.solver = BZ_SOLVER_OCTREE_REFERENCE;
    } else if (rc.treepm && !lookup(kv, {"treepm_box_length", "box_length"})) {
        // the reference's TreePM keys (CfgEntriesCore.cpp:75-117, defaults CfgConfig.hpp:49-62)
        // through the reference's setter: the isolated TreePM of octree_gpu
        std::string model = "auto", layout = "auto", precision = "fp32", assignment = "cic";
        bool local_grid = true, gravity_only = true;
        int grid = 64, jacobi = 12, max_neighbors = 64, particle_limit = 0, dense = 64;
        float cutoff = 1.0f;
        if (const std::string* s = lookup(kv, {"treepm_model"}))
            model = *s;
        if (const std::string* s = lookup(kv, {"treepm_layout"}))
            layout = *s;
        if (const std::string* s = lookup(kv, {"treepm_precision"}))
            precision = *s;
        if (const std::string* s = lookup(kv, {"treepm_assignment"}))
            assignment = *s;
        if (const std::string* s = lookup(kv, {"treepm_local_grid"}))
            local_grid = truthy(*s);
        if (const std::string* s = lookup(kv, {"treepm_gravity_only_buffers"}))
            gravity_only = truthy(*s);
        get_num(kv, {"treepm_grid_size"}, grid);
        get_num(kv, {"treepm_jacobi_iterations"}, jacobi);
        get_num(kv, {"treepm_cutoff_factor"}, cutoff);
        get_num(kv, {"treepm_max_local_neighbors"}, max_neighbors);
        get_num(kv, {"treepm_particle_limit"}, particle_limit);
        get_num(kv, {"treepm_dense_cell_threshold"}, dense);
        sys.setTreePmParameters(true, model, layout, precision, assignment, local_grid, grid, jacobi,
                                cutoff, max_neighbors, particle_limit, dense, gravity_only);
    } else if (rc.treepm) {
        // this engine's periodic TreePM (a box length given): grid, split and cutoff in cells
        c.solver = BZ_SOLVER_TREEPM;
        get_num(kv, {"treepm_grid_size"}, c.treepm_grid_size);
        get_num(kv, {"treepm_r_split_cells"}, c.treepm_r_split_cells);
        get_num(kv, {"treepm_r_cut_factor"}, c.treepm_r_cut_factor);
        get_num(kv, {"treepm_node_size_factor"}, c.treepm_node_size_factor);
        get_num(kv, {"treepm_box_length", "box_length"}, c.box_length);
        if (c.box_length <= 0.0) {
            err = "treepm box_length must be positive (omit it for the isolated TreePM)";
            return false;
        }
        if (const std::string* s = lookup(kv, {"treepm_assignment"})) {
            if (*s == "cic")
                c.treepm_assignment = 0;
            else if (*s == "tsc")
                c.treepm_assignment = 1;
            else if (*s == "pcs")
                c.treepm_assignment = 2;
            else {
                err = "treepm_assignment=" + *s + " (cic, tsc or pcs)";
                return false;
            }
        }
        if (const std::string* s = lookup(kv, {"treepm_gradient"})) {
            c.treepm_gradient = *s == "spectral" ? 1 : (*s == "analytic" ? 2 : 0);
            c.treepm_window_floor = c.treepm_gradient ? 0.0f : 0.08f;
        }
    } else {
        c.solver = BZ_SOLVER_OCTREE;
    }
    return true;
}

void print_json(const RunConfig& rc, const bz_config& c)
{
    std::printf("{\"solver\": %d, \"integrator\": \"%s\", \"dt\": %.17g, \"octree_theta\": %.9g, "
                "\"octree_softening\": %.9g, \"leaf_capacity\": %d, \"multipole_order\": %d, "
                "\"physics_max_acceleration\": %.9g, \"treepm_grid_size\": %d, "
                "\"treepm_r_split_cells\": %.9g, \"treepm_r_cut_factor\": %.9g, "
                "\"treepm_assignment\": %d, \"treepm_gradient\": %d, \"box_length\": %.17g, "
                "\"treepm_cell_floor\": %.9g, \"input\": \"%s\"}\n",
                c.solver, rc.integrator.c_str(), rc.dt, c.octree_theta, c.octree_softening,
                c.leaf_capacity, c.multipole_order, c.physics_max_acceleration, c.treepm_grid_size,
                c.treepm_r_split_cells, c.treepm_r_cut_factor, c.treepm_assignment,
                c.treepm_gradient, c.box_length, c.treepm_cell_floor, rc.input.c_str());
}

} // namespace

int main(int argc, char** argv)
{
    std::string config, export_path, export_format = "bin", input_override;
    uint64_t target_steps = 0;
    bool run = false, export_on_exit = true, dry = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](const char* what) -> std::string {
            if (i + 1 >= argc) {
                std::cerr << "[headless] error: " << what << " needs a value\n";
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--config")
            config = next("--config");
        else if (a == "--run")
            run = true;
        else if (a == "--target-steps")
            target_steps = std::stoull(next("--target-steps"));
        else if (a == "--export-on-exit")
            export_on_exit = truthy(next("--export-on-exit"));
        else if (a == "--export-format")
            export_format = next("--export-format");
        else if (a == "--export-path")
            export_path = next("--export-path");
        else if (a == "--input")
            input_override = next("--input");
        else if (a == "--dry-run")
            dry = true;
        else if (a == "--convert") {
            if (i + 2 >= argc)
                return fail("--convert IN OUT");
            const std::string in = argv[++i], out = argv[++i];
            std::vector<Particle> ps;
            std::string err;
            if (!load(in, "auto", ps, err))
                return fail(err);
            if (!save(out, "auto", ps, "octree_gpu", "leapfrog", 0))
                return fail("cannot write " + out);
            return 0;
        } else if (a == "--help" || a == "-h") {
            std::cout << "usage: bz_headless --config FILE [--input FILE] [--run] [--target-steps K]\n"
                         "       [--export-on-exit true|false] [--export-format bin|xyz] "
                         "[--export-path FILE] [--dry-run]\n"
                         "       bz_headless --convert IN OUT\n";
            return 0;
        } else {
            return fail("unknown argument " + a);
        }
    }
    std::map<std::string, std::string> kv;
    std::string err;
    if (!config.empty() && !parse_config(config, kv, err))
        return fail(err);
    RunConfig rc;
    GravitySystem probe({});
    if (!resolve(kv, probe, rc, err))
        return fail(err);
    if (!input_override.empty())
        rc.input = input_override;
    if (dry) {
        print_json(rc, probe.config());
        return 0;
    }
    if (rc.input.empty())
        return fail("no input state (input_file=... or --input)");
    std::vector<Particle> ps;
    if (!load(rc.input, rc.input_format, ps, err))
        return fail(err);
    GravitySystem sys(std::move(ps));
    sys.config() = probe.config();
    uint64_t done = 0;
    double ms = 0.0;
    if (run && target_steps > 0) {
        const auto t0 = std::chrono::steady_clock::now();
        if (!sys.step(rc.dt, static_cast<uint32_t>(target_steps)))
            return fail(sys.lastError());
        if (!sys.syncHostState())
            return fail(sys.lastError());
        ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        done = target_steps;
    }
    const std::string solver = rc.treepm ? "octree_gpu+treepm" : rc.solver;
    std::printf("[headless] done steps=%llu integrate_ms=%.3f particles=%zu solver=%s\n",
                static_cast<unsigned long long>(done), ms, sys.getParticles().size(), solver.c_str());
    if (export_on_exit && !export_path.empty()) {
        if (!save(export_path, export_format, sys.getParticles(), rc.solver, rc.integrator, done))
            return fail("cannot write " + export_path);
    }
    return 0;
}
