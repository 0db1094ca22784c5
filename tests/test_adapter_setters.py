"""The C++ ParticleSystem adapter (blitzar_b200/host/bz_particle_system.hpp) as a reference caller
uses it: a small program built against the header and libbzgrav.so calls the reference's
13-argument setTreePmParameters (engine/physics/core/particle/PhyParticleSystem.hpp:204-207) and
the other setters, and prints the engine configuration they produce.  The handle is created only
at the first update(), so nothing here touches a GPU."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "blitzar_b200")

PROGRAM = r"""
#include <cstdio>
#include "bz_particle_system.hpp"

static void dump(const char* tag, bzhost::GravitySystem& s, bool ok)
{
    const bz_config& c = s.config();
    const auto& t = s.treePmSettings();
    std::printf("{\"tag\":\"%s\",\"ok\":%d,\"solver\":%d,\"box\":%.9g,\"grid\":%d,\"floor\":%.9g,"
                "\"rs_cells\":%.9g,\"rcut\":%.9g,\"assign\":%d,\"grad\":%d,\"wfloor\":%.9g,"
                "\"t_grid\":%d,\"t_cut\":%.9g,\"t_assign\":\"%s\",\"t_prec\":\"%s\",\"t_jacobi\":%d,"
                "\"t_neigh\":%d,\"t_limit\":%d,\"t_dense\":%d,\"amax\":%.9g,\"integ\":%d}\n",
                tag, ok ? 1 : 0, c.solver, c.box_length, c.treepm_grid_size, c.treepm_cell_floor,
                c.treepm_r_split_cells, c.treepm_r_cut_factor, c.treepm_assignment,
                c.treepm_gradient, c.treepm_window_floor, t.gridSize, t.cutoffFactor,
                t.assignment.c_str(), t.precision.c_str(), t.jacobiIterations,
                t.maxLocalNeighbors, t.particleLimit, t.denseCellThreshold,
                c.physics_max_acceleration, c.integrator);
}

int main()
{
    std::vector<bzhost::Particle> ps(8);
    bzhost::GravitySystem s(ps);
    dump("init", s, true);
    bool ok = s.setTreePmParameters(true, "auto", "auto", "fp32", "tsc", true, 96, 12, 1.5f,
                                    64, 0, 64, true);
    dump("tsc96", s, ok);
    ok = s.setTreePmParameters(true, "tree", "soa", "fp64", "pcs", false, 512, 100, 3.0f,
                               999, -5, 0, false);
    dump("clamped_high", s, ok);
    ok = s.setTreePmParameters(true, "auto", "auto", "fp32", "ngp", true, 8, 1, 0.25f,
                               -1, 10, 5, true);
    dump("clamped_low", s, ok);
    ok = s.setTreePmParameters(true, "exact_tree", "auto", "fp64", "cic", true, 64, 12, 1.0f,
                               64, 0, 64, true);
    dump("exact_tree", s, ok);
    ok = s.setTreePmParameters(false, "auto", "auto", "fp32", "cic", true, 64, 12, 1.0f,
                               64, 0, 64, true);
    dump("disabled", s, ok);
    s.setPhysicsStabilityConstants(32.0f, 1e-4f, 1e-12f, 0.05f);
    ok = s.setIntegratorMode(bzhost::GravitySystem::IntegratorMode::Rk4);
    dump("rk4", s, ok);
    ok = s.setIntegratorMode(bzhost::GravitySystem::IntegratorMode::Leapfrog);
    dump("leapfrog", s, ok);
    return 0;
}
"""


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    if not os.path.exists(os.path.join(LIB_DIR, "libbzgrav.so")):
        pytest.skip("libbzgrav.so not built")
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("adapter")
    src, exe = d / "adapter.cpp", d / "adapter"
    src.write_text(PROGRAM)
    subprocess.run([cxx, "-O1", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(LIB_DIR, "host"), str(src), "-L", LIB_DIR, "-lbzgrav",
                    f"-Wl,-rpath,{LIB_DIR}", "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {d["tag"]: d for d in map(json.loads, out.splitlines())}


def test_adapter_defaults_follow_the_reference(results):
    r = results["init"]
    # octree solver, the reference's clamp default 64, symplectic Euler (BZ_INTEGRATOR_EULER)
    assert r["solver"] == 0 and r["amax"] == 64.0 and r["integ"] == 1


def test_thirteen_argument_setter_maps_onto_the_isolated_treepm(results):
    r = results["tsc96"]
    assert r["ok"] == 1 and r["solver"] == 1 and r["box"] == 0.0
    assert r["grid"] == 96 and r["floor"] == pytest.approx(0.25)
    assert r["rs_cells"] == pytest.approx(1.5 / 4.5) and r["rcut"] == pytest.approx(4.5)
    assert r["assign"] == 1 and r["grad"] == 0 and r["wfloor"] == pytest.approx(0.08)


def test_thirteen_argument_setter_clamps_as_the_reference(results):
    hi, lo = results["clamped_high"], results["clamped_low"]
    # gridSize to [32, 128], cutoffFactor to [1, 2] cells, the Jacobi and neighbour limits too
    assert hi["grid"] == hi["t_grid"] == 128 and hi["t_cut"] == pytest.approx(2.0)
    assert hi["rs_cells"] == pytest.approx(2.0 / 4.5) and hi["assign"] == 2
    assert hi["t_prec"] == "fp64" and hi["t_jacobi"] == 64 and hi["t_neigh"] == 256
    assert hi["t_limit"] == 0 and hi["t_dense"] == 1
    assert lo["grid"] == lo["t_grid"] == 32 and lo["t_cut"] == pytest.approx(1.0)
    # an unknown assignment name is CIC, as in the reference
    assert lo["assign"] == 0 and lo["t_assign"] == "cic"
    assert lo["t_jacobi"] == 4 and lo["t_neigh"] == 0 and lo["t_limit"] == 10 and lo["t_dense"] == 5


def test_exact_tree_and_disabled_keep_the_octree(results):
    assert results["exact_tree"]["ok"] == 1 and results["exact_tree"]["solver"] == 0
    assert results["disabled"]["ok"] == 1 and results["disabled"]["solver"] == 0


def test_integrator_and_stability_setters(results):
    r = results["rk4"]
    assert r["ok"] == 0 and r["integ"] == 1  # rk4 refused, Euler kept
    assert r["amax"] == pytest.approx(32.0)
    assert results["leapfrog"]["ok"] == 1 and results["leapfrog"]["integ"] == 0
