"""CPU-side checks of the product: the C-ABI library loads and exports every symbol its header
declares, argument validation happens before any CUDA call, and the snapshot formats and IC
generators behave."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    from blitzar_b200 import _lib
    from blitzar_b200 import build as b

    if not os.path.exists(_lib.LIB_PATH):
        b.build()
    L = _lib.load()
    header = open(os.path.join(ROOT, "include", "bzgrav.h")).read()
    declared = set(re.findall(r"\b(bz_[a-z0-9_]+)\s*\(", header))
    assert declared >= {"bz_create", "bz_step", "bz_accelerations", "bz_morton_keys"}
    for name in sorted(declared):
        assert hasattr(L, name), name
    assert set(_lib.EXPORTS) == declared
    assert L.bz_version().startswith(b"bzgrav")


def test_reference_gpu_comparator_exports():
    """The reference's GPU octree comparator (oracle/_ref/libbzrefgpu.so, built where a reference
    checkout was at hand) loads and exports its entry points; no GPU call is made here."""
    from oracle import oracle as O

    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libbzrefgpu.so")):
        pytest.skip("reference GPU comparator not built (no reference checkout at build time)")
    R = O.ref_gpu()
    for name in ("refgpu_create", "refgpu_destroy", "refgpu_step", "refgpu_time_steps",
                 "refgpu_accel", "refgpu_get_state"):
        assert hasattr(R, name), name


def test_config_defaults_and_argument_checks():
    import ctypes as C

    from blitzar_b200 import _lib

    L = _lib.load()
    cfg = _lib.default_config()
    assert cfg.octree_theta == pytest.approx(0.5) and cfg.leaf_capacity == 16
    assert cfg.struct_size == C.sizeof(_lib.BzConfig)
    h = C.c_void_p()
    assert L.bz_create(C.byref(cfg), 0, C.byref(h)) == _lib.BZ_INVALID_ARGUMENT
    bad = _lib.default_config()
    bad.struct_size = 4
    assert L.bz_create(C.byref(bad), 10, C.byref(h)) == _lib.BZ_INVALID_ARGUMENT
    assert L.bz_destroy(None) == _lib.BZ_INVALID_ARGUMENT
    assert L.bz_status_string(_lib.BZ_DEVICE_LIMIT) == b"device limit"


def test_nbsimbin_round_trip(tmp_path):
    from blitzar_b200 import snapshot

    rng = np.random.default_rng(0)
    pos = rng.standard_normal((100, 3)).astype(np.float32)
    vel = rng.standard_normal((100, 3)).astype(np.float32)
    m = rng.random(100).astype(np.float32)
    f = tmp_path / "s.bin"
    snapshot.write_bin(f, pos, vel, m)
    raw = f.read_bytes()
    assert raw[:8] == b"NBSIMBIN" and len(raw) == 16 + 32 * 100
    p2, v2, m2, t2 = snapshot.read_bin(f)
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel) and np.array_equal(m2, m)
    assert np.all(t2 == 0)


def test_xyz_format(tmp_path):
    from blitzar_b200 import snapshot

    pos = np.array([[1.0, -2.5, 3.14159265], [1e-7, 123456789.0, 0.0]], np.float32)
    m = np.array([1.0, 0.5], np.float32)
    f = tmp_path / "s.xyz"
    snapshot.write_xyz(f, pos, m, step=7)
    lines = f.read_text().splitlines()
    assert lines[0] == "2" and lines[1] == "solver=octree_gpu integrator=leapfrog step=7"
    assert lines[2] == "P 1 -2.5 3.14159 1 0"
    assert lines[3] == "P 1e-07 1.23457e+08 0 0.5 0"


def test_ic_generators():
    from blitzar_b200 import ics

    pos, vel, m = ics.grf_grid(16, 2)
    assert pos.shape == (4096, 3) and pos.min() >= 0 and pos.max() < 1
    g = (np.arange(16) + 0.5) / 16
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    d = pos - grid
    d -= np.rint(d)
    assert abs(np.sqrt((d ** 2).sum(1).mean()) * 16 - 0.2) < 1e-9
    pos, vel, m = ics.plummer(20000, 1)
    assert abs((m * (vel ** 2).sum(1)).sum() - 3 * np.pi / 32) < 0.02  # 2T for G = M = a = 1
    pos, vel, m = ics.hernquist(20000, 3)
    r = np.linalg.norm(pos, axis=1)
    assert abs(np.median(r) - (1 + np.sqrt(2))) < 0.1  # half-mass radius (untruncated)
    assert r.max() <= 100.0
    pos, vel, m = ics.king(3000, 5, 6.0)
    assert np.isfinite(vel).all() and abs(m.sum() - 1.0) < 1e-12


def _headless():
    from blitzar_b200 import build as b

    if not os.path.exists(b.HEADLESS):
        b.build()
    return b.HEADLESS


def test_headless_resolves_reference_config(tmp_path):
    """The C++ headless driver reads the reference's directive config (and flat keys) into the
    engine configuration without touching a GPU."""
    import json
    import subprocess

    cfg = tmp_path / "sim.ini"
    cfg.write_text(
        "# directive form\n"
        "simulation(particle_count=3073, dt=0.002, solver=octree_gpu, integrator=leapfrog)\n"
        "octree(theta=0.7, softening=0.05, criterion=com, leaf_capacity=256)\n"
        "physics(max_acceleration=64, min_softening=0.0001, min_distance2=1e-12, min_theta=0.05)\n"
        "treepm(enabled=true, assignment=pcs, grid_size=256, cutoff_factor=1.5, model=auto)\n"
        "input_file=state.bin\n")
    out = subprocess.run([_headless(), "--config", str(cfg), "--dry-run"], capture_output=True,
                         text=True, check=True).stdout
    d = json.loads(out)
    # the reference's TreePM keys: the isolated TreePM, grid clamped to 128 (mesh 256), the
    # cutoff in cells clamped to [1, 2] with r_s = cutoff / 4.5, centred differences
    assert d["solver"] == 1 and d["treepm_grid_size"] == 128 and d["treepm_assignment"] == 2
    assert d["box_length"] == 0.0 and d["treepm_gradient"] == 0 and d["dt"] == 0.002
    assert abs(d["treepm_r_split_cells"] - 1.5 / 4.5) < 1e-7 and d["treepm_r_cut_factor"] == 4.5
    assert abs(d["treepm_cell_floor"] - 0.25) < 1e-7
    assert abs(d["octree_theta"] - 0.7) < 1e-7 and abs(d["physics_max_acceleration"] - 64) < 1e-6
    assert d["input"] == "state.bin"
    # exact_tree names the reference's CPU FP64 pairwise sum: octree_gpu keeps the octree
    cfg.write_text("simulation(solver=octree_gpu, integrator=leapfrog)\ntreepm(enabled=true, model=exact_tree)\n")
    d = json.loads(subprocess.run([_headless(), "--config", str(cfg), "--dry-run"], capture_output=True,
                                  text=True, check=True).stdout)
    assert d["solver"] == 0
    # a box length selects this engine's periodic TreePM with its own keys
    cfg.write_text("simulation(solver=octree_gpu, integrator=leapfrog)\n"
                   "treepm(enabled=true, box_length=1, assignment=pcs, grid_size=64, gradient=spectral)\n")
    d = json.loads(subprocess.run([_headless(), "--config", str(cfg), "--dry-run"], capture_output=True,
                                  text=True, check=True).stdout)
    assert d["solver"] == 1 and d["box_length"] == 1.0 and d["treepm_gradient"] == 1
    assert d["treepm_grid_size"] == 64
    # the integrator: the reference's default is symplectic Euler; rk4 is not provided with
    # octree_gpu (the reference rejects the pair too)
    cfg.write_text("simulation(solver=octree_gpu)\n")
    d = json.loads(subprocess.run([_headless(), "--config", str(cfg), "--dry-run"], capture_output=True,
                                  text=True, check=True).stdout)
    assert d["integrator"] == "euler"
    bad = tmp_path / "bad.ini"
    bad.write_text("simulation(solver=octree_gpu, integrator=rk4)\n")
    r = subprocess.run([_headless(), "--config", str(bad), "--dry-run"], capture_output=True, text=True)
    assert r.returncode == 2 and "not provided" in r.stderr
    bad.write_text("solver=pairwise_cuda\n")
    r = subprocess.run([_headless(), "--config", str(bad), "--dry-run"], capture_output=True, text=True)
    assert r.returncode == 2 and "not provided" in r.stderr


def test_headless_snapshot_conversion_matches_python(tmp_path):
    """C++ and Python writers agree byte for byte on .bin and .xyz."""
    import subprocess

    from blitzar_b200 import snapshot

    rng = np.random.default_rng(3)
    pos = (rng.standard_normal((257, 3)) * 10).astype(np.float32)
    vel = rng.standard_normal((257, 3)).astype(np.float32)
    m = rng.random(257).astype(np.float32)
    src = tmp_path / "a.bin"
    snapshot.write_bin(src, pos, vel, m)
    subprocess.run([_headless(), "--convert", str(src), str(tmp_path / "b.bin")], check=True)
    assert (tmp_path / "b.bin").read_bytes() == src.read_bytes()
    subprocess.run([_headless(), "--convert", str(src), str(tmp_path / "c.xyz")], check=True)
    snapshot.write_xyz(tmp_path / "d.xyz", pos, m, solver="octree_gpu", integrator="leapfrog", step=0)
    assert (tmp_path / "c.xyz").read_text() == (tmp_path / "d.xyz").read_text()
