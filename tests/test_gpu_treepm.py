"""Periodic TreePM: mesh density and potential against the oracle (the reference CPU
templates' formulas driven with a periodic grid), and full forces against oracle PM + the
oracle's periodic split walk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    return Engine(n, **kw)


def _box_particles(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, 3)).astype(np.float32)


@pytest.mark.parametrize("mesh", [16, 32])
def test_density_and_potential(gpu, oracle, mesh):
    n = 30_000
    pos = _box_particles(n, 2)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh) as e:
        e.set_state(pos, None, m)
        rho = e.pm_mesh(0).astype(np.float64)
        phi = e.pm_mesh(1).astype(np.float64)
    _, orho, ophi = oracle.pm_periodic(oracle.pos4(pos, m), mesh, 1.0, 1.25 / mesh, want_fields=True)
    assert np.abs(rho - orho).max() / np.abs(orho).max() < 1e-5
    assert np.abs(phi - ophi).max() / np.abs(ophi).max() < 1e-4


def test_treepm_forces_match_oracle(gpu, oracle):
    n = 16_384
    mesh = 32
    pos = _box_particles(n, 4)
    m = np.full(n, 1.0 / n, np.float32)
    rs = 1.25 / mesh
    rc = 4.5 * rs
    eps = 0.02 / mesh
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, octree_softening=eps) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
    p4 = oracle.pos4(pos, m)
    apm = oracle.pm_periodic(p4, mesh, 1.0, rs)
    keys = oracle.morton63(pos.astype(np.float64), [0, 0, 0], 1.0)
    perm = oracle.stable_sort(keys)
    t = oracle.build_tree(keys[perm], p4[perm], leaf_cap=16)
    w = oracle.walk(p4[perm], t, theta=0.5, eps=eps, rcut=rc, box=1.0, rsplit=rs)
    asr = np.empty_like(w["acc"])
    asr[perm] = w["acc"]
    ref = apm + asr
    err = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(err) < 1e-5 and err.max() < 1e-3, (np.median(err), err.max())


def test_treepm_accuracy_vs_ewald(gpu, oracle):
    n = 4096
    mesh = 16
    rng = np.random.default_rng(6)
    g = (np.arange(16) + 0.5) / 16
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = ((grid + rng.normal(0, 0.3 / 16, grid.shape)) % 1.0).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    eps = 0.02 / mesh
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, octree_softening=eps) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
        fe = e.force_errors(nsample=256, seed=3)
    tg = fe["idx"].astype(np.int64)
    ref = oracle.ewald(oracle.pos4(pos, m), tg, eps=eps, box=1.0, kmax=8)
    err = np.linalg.norm(acc[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    # the device Ewald agrees with the oracle's Ewald
    assert np.allclose(np.sort(err), np.sort(fe["errs"]), rtol=1e-3, atol=1e-6)
    # plain CIC + centred-difference mesh at r_s = 1.25 cells on a 16^3 mesh
    assert np.median(err) < 1.5e-2
