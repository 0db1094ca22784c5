"""Periodic TreePM: mesh density and potential against the oracle (the reference CPU
templates' formulas driven with a periodic grid), and full forces against oracle PM + the
oracle's periodic split walk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
    return Engine(n, **kw)


def _box_particles(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, 3)).astype(np.float32)


ASSIGN = {"cic": 0, "tsc": 1, "pcs": 2}


@pytest.mark.parametrize("mesh", [16, 32])
@pytest.mark.parametrize("assignment", ["cic", "tsc", "pcs"])
def test_density_and_potential(gpu, oracle, mesh, assignment):
    n = 30_000
    pos = _box_particles(n, 2)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh,
                 treepm_assignment=ASSIGN[assignment]) as e:
        e.set_state(pos, None, m)
        rho = e.pm_mesh(0).astype(np.float64)
        phi = e.pm_mesh(1).astype(np.float64)
    _, orho, ophi = oracle.pm_periodic(oracle.pos4(pos, m), mesh, 1.0, 1.25 / mesh, want_fields=True,
                                       assignment=assignment)
    assert np.abs(rho - orho).max() / np.abs(orho).max() < 1e-5
    assert np.abs(phi - ophi).max() / np.abs(ophi).max() < 1e-4


@pytest.mark.parametrize("gradient", [1, 2])
@pytest.mark.parametrize("assignment", ["cic", "tsc", "pcs"])
def test_spectral_force_mesh(gpu, oracle, assignment, gradient):
    """Mesh forces of the fused Green x i k gradient (1) and of analytic differentiation (2: the
    potential interpolated with the gradient of the assignment weights) match the oracle."""
    n, mesh = 20_000, 32
    pos = _box_particles(n, 12)
    m = np.full(n, 1.0 / n, np.float32)
    rs = 1.25 / mesh
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, treepm_assignment=ASSIGN[assignment],
                 treepm_gradient=gradient, treepm_window_floor=0.0, treepm_r_cut_factor=1e-3) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
    ref = oracle.pm_periodic(oracle.pos4(pos, m), mesh, 1.0, rs, assignment=assignment,
                             window_floor=0.0, gradient=gradient)
    dev = np.linalg.norm(acc - ref, axis=1)
    net = np.linalg.norm(ref, axis=1)
    # FP32 transforms (cuFFT) against FP64 ones: 1e-5 relative, or 1e-5 of the rms mesh force
    # for particles whose mesh force is far below it (the transforms' rounding is global)
    rms = np.sqrt((net ** 2).mean())
    assert np.median(dev / net) < 1e-5
    assert (dev <= 1e-5 * np.maximum(net, rms)).all(), ((dev / np.maximum(net, rms)).max())


@pytest.mark.parametrize("variant", ["reference", "production", "analytic"])
def test_treepm_forces_match_oracle(gpu, oracle, variant):
    """reference: CIC, centred differences; production: PCS with the spectral gradient;
    analytic: PCS with analytic differentiation of the assignment weights."""
    n = 16_384
    mesh = 32
    pos = _box_particles(n, 4)
    m = np.full(n, 1.0 / n, np.float32)
    rs = 1.25 / mesh
    prod = variant != "reference"
    grad = {"reference": 0, "production": 1, "analytic": 2}[variant]
    rcf = 5.5 if prod else 4.5
    rc = rcf * rs
    eps = 0.02 / mesh
    kw = dict(treepm_assignment=2, treepm_gradient=grad, treepm_window_floor=0.0) if prod else {}
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, octree_softening=eps,
                 treepm_r_cut_factor=rcf, **kw) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
    p4 = oracle.pos4(pos, m)
    apm = oracle.pm_periodic(p4, mesh, 1.0, rs, assignment="pcs" if prod else "cic", gradient=grad,
                             window_floor=0.0 if prod else 0.08)
    keys = oracle.morton63(pos.astype(np.float64), [0, 0, 0], 1.0)
    perm = oracle.stable_sort(keys)
    t = oracle.build_tree(keys[perm], p4[perm], leaf_cap=16)
    a_s, s_s = oracle.walk_targets(p4[perm], t, np.arange(n), theta=0.5, eps=eps, rcut=rc, box=1.0,
                                   rsplit=rs, quadrupole=True)
    asr = np.empty_like(a_s)
    asr[perm] = a_s
    asum = np.empty_like(s_s)
    asum[perm] = s_s
    ref = apm + asr
    dev = np.linalg.norm(acc - ref, axis=1)
    net = np.linalg.norm(ref, axis=1)
    # 1e-5 relative, or the worst-case rounding of an FP32 sum of 64 terms of total magnitude
    # S = sum |a_j| + |a_mesh| where the net force is a cancellation (see test_gpu_treepm_scale)
    bound = 64.0 * 2.0 ** -24 * (asum + np.linalg.norm(apm, axis=1))
    assert np.median(dev / net) < 1e-5
    assert (dev <= np.maximum(1e-5 * net, bound)).all(), (dev / net).max()


@pytest.mark.parametrize("schedule", [0, 2])
def test_treepm_acceleration_clamp(gpu, oracle, schedule):
    """TreePM with the reference's default clamp (64): the walk's sum is clamped, then its sum
    with the mesh force (treePmComputeAcceleration, TpmTreeForce.inl:9-25), whether the mesh
    force is computed in line (schedule 0: the walk clamps the total) or concurrently (schedule
    2: the sum is completed and clamped after the join)."""
    n, mesh = 16_384, 32
    pos = _box_particles(n, 33)
    rng = np.random.default_rng(34)
    pick = rng.choice(n, 40, replace=False)
    pos[pick[20:]] = (pos[pick[:20]] + np.float32(2e-4) * rng.standard_normal((20, 3)).astype(np.float32)) % 1.0
    m = np.full(n, 1.0 / n, np.float32)
    rs = 1.25 / mesh
    rc = 5.5 * rs
    eps = 2e-4
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, octree_softening=eps,
                 treepm_r_cut_factor=5.5, treepm_assignment=2, treepm_gradient=1,
                 treepm_window_floor=0.0, physics_max_acceleration=64.0) as e:
        e.set_state(pos, None, m)
        e.set_mesh_schedule(schedule)
        acc = e.accelerations().astype(np.float64)
    p4 = oracle.pos4(pos, m)
    apm = oracle.pm_periodic(p4, mesh, 1.0, rs, assignment="pcs", spectral=True, window_floor=0.0)
    keys = oracle.morton63(pos.astype(np.float64), [0, 0, 0], 1.0)
    perm = oracle.stable_sort(keys)
    t = oracle.build_tree(keys[perm], p4[perm], leaf_cap=16)
    w = oracle.walk(p4[perm], t, theta=0.5, eps=eps, rcut=rc, box=1.0, rsplit=rs)
    asr = np.empty_like(w["acc"])
    asr[perm] = w["acc"]
    assert (np.linalg.norm(asr, axis=1) > 64.0).sum() >= 10
    ref = oracle.clamp_acceleration(apm + oracle.clamp_acceleration(asr, 64.0), 64.0)
    clamped = np.linalg.norm(asr, axis=1) > 64.0
    err = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err[clamped].max() < 1e-5, err[clamped].max()
    assert np.median(err) < 1e-5
    assert np.linalg.norm(acc, axis=1).max() <= 64.0 * (1 + 1e-6)


@pytest.mark.parametrize("variant", ["reference", "production"])
def test_treepm_accuracy_vs_ewald(gpu, oracle, variant):
    """32^3 GRF-displaced grid against FP64 Ewald.  reference: the reference mesh (CIC, centred
    differences, mesh = particle lattice, r_cut 4.5 r_s).  production: PCS, spectral gradient,
    mesh = 2x the lattice, r_s = 1.25 mesh cells, r_cut 5 r_s, no multipoles inside the cutoff."""
    from blitzar_b200 import ics

    pos, _, m = ics.grf_grid(32, 2)
    pos, m = pos.astype(np.float32), m.astype(np.float32)
    n = len(m)
    eps = 0.02 / 32
    prod = variant == "production"
    if prod:
        kw = dict(treepm_grid_size=64, treepm_assignment=2, treepm_gradient=1, treepm_window_floor=0.0,
                  treepm_r_cut_factor=5.0, treepm_node_size_factor=0.5)
    else:
        kw = dict(treepm_grid_size=32)
    with _engine(n, solver=1, box_length=1.0, octree_softening=eps, **kw) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
        fe = e.force_errors(nsample=256, seed=3)
    tg = fe["idx"].astype(np.int64)
    ref = oracle.ewald(oracle.pos4(pos, m), tg, eps=eps, box=1.0, kmax=8)
    err = np.linalg.norm(acc[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    # the device Ewald agrees with the oracle's Ewald
    assert np.allclose(np.sort(err), np.sort(fe["errs"]), rtol=1e-3, atol=1e-6)
    if prod:
        assert np.median(err) < 1e-3 and np.percentile(err, 99) < 1e-2, (np.median(err), np.percentile(err, 99))
    else:
        assert np.median(err) < 5e-2


def test_node_size_cap_matches_oracle(gpu, oracle):
    """The short-range node-size cap gives the oracle's interaction lists exactly."""
    n, mesh = 16_384, 32
    pos = _box_particles(n, 21)
    m = np.full(n, 1.0 / n, np.float32)
    rs = np.float32(1.25 * 1.0 / mesh)
    eps = 0.02 / mesh
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=mesh, octree_softening=eps,
                 treepm_node_size_factor=1.5, treepm_r_cut_factor=5.0) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
        npp, npn = e.interaction_counts()
    p4 = oracle.pos4(pos, m)
    keys = oracle.morton63(pos.astype(np.float64), [0, 0, 0], 1.0)
    perm = oracle.stable_sort(keys)
    t = oracle.build_tree(keys[perm], p4[perm], leaf_cap=16)
    w = oracle.walk(p4[perm], t, theta=0.5, eps=eps, rcut=np.float32(5.0) * rs, box=1.0, rsplit=rs,
                    max_node_size=np.float32(1.5) * rs)
    sizes = w["group_sizes"]
    assert npp == int((w["n_pp"] * sizes).sum())
    assert npn == int((w["n_pn"] * sizes).sum())


def _treepm_run(schedule, pos, vel, m, steps, use_graph=1, tune=False):
    n = len(m)
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=64, treepm_assignment=2,
                 treepm_gradient=1, treepm_window_floor=0.0, treepm_r_cut_factor=5.0,
                 treepm_node_size_factor=0.5, octree_softening=0.02 / 64, use_graph=use_graph) as e:
        e.set_state(pos, vel, m, f64=True)
        if tune:
            before = e.get_state(f64=True)
            e.autotune(trials=1)
            after = e.get_state(f64=True)
            return before, after, e.last_tune
        e.set_mesh_schedule(schedule)
        e.step(1e-3, steps)
        return e.get_state(f64=True)


@pytest.mark.parametrize("use_graph", [0, 1])
def test_mesh_schedules_agree(gpu, use_graph):
    """The three mesh-leg schedules (in line; concurrent with the tree build and walk; deposit and
    field solve forked at the drift) compute the same step: they differ only in the order of the
    float mass sums of the deposit."""
    n = 32 ** 3
    rng = np.random.default_rng(41)
    g = (np.indices((32, 32, 32)).reshape(3, -1).T + 0.5) / 32.0
    pos = (g + 0.2 / 32 * rng.standard_normal(g.shape)) % 1.0
    vel = 0.05 * rng.standard_normal(g.shape)
    m = np.full(n, 1.0 / n, np.float32)
    runs = [_treepm_run(s, pos, vel, m, 6, use_graph) for s in (0, 1, 2)]
    for p, v in runs[1:]:
        assert np.abs(p - runs[0][0]).max() < 1e-9
        assert np.abs(v - runs[0][1]).max() < 1e-6 * np.abs(runs[0][1]).max()


def test_autotune_leaves_state_unchanged(gpu):
    """The autotuner times zero-length steps: positions and velocities come out bit for bit."""
    n = 16 ** 3
    rng = np.random.default_rng(42)
    pos = rng.random((n, 3))
    vel = 0.1 * rng.standard_normal((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    before, after, tune = _treepm_run(None, pos, vel, m, 0, tune=True)
    assert tune["mesh_schedule"] in (0, 1, 2)
    for a, b in zip(before, after):  # caller order
        assert np.array_equal(a, b)


def test_walk_block_cap_does_not_change_results(gpu):
    """Capping the persistent walk's resident blocks per SM (room for the concurrent mesh leg)
    changes only the grid: every group is still walked by one warp in the same way (bit for bit
    in the tree-only solver; TreePM adds mesh forces whose float atomics sum in any order)."""
    n = 24 ** 3
    rng = np.random.default_rng(43)
    pos = rng.random((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    for treepm in (False, True):
        kw = dict(solver=1, box_length=1.0, treepm_grid_size=32, treepm_assignment=2,
                  treepm_gradient=1, treepm_window_floor=0.0, treepm_r_cut_factor=5.0,
                  treepm_node_size_factor=0.5, octree_softening=0.02 / 32) if treepm else {}
        out = []
        for cap in (0, 2, 5):
            with _engine(n, **kw) as e:
                e.set_state(pos, None, m, f64=True)
                assert e.walk_blocks_per_sm(cap) == cap
                out.append(e.accelerations().astype(np.float64))
        for a in out[1:]:
            if treepm:
                scale = np.linalg.norm(out[0], axis=1).max()
                assert np.abs(a - out[0]).max() < 1e-5 * scale
            else:
                assert np.array_equal(a, out[0])


def test_node_cap_walk_needs_no_multipoles(gpu):
    """With the node-size cap no node is accepted inside the cutoff on a near-uniform box, so the
    monopole walk (which also skips the tree's second moments) gives the quadrupole walk's
    forces; only the mesh's float reductions may order differently."""
    n = 32 ** 3
    rng = np.random.default_rng(44)
    g = (np.indices((32, 32, 32)).reshape(3, -1).T + 0.5) / 32.0
    pos = (g + 0.2 / 32 * rng.standard_normal(g.shape)) % 1.0
    m = np.full(n, 1.0 / n, np.float32)
    out = []
    for order in (2, 1):
        with _engine(n, solver=1, box_length=1.0, treepm_grid_size=64, treepm_assignment=2,
                     treepm_gradient=1, treepm_window_floor=0.0, treepm_r_cut_factor=5.0,
                     treepm_node_size_factor=0.5, octree_softening=0.02 / 32,
                     multipole_order=order) as e:
            e.set_state(pos, None, m, f64=True)
            out.append(e.accelerations().astype(np.float64))
            pp, pn = e.interaction_counts()
            assert pn == 0 and pp > 0
    scale = np.linalg.norm(out[0], axis=1).max()
    assert np.abs(out[1] - out[0]).max() < 1e-6 * scale


@pytest.mark.parametrize("assignment,gradient", [("cic", 0), ("tsc", 0), ("pcs", 0), ("pcs", 2)])
def test_isolated_treepm_matches_oracle(gpu, oracle, assignment, gradient):
    """Open-boundary TreePM (box_length 0), the reference's GPU TreePM: a doubled mesh of 2G
    cells of max(0.25, extent / (G - 2)), centred on the particles, r_s = cutoffFactor x cell
    / 4.5 (here cutoffFactor 1.5), r_cut = 4.5 r_s.  The device-computed grid equals the
    oracle's FP32 grid; density, and forces (isolated PM + open cutoff walk), match."""
    n, G = 20_000, 32
    rng = np.random.default_rng(51)
    pos = (rng.standard_normal((n, 3)) * 1.5).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    eps = 0.01
    rs_cells = np.float32(1.5 / 4.5)
    with _engine(n, solver=1, box_length=0.0, treepm_grid_size=G, treepm_r_split_cells=rs_cells,
                 treepm_r_cut_factor=4.5, treepm_assignment=ASSIGN[assignment],
                 treepm_gradient=gradient, treepm_window_floor=0.08 if gradient == 0 else 0.0,
                 octree_softening=eps) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
        grid = e.pm_grid()
        rho = e.pm_mesh(0).astype(np.float64)
    p4 = oracle.pos4(pos, m)
    apm, par, orho, _ = oracle.pm_isolated(p4, G, float(rs_cells), assignment=assignment,
                                           gradient=gradient,
                                           window_floor=0.08 if gradient == 0 else 0.0,
                                           cell_floor=0.25, softening=eps, want_fields=True)
    assert np.float32(grid["cell"]) == np.float32(par["cell"])
    assert np.array_equal(np.asarray(grid["origin"], np.float32), np.asarray(par["origin"], np.float32))
    assert np.abs(rho - orho).max() < 1e-5 * np.abs(orho).max()
    rs = np.float32(rs_cells) * np.float32(grid["cell"])
    assert np.float32(grid["rsplit"]) == rs
    p64 = pos.astype(np.float64)
    lo = p64.min(0)
    size = float((p64.max(0) - lo).max())
    keys = oracle.morton63(p64, lo, size)
    perm = oracle.stable_sort(keys)
    t = oracle.build_tree(keys[perm], p4[perm], leaf_cap=16)
    a_s, s_s = oracle.walk_targets(p4[perm], t, np.arange(n), theta=0.5, eps=eps,
                                   rcut=np.float32(4.5) * rs, box=0.0, rsplit=rs, quadrupole=True)
    asr = np.empty_like(a_s)
    asr[perm] = a_s
    asum = np.empty_like(s_s)
    asum[perm] = s_s
    ref = apm + asr
    dev = np.linalg.norm(acc - ref, axis=1)
    net = np.linalg.norm(ref, axis=1)
    bound = 64.0 * 2.0 ** -24 * (asum + np.linalg.norm(apm, axis=1))
    # the mesh force in FP32 transforms: 1e-5 of the rms mesh force as a floor
    rms_pm = np.sqrt((np.linalg.norm(apm, axis=1) ** 2).mean())
    assert np.median(dev / net) < 1e-5
    assert (dev <= np.maximum(np.maximum(1e-5 * net, bound), 1e-5 * rms_pm)).all(), (dev / net).max()
