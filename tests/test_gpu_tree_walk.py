"""Production octree (bit-exact topology and moments) and the group walk (same decisions as
the oracle, forces within 1e-5), plus the reference-formulation parity mode."""
import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
    return Engine(n, **kw)


def _sorted_inputs(oracle, pos, m, box=None):
    p64 = pos.astype(np.float64)
    if box:
        keys = oracle.morton63(p64, [0.0, 0.0, 0.0], box)
    else:
        lo = p64.min(0)
        size = float((p64.max(0) - lo).max()) or 1.0
        keys = oracle.morton63(p64, lo, size)
    perm = oracle.stable_sort(keys)
    return keys[perm], oracle.pos4(pos[perm], m[perm]), perm


@pytest.mark.parametrize("n,leaf", [(1, 16), (40, 16), (20_000, 16), (100_000, 8), (65_536, 1)])
def test_tree_bit_exact(gpu, oracle, n, leaf):
    pos = plummer(n, seed=3 + n)
    m = (np.random.default_rng(n).random(n) + 0.5).astype(np.float32) / n
    with _engine(n, leaf_capacity=leaf) as e:
        e.set_state(pos, None, m)
        t = e.tree()
    sk, sp4, _ = _sorted_inputs(oracle, pos, m)
    o = oracle.build_tree(sk, sp4, leaf_cap=leaf)
    assert t["nodes"] == o["nodes"]
    for k in ("start", "count", "child", "nchild"):
        assert np.array_equal(t[k], o[k]), k
    for k in ("mono", "bmin", "bmax", "quad"):
        assert np.array_equal(t[k], o[k]), k


def test_tree_duplicates_deep(gpu, oracle):
    """Clusters of identical positions force splits down to the deepest level."""
    n = 3000
    rng = np.random.default_rng(9)
    base = rng.random((30, 3)).astype(np.float32)
    pos = base[rng.integers(0, 30, n)]
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, leaf_capacity=4) as e:
        e.set_state(pos, None, m)
        t = e.tree()
    sk, sp4, _ = _sorted_inputs(oracle, pos, m)
    o = oracle.build_tree(sk, sp4, leaf_cap=4)
    assert t["nodes"] == o["nodes"]
    for k in ("start", "count", "child", "nchild", "mono", "quad"):
        assert np.array_equal(t[k], o[k]), k


def _rel(a, b):
    scale = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.maximum(scale, 1e-30)


@pytest.mark.parametrize("quad", [True, False])
@pytest.mark.parametrize("theta", [0.3, 0.5, 0.8])
def test_walk_matches_oracle_open(gpu, oracle, quad, theta):
    n = 30_000
    pos = plummer(n, seed=21)
    m = np.full(n, 1.0 / n, np.float32)
    eps = 0.01
    with _engine(n, octree_theta=theta, octree_softening=eps, multipole_order=2 if quad else 1) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations()
        npp, npn = e.interaction_counts()
    sk, sp4, perm = _sorted_inputs(oracle, pos, m)
    o = oracle.build_tree(sk, sp4, leaf_cap=16)
    w = oracle.walk(sp4, o, theta=theta, eps=eps, quadrupole=quad)
    oacc = np.empty_like(w["acc"])
    oacc[perm] = w["acc"]
    err = _rel(acc.astype(np.float64), oacc)
    assert err.max() < 1e-5, err.max()
    # identical interaction lists: the device counters equal the oracle's
    sizes = w["group_sizes"]
    assert npp == int((w["n_pp"] * sizes).sum())
    assert npn == int((w["n_pn"] * sizes).sum())


def test_acceleration_clamp_matches_reference_rule(gpu, oracle):
    """physics_max_acceleration (reference default 64) clamps every particle's walk sum, as
    clampAcceleration does at the end of the reference walk (OctGpu.inl:227).  Close pairs
    planted in a Plummer sphere exceed the limit; the clamped forces equal the oracle's walk
    passed through the reference's clamp rule, and unclamped particles are untouched."""
    n = 20_000
    pos = plummer(n, seed=31)
    rng = np.random.default_rng(32)
    pick = rng.choice(n, 40, replace=False)
    pos[pick[20:]] = pos[pick[:20]] + np.float32(2e-4) * rng.standard_normal((20, 3)).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    eps = 1e-4
    with _engine(n, octree_theta=0.5, octree_softening=eps, physics_max_acceleration=64.0) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations().astype(np.float64)
    sk, sp4, perm = _sorted_inputs(oracle, pos, m)
    o = oracle.build_tree(sk, sp4, leaf_cap=16)
    w = oracle.walk(sp4, o, theta=0.5, eps=eps, quadrupole=True)
    raw = np.empty_like(w["acc"])
    raw[perm] = w["acc"]
    assert (np.linalg.norm(raw, axis=1) > 64.0).sum() >= 10  # the planted pairs exceed the limit
    ref = oracle.clamp_acceleration(raw, 64.0)
    err = _rel(acc, ref)
    assert err.max() < 1e-5, err.max()
    assert np.linalg.norm(acc, axis=1).max() <= 64.0 * (1 + 1e-6)


def test_walk_accuracy_vs_fp64_direct(gpu, oracle):
    n = 20_000
    pos = plummer(n, seed=5)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, octree_theta=0.5, octree_softening=0.01) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations()
    tg = np.arange(0, n, 7)
    ref = oracle.direct(oracle.pos4(pos, m), tg, eps=0.01)
    err = _rel(acc[tg].astype(np.float64), ref)
    assert np.median(err) < 1e-3 and np.percentile(err, 99) < 1e-2


def test_potential(gpu, oracle):
    n = 8000
    pos = plummer(n, seed=8)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, octree_theta=0.4) as e:
        e.set_state(pos, None, m)
        acc, pot = e.accelerations(want_pot=True)
    _, ref_pot = oracle.direct(oracle.pos4(pos, m), None, eps=0.01, want_pot=True)
    rel = np.abs(pot - ref_pot) / np.abs(ref_pot)
    assert np.median(rel) < 1e-4


def test_reference_mode_forces_and_topology(gpu, oracle):
    """Reference formulation: one-leaf tree bit-exact, forces within 1e-5 of its walk."""
    n = 12_000
    pos = plummer(n, seed=13)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=2, octree_softening=0.01) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations()
        rt = e.reference_tree()
    o = oracle.ref_linear_octree(pos, m, 256, fused=True)
    assert rt["nodes"] == o["nodes"] == 1
    assert np.array_equal(rt["hot"], o["hot"])
    assert rt["lcount"][0] == n and rt["next"][0] == -1 and rt["first"][0] == -1
    oacc = oracle.ref_walk(pos, m, o, theta=0.5, softening=0.01)
    err = _rel(acc.astype(np.float64), oacc)
    assert err.max() < 1e-5, err.max()


@pytest.mark.parametrize("gsize", [16, 24])
def test_walk_group_size_matches_oracle(gpu, oracle, gsize):
    """Smaller walk groups (an autotuner choice) follow the same tree-cut rule as the oracle."""
    n = 20_000
    pos = plummer(n, seed=23)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, octree_theta=0.5, octree_softening=0.01, walk_group_size=gsize) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations()
        npp, npn = e.interaction_counts()
    sk, sp4, perm = _sorted_inputs(oracle, pos, m)
    o = oracle.build_tree(sk, sp4, leaf_cap=16)
    w = oracle.walk(sp4, o, theta=0.5, eps=0.01, gmax=gsize)
    oacc = np.empty_like(w["acc"])
    oacc[perm] = w["acc"]
    assert _rel(acc.astype(np.float64), oacc).max() < 1e-5
    assert w["group_sizes"].max() <= gsize
    assert npp == int((w["n_pp"] * w["group_sizes"]).sum())
    assert npn == int((w["n_pn"] * w["group_sizes"]).sum())


def test_autotune_picks_a_candidate_and_keeps_accuracy(gpu, oracle):
    n = 40_000
    pos = plummer(n, seed=24)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, octree_theta=0.5, octree_softening=0.01) as e:
        e.set_state(pos, None, m)
        leaf, grp, ms = e.autotune(trials=2)
        assert leaf in (8, 12, 16, 24, 32, 48) and grp in (16, 24, 32) and ms > 0
        acc = e.accelerations()
        e.step(1e-3, 3)  # the step graph is captured again with the tuned parameters
        p, _ = e.get_state(f64=True)
    assert np.isfinite(p).all()
    tg = np.arange(0, n, 13)
    ref = oracle.direct(oracle.pos4(pos, m), tg, eps=0.01)
    assert np.median(_rel(acc[tg].astype(np.float64), ref)) < 2e-3
