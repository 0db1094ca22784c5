"""Properties of the oracle itself: tree invariants, walk convergence to the direct sum,
Ewald consistency, mesh momentum conservation, split-kernel identities."""
import numpy as np
import pytest

from conftest import plummer


def _tree(oracle, pos, m, leaf=16):
    p64 = pos.astype(np.float64)
    lo = p64.min(0)
    keys = oracle.morton63(p64, lo, float((p64.max(0) - lo).max()) or 1.0)
    perm = oracle.stable_sort(keys)
    sp4 = oracle.pos4(pos[perm], m[perm])
    return keys[perm], sp4, perm, oracle.build_tree(keys[perm], sp4, leaf)


def test_tree_invariants(oracle):
    n = 5000
    pos = plummer(n, 3)
    m = np.full(n, 1.0 / n, np.float32)
    sk, sp4, _, t = _tree(oracle, pos, m, 8)
    assert t["start"][0] == 0 and t["count"][0] == n
    for k in range(t["nodes"]):
        if t["nchild"][k]:
            c = np.arange(t["child"][k], t["child"][k] + t["nchild"][k])
            assert t["count"][c].sum() == t["count"][k]
            assert t["start"][c[0]] == t["start"][k]
            assert np.all(np.diff(t["start"][c]) == t["count"][c[:-1]])
            assert np.all(t["parent"][c] == k)
            assert t["count"][k] > 8
        else:
            assert t["count"][k] <= 8 or t["level"][k] == 21
    assert np.isclose(t["mono"][0, 3], m.sum(), rtol=1e-6)
    com = (sp4[:, :3].astype(np.float64) * sp4[:, 3:4]).sum(0) / sp4[:, 3].sum()
    assert np.allclose(t["mono"][0, :3], com, atol=1e-6)


def test_walk_converges_to_direct_sum(oracle):
    n = 3000
    pos = plummer(n, 4)
    m = np.full(n, 1.0 / n, np.float32)
    _, sp4, _, t = _tree(oracle, pos, m)
    ref = oracle.direct(sp4, None, eps=0.01)
    errs = []
    for theta in (0.8, 0.4, 0.2):
        w = oracle.walk(sp4, t, theta=theta, eps=0.01)
        errs.append(np.median(np.linalg.norm(w["acc"] - ref, axis=1) / np.linalg.norm(ref, axis=1)))
    assert errs[0] > errs[1] > errs[2]
    w = oracle.walk(sp4, t, theta=1e-3, eps=0.01)
    err = np.linalg.norm(w["acc"] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 1e-6  # every source taken particle by particle; FP32 separations


def test_quadrupole_beats_monopole(oracle):
    n = 4000
    pos = plummer(n, 6)
    m = np.full(n, 1.0 / n, np.float32)
    _, sp4, _, t = _tree(oracle, pos, m)
    ref = oracle.direct(sp4, None, eps=0.01)
    e = {}
    for q in (False, True):
        w = oracle.walk(sp4, t, theta=0.6, eps=0.01, quadrupole=q)
        e[q] = np.median(np.linalg.norm(w["acc"] - ref, axis=1) / np.linalg.norm(ref, axis=1))
    assert e[True] < 0.5 * e[False]


def test_potential_matches_direct(oracle):
    n = 2000
    pos = plummer(n, 8)
    m = np.full(n, 1.0 / n, np.float32)
    _, sp4, _, t = _tree(oracle, pos, m)
    w = oracle.walk(sp4, t, theta=0.3, eps=0.01, want_pot=True)
    _, ref = oracle.direct(sp4, None, eps=0.01, want_pot=True)
    assert np.median(np.abs(w["pot"] - ref) / np.abs(ref)) < 1e-4


def test_ewald_parameters_agree(oracle):
    rng = np.random.default_rng(1)
    n = 600
    p4 = oracle.pos4(rng.random((n, 3)).astype(np.float32), np.full(n, 1.0 / n, np.float32))
    tg = np.arange(0, n, 10)
    a = oracle.ewald(p4, tg, eps=0.0, box=1.0, alpha=7.0, kmax=10)
    b = oracle.ewald(p4, tg, eps=0.0, box=1.0, alpha=8.0, kmax=12)
    assert np.median(np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)) < 1e-5


def test_ewald_sum_of_forces_vanishes(oracle):
    rng = np.random.default_rng(2)
    n = 500
    p4 = oracle.pos4(rng.random((n, 3)).astype(np.float32), np.full(n, 1.0 / n, np.float32))
    a = oracle.ewald(p4, None, eps=0.0, box=1.0, alpha=7.0, kmax=10)
    assert np.abs(a.sum(0)).max() < 1e-6 * np.abs(a).sum()


@pytest.mark.parametrize("assignment,spectral", [("cic", False), ("pcs", True)])
def test_mesh_momentum_conservation(oracle, assignment, spectral):
    rng = np.random.default_rng(3)
    n = 3000
    m = np.full(n, 1.0 / n, np.float32)
    p4 = oracle.pos4(rng.random((n, 3)).astype(np.float32), m)
    a = oracle.pm_periodic(p4, 16, 1.0, 1.25 / 16, assignment=assignment, spectral=spectral)
    assert np.abs((a * m[:, None]).sum(0)).max() < 1e-8 * np.abs(a * m[:, None]).sum()


def test_split_kernel_identity(oracle):
    """w(r) is the fraction of the Newtonian pair force the short range keeps: 1 at r = 0,
    erfc-dominated decay, 0.0175 at 4.5 r_s."""
    assert abs(oracle.split_weight(1e-9, 1.0) - 1.0) < 1e-12
    assert abs(oracle.split_weight(4.5, 1.0) - 0.0175329) < 1e-6
    assert oracle.split_weight(10.0, 1.0) < 1e-10


def test_tree_groups_cover_and_stay_compact(oracle):
    """Walk groups cut from the tree: they tile [0, n) in order, hold at most 32 targets, and
    each lies inside one node's box (its box is never larger than the parent node of the run)."""
    from blitzar_b200 import ics

    pos, _, m = ics.hernquist(20000, 9)
    m = m.astype(np.float32)
    sk, sp4, _, t = _tree(oracle, pos.astype(np.float32), m)
    g = oracle.tree_groups(t)
    sizes = np.diff(g)
    assert g[0] == 0 and g[-1] == len(m)
    assert sizes.min() >= 1 and sizes.max() <= 32
    fixed = np.arange(0, len(m), 32)
    # fixed chunks straddle sparse branches: the largest tree group box is far smaller
    ext = lambda a, b: float((sp4[a:b, :3].max(0) - sp4[a:b, :3].min(0)).max())
    worst_tree = max(ext(a, b) for a, b in zip(g[:-1], g[1:]))
    worst_fixed = max(ext(a, min(a + 32, len(m))) for a in fixed)
    assert worst_tree < 0.5 * worst_fixed
    # a root of at most 32 particles is a single group
    sk2, sp42, _, t2 = _tree(oracle, pos[:20].astype(np.float32), m[:20])
    assert list(oracle.tree_groups(t2)) == [0, 20]


@pytest.mark.parametrize("gradient", [0, 1, 2])
def test_isolated_pm_is_the_long_range_force(oracle, gradient):
    """The oracle's isolated PM (the reference GPU TreePM's doubled mesh) approximates the long-
    range part of the split Newtonian force, sum m d / r^3 (1 - w(r)), on a small open cluster:
    the empty half of the doubled domain isolates the periodic convolution."""
    rng = np.random.default_rng(12)
    n = 3000
    pos = (rng.standard_normal((n, 3)) * 2.0).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    p4 = oracle.pos4(pos, m)
    acc, par = oracle.pm_isolated(p4, 32, 1.25, assignment="pcs", gradient=gradient,
                                  window_floor=0.0 if gradient else 0.08, cell_floor=0.25)
    assert par["mesh"] == 64 and par["cell"] >= 0.25
    rs = par["rsplit"]
    tg = rng.choice(n, 200, replace=False)
    d = pos[None, :, :].astype(np.float64) - pos[tg][:, None, :]
    r = np.sqrt((d * d).sum(-1))
    r[r == 0] = np.inf
    w = np.array([[oracle.split_weight(v, rs) if np.isfinite(v) else 1.0 for v in row] for row in r])
    ref = (m[None, :, None] * d * ((1.0 - w) / r ** 3)[:, :, None]).sum(1)
    err = np.linalg.norm(acc[tg] - ref, axis=1) / np.linalg.norm(ref, axis=1)
    # the doubled mesh only approximately isolates the periodic convolution (images of the
    # cluster two extents away), about 1 %; centred differences (the reference's) add more
    assert np.median(err) < (4e-2 if gradient == 0 else 2e-2), np.median(err)
