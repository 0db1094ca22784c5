"""Ensembles of independent systems in one handle: no interaction between systems (all
systems share one origin, so any cross term would be large), per-system accuracy against the
FP64 direct sum, and agreement with each system stepped alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(sizes, seed):
    from blitzar_b200 import ics

    out = []
    for i, n in enumerate(sizes):
        W0 = 3.0 + 6.0 * ((seed + i) % 7) / 6.0
        p, v, m = ics.king(n, seed + i, W0)
        out.append((p, v, m.astype(np.float32)))
    return out


def test_ensemble_forces_are_per_system(gpu, oracle):
    from blitzar_b200._lib import Engine

    systems = _systems([1500, 40, 7000, 1, 3200, 33], seed=3)
    n = sum(len(m) for _, _, m in systems)
    with Engine(n, octree_theta=0.4, octree_softening=0.01, physics_max_acceleration=1e30) as e:
        offs = e.set_ensemble(systems)
        acc = e.accelerations().astype(np.float64)
        errs = e.force_errors(nsample=min(2000, n), seed=4)
    for i, (p, _, m) in enumerate(systems):
        a = acc[offs[i]:offs[i + 1]]
        if len(m) == 1:
            assert np.abs(a).max() == 0.0  # alone in its system
            continue
        ref = oracle.direct(oracle.pos4(p.astype(np.float32), m), None, eps=0.01)
        err = np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert np.median(err) < 2e-3, (i, np.median(err))
        assert np.percentile(err, 99) < 2e-2, (i, np.percentile(err, 99))
    assert errs["median"] < 2e-3  # the library's own per-system direct reference


def test_ensemble_steps_like_separate_runs(gpu):
    """Stepping the ensemble moves every system as it moves alone (same physics; the trees
    differ in key resolution, so agreement is to the tree's accuracy)."""
    from blitzar_b200._lib import Engine

    systems = _systems([3000, 800, 5000], seed=9)
    n = sum(len(m) for _, _, m in systems)
    with Engine(n, octree_theta=0.3, octree_softening=0.01, physics_max_acceleration=1e30) as e:
        offs = e.set_ensemble(systems)
        e.step(1e-3, 20)
        pe, ve = e.get_state(f64=True)
        k, w, _ = e.energy()
    ke_sum = w_sum = 0.0
    for i, (p, v, m) in enumerate(systems):
        with Engine(len(m), octree_theta=0.3, octree_softening=0.01,
                    physics_max_acceleration=1e30) as s:
            s.set_state(p, v, m, f64=True)
            k0, w0, _ = s.energy()
            s.step(1e-3, 20)
            ps, vs = s.get_state(f64=True)
            k1, w1, _ = s.energy()
        ke_sum += k1
        w_sum += w1
        d = np.abs(pe[offs[i]:offs[i + 1]] - ps).max() / np.abs(ps).max()
        assert d < 1e-5, (i, d)
    assert abs(k - ke_sum) < 1e-4 * abs(ke_sum) and abs(w - w_sum) < 1e-4 * abs(w_sum)


def test_ensemble_rejects_bad_offsets(gpu):
    import ctypes as C

    from blitzar_b200._lib import BZ_INVALID_ARGUMENT, BZ_UNSUPPORTED, Engine

    with Engine(100) as e:
        pos = np.zeros(300)
        m = np.ones(100, np.float32)
        bad = np.array([0, 50, 50, 100], np.int64)  # an empty system
        st = e.L.bz_set_ensemble(e.h, pos.ctypes.data, None, m.ctypes.data, bad.ctypes.data, 3)
        assert st == BZ_INVALID_ARGUMENT
        big = np.array([0, 200], np.int64)  # beyond the capacity
        assert e.L.bz_set_ensemble(e.h, pos.ctypes.data, None, m.ctypes.data, big.ctypes.data, 1) == BZ_INVALID_ARGUMENT
    with Engine(100, solver=1, box_length=1.0, treepm_grid_size=16) as e:
        ok = np.array([0, 100], np.int64)
        assert e.L.bz_set_ensemble(e.h, pos.ctypes.data, None, m.ctypes.data, ok.ctypes.data, 1) == BZ_UNSUPPORTED
