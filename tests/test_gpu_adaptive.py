"""Adaptive power-of-two block steps: a block with every particle on level 0 is exactly the
plain leapfrog step; levels follow the local dynamical time; energy is conserved."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
    return Engine(n, **kw)


def test_level_zero_blocks_equal_plain_leapfrog(gpu):
    from blitzar_b200 import ics

    n = 6000
    pos, vel, m = ics.plummer(n, seed=2)
    out = []
    for kw in (dict(), dict(adaptive_max_level=3, adaptive_eta=1e6)):
        with _engine(n, octree_theta=0.5, octree_softening=0.01, **kw) as e:
            e.set_state(pos, vel, m.astype(np.float32), f64=True)
            e.step(1e-3, 5)
            out.append(e.get_state(f64=True))
            if kw:
                assert (e.adaptive_levels() == 0).all()
                assert e.adaptive_updates() == 5 * n
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_levels_follow_the_core(gpu):
    from blitzar_b200 import ics

    n = 20000
    pos, vel, m = ics.king(n, 4, 9.0)
    with _engine(n, octree_theta=0.5, octree_softening=0.01, adaptive_max_level=6, adaptive_eta=0.02) as e:
        e.set_state(pos, vel, m.astype(np.float32), f64=True)
        e.step(2e-3, 2)
        lv = e.adaptive_levels().astype(int)
        upd = e.adaptive_updates()
    r = np.linalg.norm(pos, axis=1)
    inner, outer = r < np.percentile(r, 10), r > np.percentile(r, 90)
    assert lv.min() >= 0 and lv.max() <= 6
    assert lv[inner].mean() > lv[outer].mean() + 0.5
    # every particle closes at least one step per block, the fine ones more
    assert upd >= 2 * n and upd > 2 * n * 1.2


def test_adaptive_energy_conservation(gpu):
    from blitzar_b200 import ics

    n = 16384
    pos, vel, m = ics.plummer(n, seed=6)
    with _engine(n, octree_theta=0.4, octree_softening=0.01, adaptive_max_level=5, adaptive_eta=0.02) as e:
        e.set_state(pos, vel, m.astype(np.float32), f64=True)
        k0, w0, _ = e.energy()
        e.step(8e-3, 25)
        k1, w1, _ = e.energy()
        lv = e.adaptive_levels()
    assert lv.max() >= 2  # the run did use several levels
    assert abs((k1 + w1) - (k0 + w0)) < 1e-3 * abs(k0 + w0)
