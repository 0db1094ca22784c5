"""Leapfrog stepping through the C ABI: graph and eager paths agree, momentum and energy
behave, and a short run matches an oracle KDK integration."""
import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    return Engine(n, **kw)


def test_graph_equals_eager(gpu):
    n = 20_000
    pos = plummer(n, seed=2)
    rng = np.random.default_rng(2)
    vel = (0.1 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    out = []
    for g in (0, 1):
        with _engine(n, use_graph=g) as e:
            e.set_state(pos, vel, m)
            e.step(1e-3, 7)
            out.append(e.get_state(f64=True))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_kdk_matches_oracle_integration(gpu, oracle):
    n = 4000
    pos = plummer(n, seed=4).astype(np.float64)
    rng = np.random.default_rng(4)
    vel = 0.2 * rng.standard_normal((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    dt, steps = 1e-3, 5
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        e.step(dt, steps)
        gp, gv = e.get_state(f64=True)

    def force(p):
        p32 = p.astype(np.float32)
        lo = p.min(0)
        size = float((p.max(0) - lo).max())
        k = oracle.morton63(p, lo, size)
        pm = oracle.stable_sort(k)
        t = oracle.build_tree(k[pm], oracle.pos4(p32[pm], m[pm]), 16)
        w = oracle.walk(oracle.pos4(p32[pm], m[pm]), t, theta=0.5, eps=0.01)
        a = np.empty((n, 3))
        a[pm] = w["acc"]
        return a

    x, v = pos.copy(), vel.copy()
    a = force(x)
    for _ in range(steps):
        v = v + 0.5 * dt * a
        x = x + dt * v
        a = force(x)
        v = v + 0.5 * dt * a
    assert np.abs(gp - x).max() < 1e-9
    assert np.abs(gv - v).max() < 1e-6


def test_periodic_wrap_and_momentum(gpu):
    n = 32_768
    rng = np.random.default_rng(1)
    pos = rng.random((n, 3)).astype(np.float32)
    vel = (0.5 * rng.standard_normal((n, 3))).astype(np.float32)
    vel -= vel.mean(0)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=32, octree_softening=0.02 / 32) as e:
        e.set_state(pos, vel, m)
        e.step(5e-4, 10)
        p, v = e.get_state(f64=True)
    assert p.min() >= 0.0 and p.max() < 1.0
    mom = (v * m[:, None]).sum(0)
    assert np.abs(mom).max() < 1e-4 * np.abs(v).mean()
