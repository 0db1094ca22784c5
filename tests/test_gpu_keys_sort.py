"""Morton keys and the stable radix sort: bit-exact against the oracle (and, in reference
mode, against the reference's own key kernel compiled on the host)."""
import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
    return Engine(n, **kw)


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 50_000, 262_145])
def test_production_keys_and_permutation(gpu, oracle, n):
    pos = plummer(n, seed=n)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    p64 = pos.astype(np.float64)
    lo, hi = p64.min(0), p64.max(0)
    size = float((hi - lo).max()) or 1.0
    ok = oracle.morton63(p64, lo, size)
    operm = oracle.stable_sort(ok)
    assert np.array_equal(perm, operm)
    assert np.array_equal(keys, ok[operm])


def test_periodic_box_keys(gpu, oracle):
    n = 20_000
    rng = np.random.default_rng(7)
    pos = rng.random((n, 3)).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=1, box_length=1.0, treepm_grid_size=32) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    ok = oracle.morton63(pos.astype(np.float64), [0.0, 0.0, 0.0], 1.0)
    operm = oracle.stable_sort(ok)
    assert np.array_equal(perm, operm)
    assert np.array_equal(keys, ok[operm])


@pytest.mark.parametrize("n", [1, 5, 4096, 65_536, 100_003])
def test_reference_keys_bit_exact(gpu, oracle, n):
    pos = plummer(n, seed=11 + n)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n, solver=2) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    ok, _ = oracle.morton_ref(pos, fused=True)
    operm = oracle.stable_sort(ok)
    assert np.array_equal(perm, operm)
    assert np.array_equal(keys, ok[operm])
    assert int(keys.max()).bit_length() <= 30  # the reference spread keeps 10 bits per axis


def test_sort_all_equal_keys(gpu, oracle):
    """Every particle at one point: every digit pass is trivial; order must stay stable."""
    n = 9000
    pos = np.zeros((n, 3), np.float32)
    m = np.full(n, 1.0, np.float32)
    with _engine(n) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    assert np.array_equal(perm, np.arange(n))
    assert np.all(keys == keys[0])


def test_sort_duplicates_and_ties(gpu, oracle):
    """Heavy ties: positions on a coarse lattice; ties must keep caller order."""
    n = 70_001
    rng = np.random.default_rng(5)
    pos = rng.integers(0, 4, size=(n, 3)).astype(np.float32)
    m = np.full(n, 1.0, np.float32)
    with _engine(n) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    p64 = pos.astype(np.float64)
    lo = p64.min(0)
    size = float((p64.max(0) - lo).max())
    ok = oracle.morton63(p64, lo, size)
    operm = oracle.stable_sort(ok)
    assert np.array_equal(perm, operm)


def _caller_order_case(oracle, kind, n, seed):
    """Positions in a chosen caller order, for the nearly-sorted fast path of the sort: the
    keys reach the sort in caller order (sorted, nearly sorted, or an order whose in-order
    part is not sorted, which must take the full sort)."""
    rng = np.random.default_rng(seed)
    pos = plummer(n, seed=seed).astype(np.float64)
    if kind == "duplicates":
        pos[rng.integers(0, n, n // 4)] = pos[rng.integers(0, n, n // 4)]
    lo, hi = pos.min(0), pos.max(0)
    size = float((hi - lo).max())
    order = oracle.stable_sort(oracle.morton63(pos, lo, size))
    if kind in ("sorted", "duplicates"):
        idx = order.copy()
        if kind == "duplicates":  # a few displaced among equal keys
            moved = rng.choice(n, n // 1500 + 3, replace=False)
            for j in moved:
                t = rng.integers(0, n)
                v = idx[j]
                idx = np.insert(np.delete(idx, j), t, v)
    elif kind == "nearly":
        idx = list(order)
        for _ in range(n // 1000 + 3):  # move single particles far away in the order
            j, t = rng.integers(0, n, 2)
            idx.insert(t, idx.pop(j))
        idx = np.array(idx)
        sw = rng.choice(n - 1, n // 600 + 2, replace=False)  # and swap some neighbours
        idx[sw], idx[sw + 1] = idx[sw + 1].copy(), idx[sw].copy()
    elif kind == "unsorted_core":
        # the run s20..s29 moved as a block before s10..s19: only the ends near the seam are
        # out of order within an 8-key window, s21 stays before s18 in the in-order part, which
        # is then not sorted, so the full sort must run
        idx = np.concatenate([order[:10], order[20:30], order[10:20], order[30:]])
    else:
        raise ValueError(kind)
    return pos[idx].astype(np.float32)


@pytest.mark.parametrize("kind", ["sorted", "nearly", "unsorted_core", "duplicates"])
@pytest.mark.parametrize("n", [5000, 300_000])
def test_nearly_sorted_inputs(gpu, oracle, kind, n):
    """The adaptive sort (only the locally out-of-order pairs radix-sorted, then merged) gives
    the stable order of the full sort bit for bit, and falls back to the full sort when the
    in-order part is not sorted."""
    pos = _caller_order_case(oracle, kind, n, seed=n + len(kind))
    p64 = pos.astype(np.float64)
    lo, hi = p64.min(0), p64.max(0)
    ok = oracle.morton63(p64, lo, float((hi - lo).max()))
    # the case exercises the path it names: fast (in-order part sorted) or the full sort
    assert _fast_path(ok) == (kind != "unsorted_core")
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, None, m)
        keys, perm = e.morton_keys()
    operm = oracle.stable_sort(ok)
    assert np.array_equal(perm, operm)
    assert np.array_equal(keys, ok[operm])


def _fast_path(k, window=8):
    """Host statement of the adaptive sort's choice: a position is out of order when its key is
    below one of the `window` keys before it or above one of the `window` keys after it; the
    fast path needs the other positions sorted and at most max(n / 8, 4096) out of order."""
    n = len(k)
    f = np.zeros(n, bool)
    for w in range(1, window + 1):
        f[w:] |= k[w:] < k[:-w]
        f[:-w] |= k[:-w] > k[w:]
    u = k[~f]
    return bool(np.all(u[1:] >= u[:-1])) and int(f.sum()) <= max(n // 8, 4096)


def test_resort_after_steps_matches_full_sort(gpu, oracle):
    """Steps re-sort the previous order (the fast path); the tree built on it must match the
    one built from a fresh full sort of the same positions."""
    n = 60_000
    pos = plummer(n, seed=77)
    rng = np.random.default_rng(77)
    vel = (0.3 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, vel, m)
        e.step(2e-3, 5)
        acc = e.accelerations()
        p, v = e.get_state(f64=True)
    with _engine(n) as e2:
        e2.set_state(p, v, m, f64=True)
        acc2 = e2.accelerations()
    assert np.array_equal(acc, acc2)
