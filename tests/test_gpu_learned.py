"""Learned TreePM pair correction through the C ABI: the tensor-core MLP's forward pass and
gradients against the oracle's restatement (same BF16 rounding points), and what the trained
network gains over the plain TreePM at the same split scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NP = 1667


def _params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(NP, np.float32)
    p[0:512] = rng.uniform(-0.5, 0.5, 512)
    p[512:1536] = rng.uniform(-0.3, 0.3, 1024)
    p[1536:1568] = rng.uniform(-0.1, 0.1, 32)
    p[1568:1664] = rng.uniform(-0.4, 0.4, 96)
    p[1664:1667] = rng.uniform(-0.1, 0.1, 3)
    return p


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n, 6), np.float32)
    x[:, :3] = rng.uniform(-4, 4, (n, 3))
    x[:, 3:] = rng.random((n, 3))
    return x


def _engine(n=4096, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
    cfg = dict(solver=1, box_length=1.0, treepm_grid_size=32, treepm_assignment=2, treepm_gradient=1,
               treepm_window_floor=0.0, octree_softening=1e-3)
    cfg.update(kw)
    e = Engine(n, **cfg)
    rng = np.random.default_rng(0)
    e.set_state(rng.random((n, 3)).astype(np.float32), None, np.full(n, 1.0 / n, np.float32))
    return e


def test_mlp_forward_matches_oracle(gpu, oracle):
    p = _params(1)
    x = _inputs(1000, 2)
    with _engine() as e:
        e.learn_set(p, 0.75)
        y = e.learn_forward(x).astype(np.float64)
        p2, sc = e.learn_get()
    assert np.array_equal(p2, p) and sc == pytest.approx(0.75)
    ref = oracle.mlp_forward(p, x, 0.75).astype(np.float64)
    err = np.linalg.norm(y - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-3)
    # identical BF16 rounding points; FP32 vs FP64 accumulation and fast exp only
    assert np.median(err) < 2e-3 and err.max() < 3e-2, (np.median(err), err.max())


def test_mlp_gradient_matches_oracle(gpu, oracle):
    p = _params(3)
    x = _inputs(512, 4)
    y = np.random.default_rng(5).standard_normal((512, 3)).astype(np.float32)
    with _engine() as e:
        e.learn_set(p, 1.0)
        g, loss = e.learn_gradient(x, y)
    gr, lr = oracle.mlp_grad(p, x, y)
    assert loss == pytest.approx(lr, rel=2e-3)
    for name, a, b in (("W1", 0, 512), ("W2", 512, 1536), ("b2", 1536, 1568), ("W3", 1568, 1664),
                       ("b3", 1664, 1667)):
        rel = np.linalg.norm(g[a:b] - gr[a:b]) / np.linalg.norm(gr[a:b])
        assert rel < 1e-2, (name, rel)


def test_learned_correction_reduces_mesh_error(gpu):
    """Plain TreePM with a small split scale (0.8 mesh cells) is limited by the mesh's
    anisotropy; the correction trained on the engine's own residuals removes a large part."""
    from blitzar_b200 import ics
    from blitzar_b200._lib import Engine

    ns, mesh = 32, 64
    pos, _, m = ics.grf_grid(ns, seed=2, rms_cells=0.2)
    cfg = dict(solver=1, box_length=1.0, treepm_grid_size=mesh, treepm_r_split_cells=0.8,
               treepm_r_cut_factor=5.0, treepm_assignment=2, treepm_gradient=1,
               treepm_window_floor=0.0, treepm_node_size_factor=0.5, octree_softening=0.02 / ns,
               physics_max_acceleration=1e30)
    with Engine(len(m), **cfg) as e:
        e.set_state(pos, None, m.astype(np.float32), f64=True)
        plain = e.force_errors(nsample=1024, seed=3)
        x, y = e.learn_generate(1 << 18, seed=7)
        loss = e.learn_train(x, y, steps=3000, batch=4096, lr=3e-3, seed=1)
        e.learn_enable(True)
        learned = e.force_errors(nsample=1024, seed=3)
    assert loss < 0.2  # normalised residual variance left
    assert learned["median"] < 0.75 * plain["median"], (plain, learned)
