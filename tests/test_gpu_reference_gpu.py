"""The reference's own GPU octree -- its CUDA kernels and octree_gpu Euler step compiled for
sm_100a from its sources (oracle/ref_gpu_shim.cu) -- as a checker: the same kernels run on the
host agree with it, and this engine's reference formulation agrees with it.  Skipped where the
reference tree was not at hand when the oracle was built."""
import ctypes as C

import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refgpu(oracle):
    R = oracle.ref_gpu()
    if R is None:
        pytest.skip("oracle/_ref/libbzrefgpu.so not built (no reference checkout at build time)")
    return R


def _soa(a):
    return [np.ascontiguousarray(a[:, k], np.float32) for k in range(3)]


class _RefGpu:
    def __init__(self, R, pos, vel, m, leaf=256):
        self.R, self.n = R, len(m)
        x, y, z = _soa(pos)
        vx, vy, vz = _soa(vel)
        self.h = R.refgpu_create(self.n, leaf, x, y, z, vx, vy, vz, np.ascontiguousarray(m))
        assert self.h

    def accel(self, theta=0.5, eps=0.01, min_d2=1e-12, amax=1e30, crit=0):
        a = [np.zeros(self.n, np.float32) for _ in range(3)]
        nodes, leaves = C.c_int(), C.c_int()
        rc = self.R.refgpu_accel(self.h, theta, eps, min_d2, amax, crit, *a, C.byref(nodes),
                                 C.byref(leaves))
        assert rc == 0, rc
        return np.stack(a, 1), nodes.value, leaves.value

    def step(self, dt, theta=0.5, eps=0.01, min_d2=1e-12, amax=1e30, crit=0):
        assert self.R.refgpu_step(self.h, dt, theta, eps, min_d2, amax, crit) == 0

    def state(self):
        s = [np.zeros(self.n, np.float32) for _ in range(6)]
        assert self.R.refgpu_get_state(self.h, *s) == 0
        return np.stack(s[:3], 1), np.stack(s[3:], 1)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.R.refgpu_destroy(self.h)


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)


@pytest.mark.parametrize("n", [1, 2, 3000])
def test_reference_gpu_kernels_match_their_host_build(gpu, oracle, refgpu, n):
    """The reference kernels on the GPU and on the host (oracle/_ref/libbzref.so) give the same
    tree size and the same accelerations to float rounding (rsqrtf on the device, 1/sqrtf on
    the host)."""
    R = oracle.ref()
    if R is None:
        pytest.skip("oracle/_ref/libbzref.so not built")
    pos = plummer(n, seed=41)
    m = np.full(n, 1.0 / n, np.float32)
    with _RefGpu(refgpu, pos, np.zeros_like(pos), m) as g:
        ga, nodes, leaves = g.accel()
    x, y, z = _soa(pos)
    ha = [np.zeros(n, np.float32) for _ in range(3)]
    hn = C.c_int()
    assert R.ref_octree_gpu_accel(x, y, z, m, n, 256, 0.5, 0.01, 1e-12, 1e30, 0, 0.0, 0.0, *ha,
                                  C.byref(hn)) == 0
    assert nodes == hn.value and leaves >= 1
    ha = np.stack(ha, 1)
    if n > 1:
        assert _rel(ga, ha).max() < 1e-5
    else:
        assert np.all(ga == 0) and np.all(ha == 0)


def test_engine_reference_mode_matches_reference_gpu(gpu, refgpu):
    """This engine's reference formulation (solver 2) against the reference's own GPU walk on
    the same particles: the reference's 10-bit key spread gives one leaf, so both are a direct
    sum over the leaf; forces agree to 1e-5."""
    from blitzar_b200._lib import Engine

    n = 12_000
    pos = plummer(n, seed=13)
    m = np.full(n, 1.0 / n, np.float32)
    with Engine(n, solver=2, octree_softening=0.01, physics_max_acceleration=1e30) as e:
        e.set_state(pos, None, m)
        acc = e.accelerations()
    with _RefGpu(refgpu, pos, np.zeros_like(pos), m) as g:
        ga, nodes, leaves = g.accel()
    assert nodes == 1 and leaves == 1
    assert _rel(acc.astype(np.float64), ga.astype(np.float64)).max() < 1e-5


def test_reference_gpu_euler_step_uses_engine_accelerations(gpu, refgpu):
    """One symplectic-Euler step of the reference's octree_gpu (the step the reference arm
    times) equals v' = v + a dt, x' = x + v' dt in FP32 with a = this engine's reference
    formulation at x, under the reference's default acceleration clamp (64)."""
    from blitzar_b200._lib import Engine

    n, dt = 8000, 1e-3
    pos = plummer(n, seed=17)
    rng = np.random.default_rng(17)
    vel = (0.2 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    with Engine(n, solver=2, octree_softening=0.01, physics_max_acceleration=64.0) as e:
        e.set_state(pos, vel, m)
        acc = e.accelerations()
    v1 = vel + acc * np.float32(dt)
    x1 = pos + v1 * np.float32(dt)
    with _RefGpu(refgpu, pos, vel, m) as g:
        g.step(dt, amax=64.0)
        gp, gv = g.state()
    assert np.abs(gv - v1).max() < 1e-5 * np.abs(v1).max()
    assert np.abs(gp - x1).max() < 1e-6 * np.abs(x1).max()
