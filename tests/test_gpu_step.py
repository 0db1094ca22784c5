"""Leapfrog stepping through the C ABI: graph and eager paths agree, momentum and energy
behave, and a short run matches an oracle KDK integration."""
import numpy as np
import pytest

from conftest import plummer

pytestmark = pytest.mark.gpu


def _engine(n, **kw):
    from blitzar_b200._lib import Engine
    kw.setdefault("physics_max_acceleration", 1e30)  # parity with the unclamped oracle
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


@pytest.mark.parametrize("case", ["octree", "treepm"])
def test_steps_in_one_call_equal_single_steps(gpu, case):
    """A leapfrog call of several steps folds each closing kick into the next step's opening
    kernel (and kicks once after the last step): the same arithmetic as single-step calls, so
    the octree state agrees bit for bit.  TreePM agrees to the mesh's run-to-run spread (its
    float reductions into the mesh run in no fixed order), and its accelerations, completed by
    the mesh leg's in the closing kick, agree too."""
    n = 16_384
    rng = np.random.default_rng(12)
    if case == "octree":
        pos = plummer(n, seed=12)
        cfg = {}
    else:
        pos = rng.random((n, 3)).astype(np.float32)
        cfg = dict(solver=1, box_length=1.0, treepm_grid_size=32, octree_softening=1e-3,
                   treepm_assignment=2, treepm_gradient=2)
    vel = (0.1 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    out = []
    for split in (False, True):
        with _engine(n, **cfg) as e:
            e.set_state(pos, vel, m)
            if split:
                for _ in range(6):
                    e.step(1e-3, 1)
            else:
                e.step(1e-3, 6)
            p, v = e.get_state(f64=True)
            a = np.empty(3 * n, np.float32)
            e.get_state_acc_soa(np.empty(3 * n, np.float32), np.empty(3 * n, np.float32), a)
            out.append((p, v, a))
    if case == "octree":
        for x, y in zip(out[0], out[1]):
            assert np.array_equal(x, y)
    else:
        assert np.abs(out[0][0] - out[1][0]).max() < 1e-10
        assert np.abs(out[0][1] - out[1][1]).max() < 1e-7
        a0, a1 = out[0][2].reshape(3, n), out[1][2].reshape(3, n)
        assert np.abs(a0 - a1).max() < 1e-4 * np.abs(a1).max()


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


def test_symplectic_euler_matches_oracle_integration(gpu, oracle):
    """integrator = Euler: v += a(x) dt, x += v dt, one force evaluation a step, as the
    reference's updateParticlesOctree (engine/physics/octree/cuda/force/OctGpu.inl:246-275)."""
    from blitzar_b200._lib import BZ_INTEGRATOR_EULER

    n = 4000
    pos = plummer(n, seed=5).astype(np.float64)
    rng = np.random.default_rng(5)
    vel = 0.2 * rng.standard_normal((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    dt, steps = 1e-3, 5
    with _engine(n, integrator=BZ_INTEGRATOR_EULER) as e:
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
    for _ in range(steps):
        v = v + dt * force(x)
        x = x + dt * v
    assert np.abs(gp - x).max() < 1e-9
    assert np.abs(gv - v).max() < 1e-6
    # and not the leapfrog result
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        e.step(dt, steps)
        lp, _ = e.get_state(f64=True)
    assert np.abs(lp - x).max() > 1e-8


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


def test_energy_diagnostics_match_oracle(gpu, oracle):
    """bz_energy: FP64 kinetic energy and momentum equal the host sums of the same state;
    the potential energy equals the oracle's direct sum within the walk's multipole error."""
    from blitzar_b200 import ics

    n = 8192
    pos, vel, m = ics.plummer(n, seed=3)
    m = m.astype(np.float32)
    with _engine(n, octree_theta=0.3) as e:
        e.set_state(pos, vel, m, f64=True)
        ke, pe, mom = e.energy()
        p, v = e.get_state(f64=True)
    md = m.astype(np.float64)
    assert abs(ke - 0.5 * (md * (v ** 2).sum(1)).sum()) < 1e-12 * abs(ke)
    assert np.allclose(mom, (md[:, None] * v).sum(0), rtol=0, atol=1e-12)
    _, phi = oracle.direct(oracle.pos4(pos.astype(np.float32), m), None, eps=0.01, want_pot=True)
    pe_ref = 0.5 * (md * phi).sum()
    assert abs(pe - pe_ref) < 2e-4 * abs(pe_ref)
    assert -1.6 < 2 * ke / pe < -0.4  # near virial equilibrium: 2T / W = -1 for the Plummer DF


def test_energy_drift_is_small(gpu):
    """A leapfrog run of a Plummer sphere conserves total energy to well below 1e-3."""
    from blitzar_b200 import ics

    n = 16384
    pos, vel, m = ics.plummer(n, seed=5)
    with _engine(n, octree_softening=0.01) as e:
        e.set_state(pos, vel, m.astype(np.float32), f64=True)
        k0, w0, p0 = e.energy()
        e.step(1e-3, 200)
        k1, w1, p1 = e.energy()
    e0, e1 = k0 + w0, k1 + w1
    assert abs(e1 - e0) < 5e-4 * abs(e0)
    assert np.abs(p1 - p0).max() < 1e-4 * np.sqrt(2 * k0 * m.sum())


@pytest.mark.parametrize("integrator", ["leapfrog", "euler"])
def test_headless_driver_matches_engine(gpu, tmp_path, integrator):
    """The C++ headless driver (reference config + NBSIMBIN in, NBSIMBIN out) steps exactly as
    the engine driven through ctypes does, with either integrator."""
    import subprocess

    from blitzar_b200 import build as b
    from blitzar_b200 import ics, snapshot
    from blitzar_b200._lib import BZ_INTEGRATOR_EULER, BZ_INTEGRATOR_LEAPFROG

    n = 4096
    pos, vel, m = ics.plummer(n, seed=8)
    pos, vel, m = pos.astype(np.float32), vel.astype(np.float32), m.astype(np.float32)
    snapshot.write_bin(tmp_path / "in.bin", pos, vel, m)
    (tmp_path / "sim.ini").write_text(
        f"simulation(dt=0.001, solver=octree_gpu, integrator={integrator})\n"
        "octree(theta=0.6, softening=0.02)\n"
        f"input_file={tmp_path / 'in.bin'}\n")
    r = subprocess.run([b.HEADLESS, "--config", str(tmp_path / "sim.ini"), "--run",
                        "--target-steps", "10", "--export-format", "bin", "--export-path",
                        str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "[headless] done steps=10" in r.stdout
    p_h, v_h, m_h, _ = snapshot.read_bin(tmp_path / "out.bin")
    # the headless run keeps the reference's default clamp (64); so does this handle
    mode = BZ_INTEGRATOR_EULER if integrator == "euler" else BZ_INTEGRATOR_LEAPFROG
    with _engine(n, octree_theta=0.6, octree_softening=0.02, physics_max_acceleration=64.0,
                 integrator=mode) as e:
        e.set_state(pos, vel, m)
        e.step(1e-3, 10)
        p_e, v_e = e.get_state()
    assert np.array_equal(p_h, p_e.astype(np.float32)) and np.array_equal(v_h, v_e.astype(np.float32))
    assert np.array_equal(m_h, m)


def test_state_with_accelerations(gpu):
    """A state uploaded with the accelerations of its positions steps exactly like the same
    state uploaded alone (whose set-up evaluation computes those forces), and the accelerations
    returned with a state are the forces at its positions."""
    n = 20_000
    pos = plummer(n, seed=8)
    rng = np.random.default_rng(8)
    vel = (0.1 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, vel, m)
        acc = e.accelerations()
    with _engine(n) as e:
        e.set_state(pos, vel, m)
        e.step(1e-3, 3)
        pa, va = e.get_state(f64=True)
    ps = np.ascontiguousarray(pos.T, np.float32).ravel()
    vs = np.ascontiguousarray(vel.T, np.float32).ravel()
    acs = np.ascontiguousarray(acc.T, np.float32).ravel()
    with _engine(n) as e:
        e.set_state_acc_soa(ps, vs, m, acs)
        e.step(1e-3, 3)
        pb, vb = e.get_state(f64=True)
        p3, v3, a3 = (np.empty(3 * n, np.float32) for _ in range(3))
        e.get_state_acc_soa(p3, v3, a3)
        again = e.accelerations()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert np.array_equal(a3.reshape(3, n).T, again)


@pytest.mark.parametrize("case", ["octree", "treepm"])
def test_step_with_overlapped_download(gpu, case):
    """bz_step_get_state_acc_f64 (the position download overlapping the step) returns, step
    after step, what bz_step followed by bz_get_state_acc_f64 returns: bit for bit for the
    octree; for TreePM to the mesh's own run-to-run spread (its deposit adds the blocks' tiles
    into the mesh with float reductions, in no fixed order: ~1e-12 in positions after a few
    steps, the same between two bz_step runs)."""
    n = 20_000
    rng = np.random.default_rng(12)
    if case == "octree":
        pos = plummer(n, seed=12).astype(np.float64)
        kw = {}
    else:  # periodic TreePM, its mesh leg on the second stream
        pos = rng.random((n, 3))
        kw = dict(solver=1, box_length=1.0, treepm_grid_size=32, octree_softening=0.02 / 32)
    vel = 0.1 * rng.standard_normal((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    outs = []
    for fused in (False, True):
        with _engine(n, **kw) as e:
            e.set_state(pos, vel, m, f64=True)
            p3, v3 = np.empty(3 * n), np.empty(3 * n)
            a3 = np.empty(3 * n, np.float32)
            got = []
            for _ in range(3):
                if fused:
                    e.step_get_state_acc_f64_soa(1e-3, p3, v3, a3)
                else:
                    e.step(1e-3, 1)
                    e.get_state_acc_f64_soa(p3, v3, a3)
                got.append((p3.copy(), v3.copy(), a3.copy()))
                e.set_state_acc_f64_soa(p3, v3, m, a3)
            outs.append(got)
    for (pa, va, aa), (pb, vb, ab) in zip(*outs):
        if case == "octree":
            assert np.array_equal(pa, pb) and np.array_equal(va, vb) and np.array_equal(aa, ab)
        else:
            assert np.abs(pa - pb).max() < 1e-10 and np.abs(va - vb).max() < 1e-7
            assert np.abs(aa - ab).max() < 1e-4 * np.abs(aa).max()


def test_state_round_trip_keeps_order(gpu):
    """Uploading a held state back (same size) keeps the device's particle order; the steps that
    follow match those of a fresh engine given the same state and accelerations."""
    n = 20_000
    pos = plummer(n, seed=9)
    rng = np.random.default_rng(9)
    vel = (0.1 * rng.standard_normal((n, 3))).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    p3, v3, a3 = (np.empty(3 * n, np.float32) for _ in range(3))
    with _engine(n) as e:
        e.set_state(pos, vel, m)
        e.step(1e-3, 2)
        e.get_state_acc_soa(p3, v3, a3)
        e.set_state_acc_soa(p3, v3, m, a3)  # same size: kept in the sorted order
        e.step(1e-3, 2)
        pa, va = e.get_state(f64=True)
    with _engine(n) as e:
        e.set_state_acc_soa(p3, v3, m, a3)
        e.step(1e-3, 2)
        pb, vb = e.get_state(f64=True)
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)


def test_state_with_accelerations_f64(gpu):
    """The FP64 state-with-accelerations calls: a host round trip after every step leaves the
    trajectory bit for bit that of a resident state (no FP32 rounding of positions and
    velocities), and the FP64 download equals bz_get_state_f64."""
    n = 20_000
    pos = plummer(n, seed=10).astype(np.float64)
    rng = np.random.default_rng(10)
    vel = 0.1 * rng.standard_normal((n, 3))
    m = np.full(n, 1.0 / n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        e.step(1e-3, 4)
        pa, va = e.get_state(f64=True)
    p3, v3 = np.empty(3 * n), np.empty(3 * n)
    a3 = np.empty(3 * n, np.float32)
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        for _ in range(4):
            e.get_state_acc_f64_soa(p3, v3, a3)
            e.set_state_acc_f64_soa(p3, v3, m, a3)  # same size: kept in the sorted order
            e.step(1e-3, 1)
        e.get_state_acc_f64_soa(p3, v3, a3)
        pb, vb = e.get_state(f64=True)
        again = e.accelerations()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert np.array_equal(p3.reshape(3, n).T, pb) and np.array_equal(v3.reshape(3, n).T, vb)
    assert np.array_equal(a3.reshape(3, n).T, again)
    # a fresh handle given the FP64 state and its accelerations steps like the resident one
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        e.step(1e-3, 2)
        pc, vc = e.get_state(f64=True)
    with _engine(n) as e:
        e.set_state(pos, vel, m, f64=True)
        p0, v0, a0 = np.empty(3 * n), np.empty(3 * n), np.empty(3 * n, np.float32)
        e.get_state_acc_f64_soa(p0, v0, a0)
    with _engine(n) as e:
        e.set_state_acc_f64_soa(p0, v0, m, a0)
        e.step(1e-3, 2)
        pd, vd = e.get_state(f64=True)
    assert np.array_equal(pc, pd) and np.array_equal(vc, vd)
