"""Generate the golden fixtures in this directory from the reference's own code.

The reference sources are compiled where they lie into oracle/_ref/libbzref.so
(`make -C oracle ref`, needs the reference tree) and run here on seeded inputs; the outputs
are stored as small .npz files that travel with the repository, so the oracle restatement can
be pinned to the reference on machines that do not have the reference tree.

Run: python tests/golden/make_golden.py [isolated]   (a name: regenerate that fixture only)
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def plummer_positions(n, seed):
    rng = np.random.default_rng(seed)
    u = rng.random(n) * 0.999
    r = 1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (r[:, None] * v).astype(np.float32)


def soa(p):
    return [np.ascontiguousarray(p[:, a]) for a in range(3)]


def isolated_treepm(R):
    """6. the reference GPU TreePM's isolated mesh (its kernels run on the host): grid, density,
    potential and the sampled mesh accelerations, CIC / TSC / PCS, for an open cluster."""
    n = 3000
    rng = np.random.default_rng(105)
    pos = (rng.standard_normal((n, 3)) * 1.5).astype(np.float32)
    mass = (rng.random(n).astype(np.float32) + 0.5) / n
    x, y, z = soa(pos)
    fn = R.ref_treepm_isolated
    fn.argtypes = [np.ctypeslib.ndpointer(np.float32)] * 4 + [C.c_int, C.c_int, C.c_float, C.c_float,
                                                              C.c_int, np.ctypeslib.ndpointer(np.float64),
                                                              C.c_void_p, C.c_void_p] + \
        [np.ctypeslib.ndpointer(np.float32)] * 3
    out = {}
    G, softening, cutoff_factor = 32, 0.01, 1.5
    for code, name in ((0, "cic"), (1, "tsc"), (2, "pcs")):
        params = np.zeros(8)
        dens = np.zeros((2 * G) ** 3, np.float32)
        phi = np.zeros((2 * G) ** 3, np.float32)
        ax, ay, az = [np.zeros(n, np.float32) for _ in range(3)]
        fn(x, y, z, mass, n, G, softening, cutoff_factor, code, params, dens.ctypes.data,
           phi.ctypes.data, ax, ay, az)
        out[f"{name}_params"] = params
        out[f"{name}_density"] = dens
        # the potential is dense: a seeded sample of its cells keeps the fixture small
        cells = np.sort(np.random.default_rng(106).choice(dens.size, 8192, replace=False))
        out[f"{name}_potential_cells"] = cells
        out[f"{name}_potential"] = phi[cells]
        out[f"{name}_acc"] = np.stack([ax, ay, az], 1)
    np.savez_compressed(os.path.join(HERE, "ref_treepm_isolated.npz"), pos=pos, mass=mass, grid=G,
                        softening=softening, cutoff_factor=cutoff_factor, **out)


def main(only=None):
    O.build(ref=True)
    R = O.ref()
    if R is None:
        raise SystemExit("oracle/_ref/libbzref.so is not built (needs the reference tree)")
    if only == "isolated":
        isolated_treepm(R)
        print("golden fixture written to", HERE)
        return

    # 1. Morton keys, stable sort permutation and topology (reference octree_gpu build)
    n = 2000
    pos = plummer_positions(n, 101)
    mass = (np.random.default_rng(102).random(n).astype(np.float32) + 0.5) / n
    x, y, z = soa(pos)
    keys = np.zeros(n, np.uint64)
    idx = np.zeros(n, np.int32)
    bbox = np.zeros(6, np.float32)
    R.ref_morton_keys(x, y, z, n, keys, idx, bbox)
    cap = 8 * n + 64
    hot = np.zeros(8 * cap, np.float32)
    nxt, mask, first, lstart, lcount = [np.zeros(cap, np.int32) for _ in range(5)]
    skeys = np.zeros(n, np.uint64)
    sidx = np.zeros(n, np.int32)
    depth = np.zeros(1, np.int32)
    nodes = R.ref_linear_octree(x, y, z, mass, n, 256, cap, hot, nxt, mask, first, lstart, lcount,
                                skeys, sidx, depth)
    np.savez_compressed(os.path.join(HERE, "ref_octree_build.npz"), pos=pos, mass=mass, keys=keys,
                        bbox=bbox, sorted_keys=skeys, sorted_index=sidx, nodes=np.int64(nodes),
                        hot=hot[: 8 * nodes].reshape(nodes, 8), next=nxt[:nodes], mask=mask[:nodes],
                        first=first[:nodes], lstart=lstart[:nodes], lcount=lcount[:nodes],
                        leaf_depth=depth)

    # 2. forces: reference GPU walk (host-compiled), octree_cpu, FP64 pairwise
    ax, ay, az = [np.zeros(n, np.float32) for _ in range(3)]
    nc = C.c_int(0)
    R.ref_octree_gpu_accel(x, y, z, mass, n, 256, 0.5, 0.01, 1e-12, 1e30, 0, 0.0, 0.0, ax, ay, az,
                           C.byref(nc))
    gpu_walk = np.stack([ax, ay, az], 1)
    bx, by, bz = [np.zeros(n, np.float32) for _ in range(3)]
    R.ref_octree_cpu_accel(x, y, z, mass, n, 0.5, 0.01, 1e-12, 1e30, 0, 0.0, 0.0, None, 0, bx, by, bz)
    cpu_walk = np.stack([bx, by, bz], 1)
    px, py, pz = [np.zeros(n, np.float32) for _ in range(3)]
    R.ref_fp64_pairwise(x, y, z, mass, n, 0.01, 1e-12, px, py, pz)
    pairwise = np.stack([px, py, pz], 1)
    np.savez_compressed(os.path.join(HERE, "ref_forces.npz"), pos=pos, mass=mass, theta=0.5,
                        softening=0.01, octree_gpu=gpu_walk, octree_cpu=cpu_walk,
                        fp64_pairwise=pairwise)

    # 3. periodic mesh templates (FP64) with explicit grid and split scale
    m_pm = 4000
    ppos = np.random.default_rng(103).random((m_pm, 3)).astype(np.float32)
    pmass = np.full(m_pm, 1.0 / m_pm, np.float32)
    qx, qy, qz = soa(ppos)
    out = {}
    for assignment in ("cic", "tsc"):
        grid = 16
        dens = np.zeros(grid ** 3)
        fx, fy, fz = [np.zeros(m_pm, np.float32) for _ in range(3)]
        R.ref_pm_periodic(qx, qy, qz, pmass, m_pm, grid, 1.0, 1.25 / grid, 1, assignment.encode(),
                          fx, fy, fz, dens.ctypes.data, None)
        out[f"{assignment}_density"] = dens
        out[f"{assignment}_acc"] = np.stack([fx, fy, fz], 1)
    np.savez_compressed(os.path.join(HERE, "ref_pm.npz"), pos=ppos, mass=pmass, grid=16,
                        rsplit=1.25 / 16, **out)

    # 4. short-range pair law of the CPU templates (FP64 Scalar)
    rng = np.random.default_rng(104)
    sep = rng.normal(0, 0.05, (64, 3)).astype(np.float32)
    pair = np.zeros((64, 3), np.float32)
    for i in range(64):
        o = np.zeros(3, np.float32)
        R.ref_short_range_pair(np.zeros(3, np.float32), sep[i].copy(), np.float32(0.7), 0.002, 1e-12,
                               0.01, o)
        pair[i] = o
    # 5. the reference radix-2 FFT on a small complex cube
    cube = rng.standard_normal((8, 8, 8)) + 1j * rng.standard_normal((8, 8, 8))
    flat = np.ascontiguousarray(np.stack([cube.real, cube.imag], -1).reshape(-1))
    R.ref_fft3d(flat, 8, 0)
    np.savez_compressed(os.path.join(HERE, "ref_misc.npz"), sep=sep, pair=pair, pair_mass=0.7,
                        pair_softening=0.002, pair_split=0.01, fft_in=cube,
                        fft_out=(flat[0::2] + 1j * flat[1::2]).reshape(8, 8, 8))
    isolated_treepm(R)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
