"""ctypes bindings for the oracle libraries -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg and reference arm
import this module, and only as the checker or the reference being timed: the product
(``blitzar_b200``) never calls into it.

* ``liboracle.so`` -- the C restatement in ``bz_oracle.c`` (built from committed sources).
* ``_ref/libbzref.so`` -- the reference's own sources compiled where they lie
  (``ref_shim.cpp``); present only where the reference tree was available at build time.
* ``_ref/libbzrefgpu.so`` -- the reference's GPU linear octree and octree_gpu Euler step
  compiled for sm_100a from its sources (``ref_gpu_shim.cu``), run on the GPU as the
  reference arm's GPU comparator and as a checker in the GPU tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None
_REF_GPU = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


class WalkParams(C.Structure):
    _fields_ = [("theta2", C.c_float), ("eps2", C.c_float), ("rcut2", C.c_float),
                ("box", C.c_float), ("rsplit", C.c_float), ("min_dist2", C.c_float),
                ("quadrupole", C.c_int), ("group", C.c_int), ("max_node_size", C.c_float)]


def reference_dir() -> str | None:
    """Root of a BLITZAR checkout to compile the reference shim from: $BZ_REFERENCE_DIR, else a
    checkout named ``reference`` beside this repository; None when neither exists."""
    env = os.environ.get("BZ_REFERENCE_DIR")
    cand = env if env else os.path.join(os.path.dirname(HERE), os.pardir, "reference")
    cand = os.path.abspath(cand)
    return cand if os.path.isdir(os.path.join(cand, "engine")) else None


def build(ref: bool = False) -> None:
    """Compile the restatement (and, with ref=True, the reference shim from reference_dir())
    in place."""
    target = ["all"]
    if ref:
        root = reference_dir()
        if root is None:
            raise RuntimeError("reference shim requested but no BLITZAR checkout was found: "
                               "set BZ_REFERENCE_DIR to its root")
        target += ["ref", f"REF={root}"]
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "bz_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        L.or_bbox_f32.argtypes = [_f32p, _f32p, _f32p, C.c_int64, _f32p]
        L.or_morton_ref.argtypes = [_f32p, _f32p, _f32p, C.c_int64, _f32p, C.c_int, _u64p]
        L.or_morton63.argtypes = [_f64p, _f64p, _f64p, C.c_int64, _f64p, C.c_double, _u64p]
        L.or_stable_sort_u64.argtypes = [_u64p, C.c_int64, _i32p]
        L.or_ref_linear_octree.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int64, C.c_int, C.c_int,
                                           C.c_int64, _f32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                                           _u64p, _i32p, _i32p]
        L.or_ref_linear_octree.restype = C.c_int64
        L.or_ref_walk.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int64, _f32p, _i32p, _i32p,
                                  _i32p, _i32p, _i32p, _i32p, C.c_int32, C.c_float, C.c_float,
                                  C.c_float, C.c_float, C.c_int, C.c_float, C.c_float, _f64p]
        L.or_build_tree.argtypes = [_u64p, _f32p, C.c_int64, C.c_int, C.c_int, C.c_int64,
                                    _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _f32p, _f32p,
                                    _f32p, _f32p]
        L.or_build_tree.restype = C.c_int64
        L.or_mlp_forward.argtypes = [_f32p, _f32p, C.c_int64, C.c_float, _f32p]
        L.or_mlp_grad.argtypes = [_f32p, _f32p, _f32p, C.c_int64, _f64p, C.POINTER(C.c_double)]
        L.or_tree_groups.argtypes = [_i32p, _i32p, _i32p, _i32p, _f32p, _f32p, _f32p, C.c_int32,
                                     _i64p]
        L.or_tree_groups.restype = C.c_int64
        L.or_walk.argtypes = [_f32p, C.c_int64, _i32p, _i32p, _i32p, _i32p, _f32p, _f32p,
                              _f32p, _f32p, C.POINTER(WalkParams), C.c_void_p, C.c_int64, _f64p,
                              C.c_void_p, _i64p, _i64p]
        L.or_walk_ex.argtypes = L.or_walk.argtypes + [C.c_void_p, C.c_int64, C.c_void_p]
        L.or_pm_periodic_at.argtypes = [_f32p, C.c_int64, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.c_int, C.c_double, C.c_void_p, C.c_int64, _f64p,
                                        C.c_void_p, C.c_void_p]
        L.or_pm_isolated.argtypes = [_f32p, C.c_int64, C.c_int, C.c_float, C.c_float, C.c_double,
                                     C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int64, _f64p,
                                     _f64p, C.c_void_p, C.c_void_p]
        L.or_direct_f64.argtypes = [_f32p, C.c_int64, C.c_void_p, C.c_int64, C.c_double,
                                    C.c_double, C.c_double, C.c_double, _f64p, C.c_void_p]
        L.or_ewald_f64.argtypes = [_f32p, C.c_int64, C.c_void_p, C.c_int64, C.c_double,
                                   C.c_double, C.c_double, C.c_int, _f64p]
        L.or_fft3d.argtypes = [_f64p, C.c_int, C.c_int]
        L.or_pm_periodic.argtypes = [_f32p, C.c_int64, C.c_int, C.c_double, C.c_double, C.c_int,
                                     C.c_int, C.c_double, _f64p, C.c_void_p, C.c_void_p]
        L.or_split_weight.argtypes = [C.c_double, C.c_double]
        L.or_split_weight.restype = C.c_double
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libbzref.so"))


def ref():
    """The reference's own code (compiled from its sources), or None when not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libbzref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_morton_keys.argtypes = [_f32p, _f32p, _f32p, C.c_int, _u64p, _i32p, _f32p]
        R.ref_linear_octree.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int,
                                        _f32p, _i32p, _i32p, _i32p, _i32p, _i32p, _u64p, _i32p,
                                        _i32p]
        R.ref_octree_gpu_accel.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                           C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                           C.c_float, C.c_float, _f32p, _f32p, _f32p,
                                           C.POINTER(C.c_int)]
        R.ref_octree_cpu_accel.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                                           C.c_float, C.c_void_p, C.c_int, _f32p, _f32p, _f32p]
        R.ref_octree_cpu_build.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                                           C.c_float]
        R.ref_octree_cpu_build.restype = C.c_void_p
        R.ref_octree_cpu_walk.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _f32p, _f32p, _f32p]
        R.ref_octree_cpu_nodes.argtypes = [C.c_void_p]
        R.ref_octree_cpu_free.argtypes = [C.c_void_p]
        R.ref_fp64_pairwise.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float,
                                        C.c_float, _f32p, _f32p, _f32p]
        R.ref_pm_periodic.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_double,
                                      C.c_double, C.c_int, C.c_char_p, _f32p, _f32p, _f32p,
                                      C.c_void_p, C.c_void_p]
        R.ref_fft3d.argtypes = [_f64p, C.c_int, C.c_int]
        R.ref_short_range_pair.argtypes = [_f32p, _f32p, C.c_float, C.c_float, C.c_float,
                                           C.c_float, _f32p]
        R.ref_omp_threads.restype = C.c_int
        _REF = R
    return _REF


# ------------------------------------------------------------------------- helpers

def _soa(pos):
    pos = np.asarray(pos, np.float32)
    return [np.ascontiguousarray(pos[:, a]) for a in range(3)]


def pos4(pos, mass):
    out = np.empty((len(mass), 4), np.float32)
    out[:, :3] = pos
    out[:, 3] = mass
    return out


def morton_ref(pos, fused=True):
    """Reference keys; fused=True models the reference CUDA kernel (nvcc contraction)."""
    x, y, z = _soa(pos)
    bb = np.zeros(6, np.float32)
    lib().or_bbox_f32(x, y, z, len(x), bb)
    keys = np.zeros(len(x), np.uint64)
    lib().or_morton_ref(x, y, z, len(x), bb, 1 if fused else 0, keys)
    return keys, bb


def morton63(pos64, origin, size):
    pos64 = np.asarray(pos64, np.float64)
    keys = np.zeros(len(pos64), np.uint64)
    lib().or_morton63(np.ascontiguousarray(pos64[:, 0]), np.ascontiguousarray(pos64[:, 1]),
                      np.ascontiguousarray(pos64[:, 2]), len(pos64),
                      np.asarray(origin, np.float64), float(size), keys)
    return keys


def stable_sort(keys):
    perm = np.zeros(len(keys), np.int32)
    lib().or_stable_sort_u64(np.ascontiguousarray(keys, np.uint64), len(keys), perm)
    return perm


def ref_linear_octree(pos, mass, leaf_capacity=256, fused=True):
    """Restated reference topology (fused=True: as its CUDA build rounds).  Returns a dict."""
    x, y, z = _soa(pos)
    n = len(x)
    cap = 8 * n + 64
    out = dict(hot=np.zeros(8 * cap, np.float32), next=np.zeros(cap, np.int32),
               mask=np.zeros(cap, np.int32), first=np.zeros(cap, np.int32),
               lstart=np.zeros(cap, np.int32), lcount=np.zeros(cap, np.int32),
               keys=np.zeros(n, np.uint64), index=np.zeros(n, np.int32))
    depth = np.zeros(1, np.int32)
    nn = lib().or_ref_linear_octree(x, y, z, np.asarray(mass, np.float32), n, leaf_capacity,
                                    1 if fused else 0, cap,
                                    out["hot"], out["next"], out["mask"], out["first"],
                                    out["lstart"], out["lcount"], out["keys"], out["index"], depth)
    if nn < 0:
        raise RuntimeError("reference octree capacity overflow")
    res = {k: (v[: 8 * nn].reshape(nn, 8) if k == "hot" else v[:nn]) for k, v in out.items()
           if k not in ("keys", "index")}
    res["keys"], res["index"], res["leaf_depth"], res["nodes"] = out["keys"], out["index"], int(depth[0]), int(nn)
    return res


def ref_walk(pos, mass, tree, theta=0.5, softening=0.01, min_distance2=1e-12,
             max_acceleration=1e30, criterion=0, split_scale=0.0, cutoff2=0.0):
    x, y, z = _soa(pos)
    acc = np.zeros(3 * len(x), np.float64)
    lib().or_ref_walk(x, y, z, np.asarray(mass, np.float32), len(x),
                      np.ascontiguousarray(tree["hot"].reshape(-1)), tree["next"], tree["mask"],
                      tree["first"], tree["lstart"], tree["lcount"], tree["index"],
                      tree["nodes"] - 1, theta, softening, min_distance2, max_acceleration,
                      criterion, split_scale, cutoff2, acc)
    return acc.reshape(-1, 3)


def build_tree(sorted_keys, sorted_pos4, leaf_cap=16, max_level=21):
    n = len(sorted_keys)
    cap = 2 * n + 64
    a = {k: np.zeros(cap, np.int32) for k in ("start", "count", "child", "nchild", "parent", "level")}
    mono = np.zeros(4 * cap, np.float32)
    bmin = np.zeros(3 * cap, np.float32)
    bmax = np.zeros(3 * cap, np.float32)
    quad = np.zeros(6 * cap, np.float32)
    nn = lib().or_build_tree(np.ascontiguousarray(sorted_keys, np.uint64),
                             np.ascontiguousarray(sorted_pos4, np.float32), n, leaf_cap, max_level,
                             cap, a["start"], a["count"], a["child"], a["nchild"], a["parent"],
                             a["level"], mono, bmin, bmax, quad)
    if nn < 0:
        raise RuntimeError("tree capacity overflow")
    t = {k: v[:nn] for k, v in a.items()}
    t["mono"] = mono[: 4 * nn].reshape(nn, 4)
    t["bmin"] = bmin[: 3 * nn].reshape(nn, 3)
    t["bmax"] = bmax[: 3 * nn].reshape(nn, 3)
    t["quad"] = quad[: 6 * nn].reshape(nn, 6)
    t["nodes"] = int(nn)
    return t


def tree_groups(tree, gmax=32):
    """Group start indices (plus the end sentinel) cut from the tree, the engine's rule."""
    n = int(tree["count"][0])
    g = np.zeros(n + 2, np.int64)
    ng = lib().or_tree_groups(tree["start"], tree["count"], tree["child"], tree["nchild"],
                              np.ascontiguousarray(tree["bmin"].reshape(-1)),
                              np.ascontiguousarray(tree["bmax"].reshape(-1)),
                              np.ascontiguousarray(tree["mono"].reshape(-1)), gmax, g)
    return g[: ng + 1].copy()


def walk(sorted_pos4, tree, theta=0.5, eps=0.01, rcut=0.0, box=0.0, rsplit=0.0,
         min_dist2=1e-12, quadrupole=True, group=None, want_pot=False, max_node_size=0.0,
         gmax=32):
    """Group walk.  group=None: groups of at most gmax targets cut from the tree (as the
    engine does); an integer: fixed groups of that many consecutive sorted targets."""
    n = len(sorted_pos4)
    prm = WalkParams(np.float32(theta) * np.float32(theta), np.float32(eps) * np.float32(eps),
                     np.float32(rcut) * np.float32(rcut), box, rsplit, min_dist2,
                     1 if quadrupole else 0, group or 32, max_node_size)
    acc = np.zeros(3 * n, np.float64)
    pot = np.zeros(n, np.float64) if want_pot else None
    if group is None:
        gstart = tree_groups(tree, gmax)
        ng = len(gstart) - 1
    else:
        gstart = np.arange(0, n + group, group, dtype=np.int64)
        gstart[-1] = n
        gstart = gstart[: (n + group - 1) // group + 1]
        ng = len(gstart) - 1
    npp = np.zeros(ng, np.int64)
    npn = np.zeros(ng, np.int64)
    lib().or_walk(np.ascontiguousarray(sorted_pos4, np.float32), n, tree["start"], tree["count"],
                  tree["child"], tree["nchild"], np.ascontiguousarray(tree["mono"].reshape(-1)),
                  np.ascontiguousarray(tree["bmin"].reshape(-1)),
                  np.ascontiguousarray(tree["bmax"].reshape(-1)),
                  np.ascontiguousarray(tree["quad"].reshape(-1)), C.byref(prm),
                  gstart.ctypes.data, ng, acc, pot.ctypes.data if pot is not None else None,
                  npp, npn)
    out = dict(acc=acc.reshape(n, 3), n_pp=npp, n_pn=npn, gstart=gstart,
               group_sizes=np.diff(gstart))
    if pot is not None:
        out["pot"] = pot
    return out


def walk_targets(sorted_pos4, tree, sorted_targets, theta=0.5, eps=0.01, rcut=0.0, box=0.0,
                 rsplit=0.0, min_dist2=1e-12, quadrupole=True, max_node_size=0.0, gmax=32):
    """Group walk (the engine's tree groups) of only the groups that hold the given sorted
    target indices.  Returns (acc[len(targets), 3], asum[len(targets)]): the short-range
    accelerations of those targets and, per target, the sum of the magnitudes of its terms."""
    n = len(sorted_pos4)
    prm = WalkParams(np.float32(theta) * np.float32(theta), np.float32(eps) * np.float32(eps),
                     np.float32(rcut) * np.float32(rcut), box, rsplit, min_dist2,
                     1 if quadrupole else 0, 32, max_node_size)
    gstart = tree_groups(tree, gmax)
    ng = len(gstart) - 1
    tg = np.asarray(sorted_targets, np.int64)
    only = np.unique(np.searchsorted(gstart, tg, side="right") - 1).astype(np.int64)
    acc = np.zeros(3 * n, np.float64)
    asum = np.zeros(n, np.float64)
    npp = np.zeros(ng, np.int64)
    npn = np.zeros(ng, np.int64)
    lib().or_walk_ex(np.ascontiguousarray(sorted_pos4, np.float32), n, tree["start"], tree["count"],
                     tree["child"], tree["nchild"], np.ascontiguousarray(tree["mono"].reshape(-1)),
                     np.ascontiguousarray(tree["bmin"].reshape(-1)),
                     np.ascontiguousarray(tree["bmax"].reshape(-1)),
                     np.ascontiguousarray(tree["quad"].reshape(-1)), C.byref(prm),
                     gstart.ctypes.data, ng, acc, None, npp, npn, only.ctypes.data, len(only),
                     asum.ctypes.data)
    return acc.reshape(n, 3)[tg], asum[tg]


def direct(pos4_, targets=None, eps=0.01, box=0.0, rsplit=0.0, rcut=0.0, want_pot=False):
    p = np.ascontiguousarray(pos4_, np.float32)
    if targets is None:
        nt, tptr, tg = len(p), None, None
    else:
        tg = np.ascontiguousarray(targets, np.int64)
        nt, tptr = len(tg), tg.ctypes.data
    acc = np.zeros(3 * nt, np.float64)
    pot = np.zeros(nt, np.float64) if want_pot else None
    lib().or_direct_f64(p, len(p), tptr, nt, eps, box, rsplit, rcut, acc,
                        pot.ctypes.data if pot is not None else None)
    return (acc.reshape(nt, 3), pot) if want_pot else acc.reshape(nt, 3)


def ewald(pos4_, targets=None, eps=0.0, box=1.0, alpha=None, kmax=8):
    p = np.ascontiguousarray(pos4_, np.float32)
    if alpha is None:
        alpha = 6.4 / box
    tg = None if targets is None else np.ascontiguousarray(targets, np.int64)
    nt = len(p) if tg is None else len(tg)
    acc = np.zeros(3 * nt, np.float64)
    lib().or_ewald_f64(p, len(p), None if tg is None else tg.ctypes.data, nt, eps, box, alpha,
                       kmax, acc)
    return acc.reshape(nt, 3)


ASSIGNMENT_ORDER = {"cic": 2, "tsc": 3, "pcs": 4}


def pm_periodic(pos4_, mesh, box, rsplit, want_fields=False, assignment="cic", spectral=False,
                window_floor=0.08, gradient=None):
    """Periodic PM accelerations; gradient: 0 centred differences, 1 spectral (spectral=True),
    2 analytic differentiation of the assignment weights (overrides spectral when given)."""
    p = np.ascontiguousarray(pos4_, np.float32)
    mode = gradient if gradient is not None else (1 if spectral else 0)
    acc = np.zeros(3 * len(p), np.float64)
    cells = mesh ** 3
    dens = np.zeros(cells, np.float64) if want_fields else None
    phi = np.zeros(cells, np.float64) if want_fields else None
    lib().or_pm_periodic(p, len(p), mesh, box, rsplit, ASSIGNMENT_ORDER[assignment],
                         mode, window_floor, acc,
                         None if dens is None else dens.ctypes.data,
                         None if phi is None else phi.ctypes.data)
    if want_fields:
        return acc.reshape(-1, 3), dens, phi
    return acc.reshape(-1, 3)


def pm_periodic_at(pos4_, targets, mesh, box, rsplit, assignment="cic", spectral=False,
                   window_floor=0.08, gradient=None):
    """pm_periodic's mesh force interpolated only at the given particle indices."""
    p = np.ascontiguousarray(pos4_, np.float32)
    mode = gradient if gradient is not None else (1 if spectral else 0)
    tg = np.ascontiguousarray(targets, np.int64)
    acc = np.zeros(3 * len(tg), np.float64)
    lib().or_pm_periodic_at(p, len(p), mesh, box, rsplit, ASSIGNMENT_ORDER[assignment],
                            mode, window_floor, tg.ctypes.data, len(tg), acc,
                            None, None)
    return acc.reshape(-1, 3)


def pm_isolated(pos4_, grid_half, rsplit_cells, assignment="cic", gradient=0, window_floor=0.08,
                cell_floor=0.25, softening=0.0, targets=None, want_fields=False):
    """The reference GPU TreePM's isolated PM (doubled mesh of 2 grid_half cells centred on the
    particle bounds, cell = max(cell_floor, extent / (grid_half - 2)), r_s = rsplit_cells x
    cell): returns (acc[n or len(targets), 3], params) with params = {cell, origin, mesh,
    rsplit, extent}, plus (density, phi) meshes when want_fields."""
    p = np.ascontiguousarray(pos4_, np.float32)
    tg = None if targets is None else np.ascontiguousarray(targets, np.int64)
    nt = len(p) if tg is None else len(tg)
    acc = np.zeros(3 * nt, np.float64)
    par = np.zeros(8, np.float64)
    M = 2 * grid_half
    dens = np.zeros(M ** 3, np.float64) if want_fields else None
    phi = np.zeros(M ** 3, np.float64) if want_fields else None
    lib().or_pm_isolated(p, len(p), grid_half, cell_floor, softening, rsplit_cells,
                         ASSIGNMENT_ORDER[assignment], gradient, window_floor,
                         None if tg is None else tg.ctypes.data, nt, acc, par,
                         None if dens is None else dens.ctypes.data,
                         None if phi is None else phi.ctypes.data)
    params = dict(cell=par[0], origin=par[1:4].copy(), mesh=int(par[4]), rsplit=par[5], extent=par[6])
    out = (acc.reshape(-1, 3), params)
    return out + (dens, phi) if want_fields else out


def fft3d(cube_complex, inverse=False):
    a = np.ascontiguousarray(np.stack([cube_complex.real, cube_complex.imag], -1).reshape(-1), np.float64)
    lib().or_fft3d(a, cube_complex.shape[0], 1 if inverse else 0)
    a = a.reshape(-1, 2)
    return (a[:, 0] + 1j * a[:, 1]).reshape(cube_complex.shape)


def clamp_acceleration(acc, max_acc):
    """The reference's acceleration clamp (clampAcceleration, engine/physics/core/cuda/prelude/
    CudForceKernels.inl:7-14) on an (n, 3) array: FP32 norm, vectors longer than max_acc
    scaled to that length."""
    a = np.asarray(acc, np.float32)
    norm = np.sqrt((a * a).sum(axis=1, dtype=np.float32)).astype(np.float32)
    m = np.float32(max_acc)
    scale = np.where((norm > m) & (norm > np.float32(1e-12)), m / np.maximum(norm, np.float32(1e-30)),
                     np.float32(1.0)).astype(np.float32)
    return (np.asarray(acc, np.float64) * scale[:, None]).astype(np.float64)


def split_weight(s, rsplit):
    return lib().or_split_weight(float(s), float(rsplit))


def mlp_forward(params, x6, scale=1.0):
    """CPU restatement of the learned-correction MLP (same BF16 rounding points)."""
    x = np.ascontiguousarray(x6, np.float32)
    out = np.zeros((len(x), 3), np.float32)
    lib().or_mlp_forward(np.ascontiguousarray(params, np.float32), x, len(x), scale, out)
    return out


def mlp_grad(params, x6, y3):
    x = np.ascontiguousarray(x6, np.float32)
    g = np.zeros(1667, np.float64)
    loss = C.c_double(0.0)
    lib().or_mlp_grad(np.ascontiguousarray(params, np.float32), x, np.ascontiguousarray(y3, np.float32),
                      len(x), g, C.byref(loss))
    return g, loss.value


def ref_gpu():
    """The reference's own GPU octree (``_ref/libbzrefgpu.so``), or None when not built.

    ``refgpu_create(n, leaf_capacity, px, py, pz, vx, vy, vz, mass)`` -> handle;
    ``refgpu_step(h, dt, theta, softening, min_distance2, max_acceleration, criterion)``;
    ``refgpu_time_steps(h, warmup, steps, dt, ..., criterion, &ms)``;
    ``refgpu_accel(h, theta, softening, min_distance2, max_acceleration, criterion, ax, ay, az,
    &nodes, &leaves)``; ``refgpu_get_state(h, px, py, pz, vx, vy, vz)``; ``refgpu_destroy(h)``.
    Status 0 is success; negative values are argument (-1), CUDA (-2), capacity (-3) or tree
    (-4) errors."""
    global _REF_GPU
    if _REF_GPU is None:
        path = os.path.join(HERE, "_ref", "libbzrefgpu.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.refgpu_create.argtypes = [C.c_int, C.c_int] + [_f32p] * 7
        R.refgpu_create.restype = C.c_void_p
        R.refgpu_destroy.argtypes = [C.c_void_p]
        law = [C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]
        R.refgpu_step.argtypes = [C.c_void_p, C.c_float] + law
        R.refgpu_time_steps.argtypes = ([C.c_void_p, C.c_int, C.c_int, C.c_float] + law +
                                        [C.POINTER(C.c_double)])
        R.refgpu_accel.argtypes = ([C.c_void_p] + law + [_f32p, _f32p, _f32p, C.POINTER(C.c_int),
                                                         C.POINTER(C.c_int)])
        R.refgpu_get_state.argtypes = [C.c_void_p] + [_f32p] * 6
        _REF_GPU = R
    return _REF_GPU
