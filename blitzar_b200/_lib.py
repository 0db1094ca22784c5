"""ctypes binding of libbzgrav.so (the C ABI declared in include/bzgrav.h).

The library is the product; this module only marshals host arrays.  Loading fails loudly if
the shared object has not been built -- there is no CPU fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbzgrav.so")

BZ_OK, BZ_INVALID_ARGUMENT, BZ_NOT_READY, BZ_TIMEOUT, BZ_INTERNAL_ERROR = 0, 1, 2, 3, 4
BZ_CUDA_ERROR, BZ_OUT_OF_MEMORY, BZ_DEVICE_LIMIT, BZ_UNSUPPORTED = 5, 6, 7, 8
BZ_INTEGRATOR_LEAPFROG, BZ_INTEGRATOR_EULER = 0, 1  # bz_integrator
SOLVER_OCTREE, SOLVER_TREEPM, SOLVER_OCTREE_REFERENCE = 0, 1, 2
KEYS_PRODUCTION, KEYS_REFERENCE = 0, 1

#: every symbol include/bzgrav.h declares
EXPORTS = (
    "bz_config_init", "bz_create", "bz_destroy", "bz_set_state", "bz_set_state_f64", "bz_step",
    "bz_accelerations", "bz_get_state", "bz_get_state_f64", "bz_morton_keys", "bz_tree_topology",
    "bz_reference_tree", "bz_interaction_counts", "bz_enable_phase_timing", "bz_phase_times",
    "bz_force_errors", "bz_pm_mesh", "bz_particle_count", "bz_device_bytes", "bz_last_error",
    "bz_status_string", "bz_version", "bz_kernel_launches", "bz_launches_per_step",
    "bz_sort_pairs_noalloc", "bz_energy", "bz_autotune", "bz_learn_generate", "bz_learn_train",
    "bz_learn_set", "bz_learn_get", "bz_learn_enable", "bz_learn_forward", "bz_learn_gradient",
    "bz_set_ensemble", "bz_adaptive_levels", "bz_adaptive_updates", "bz_set_mesh_schedule",
    "bz_walk_blocks_per_sm", "bz_set_state_acc", "bz_get_state_acc", "bz_set_state_acc_f64",
    "bz_get_state_acc_f64", "bz_step_get_state_acc_f64", "bz_walk_counts", "bz_pm_grid",
)

PHASES = ("keys", "sort", "permute", "tree", "mesh", "walk", "integrate", "total")


class BzConfig(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("solver", C.c_int32),
        ("octree_theta", C.c_float),
        ("octree_softening", C.c_float),
        ("octree_opening_criterion", C.c_int32),
        ("linear_octree_leaf_capacity", C.c_int32),
        ("leaf_capacity", C.c_int32),
        ("multipole_order", C.c_int32),
        ("physics_max_acceleration", C.c_float),
        ("physics_min_softening", C.c_float),
        ("physics_min_distance2", C.c_float),
        ("physics_min_theta", C.c_float),
        ("treepm_grid_size", C.c_int32),
        ("treepm_r_split_cells", C.c_float),
        ("treepm_r_cut_factor", C.c_float),
        ("treepm_assignment", C.c_int32),
        ("treepm_gradient", C.c_int32),
        ("treepm_window_floor", C.c_float),
        ("treepm_node_size_factor", C.c_float),
        ("box_length", C.c_double),
        ("key_mode", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_uint64),
        ("use_graph", C.c_int32),
        ("walk_group_size", C.c_int32),
        ("adaptive_max_level", C.c_int32),
        ("adaptive_eta", C.c_float),
        ("treepm_cell_floor", C.c_float),
        ("integrator", C.c_int32),
    ]


class BzError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_LIB = None
_vp = C.c_void_p


def load():
    """Load libbzgrav.so; raise if it is missing (build it with ``python -m blitzar_b200.build``)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run `python -m blitzar_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.bz_config_init.argtypes = [C.POINTER(BzConfig)]
    L.bz_create.argtypes = [C.POINTER(BzConfig), C.c_size_t, C.POINTER(_vp)]
    L.bz_destroy.argtypes = [_vp]
    L.bz_set_state.argtypes = [_vp, _vp, _vp, _vp, C.c_size_t]
    L.bz_set_state_f64.argtypes = [_vp, _vp, _vp, _vp, C.c_size_t]
    L.bz_step.argtypes = [_vp, C.c_double, C.c_uint32]
    L.bz_accelerations.argtypes = [_vp, _vp, _vp]
    L.bz_get_state.argtypes = [_vp, _vp, _vp]
    L.bz_get_state_f64.argtypes = [_vp, _vp, _vp]
    L.bz_morton_keys.argtypes = [_vp, _vp, _vp]
    L.bz_tree_topology.argtypes = [_vp, C.POINTER(C.c_int64)] + [_vp] * 8
    L.bz_reference_tree.argtypes = [_vp, C.POINTER(C.c_int64)] + [_vp] * 6
    L.bz_interaction_counts.argtypes = [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.bz_walk_counts.argtypes = [_vp] + [C.POINTER(C.c_uint64)] * 3
    L.bz_enable_phase_timing.argtypes = [_vp, C.c_int]
    L.bz_phase_times.argtypes = [_vp, _vp, C.c_int]
    L.bz_force_errors.argtypes = [_vp, C.c_int32, C.c_uint64, _vp, _vp, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
    L.bz_pm_mesh.argtypes = [_vp, C.c_int, _vp]
    L.bz_pm_grid.argtypes = [_vp, _vp]
    L.bz_particle_count.argtypes = [_vp]
    L.bz_particle_count.restype = C.c_size_t
    L.bz_device_bytes.argtypes = [_vp]
    L.bz_device_bytes.restype = C.c_size_t
    L.bz_last_error.argtypes = [_vp, C.c_char_p, C.c_size_t]
    L.bz_last_error.restype = C.c_size_t
    L.bz_status_string.argtypes = [C.c_int]
    L.bz_status_string.restype = C.c_char_p
    L.bz_version.restype = C.c_char_p
    L.bz_kernel_launches.restype = C.c_uint64
    L.bz_launches_per_step.argtypes = [_vp, C.POINTER(C.c_uint64)]
    L.bz_energy.argtypes = [_vp, _vp, _vp, _vp]
    L.bz_autotune.argtypes = [_vp, C.c_int32, _vp, _vp, _vp, _vp]
    L.bz_set_mesh_schedule.argtypes = [_vp, C.c_int32]
    L.bz_walk_blocks_per_sm.argtypes = [_vp, C.c_int32, _vp]
    L.bz_set_state_acc.argtypes = [_vp, _vp, _vp, _vp, _vp, C.c_size_t]
    L.bz_get_state_acc.argtypes = [_vp, _vp, _vp, _vp]
    L.bz_set_state_acc_f64.argtypes = [_vp, _vp, _vp, _vp, _vp, C.c_size_t]
    L.bz_get_state_acc_f64.argtypes = [_vp, _vp, _vp, _vp]
    L.bz_step_get_state_acc_f64.argtypes = [_vp, C.c_double, _vp, _vp, _vp]
    L.bz_adaptive_levels.argtypes = [_vp, _vp]
    L.bz_adaptive_updates.argtypes = [_vp, C.POINTER(C.c_uint64)]
    L.bz_set_ensemble.argtypes = [_vp, _vp, _vp, _vp, _vp, C.c_int32]
    L.bz_learn_generate.argtypes = [_vp, C.c_int64, C.c_uint64, _vp, _vp]
    L.bz_learn_train.argtypes = [_vp, _vp, _vp, C.c_int64, C.c_int32, C.c_int32, C.c_float,
                                 C.c_uint64, _vp]
    L.bz_learn_set.argtypes = [_vp, _vp, C.c_float]
    L.bz_learn_get.argtypes = [_vp, _vp, _vp]
    L.bz_learn_enable.argtypes = [_vp, C.c_int32]
    L.bz_learn_forward.argtypes = [_vp, _vp, C.c_int64, _vp]
    L.bz_learn_gradient.argtypes = [_vp, _vp, _vp, C.c_int64, _vp, _vp]
    L.bz_sort_pairs_noalloc.argtypes = [_vp, _vp, C.c_int64, C.c_int, C.c_uint64]
    _LIB = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def default_config(**kw) -> BzConfig:
    cfg = BzConfig()
    load().bz_config_init(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


class Engine:
    """One engine handle (one particle system on one GPU)."""

    def __init__(self, capacity: int, **cfg):
        self.L = load()
        self.cfg = default_config(**cfg)
        h = _vp()
        st = self.L.bz_create(C.byref(self.cfg), capacity, C.byref(h))
        if st != BZ_OK:
            raise BzError(st, f"bz_create: {self.L.bz_status_string(st).decode()}")
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.bz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st != BZ_OK:
            buf = C.create_string_buffer(1024)
            self.L.bz_last_error(self.h, buf, 1024)
            raise BzError(st, f"{what}: {buf.value.decode(errors='replace')}")

    # -- state
    def set_state(self, pos, vel=None, mass=None, f64=False):
        pos = np.asarray(pos)
        n = pos.shape[0]
        if f64:
            p = np.ascontiguousarray(pos.T, np.float64)
            v = None if vel is None else np.ascontiguousarray(np.asarray(vel).T, np.float64)
            m = np.ascontiguousarray(mass, np.float32)
            self._check(self.L.bz_set_state_f64(self.h, _ptr(p), _ptr(v), _ptr(m), n), "bz_set_state_f64")
        else:
            p = np.ascontiguousarray(pos.T, np.float32)
            v = None if vel is None else np.ascontiguousarray(np.asarray(vel).T, np.float32)
            m = np.ascontiguousarray(mass, np.float32)
            self._check(self.L.bz_set_state(self.h, _ptr(p), _ptr(v), _ptr(m), n), "bz_set_state")
        self.n = n

    def adaptive_levels(self):
        lv = np.empty(self.n, np.uint8)
        self._check(self.L.bz_adaptive_levels(self.h, _ptr(lv)), "bz_adaptive_levels")
        return lv

    def adaptive_updates(self):
        u = C.c_uint64(0)
        self._check(self.L.bz_adaptive_updates(self.h, C.byref(u)), "bz_adaptive_updates")
        return u.value

    def set_ensemble(self, systems):
        """systems: list of (pos[n,3], vel[n,3] or None, mass[n]) of independent systems."""
        offs = np.zeros(len(systems) + 1, np.int64)
        for i, (_, _, m) in enumerate(systems):
            offs[i + 1] = offs[i] + len(m)
        n = int(offs[-1])
        pos = np.concatenate([np.asarray(p, np.float64) for p, _, _ in systems])
        vel = np.concatenate([np.zeros((len(m), 3)) if v is None else np.asarray(v, np.float64)
                              for _, v, m in systems])
        mass = np.concatenate([np.asarray(m, np.float32) for _, _, m in systems])
        ps = np.ascontiguousarray(pos.T.reshape(-1))
        vs = np.ascontiguousarray(vel.T.reshape(-1))
        self._check(self.L.bz_set_ensemble(self.h, _ptr(ps), _ptr(vs), _ptr(mass), _ptr(offs),
                                           len(systems)), "bz_set_ensemble")
        self.n = n
        return offs

    def set_state_soa(self, pos_soa3, vel_soa3, mass):
        """Upload from caller-owned SoA float32 buffers (no copies on the Python side)."""
        n = mass.shape[0]
        self._check(self.L.bz_set_state(self.h, _ptr(pos_soa3), _ptr(vel_soa3), _ptr(mass), n),
                    "bz_set_state")
        self.n = n

    def get_state(self, f64=False, with_vel=True):
        n = self.n
        dt = np.float64 if f64 else np.float32
        p = np.empty(3 * n, dt)
        v = np.empty(3 * n, dt) if with_vel else None
        fn = self.L.bz_get_state_f64 if f64 else self.L.bz_get_state
        self._check(fn(self.h, _ptr(p), _ptr(v)), "bz_get_state")
        return p.reshape(3, n).T.copy(), (None if v is None else v.reshape(3, n).T.copy())

    def set_state_acc_soa(self, pos_soa3, vel_soa3, mass, acc_soa3):
        """Upload a leapfrog state with the accelerations of its positions (caller-owned SoA
        float32 buffers): the next step needs no set-up force evaluation."""
        n = mass.shape[0]
        self._check(self.L.bz_set_state_acc(self.h, _ptr(pos_soa3), _ptr(vel_soa3), _ptr(mass),
                                            _ptr(acc_soa3), n), "bz_set_state_acc")
        self.n = n

    def get_state_acc_soa(self, pos_soa3, vel_soa3, acc_soa3):
        """Download positions, velocities and the accelerations of the positions (SoA)."""
        self._check(self.L.bz_get_state_acc(self.h, _ptr(pos_soa3), _ptr(vel_soa3), _ptr(acc_soa3)),
                    "bz_get_state_acc")

    def set_state_acc_f64_soa(self, pos_soa3, vel_soa3, mass, acc_soa3):
        """As set_state_acc_soa with FP64 positions and velocities (accelerations FP32)."""
        n = mass.shape[0]
        self._check(self.L.bz_set_state_acc_f64(self.h, _ptr(pos_soa3), _ptr(vel_soa3), _ptr(mass),
                                                _ptr(acc_soa3), n), "bz_set_state_acc_f64")
        self.n = n

    def get_state_acc_f64_soa(self, pos_soa3, vel_soa3, acc_soa3):
        """FP64 positions and velocities with the FP32 accelerations of the positions (SoA)."""
        self._check(self.L.bz_get_state_acc_f64(self.h, _ptr(pos_soa3), _ptr(vel_soa3),
                                                _ptr(acc_soa3)), "bz_get_state_acc_f64")

    def step_get_state_acc_f64_soa(self, dt, pos_soa3, vel_soa3, acc_soa3):
        """One step, then the FP64 state and FP32 accelerations (SoA), the position download
        overlapping the step (bz_step_get_state_acc_f64)."""
        self._check(self.L.bz_step_get_state_acc_f64(self.h, dt, _ptr(pos_soa3), _ptr(vel_soa3),
                                                     _ptr(acc_soa3)), "bz_step_get_state_acc_f64")

    def get_state_soa(self, pos_soa3, vel_soa3):
        self._check(self.L.bz_get_state(self.h, _ptr(pos_soa3), _ptr(vel_soa3)), "bz_get_state")

    def step(self, dt, nsteps=1):
        self._check(self.L.bz_step(self.h, dt, nsteps), "bz_step")

    def accelerations(self, want_pot=False):
        a = np.empty(3 * self.n, np.float32)
        p = np.empty(self.n, np.float32) if want_pot else None
        self._check(self.L.bz_accelerations(self.h, _ptr(a), _ptr(p)), "bz_accelerations")
        acc = a.reshape(3, self.n).T.copy()
        return (acc, p) if want_pot else acc

    # ---- learned pair correction
    MLP_PARAMS = 1667

    def learn_generate(self, nsamples, seed=1):
        x = np.empty((nsamples, 6), np.float32)
        y = np.empty((nsamples, 3), np.float32)
        self._check(self.L.bz_learn_generate(self.h, nsamples, seed, _ptr(x), _ptr(y)), "bz_learn_generate")
        return x, y

    def learn_train(self, x, y, steps=3000, batch=4096, lr=3e-3, seed=1):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float(0.0)
        self._check(self.L.bz_learn_train(self.h, _ptr(x), _ptr(y), len(x), steps, batch, lr, seed,
                                          C.byref(loss)), "bz_learn_train")
        return loss.value

    def learn_set(self, params, scale):
        p = np.ascontiguousarray(params, np.float32)
        self._check(self.L.bz_learn_set(self.h, _ptr(p), scale), "bz_learn_set")

    def learn_get(self):
        p = np.empty(self.MLP_PARAMS, np.float32)
        sc = C.c_float(0.0)
        self._check(self.L.bz_learn_get(self.h, _ptr(p), C.byref(sc)), "bz_learn_get")
        return p, sc.value

    def learn_enable(self, on=True):
        self._check(self.L.bz_learn_enable(self.h, 1 if on else 0), "bz_learn_enable")

    def learn_forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((len(x), 3), np.float32)
        self._check(self.L.bz_learn_forward(self.h, _ptr(x), len(x), _ptr(y)), "bz_learn_forward")
        return y

    def learn_gradient(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.empty(self.MLP_PARAMS, np.float32)
        loss = C.c_float(0.0)
        self._check(self.L.bz_learn_gradient(self.h, _ptr(x), _ptr(y), len(x), _ptr(g), C.byref(loss)),
                    "bz_learn_gradient")
        return g, loss.value

    def autotune(self, trials=3):
        """Pick the fastest (leaf capacity, walk group size, TreePM mesh schedule) for the current
        state; the schedule is 0 in line, 1 concurrent with the tree build and walk, 2 also
        concurrent with the sort."""
        leaf = C.c_int32(0)
        grp = C.c_int32(0)
        ms = C.c_float(0.0)
        ov = C.c_int32(0)
        self._check(self.L.bz_autotune(self.h, trials, C.byref(leaf), C.byref(grp), C.byref(ms),
                                       C.byref(ov)), "bz_autotune")
        self.last_tune = dict(leaf_capacity=leaf.value, walk_group_size=grp.value,
                              mesh_schedule=ov.value, walk_blocks_per_sm=self.walk_blocks_per_sm(),
                              ms_per_evaluation=ms.value)
        return leaf.value, grp.value, ms.value

    def walk_blocks_per_sm(self, value=-1):
        """Cap on resident walk blocks per SM (0: as many as fit); value < 0 only queries."""
        cur = C.c_int32(0)
        self._check(self.L.bz_walk_blocks_per_sm(self.h, int(value), C.byref(cur)),
                    "bz_walk_blocks_per_sm")
        return cur.value

    def set_mesh_schedule(self, schedule):
        """Pin the TreePM mesh-leg schedule (0 in line, 1 concurrent with the tree build and
        walk, 2 also concurrent with the sort)."""
        self._check(self.L.bz_set_mesh_schedule(self.h, int(schedule)), "bz_set_mesh_schedule")

    def energy(self, potential=True):
        """FP64 (kinetic, potential or None, momentum[3]) of the current state."""
        ke = C.c_double(0.0)
        pe = C.c_double(0.0)
        mom = np.zeros(3, np.float64)
        self._check(self.L.bz_energy(self.h, C.byref(ke), C.byref(pe) if potential else None,
                                     _ptr(mom)), "bz_energy")
        return ke.value, (pe.value if potential else None), mom

    def morton_keys(self):
        k = np.empty(self.n, np.uint64)
        p = np.empty(self.n, np.int32)
        self._check(self.L.bz_morton_keys(self.h, _ptr(k), _ptr(p)), "bz_morton_keys")
        return k, p

    def tree(self):
        nn = C.c_int64(0)
        self._check(self.L.bz_tree_topology(self.h, C.byref(nn), *([None] * 8)), "bz_tree_topology")
        k = nn.value
        t = {name: np.empty(k, np.int32) for name in ("start", "count", "child", "nchild")}
        t["mono"] = np.empty((k, 4), np.float32)
        t["bmin"] = np.empty((k, 3), np.float32)
        t["bmax"] = np.empty((k, 3), np.float32)
        t["quad"] = np.empty((k, 6), np.float32)
        self._check(self.L.bz_tree_topology(self.h, C.byref(nn), _ptr(t["start"]), _ptr(t["count"]),
                                            _ptr(t["child"]), _ptr(t["nchild"]), _ptr(t["mono"]),
                                            _ptr(t["bmin"]), _ptr(t["bmax"]), _ptr(t["quad"])),
                    "bz_tree_topology")
        t["nodes"] = k
        return t

    def reference_tree(self):
        nn = C.c_int64(0)
        hot = np.empty(8, np.float32)
        arrs = [np.empty(1, np.int32) for _ in range(5)]
        self._check(self.L.bz_reference_tree(self.h, C.byref(nn), _ptr(hot), *[_ptr(a) for a in arrs]),
                    "bz_reference_tree")
        return dict(nodes=nn.value, hot=hot.reshape(1, 8), next=arrs[0], mask=arrs[1],
                    first=arrs[2], lstart=arrs[3], lcount=arrs[4])

    def interaction_counts(self):
        a, b = C.c_uint64(0), C.c_uint64(0)
        self._check(self.L.bz_interaction_counts(self.h, C.byref(a), C.byref(b)), "bz_interaction_counts")
        return a.value, b.value

    def walk_counts(self):
        """(listed pairs, pairs through the pair law, multipole terms) of the last walk."""
        a, b, c = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        self._check(self.L.bz_walk_counts(self.h, C.byref(a), C.byref(b), C.byref(c)), "bz_walk_counts")
        return a.value, b.value, c.value

    def enable_timing(self, on=True):
        self._check(self.L.bz_enable_phase_timing(self.h, 1 if on else 0), "bz_enable_phase_timing")

    def phase_times(self):
        ms = np.zeros(len(PHASES), np.float32)
        self._check(self.L.bz_phase_times(self.h, _ptr(ms), len(PHASES)), "bz_phase_times")
        return dict(zip(PHASES, ms.tolist()))

    def force_errors(self, nsample=4096, seed=1):
        errs = np.empty(nsample, np.float32)
        idx = np.empty(nsample, np.int32)
        med, p99 = C.c_double(0), C.c_double(0)
        self._check(self.L.bz_force_errors(self.h, nsample, seed, _ptr(errs), _ptr(idx), C.byref(med),
                                           C.byref(p99)), "bz_force_errors")
        return dict(median=med.value, p99=p99.value, errs=errs, idx=idx)

    def pm_mesh(self, which):
        M = self.cfg.treepm_grid_size * (2 if self.cfg.box_length <= 0.0 else 1)
        out = np.empty(M ** 3, np.float32)
        self._check(self.L.bz_pm_mesh(self.h, which, _ptr(out)), "bz_pm_mesh")
        return out

    def pm_grid(self):
        """Mesh grid of the last force evaluation: dict(origin, cell, rsplit, rcut)."""
        v = np.zeros(6, np.float64)
        self._check(self.L.bz_pm_grid(self.h, _ptr(v)), "bz_pm_grid")
        return dict(origin=v[:3].copy(), cell=v[3], rsplit=v[4], rcut=v[5])

    def launches_per_step(self):
        k = C.c_uint64(0)
        self._check(self.L.bz_launches_per_step(self.h, C.byref(k)), "bz_launches_per_step")
        return k.value

    def device_bytes(self):
        return self.L.bz_device_bytes(self.h)
