#!/usr/bin/env python
"""Benchmark: particle-steps/s of the periodic TreePM leapfrog step on one B200.

Workload (default ``treepm256``, the box the metric's learned-vs-plain target is stated on):
N = 256^3 = 16,777,216 equal-mass particles on a unit periodic box, grid positions displaced by
a Zel'dovich field of a Gaussian random field with P(k) ~ k^-2 (3-D rms displacement 0.2 cell,
seed 4), zero velocities, theta = 0.5, Plummer softening 0.02 lattice cell, FP64 leapfrog with
dt = 5e-4.  Inputs are seeded synthetic data.  The mesh settings (512^3 PCS mesh, spectral
gradient, r_s = 1.0 mesh cell, cutoff 5 r_s, no multipoles inside the cutoff) are the cheapest
found that hold the median force error under 1e-3 against FP64 Ewald on this box (r_s = 0.9
and 0.8 cells miss it; 4.5 r_s misses it); ``treepm128`` is the same recipe at 128^3 (seed 2)
and ``treepm128_cic`` runs the reference mesh (128^3 CIC, centred differences, cutoff 4.5 r_s).

A "step" is one KDK leapfrog step of the whole system (keys, sort, permutation, octree,
mesh, group walk, kicks and drift), replayed from a CUDA graph.  The state (about 230 B per
particle: ~3.9 GB at 256^3, ~480 MB at 128^3) is larger than the 126 MB L2, so no flush is
needed between steps.

Under torchrun (N > 1) every rank steps an independent replica (the force evaluation of one
system does not shard) and `value` sums all ranks' particle-steps over the slowest rank's
device time.  ``--impl reference`` times the reference's CPU TreePM path instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PP = {True: 35, False: 20}          # pair: monopole 20 (rsqrt = 1), + 15 with the split
FLOP_PN = {(True, True): 80, (True, False): 35, (False, True): 65, (False, False): 20}
FP32_LANES_PER_SM = 128
SMS = 148
NOMINAL_SM_MHZ = 1965.0

# treepm128: the 128^3 periodic box at <= 1e-3 median force error against FP64 Ewald: PCS
# assignment, spectral gradient, a 256^3 mesh (twice the particle lattice) with r_s = 1.0 mesh
# cell, r_cut = 5 r_s (4.5 r_s misses the target), and no multipoles inside the cutoff (the split kernel's expansion error
# is large next to the small net forces of this near-uniform box).  treepm128_cic runs the
# reference-style mesh (CIC, centred differences, 128^3, r_cut 4.5 r_s, theta 0.5 multipoles),
# which stays near 2e-2 median error on this box.
WORKLOADS = {
    "treepm128": dict(kind="treepm", n_side=128, mesh=256, r_split_cells=1.0, r_cut_factor=5.0,
                      theta=0.5, eps_lattice=0.02, dt=5e-4, seed=2, rms_cells=0.2,
                      assignment="pcs", gradient="analytic", node_size_factor=0.5),
    "treepm256": dict(kind="treepm", n_side=256, mesh=512, r_split_cells=0.95, r_cut_factor=5.0,
                      theta=0.5, eps_lattice=0.02, dt=5e-4, seed=4, rms_cells=0.2,
                      assignment="pcs", gradient="analytic", node_size_factor=0.5),
    "treepm128_cic": dict(kind="treepm", n_side=128, mesh=128, r_split_cells=1.25, r_cut_factor=4.5,
                          theta=0.5, eps_lattice=0.02, dt=5e-4, seed=2, rms_cells=0.2,
                          assignment="cic", gradient="centred-difference", node_size_factor=0.0),
    "treepm64": dict(kind="treepm", n_side=64, mesh=128, r_split_cells=1.0, r_cut_factor=5.0,
                     theta=0.5, eps_lattice=0.02, dt=5e-4, seed=2, rms_cells=0.2,
                     assignment="pcs", gradient="analytic", node_size_factor=0.5),
    # the reference's own GPU TreePM (isolated doubled mesh) at its defaults for the 13 TreePM
    # parameters (grid 64 -> mesh 128, cutoff 1 cell, CIC, centred differences) on a Plummer
    # sphere of 1M particles
    "treepm_open": dict(kind="treepm_open", ic="plummer", n=1 << 20, grid=64, cutoff_factor=1.0,
                        assignment="cic", theta=0.5, eps=0.01, dt=1e-3, seed=1),
    "plummer65k": dict(kind="octree", ic="plummer", n=65536, theta=0.5, eps=0.01, dt=1e-3, seed=1),
    "hernquist4m": dict(kind="octree", ic="hernquist", n=4194304, theta=0.4, eps=0.005, dt=2e-4,
                        seed=3),
    "ensemble256": dict(kind="ensemble", clusters=256, n_min=1024, n_max=65536, w0_min=3.0,
                        w0_max=9.0, theta=0.5, eps=0.01, dt=1e-3, seed=5, adaptive_levels=7,
                        adaptive_eta=0.02),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="treepm256")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--error-sample", type=int, default=2048)
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of reference CPU work for the cpu_baseline object")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default leaf capacity, group size and mesh overlap")
    ap.add_argument("--tune", default="",
                    help="LEAF,GROUP,SCHEDULE: pin the autotuner's three choices instead of "
                         "tuning (to profile the configuration a tuned run picked)")
    ap.add_argument("--learned-experiment", choices=["split", "cut"], default="split",
                    help="split: plain and learned at a smaller split scale; cut: plain at "
                         "r_cut 4.5 r_s against learned at 3.0 r_s")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-correction comparison (TreePM workloads)")
    return ap.parse_args()


# --------------------------------------------------------------------------- setup

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local, backend="nccl"):
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def make_ensemble(w, rank):
    """King clusters with N log-uniform in [n_min, n_max] and W0 uniform in [w0_min, w0_max]."""
    from blitzar_b200 import ics

    rng = np.random.default_rng(w["seed"] + rank)
    sizes = np.rint(np.exp(rng.uniform(np.log(w["n_min"]), np.log(w["n_max"]), w["clusters"])))
    w0 = rng.uniform(w["w0_min"], w["w0_max"], w["clusters"])
    systems = []
    for i, (n, W0) in enumerate(zip(sizes.astype(int), w0)):
        p, v, m = ics.king(int(n), 1000 * (w["seed"] + rank) + i, float(W0))
        systems.append((p, v, m.astype(np.float32)))
    return systems


def make_ics(w, rank):
    from blitzar_b200 import ics

    if w["kind"] == "ensemble":
        systems = make_ensemble(w, rank)
        pos = np.concatenate([p for p, _, _ in systems])
        vel = np.concatenate([v for _, v, _ in systems])
        mass = np.concatenate([m for _, _, m in systems])
        return pos, vel, mass
    if w["kind"] == "treepm":
        pos, vel, mass = ics.grf_grid(w["n_side"], seed=w["seed"] + rank, rms_cells=w["rms_cells"])
    elif w["kind"] == "treepm_open" or w["ic"] == "plummer":
        pos, vel, mass = ics.plummer(w["n"], seed=w["seed"] + rank)
    elif w["ic"] == "hernquist":
        pos, vel, mass = ics.hernquist(w["n"], seed=w["seed"] + rank)
    else:
        pos, vel, mass = ics.plummer(w["n"], seed=w["seed"] + rank)
    return pos, vel, mass.astype(np.float32)


def engine_config(w):
    if w["kind"] == "treepm":
        grad = {"centred-difference": 0, "spectral": 1, "analytic": 2}[w["gradient"]]
        return dict(solver=1, box_length=1.0, treepm_grid_size=w["mesh"],
                    treepm_r_split_cells=w["r_split_cells"], treepm_r_cut_factor=w["r_cut_factor"],
                    treepm_assignment={"cic": 0, "tsc": 1, "pcs": 2}[w["assignment"]],
                    treepm_gradient=grad,
                    treepm_window_floor=0.0 if grad else 0.08,
                    treepm_node_size_factor=w["node_size_factor"],
                    octree_theta=w["theta"], octree_softening=w["eps_lattice"] / w["n_side"],
                    # with the node-size cap no node is accepted inside the cutoff on these
                    # boxes (particle_node = 0 in the counters), so the walk needs no multipoles
                    # and the tree no second moments; the cic workload (no cap) keeps them
                    multipole_order=1 if w["node_size_factor"] > 0 else 2)
    if w["kind"] == "treepm_open":
        # the reference's isolated TreePM: setTreePmParameters(grid, cutoffFactor, assignment)
        # maps to this mesh of 2 x grid cells, r_s = cutoff / 4.5, r_cut = 4.5 r_s
        return dict(solver=1, box_length=0.0, treepm_grid_size=w["grid"],
                    treepm_r_split_cells=w["cutoff_factor"] / 4.5, treepm_r_cut_factor=4.5,
                    treepm_assignment={"cic": 0, "tsc": 1, "pcs": 2}[w["assignment"]],
                    treepm_gradient=0, treepm_window_floor=0.08, octree_theta=w["theta"],
                    octree_softening=w["eps"], multipole_order=2)
    cfg = dict(solver=0, octree_theta=w["theta"], octree_softening=w["eps"], multipole_order=2)
    if w.get("adaptive_levels"):
        cfg.update(adaptive_max_level=w["adaptive_levels"], adaptive_eta=w["adaptive_eta"])
    return cfg


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples taken while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100",
                                          "-i", str(self.dev)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_traffic(name):
    path = os.path.join(ROOT, "profiles", f"{name}.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


# --------------------------------------------------------------------------- CPU baseline

def cpu_reference_step(w, pos, mass, budget_s, seed=7, chunk=65536):
    """One force evaluation of the reference's CPU code on the box's host cores, measured, not
    modelled, as far as `budget_s` seconds allow.

    TreePM: the reference's periodic PM templates (TpmAssignment/TpmField, FP32, CIC) over all
    N particles, then its octree_cpu build over all N (Octree::build, serial in the reference),
    then its cutoff/erfc-split walk (Octree::computeForceOn, OpenMP) over the targets in seeded
    random chunks.  Octree: the build, then the walk over the targets.  Ensembles: build and
    walk of whole clusters, one after another.  The PM and the build always run in full; only
    walk chunks (or clusters) left when the budget runs out are extrapolated, by target (or
    particle) count, and the result says so.  Returns a dict or None without the reference
    library."""
    from oracle import oracle as O

    n = len(mass)
    rng = np.random.default_rng(seed)
    R = O.ref() if O.ref_available() else None
    t_start = time.perf_counter()
    pieces = {}
    if w["kind"] == "ensemble":
        if R is None:
            return None
        systems = make_ensemble(w, 0)
        order = rng.permutation(len(systems))
        t_s, n_s, done = 0.0, 0, 0
        for i in order:
            p, _, mm = systems[i]
            q = p.astype(np.float32)
            cx, cy, cz = [np.ascontiguousarray(q[:, a]) for a in range(3)]
            mm = np.ascontiguousarray(mm, np.float32)
            k = len(mm)
            bx, by, bz = [np.zeros(k, np.float32) for _ in range(3)]
            t0 = time.perf_counter()
            R.ref_octree_cpu_accel(cx, cy, cz, mm, k, w["theta"], w["eps"], 1e-12, 1e30, 0, 0.0,
                                   0.0, None, 0, bx, by, bz)
            t_s += time.perf_counter() - t0
            n_s += k
            done += 1
            if time.perf_counter() - t_start > budget_s:
                break
        t_step = t_s * n / n_s
        pieces["clusters_s"] = t_s
        text = (f"reference octree_cpu (build + walk of every particle of a cluster) on {done} of "
                f"{len(systems)} clusters in seeded random order ({n_s} of {n} particles)")
        extrapolated = n_s < n
        cores, kind = int(R.ref_omp_threads()), "reference"
    else:
        p32 = pos.astype(np.float32)
        x, y, z = [np.ascontiguousarray(p32[:, a]) for a in range(3)]
        m = np.ascontiguousarray(mass, np.float32)
        targets = rng.permutation(n).astype(np.int32)
        treepm = w["kind"] == "treepm"
        iso = w["kind"] == "treepm_open"
        if iso:
            # grid of the reference's isolated mesh: the cell follows the bounds
            ext = max(float((p32[:, a].max() - p32[:, a].min())) for a in range(3))
            cell = max(0.25, max(ext, w["eps"]) / (w["grid"] - 2))
            rc = min(max(w["cutoff_factor"], 1.0), 2.0) * cell
            rs = rc / 4.5
            eps, theta = w["eps"], w["theta"]
        elif treepm:
            M = w["mesh"]
            rs = w["r_split_cells"] / M
            rc = w["r_cut_factor"] * rs
            eps = w["eps_lattice"] / w["n_side"]
            theta = w["theta"]
        else:
            rs = rc = 0.0
            eps, theta = w["eps"], w["theta"]
        if R is not None:
            if treepm:
                ax, ay, az = [np.zeros(n, np.float32) for _ in range(3)]
                t0 = time.perf_counter()
                R.ref_pm_periodic(x, y, z, m, n, M, 1.0, rs, 0, b"cic", ax, ay, az, None, None)
                pieces["pm_s"] = time.perf_counter() - t0
            elif iso:
                import ctypes as C
                fn = R.ref_treepm_isolated
                fn.argtypes = [np.ctypeslib.ndpointer(np.float32)] * 4 + [
                    C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                    np.ctypeslib.ndpointer(np.float64), C.c_void_p, C.c_void_p] + \
                    [np.ctypeslib.ndpointer(np.float32)] * 3
                ax, ay, az = [np.zeros(n, np.float32) for _ in range(3)]
                t0 = time.perf_counter()
                fn(x, y, z, m, n, w["grid"], w["eps"], w["cutoff_factor"],
                   {"cic": 0, "tsc": 1, "pcs": 2}[w["assignment"]], np.zeros(8), None, None, ax, ay, az)
                pieces["pm_s"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            tree = R.ref_octree_cpu_build(x, y, z, m, n, theta, eps, 1e-12, 1e30, 0, rs, rc * rc)
            pieces["build_s"] = time.perf_counter() - t0
            t_walk, walked = 0.0, 0
            try:
                while walked < n:
                    tg = np.ascontiguousarray(np.sort(targets[walked:walked + chunk]))
                    bx, by, bz = [np.zeros(len(tg), np.float32) for _ in range(3)]
                    t0 = time.perf_counter()
                    R.ref_octree_cpu_walk(tree, tg.ctypes.data, len(tg), bx, by, bz)
                    t_walk += time.perf_counter() - t0
                    walked += len(tg)
                    if time.perf_counter() - t_start > budget_s:
                        break
            finally:
                R.ref_octree_cpu_free(tree)
            pieces["walk_s"] = t_walk
            pieces["walk_targets"] = walked
            t_step = pieces.get("pm_s", 0.0) + pieces["build_s"] + t_walk * n / walked
            cores, kind = int(R.ref_omp_threads()), "reference"
            text = ("reference CPU code built from its sources: " +
                    (f"periodic PM templates (TpmAssignment/TpmField, FP32 CIC, mesh {M}^3) over all "
                     f"{n} particles, " if treepm else "") +
                    (f"its GPU TreePM's isolated-mesh kernels run on one host core (deposit, "
                     f"cuFFT replaced by its CPU fft3d, gradient, sampling; mesh {2 * w['grid']}^3) "
                     f"over all {n} particles, " if iso else "") +
                    f"octree_cpu build over all {n} (Octree::build) and its "
                    + ("cutoff/erfc-split " if treepm or iso else "") +
                    f"walk (Octree::computeForceOn) for {walked} seeded targets"
                    + (f", walk time scaled to all {n}" if walked < n else "")
                    + (" (open-boundary short range: the reference has no periodic split)"
                       if treepm else ""))
        else:
            p4 = O.pos4(p32, m)
            if treepm:
                t0 = time.perf_counter()
                O.pm_periodic(p4, M, 1.0, rs)
                pieces["pm_s"] = time.perf_counter() - t0
            t_walk, walked = 0.0, 0
            while walked < n:
                tg = np.sort(targets[walked:walked + 1024]).astype(np.int64)
                t0 = time.perf_counter()
                O.direct(p4, tg, eps=eps, box=1.0 if treepm else 0.0, rsplit=rs, rcut=rc)
                t_walk += time.perf_counter() - t0
                walked += len(tg)
                if time.perf_counter() - t_start > budget_s:
                    break
            pieces["direct_s"] = t_walk
            pieces["direct_targets"] = walked
            t_step = pieces.get("pm_s", 0.0) + t_walk * n / walked
            cores, kind = os.cpu_count() or 1, "port"
            text = (f"oracle port: " + ("FP64 PM over all particles + " if treepm else "") +
                    f"FP64 direct sum for {walked} seeded targets"
                    + (f", scaled to all {n}" if walked < n else ""))
        extrapolated = pieces.get("walk_targets", pieces.get("direct_targets", n)) < n
    return {"value": n / t_step, "unit": "particle-steps/s", "cores": cores, "kind": kind,
            "sample": text, "step_s": t_step, "measured_s": time.perf_counter() - t_start,
            "extrapolated": bool(extrapolated), "pieces": pieces}


def reference_gpu_step(w, pos, vel, mass, warmup=2, steps=5):
    """The reference's own GPU octree on the same particles: its CUDA kernels and octree_gpu
    symplectic-Euler step compiled for sm_100a from its sources (oracle/_ref/libbzrefgpu.so),
    at its defaults (leaf capacity 256, minimum distance² 1e-12, acceleration clamp 64), timed
    with CUDA events on the stream it launches on.  Octree workloads of at most 2^18 particles:
    the reference's 10-bit key spread puts every particle in one leaf, so its walk is a direct
    sum, O(N^2) a step.  None for other workloads or without the library."""
    if w["kind"] != "octree" or len(mass) > 1 << 18:
        return None
    import ctypes as C

    from oracle import oracle as O

    R = O.ref_gpu()
    if R is None:
        return None
    n = len(mass)
    soa = [np.ascontiguousarray(a[:, k], np.float32) for a in (pos, vel) for k in range(3)]
    m = np.ascontiguousarray(mass, np.float32)
    h = R.refgpu_create(n, 256, *soa, m)
    if not h:
        return None
    try:
        law = (w["theta"], w["eps"], 1e-12, 64.0, 0)
        acc = [np.zeros(n, np.float32) for _ in range(3)]
        nodes, leaves = C.c_int(), C.c_int()
        if R.refgpu_accel(h, *law, *acc, C.byref(nodes), C.byref(leaves)) != 0:
            return None
        ms = C.c_double()
        rc = R.refgpu_time_steps(h, warmup, steps, w["dt"], *law, C.byref(ms))
    finally:
        R.refgpu_destroy(h)
    if rc != 0:
        return None
    return {"value": n / (ms.value * 1e-3), "unit": "particle-steps/s", "ms_per_step": ms.value,
            "steps": steps, "warmup": warmup, "tree_nodes": nodes.value,
            "tree_leaves": leaves.value,
            "kind": "reference octree_gpu: its linear-octree build and updateParticlesOctree "
                    "kernels compiled for sm_100a from its sources",
            "note": "one leaf holds every particle (10-bit key spread), so the walk is an "
                    "O(N^2) direct sum; CUDA events on the legacy default stream"}


# --------------------------------------------------------------------------- arms

def run_reference(args, w, rank, world):
    """The reference's own CPU implementation of the path on this box's host cores: whole
    force evaluations (cpu_reference_step) repeated while they fit in a few minutes; rank 0
    only.  "steps" is the number actually timed; a step whose walk did not finish within the
    budget is extrapolated and marked so.  Octree workloads add "reference_gpu", the
    reference's own GPU octree timed on this GPU (reference_gpu_step)."""
    if rank != 0:
        return 0
    pos, vel, mass = make_ics(w, 0)
    n = len(mass)
    budget = float(os.environ.get("BZ_REFERENCE_BUDGET_S", "240"))
    results = []
    t0 = time.perf_counter()
    while len(results) < max(1, args.steps):
        res = cpu_reference_step(w, pos, mass, budget)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU library not built "
                              "(oracle/_ref/libbzref.so needs a BLITZAR checkout at build time)"}))
            return 0
        results.append(res)
        # another step only if it surely fits in the budget too
        if res["extrapolated"] or (time.perf_counter() - t0) + res["measured_s"] > budget:
            break
    step_s = float(np.median([r["step_s"] for r in results]))
    value = n / step_s
    last = results[-1]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": len(results), "steps_requested": args.steps, "warmup": 0,
        "ms_per_step": 1e3 * step_s, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "extrapolated": any(r["extrapolated"] for r in results),
        "measured_s": time.perf_counter() - t0,
        "config": config_dict(w, args, n),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": last["cores"],
                         "kind": last["kind"], "sample": last["sample"],
                         "extrapolated": last["extrapolated"], "pieces": last["pieces"]},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu_step(w, pos, vel, mass)
    if gpu is not None:
        line["reference_gpu"] = gpu
    print(json.dumps(line))
    return 0


METRIC = "particle-steps/s at <=1e-3 median force err: learned/mixed vs plain GPU TreePM"


def config_dict(w, args, n):
    c = {"workload": args.workload, "particles": n, "parallelism": f"replicas{args.gpus}",
         "l2": "inputs larger than L2 (state ~230 B/particle)"}
    c.update({k: v for k, v in w.items() if k != "kind"})
    return c


LEARNED_RS = 0.8  # split scale (mesh cells) at which the learned correction is compared
LEARNED_SAMPLES = 1 << 22  # training residuals


def learned_comparison(w, pos, vel, mass, stream, local, dt, nsample, experiment="split"):
    """Plain TreePM against the learned pair correction: force errors against FP64 Ewald and
    device time per step of each, plus the training cost.  The correction is trained here, on
    the GPU, on residuals the engine generates for this mesh.

    experiment "split": both at a smaller split scale (fewer short-range pairs, larger mesh
    error), the same cutoff.  experiment "cut": the workload's split scale, plain at
    r_cut = 4.5 r_s against the corrected walk at r_cut = 3.0 r_s."""
    import torch

    from blitzar_b200._lib import Engine

    if experiment == "cut":
        rs, rcf_plain, rcf_learned = w["r_split_cells"], 4.5, 3.0
    else:
        rs, rcf_plain, rcf_learned = LEARNED_RS, w["r_cut_factor"], w["r_cut_factor"]
    out = {"experiment": experiment, "r_split_cells": rs, "r_cut_factor": rcf_plain,
           "r_cut_factor_learned": rcf_learned}
    n = len(mass)

    def timed(eng, steps=5):
        eng.step(dt, 2)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.step(dt, steps)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    with Engine(n, stream=stream.cuda_stream, device=local,
                **engine_config(dict(w, r_split_cells=rs, r_cut_factor=rcf_plain))) as e:
        e.set_state(pos, vel, mass, f64=True)
        pe = e.force_errors(nsample=nsample, seed=11)
        ms_plain = timed(e)
    with Engine(n, stream=stream.cuda_stream, device=local,
                **engine_config(dict(w, r_split_cells=rs, r_cut_factor=rcf_learned))) as e:
        e.set_state(pos, vel, mass, f64=True)
        if rcf_learned != rcf_plain:  # the shorter cutoff before its correction
            ue = e.force_errors(nsample=nsample, seed=11)
            out["uncorrected"] = {"median": ue["median"], "p99": ue["p99"], "ms_per_step": timed(e)}
            e.set_state(pos, vel, mass, f64=True)
        t0 = time.perf_counter()
        x, y = e.learn_generate(LEARNED_SAMPLES, seed=7)
        t1 = time.perf_counter()
        loss = e.learn_train(x, y, steps=12000, batch=4096, lr=3e-3, seed=1)
        t2 = time.perf_counter()
        e.learn_enable(True)
        le = e.force_errors(nsample=nsample, seed=11)
        ms_learned = timed(e)
    out["plain"] = {"median": pe["median"], "p99": pe["p99"], "ms_per_step": ms_plain}
    out["learned"] = {"median": le["median"], "p99": le["p99"], "ms_per_step": ms_learned,
                      "value": n / (ms_learned * 1e-3), "samples": int(len(x)),
                      "generate_s": t1 - t0, "train_s": t2 - t1, "train_steps": 12000,
                      "final_loss": loss}
    out["meets_target"] = bool(le["median"] <= 1e-3 and le["p99"] <= 1e-2)
    return out


def run_ours(args, w, rank, world, local):
    import torch

    dist = init_dist(world, local)
    torch.cuda.set_device(local)
    from blitzar_b200._lib import Engine

    systems = None
    if w["kind"] == "ensemble":
        # one ensemble for the whole job: its clusters are split over the ranks by cost (LPT on
        # particle count), each rank steps its share as one ensemble handle, no collective
        from blitzar_b200 import sharding

        everything = make_ensemble(w, 0)
        share = sharding.lpt_partition([len(m) for _, _, m in everything], world)[rank]
        systems = [everything[i] for i in share]
        pos = np.concatenate([p for p, _, _ in systems])
        vel = np.concatenate([v for _, v, _ in systems])
        mass = np.concatenate([m for _, _, m in systems])
    else:
        pos, vel, mass = make_ics(w, rank)
    n = len(mass)
    stream = torch.cuda.Stream()
    cfg = engine_config(w)
    pinned = None
    if args.tune:
        leaf, group, schedule = (int(v) for v in args.tune.split(","))
        cfg.update(leaf_capacity=leaf, walk_group_size=group)
        pinned = dict(leaf_capacity=leaf, walk_group_size=group, mesh_schedule=schedule,
                      walk_blocks_per_sm=0, pinned=True)
    eng = Engine(n, stream=stream.cuda_stream, device=local, **cfg)
    if systems is not None:
        offsets = eng.set_ensemble(systems)
    else:
        eng.set_state(pos, vel, mass, f64=True)
    dt = w["dt"]
    tuned = None
    if pinned is not None:
        if cfg.get("solver") == 1:
            eng.set_mesh_schedule(pinned["mesh_schedule"])
        tuned = pinned
    elif not args.no_autotune and not w.get("adaptive_levels"):
        eng.autotune(trials=5)  # untimed: picks leaf capacity, group size, mesh schedule
        tuned = eng.last_tune
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            eng.step(dt, 1)
    torch.cuda.synchronize()
    energy0 = eng.energy() if w["kind"] in ("octree", "ensemble") else None

    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    adaptive = bool(w.get("adaptive_levels"))
    upd0 = eng.adaptive_updates() if adaptive else 0
    start.record(stream)
    eng.step(dt, args.steps)
    end.record(stream)
    torch.cuda.synchronize()
    updates = (eng.adaptive_updates() - upd0) if adaptive else n * args.steps
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = start.elapsed_time(end)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # particle-steps: with adaptive block steps, every closed step of every particle (one force
    # evaluation and one kick each); otherwise N per step
    if w["kind"] == "ensemble" and dist:
        t = torch.tensor([float(updates)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        value = float(t.item()) / (ms / 1e3)   # the ranks share one ensemble
    else:
        value = updates * world / (ms / 1e3)
    drift = None
    if energy0 is not None:
        k1, w1, p1 = eng.energy()
        e0 = energy0[0] + energy0[1]
        drift = {"relative_energy_drift": (k1 + w1 - e0) / abs(e0), "steps": args.steps,
                 "momentum_change": float(np.abs(p1 - energy0[2]).max()),
                 "note": "total energy (FP64 kinetic + tree potential) before and after the timed steps"}

    launches_step = eng.launches_per_step()
    # phase-timed eager pass for the per-kernel roofline
    eng.enable_timing(True)
    eng.step(dt, 3)
    ph = eng.phase_times()
    listed, evaluated, nodes = eng.walk_counts()
    eng.enable_timing(False)
    split = w["kind"] in ("treepm", "treepm_open")
    # algorithmic flops: pairs that went through the pair law (inside the cutoff) and
    # multipole terms; the distance tests of listed pairs outside the cutoff are not counted
    flops = evaluated * FLOP_PP[split] + nodes * FLOP_PN[(split, True)]
    walk_ms = ph["walk"]
    achieved_tf = flops / (walk_ms * 1e-3) / 1e12 if walk_ms > 0 else 0.0
    peak_tf = SMS * FP32_LANES_PER_SM * 2 * NOMINAL_SM_MHZ * 1e6 / 1e12
    # DRAM traffic and issue utilisation come from an ncu capture committed under profiles/;
    # they are quoted only when that capture used this run's walk settings
    leaf_now = tuned["leaf_capacity"] if tuned else cfg.get("leaf_capacity", 16)
    group_now = tuned["walk_group_size"] if tuned else 32
    prof = None
    for cap in (load_traffic(f"walk_{args.workload}") or {}).get("captures", []):
        if cap.get("leaf_capacity") == leaf_now and cap.get("walk_group_size") == group_now:
            prof = cap
    prof_ok = prof is not None
    roofline = {
        "kernel": "k_walk (group tree walk + pair/multipole arithmetic)",
        "bound": "fp32", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
        "frac": achieved_tf / peak_tf,
        "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 x 1965 MHz); no measured FP32 peak is provided",
        "traffic": prof.get("dram_bytes_per_launch") if prof_ok else None,
        "ncu_issue_active_pct": prof.get("issue_active_pct") if prof_ok else None,
        "traffic_source": (f"profiles/walk_{args.workload}.json: ncu capture of one launch at leaf "
                           f"{prof.get('leaf_capacity')}, group {prof.get('walk_group_size')}"
                           if prof_ok else
                           "none: no committed ncu capture of this workload at this run's leaf "
                           "capacity and group size"),
        "interactions_per_launch": {"listed_pairs": listed, "evaluated_pairs": evaluated,
                                    "particle_node": nodes},
        "listed_per_evaluated": (listed / evaluated) if evaluated else None,
        "flops_per_interaction": {"pp": FLOP_PP[split], "pn": FLOP_PN[(split, True)]},
        "launch_ms": walk_ms,
    }
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    # The step's re-sort sees the previous sorted order: the nearly-sorted path reads the keys
    # for the out-of-order flags (8 B + 1 B flag written), splits (1 + 12 B read, 12 B written),
    # checks the in-order part (8 B) and merges (12 B read, 12 B written) = 66 B per particle;
    # a full radix sort would be 8 B + 8 passes x 24 B = 200 B per particle.
    sort_bytes = n * (9 + 25 + 8 + 24)
    keys_bytes = n * (24 + 12)
    permute_bytes = n * (2 * (48 + 4 + 4) + 16)
    secondary = {
        "sort": {"bound": "hbm", "achieved": sort_bytes / (ph["sort"] * 1e-3) / 1e9, "peak": hbm_peak,
                 "unit": "GB/s", "ms": ph["sort"], "bytes_per_particle": 66,
                 "note": "nearly sorted re-sort of a step (a full radix sort moves 200 B/particle)"},
        "keys": {"bound": "hbm", "achieved": keys_bytes / (ph["keys"] * 1e-3) / 1e9, "peak": hbm_peak,
                 "unit": "GB/s", "ms": ph["keys"]},
        "permute": {"bound": "hbm", "achieved": permute_bytes / (ph["permute"] * 1e-3) / 1e9,
                    "peak": hbm_peak, "unit": "GB/s", "ms": ph["permute"]},
    }
    for k in secondary.values():
        k["frac"] = k["achieved"] / k["peak"]

    errs = eng.force_errors(nsample=args.error_sample, seed=11)

    # end to end through the C ABI with pinned host buffers: upload state, one step, download
    e2e = None
    if args.e2e_steps > 0 and systems is not None:
        # ensembles: FP64 SoA state and the system offsets through bz_set_ensemble
        import ctypes as C

        hp = torch.empty(3 * n, dtype=torch.float64, pin_memory=True).numpy()
        hv = torch.empty(3 * n, dtype=torch.float64, pin_memory=True).numpy()
        hm = torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
        hm[:] = mass
        offs = np.ascontiguousarray(offsets, np.int64)

        def up():
            eng._check(eng.L.bz_set_ensemble(eng.h, hp.ctypes.data, hv.ctypes.data, hm.ctypes.data,
                                              offs.ctypes.data, len(systems)), "bz_set_ensemble")

        def down():
            eng._check(eng.L.bz_get_state_f64(eng.h, hp.ctypes.data, hv.ctypes.data), "bz_get_state_f64")

        down()
        up()
        eng.step(dt, 1)
        down()
        torch.cuda.synchronize()
        steps_done = 0
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            up()
            eng.step(dt, 1)
            steps_done += eng.adaptive_updates() if adaptive else n  # counter restarts per upload
            down()
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        e2e = {"value": steps_done * world / sec, "unit": "particle-steps/s",
               "h2d_bytes_per_step": 6 * 8 * n + 4 * n + 8 * len(offs), "d2h_bytes_per_step": 6 * 8 * n,
               "note": "each step uploads the full FP64 ensemble state, which forces a fresh force "
                       "evaluation before the leapfrog step (two evaluations per step)"}
    elif args.e2e_steps > 0:
        # the host keeps the FP64 leapfrog state (positions, velocities, masses and the FP32
        # accelerations of the positions) in pinned memory and round-trips it through the C ABI
        # every step
        hp = torch.empty(3 * n, dtype=torch.float64, pin_memory=True).numpy()
        hv = torch.empty(3 * n, dtype=torch.float64, pin_memory=True).numpy()
        ha = torch.empty(3 * n, dtype=torch.float32, pin_memory=True).numpy()
        hm = torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
        hm[:] = mass
        eng.get_state_acc_f64_soa(hp, hv, ha)
        eng.set_state_acc_f64_soa(hp, hv, hm, ha)
        eng.step_get_state_acc_f64_soa(dt, hp, hv, ha)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            eng.set_state_acc_f64_soa(hp, hv, hm, ha)
            eng.step_get_state_acc_f64_soa(dt, hp, hv, ha)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        if dist:
            t = torch.tensor([sec], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec = float(t.item())
        e2e = {"value": n * world * args.e2e_steps / sec, "unit": "particle-steps/s",
               "h2d_bytes_per_step": (6 * 8 + 4 + 3 * 4) * n, "d2h_bytes_per_step": (6 * 8 + 3 * 4) * n,
               "note": "each step uploads the FP64 leapfrog state with the FP32 accelerations of "
                       "its positions (bz_set_state_acc_f64), steps once (one force evaluation, "
                       "as for a resident state) and downloads state and accelerations, the "
                       "positions while the step runs (bz_step_get_state_acc_f64); wall clock "
                       "over the steps"}

    learned = None
    if w["kind"] == "treepm" and not args.no_learned:
        learned = learned_comparison(w, pos, vel, mass, stream, local, dt, args.error_sample,
                                     args.learned_experiment)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_step(w, pos, mass, args.cpu_budget)

    line = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong" if w["kind"] == "ensemble" else "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": ("synthetic (seeded GRF-displaced grid)" if w["kind"] == "treepm"
                 else "synthetic (seeded King clusters)" if w["kind"] == "ensemble"
                 else f"synthetic (seeded {w['ic'].capitalize()} sphere)"),
        "config": config_dict(w, args, n),
        "force_error": {"median": errs["median"], "p99": errs["p99"], "sample": args.error_sample,
                        "reference": "FP64 Ewald" if w["kind"] == "treepm" else
                        "FP64 direct sum within each system" if w["kind"] == "ensemble" else "FP64 direct sum"},
        "roofline": roofline, "roofline_secondary": secondary,
        "phase_ms": ph, "gpu_launches": launches_step * args.steps, "launches_per_step": launches_step,
        "clocks": clk, "e2e": e2e, "cpu_baseline": cpu,
    }
    if drift is not None:
        line["energy"] = drift
    if learned is not None:
        line["learned"] = learned
    if tuned is not None:
        line["autotune"] = tuned
    if adaptive:
        line["adaptive"] = {"max_level": w["adaptive_levels"], "eta": w["adaptive_eta"],
                            "block_steps": args.steps, "particle_steps": int(updates),
                            "mean_steps_per_particle_per_block": updates / (n * args.steps),
                            "note": "ms_per_step is per block step of dt_max; phase_ms covers "
                                    "one substep"}
    eng.close()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    rank, world, local = dist_env()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, w, rank, world)
    return run_ours(args, w, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
