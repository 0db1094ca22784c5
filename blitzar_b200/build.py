"""Build libbzgrav.so (the engine's C-ABI library) in-tree for sm_100a.

Every translation unit is compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``;
the octree moments file is compiled without FMA contraction so that its FP64 sums round
exactly as written.  Output: ``blitzar_b200/libbzgrav.so`` (git-ignored; it travels with the
working tree).  Usage: ``python -m blitzar_b200.build [--force]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libbzgrav.so")
HEADLESS = os.path.join(HERE, "bz_headless")  # C++ headless driver (links libbzgrav.so)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
SOURCES = {
    "bz_keys.cu": [],
    "bz_sort.cu": [],
    "bz_tree.cu": ["--fmad=false"],
    "bz_groups.cu": [],
    "bz_mlp.cu": [],
    "bz_adaptive.cu": [],
    "bz_walk.cu": [],
    "bz_pm.cu": [],
    "bz_state.cu": [],
    "bz_diag.cu": [],
    "bz_api.cu": [],
    "bz_noalloc.cu": [],
}
HEADERS = ["bz_common.cuh", "bz_kernels.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbzgrav")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "bzgrav.h")]
    objs, jobs = [], []
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            jobs.append([cc] + ARCH + COMMON + extra + ["-c", path, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            sys.stdout.write(r.stdout + r.stderr)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    host_src = os.path.join(HERE, "host", "bz_headless.cpp")
    host_hdr = os.path.join(HERE, "host", "bz_particle_system.hpp")
    if force or _stale(HEADLESS, [host_src, host_hdr, LIB, os.path.join(ROOT, "include", "bzgrav.h")]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
               "-I", os.path.join(HERE, "host"), host_src, "-L", HERE, "-lbzgrav",
               "-Wl,-rpath,$ORIGIN", "-o", HEADLESS]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("headless driver build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
