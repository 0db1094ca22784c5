"""Snapshot formats of the reference, byte-compatible.

* ``.bin`` (NBSIMBIN v1): 8-byte magic "NBSIMBIN", u32 version = 1, u32 count, then per
  particle 8 float32 {px, py, pz, vx, vy, vz, mass, temperature}
  (engine/server/simulation/persistence/SrvPersistenceInternal.hpp:21-39, writer
  engine/server/simulation/persistence/SrvIO.cpp:139-165).
* ``.xyz``: line 1 the count, line 2 ``solver=<s> integrator=<i> step=<k>``, then
  ``P x y z mass temperature`` per particle with C++ ostream default formatting (6
  significant digits) (SrvIO.cpp:173-181).  It carries no velocities.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"NBSIMBIN"
VERSION = 1


def write_bin(path, pos, vel, mass, temperature=None):
    n = len(mass)
    rec = np.zeros((n, 8), np.float32)
    rec[:, 0:3] = pos
    rec[:, 3:6] = vel
    rec[:, 6] = mass
    rec[:, 7] = 0.0 if temperature is None else temperature
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<II", VERSION, n))
        f.write(rec.astype("<f4").tobytes())


def read_bin(path):
    with open(path, "rb") as f:
        head = f.read(16)
        if head[:8] != MAGIC:
            raise ValueError("not an NBSIMBIN file")
        version, n = struct.unpack("<II", head[8:16])
        if version != VERSION:
            raise ValueError(f"unsupported NBSIMBIN version {version}")
        rec = np.frombuffer(f.read(32 * n), "<f4").reshape(n, 8)
    return rec[:, 0:3].copy(), rec[:, 3:6].copy(), rec[:, 6].copy(), rec[:, 7].copy()


def _g6(v: float) -> str:
    """C++ ostream default float formatting: %g with 6 significant digits."""
    return "%g" % v


def write_xyz(path, pos, mass, temperature=None, solver="octree_gpu", integrator="leapfrog",
              step=0):
    n = len(mass)
    t = np.zeros(n, np.float32) if temperature is None else temperature
    p = np.asarray(pos, np.float32)
    m = np.asarray(mass, np.float32)
    lines = [str(n), f"solver={solver} integrator={integrator} step={step}"]
    for i in range(n):
        lines.append("P %s %s %s %s %s" % (_g6(p[i, 0]), _g6(p[i, 1]), _g6(p[i, 2]), _g6(m[i]), _g6(t[i])))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_xyz(path):
    with open(path) as f:
        n = int(f.readline())
        f.readline()
        data = np.array([list(map(float, f.readline().split()[1:6])) for _ in range(n)], np.float32)
    return data[:, 0:3], data[:, 3], data[:, 4]
