"""Seeded initial conditions for the benchmark workloads (FP64, numpy).

None of these exist in the reference (its Plummer generator draws Gaussian velocities,
engine/server/simulation/state/SrvPlummer.cpp:17-106); they are written from the published
models:

* ``grf_grid``   -- particles on a regular grid displaced by a Gaussian random field
                    (Zel'dovich: psi_k = i k delta_k / k^2 with P_delta(k) ~ k^n), periodic box;
* ``plummer``    -- Plummer sphere: radii by inverse CDF, speeds from the isotropic
                    distribution function f(E) ~ (-E)^{7/2} by rejection (Aarseth, Henon &
                    Wielen 1974);
* ``hernquist``  -- Hernquist (1990) profile truncated at r_max, radii by inverse CDF, speeds
                    by rejection from the isotropic DF;
* ``king``       -- King (1966) model of concentration W0: Poisson-equation integration of the
                    lowered-isothermal DF, radii and speeds by rejection.

All generators take an explicit seed (numpy default_rng) and return float64 arrays.
"""
from __future__ import annotations

import math

import numpy as np


def grf_grid(n_side: int, seed: int, rms_cells: float = 0.2, spectral_index: float = -2.0,
             box: float = 1.0):
    """Grid of n_side^3 particles displaced by a Zel'dovich field of a Gaussian random
    density field with P(k) ~ k^spectral_index; displacement rms (3-D) = rms_cells cells.
    Returns (pos, vel, mass): vel = 0, total mass 1, positions wrapped into [0, box)."""
    rng = np.random.default_rng(seed)
    n = n_side
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz = np.fft.rfftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k2[0, 0, 0] = 1.0
    amp = np.sqrt(k2 ** (spectral_index / 2.0))
    amp[0, 0, 0] = 0.0
    white = rng.standard_normal((n, n, n))
    delta_k = np.fft.rfftn(white) * amp
    disp = np.empty((3, n, n, n))
    for a, K in enumerate((KX, KY, KZ)):
        disp[a] = np.fft.irfftn(1j * K / k2 * delta_k, s=(n, n, n), axes=(0, 1, 2))
    rms = math.sqrt(float((disp ** 2).sum(0).mean()))
    cell = box / n
    disp *= rms_cells * cell / rms
    g = (np.arange(n) + 0.5) * cell
    GX, GY, GZ = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([GX + disp[0], GY + disp[1], GZ + disp[2]], -1).reshape(-1, 3)
    pos %= box
    pos[pos >= box] = 0.0
    npart = n ** 3
    return pos, np.zeros_like(pos), np.full(npart, 1.0 / npart)


def _isotropic(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def plummer(n: int, seed: int, a: float = 1.0, mass: float = 1.0, G: float = 1.0,
            r_cut: float | None = None):
    """Plummer sphere with the isotropic DF.  Returns (pos, vel, mass)."""
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    filled = 0
    while filled < n:
        u = rng.random(n - filled)
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        if r_cut is not None:
            rr = rr[rr <= r_cut]
        r[filled:filled + len(rr)] = rr
        filled += len(rr)
    pos = r[:, None] * _isotropic(rng, n)
    # speed q = v / v_esc with g(q) ~ q^2 (1 - q^2)^{7/2}, max 0.1 at q^2 = 2/9
    q = np.empty(n)
    todo = np.arange(n)
    while len(todo):
        x = rng.random(len(todo))
        y = rng.random(len(todo)) * 0.1
        ok = y < x * x * (1.0 - x * x) ** 3.5
        q[todo[ok]] = x[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0 * G * mass / np.sqrt(r * r + a * a))
    vel = (q * vesc)[:, None] * _isotropic(rng, n)
    return pos, vel, np.full(n, mass / n)


def hernquist(n: int, seed: int, a: float = 1.0, mass: float = 1.0, r_max: float = 100.0,
              G: float = 1.0):
    """Hernquist sphere truncated at r_max * a with speeds from the isotropic DF."""
    rng = np.random.default_rng(seed)
    # M(<r) = M r^2 / (r + a)^2, normalised to the truncation radius
    fmax = r_max ** 2 / (1.0 + r_max) ** 2
    u = rng.random(n) * fmax
    s = np.sqrt(u)
    r = a * s / (1.0 - s)
    pos = r[:, None] * _isotropic(rng, n)
    # isotropic DF f(E) (Hernquist 1990, eq. 17) in units G = M = a = 1
    def f_of(eps):
        q = np.sqrt(eps)
        return (1.0 / (1.0 - eps) ** 2.5) * (3.0 * np.arcsin(q) + q * np.sqrt(1.0 - eps) * (1.0 - 2.0 * eps)
                                             * (8.0 * eps * eps - 8.0 * eps - 3.0))
    psi = G * mass / (r + a)  # relative potential (untruncated model)
    vesc = np.sqrt(2.0 * psi)
    vel_mag = np.empty(n)
    todo = np.arange(n)
    while len(todo):
        ps = psi[todo]
        # p(v) ~ v^2 f(psi - v^2/2); bound by the maximum on a coarse grid per particle
        grid = np.linspace(0.0, 1.0, 64)[None, :] * vesc[todo, None]
        e = np.clip(ps[:, None] - 0.5 * grid ** 2, 1e-12, 1.0 - 1e-12)
        pmax = (grid ** 2 * f_of(e)).max(1) * 1.1 + 1e-30
        v = rng.random(len(todo)) * vesc[todo]
        e1 = np.clip(ps - 0.5 * v ** 2, 1e-12, 1.0 - 1e-12)
        ok = rng.random(len(todo)) * pmax < v ** 2 * f_of(e1)
        vel_mag[todo[ok]] = v[ok]
        todo = todo[~ok]
    vel = vel_mag[:, None] * _isotropic(rng, n)
    return pos, vel, np.full(n, mass / n)


def _king_profile(W0: float, npts: int = 4000):
    """Dimensionless King model: integrate Poisson's equation for W(r) with rho(W)."""
    from math import erf, exp, pi, sqrt

    def rho(W):
        if W <= 0.0:
            return 0.0
        return exp(W) * erf(sqrt(W)) - sqrt(4.0 * W / pi) * (1.0 + 2.0 * W / 3.0)

    rho0 = rho(W0)
    # d2W/dr2 + 2/r dW/dr = -9 rho(W)/rho0 (r in core radii)
    dr = 1e-3
    r, W, dW = dr, W0 - 1.5 * dr * dr, -3.0 * dr
    rs, Ws, Ms = [0.0], [W0], [0.0]
    M = 0.0
    while W > 0.0 and len(rs) < 2_000_000:
        def acc(rr, w, dw):
            return -9.0 * rho(w) / rho0 - 2.0 / rr * dw
        k1w, k1d = dW, acc(r, W, dW)
        k2w, k2d = dW + 0.5 * dr * k1d, acc(r + 0.5 * dr, W + 0.5 * dr * k1w, dW + 0.5 * dr * k1d)
        k3w, k3d = dW + 0.5 * dr * k2d, acc(r + 0.5 * dr, W + 0.5 * dr * k2w, dW + 0.5 * dr * k2d)
        k4w, k4d = dW + dr * k3d, acc(r + dr, W + dr * k3w, dW + dr * k3d)
        W += dr / 6.0 * (k1w + 2 * k2w + 2 * k3w + k4w)
        dW += dr / 6.0 * (k1d + 2 * k2d + 2 * k3d + k4d)
        M += 4.0 * math.pi * r * r * max(rho(W), 0.0) / rho0 * dr
        r += dr
        rs.append(r)
        Ws.append(max(W, 0.0))
        Ms.append(M)
        if r > 5.0:
            dr = 1e-2
    return np.array(rs), np.array(Ws), np.array(Ms)


def king(n: int, seed: int, W0: float, mass: float = 1.0, r_scale: float = 1.0, G: float = 1.0):
    """King (1966) model with central potential W0: radii from the cumulative mass profile,
    speeds by rejection from f ~ e^{W - v^2/2} - 1; returned with total mass `mass` and the
    core radius scaled to `r_scale`."""
    rng = np.random.default_rng(seed)
    rs, Ws, Ms = _king_profile(W0)
    u = rng.random(n) * Ms[-1]
    r = np.interp(u, Ms, rs)
    pos = r[:, None] * _isotropic(rng, n)
    W = np.interp(r, rs, Ws)
    vmax = np.sqrt(2.0 * np.maximum(W, 1e-12))
    v = np.empty(n)
    todo = np.arange(n)
    while len(todo):
        vv = rng.random(len(todo)) * vmax[todo]
        g = vv * vv * (np.exp(W[todo] - 0.5 * vv * vv) - 1.0)
        gmax = np.max(np.stack([(x * x * (np.exp(W[todo] - 0.5 * x * x) - 1.0))
                                for x in np.linspace(0, 1, 32)[:, None] * vmax[todo]]), 0) * 1.1 + 1e-30
        ok = rng.random(len(todo)) * gmax < g
        v[todo[ok]] = vv[ok]
        todo = todo[~ok]
    vel = v[:, None] * _isotropic(rng, n)
    # Model units: G = 1, velocity dispersion parameter 1, core radius 1, so G rho0 = 9/(4 pi)
    # and the model mass is rho0 * Ms.  Scaling mass by mu and length by L scales velocities
    # by sqrt(mu / L).
    m_model = 9.0 / (4.0 * math.pi) * Ms[-1]
    vscale = math.sqrt((G * mass / m_model) / r_scale)
    return pos * r_scale, vel * vscale, np.full(n, mass / n)
