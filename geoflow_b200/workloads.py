"""Seeded synthetic inputs of the benchmark configurations.

One definition shared by bench.py, the tests and the fixture scripts, so a
workload means the same field everywhere:

* 2-d periodic advection (16^2 elements, p = 4): the Gaussian lump
  exp(-((x-.5)^2 + (y-.5)^2)/0.01) plus U(-1e-3, 1e-3) noise drawn per
  unique node (so the field stays continuous), seed 20261203 + 1.
* 3-d Helmholtz right-hand side: f = sum_m a_m sin(pi k_mx x) sin(pi k_my y)
  sin(pi k_mz z), k ~ U{1..8}, a ~ N(0, 1), 8 modes, seed 20261203 + 2.
* 3-d Burgers velocity on [0, 2pi)^3: 4 random Fourier modes per integer
  shell 1 <= |k| <= 6, amplitude |k|^(-5/3), random phase and direction,
  zero mean, seed 20261203 + 3; dt = 0.3 h_min / (p^2 max|u|).
"""
from __future__ import annotations

import numpy as np

SEED = 20261203


def advection2d_initial(xyz, node_class, nclass, seed=SEED + 1):
    """Gaussian lump plus per-unique-node noise (numpy FP64)."""
    rng = np.random.default_rng(seed)
    x, y = xyz[0], xyz[1]
    u = np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / 0.01)
    return u + rng.uniform(-1e-3, 1e-3, nclass)[node_class]


def helmholtz_rhs_modes(seed=SEED + 2, nmodes=8):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 9, size=(nmodes, 3))
    a = rng.standard_normal(nmodes)
    return k, a


def burgers_modes(seed=SEED + 3):
    """[(k vector, amplitude, phase, direction)] of the 3-d Burgers
    velocity: 4 modes on each integer shell |k| = 1..6."""
    rng = np.random.default_rng(seed)
    modes = []
    for kk in range(1, 7):
        for _ in range(4):
            kv = rng.standard_normal(3)
            kv = np.round(kv / np.linalg.norm(kv) * kk).astype(int)
            if not kv.any():
                kv[0] = kk
            amp = float(np.linalg.norm(kv)) ** (-5.0 / 3.0)
            ph = float(rng.uniform(0, 2 * np.pi))
            d = rng.standard_normal(3)
            modes.append((kv, amp, ph, d))
    return modes


def burgers_velocity(xyz, modes, xp=np):
    """u_c = sum_modes amp d_c sin(k.x + phase), for numpy or torch arrays
    (xp the array module)."""
    x, y, z = xyz
    u = [xp.zeros_like(x) for _ in range(3)]
    for kv, amp, ph, d in modes:
        s = xp.sin(kv[0] * x + kv[1] * y + kv[2] * z + ph)
        for c in range(3):
            u[c] += amp * d[c] * s
    return u


def burgers_dt(umax, ne, p, xi, length=2 * np.pi, cfl=0.3):
    """dt = cfl * h_min / (p^2 max|u|), h_min the smallest GLL spacing
    (the formula of GBurgers::dt_impl with its pmax set)."""
    h = length / ne
    hmin = h * 0.5 * (xi[1] - xi[0])
    return cfl * hmin / (p * p * umax)


# ---- the icosahedral-sphere advection members of the ensemble ----
def icos_solid_body_wind(xyz, u0=1.0, alpha=0.0):
    """Cartesian components of the solid-body rotation wind of the
    reference's icosahedral advection tests: physical spherical components
    u_theta = -u0 sin(lon) sin(alpha), u_lambda = u0 (cos(lat) cos(alpha) +
    sin(lat) cos(lon) sin(alpha)), converted as GMTK::vsphere2cart
    (blas/gmtk.ipp:2998-3040, physical components)."""
    x, y, z = xyz
    r = np.sqrt(x * x + y * y + z * z)
    lat = np.arcsin(z / r)
    lon = np.arctan2(y, x)
    vth = -u0 * np.sin(lon) * np.sin(alpha)
    vph = u0 * (np.cos(lat) * np.cos(alpha) + np.sin(lat) * np.cos(lon) * np.sin(alpha))
    cx = -vth * np.sin(lat) * np.cos(lon) - vph * np.sin(lon)
    cy = -vth * np.sin(lat) * np.sin(lon) + vph * np.cos(lon)
    cz = vth * np.cos(lat)
    return [cx, cy, cz]


def icos_cosine_bell(xyz, lat0, lon0, u0=1.0):
    """The cosine bell of compute_icosbell (test/sandbox/cdg/src/
    gtest_burgers.cpp:943-1033) at t = 0: u = u0 (1 + cos(pi s / R)) / 2 for
    great-circle distance s < R = r/3 from (lat0, lon0) (radians), else 0.
    (The reference's amplitude factor (sig0/sig)^GDIM is 0/0 at t = 0 with
    its sig0 = 0; it is left out.)"""
    x, y, z = xyz
    r = np.sqrt(x * x + y * y + z * z)
    lat = np.arcsin(z / r)
    lon = np.arctan2(y, x)
    R = r / 3.0
    cosd = np.sin(lat0) * np.sin(lat) + np.cos(lat0) * np.cos(lat) * np.cos(lon - lon0)
    s = r * np.arccos(np.clip(cosd, -1.0, 1.0))
    return np.where(s < R, 0.5 * u0 * (1.0 + np.cos(np.pi * s / R)), 0.0)


def icos_members(seed=SEED + 5, n=16):
    """The 16 icosahedral members: (level 3..5, p 4..8, bell centre) drawn
    by seed."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        level = int(rng.integers(3, 6))
        p = int(rng.integers(4, 9))
        lat0 = float(rng.uniform(-np.pi / 3, np.pi / 3))
        lon0 = float(rng.uniform(0.0, 2 * np.pi))
        out.append((level, p, lat0, lon0))
    return out


def box_members(seed=SEED + 6, n=16):
    """The 16 2-d box Helmholtz members: (elements per direction 8..64,
    p 3..8) drawn by seed; the right-hand side is helmholtz2d_rhs."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice([8, 16, 24, 32, 48, 64])), int(rng.integers(3, 9)))
            for _ in range(n)]


def helmholtz2d_rhs(xyz, seed, nmodes=4):
    """f = sum_m a_m sin(pi kx_m x) sin(pi ky_m y), k ~ U{1..8}, a ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 9, size=(nmodes, 2))
    a = rng.standard_normal(nmodes)
    x, y = xyz[0], xyz[1]
    f = np.zeros_like(x)
    for m in range(nmodes):
        f += a[m] * np.sin(np.pi * k[m, 0] * x) * np.sin(np.pi * k[m, 1] * y)
    return f
