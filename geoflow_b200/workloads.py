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
