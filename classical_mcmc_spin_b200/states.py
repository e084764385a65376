"""Seeded initial spin states.

The reference seeds its generator from the wall clock (lattice.h:649), so its
random states cannot be reproduced; every state here comes from an explicit
seed and is written/read in the reference's initial_spin_config text format
(Lattice.save_spin_config / load_spin_config).
"""
from __future__ import annotations

import numpy as np


def random_unit_spins(n: int, seed: int) -> np.ndarray:
    """i.i.d. uniform on S^2, Marsaglia (1972) rejection as in lattice.h:1115-1124."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, 3))
    filled = 0
    while filled < n:
        m = max(16, int((n - filled) * 1.35) + 8)
        u = 2.0 * rng.random((m, 2)) - 1.0
        s = (u * u).sum(axis=1)
        u = u[s < 1.0]
        s = s[s < 1.0]
        k = min(len(s), n - filled)
        f = 2.0 * np.sqrt(1.0 - s[:k])
        out[filled:filled + k, 0] = f * u[:k, 0]
        out[filled:filled + k, 1] = f * u[:k, 1]
        out[filled:filled + k, 2] = 1.0 - 2.0 * s[:k]
        filled += k
    return out


ZIGZAG_AXIS = np.array([1.0, 1.0, 1.0]) / np.sqrt(3.0)


def zigzag_honeycomb(d1: int, d2: int, d3: int = 1, axis=ZIGZAG_AXIS, tilt_sigma: float = 0.0,
                     seed: int = 0) -> np.ndarray:
    """Zigzag order on the 2-atom honeycomb: ferromagnetic chains along the
    x-bond direction (a2), antiparallel between neighbouring chains along a1:
    site (i, j, k, atom) gets (-1)^i * axis.  With tilt_sigma > 0 each spin is
    tilted by i.i.d. Gaussian components of that width and renormalised.
    (The reference has no zigzag initialiser; this one is defined here.)"""
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    i = np.arange(d1).repeat(d2 * d3 * 2)
    sign = np.where(i % 2 == 0, 1.0, -1.0)
    s = sign[:, None] * axis[None, :]
    if tilt_sigma > 0:
        rng = np.random.default_rng(seed)
        s = s + tilt_sigma * rng.standard_normal(s.shape)
        s /= np.linalg.norm(s, axis=1, keepdims=True)
    return s
