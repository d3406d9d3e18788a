"""Moment-tensor helpers for the ElasticWAVE sources.

The reference injects a moment tensor as sigma_ab += w(t) * (-M_ab) at the
source cell (Elastic3D_SSG_Tensor.py:186-193) and takes M as a (3, 3) field;
these helpers build such M arrays.  Axes follow the grid: x (first index),
y (second), z (last index, positive downwards).
"""
from __future__ import annotations

import math

import numpy as np


def double_couple(strike: float, dip: float, rake: float, m0: float = 1.0) -> np.ndarray:
    """Double-couple moment tensor (Aki & Richards, Quantitative Seismology,
    eq. 4.88) for strike/dip/rake in degrees, x = north, y = east, z = down."""
    phi, delta, lam = (math.radians(v) for v in (strike, dip, rake))
    sd, cd = math.sin(delta), math.cos(delta)
    s2d, c2d = math.sin(2 * delta), math.cos(2 * delta)
    sl, cl = math.sin(lam), math.cos(lam)
    sp, cp = math.sin(phi), math.cos(phi)
    s2p, c2p = math.sin(2 * phi), math.cos(2 * phi)
    mxx = -(sd * cl * s2p + s2d * sl * sp * sp)
    mxy = sd * cl * c2p + 0.5 * s2d * sl * s2p
    mxz = -(cd * cl * cp + c2d * sl * sp)
    myy = sd * cl * s2p - s2d * sl * cp * cp
    myz = -(cd * cl * sp - c2d * sl * cp)
    mzz = s2d * sl
    M = np.array([[mxx, mxy, mxz], [mxy, myy, myz], [mxz, myz, mzz]], dtype=np.float64) * m0
    return M.astype(np.float32)


def explosive(m0: float = 1.0) -> np.ndarray:
    """Isotropic source M = m0 * I."""
    return (np.eye(3) * m0).astype(np.float32)


def random_tensor(seed: int = 0, m0: float = 1.0) -> np.ndarray:
    """General symmetric moment tensor with six N(0,1) components."""
    g = np.random.default_rng(seed).standard_normal(6)
    M = np.array([[g[0], g[3], g[4]], [g[3], g[1], g[5]], [g[4], g[5], g[2]]]) * m0
    return M.astype(np.float32)
