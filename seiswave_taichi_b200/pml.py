"""Finite-difference coefficients and ADE-CPML / split-PML profiles.

Host-side restatement of the reference's set-up routines:

* ``diff_coff``     -- Elastic2D_CPML.py:355-366 (identical copies in the 3D
  classes): solve A c = e1 with A[i, j] = (2j+1)^(2i+1) in float64 and store
  the coefficients as float32.
* ``diff_coff_op``  -- Elastic2D_CPML.py:368-390, the hard-coded optimised sets.
* ``axis_profile``  -- one axis of SetADEPML2D (Elastic2D_CPML.py:392-528) and
  SetADEPML3D (Elastic3D_SSG_Tensor.py:361-568): d, alpha, kappa at integer
  and half points evaluated in double precision, stored in the field type,
  alpha clamped at 0 after storing, then b and a recomputed in double
  precision from the stored values (a only where |d| > 1e-6).

Two derived tables feed the kernels:

* ``axis_flags``  -- per index, whether the integer (bit 0) and half (bit 1)
  point satisfies the reference's PML predicate ``x <= xmin_pml or x >=
  xmax_pml``, evaluated in the field type exactly as the Taichi kernel does.
* ``slab_extent`` -- the leading/trailing index ranges where the CPML
  correction is not the identity (a != 0 or kappa != 1).  Outside them the
  reference's memory-variable update leaves psi at 0 and the derivative
  unchanged, so the memory variables are stored only on these slabs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PROFILE_NAMES = ("pml", "pml_half", "alpha", "alpha_half", "k", "k_half",
                 "b", "b_half", "a", "a_half")


def diff_coff(order: int) -> np.ndarray:
    """Staggered first-derivative coefficients c_0..c_{N-1} (float32)."""
    order = int(order)
    if order < 1:
        raise ValueError("accuracy (half stencil length) must be >= 1")
    b = np.zeros(order)
    b[0] = 1
    A = np.zeros((order, order))
    for i in range(order):
        for j in range(order):
            A[i, j] = (2 * j + 1) ** (2 * i + 1)
    return np.linalg.solve(A, b).astype(np.float32)


def diff_coff_op(order: int) -> np.ndarray:
    """The reference's optimised coefficient sets for N = 2..5 (float32)."""
    table = {
        2: [1.129042, -0.0430142],
        3: [2.081695391597685, -0.01139368190892791, -0.2095028691741802],
        4: [1.231666, -1.041182e-1, 2.063707e-2, -3.570998e-3],
        5: [1.236425, -0.10811, 0.02339911, -0.005061550, 0.0007054313],
    }
    c = np.zeros(int(order), dtype=np.float32)
    if int(order) in table:
        c[:] = np.asarray(table[int(order)], dtype=np.float32)
    return c


@dataclass
class AxisProfile:
    """The ten profile arrays of one axis plus the predicate bounds."""
    arrays: dict
    pml_min: float   # xmin_pml = xmin + thick
    pml_max: float   # xmax_pml = xmax - thick
    thick: float

    def __getitem__(self, name):
        return self.arrays[name]


def axis_profile(n: int, star: int, d: float, thick: float, use_lo: bool, use_hi: bool,
                 vp_max: float, Rcoef: float, alpha_max: float, kmax: float, theta: float,
                 dt: float, dtype=np.float32) -> AxisProfile:
    """One axis of SetADEPML2D/3D.

    Elastic2D_CPML.py:410-528 with xmin = 0 and xmax = d*(n-1-2*star)
    (Elastic2D_CPML.py:37-38, Elastic3D_SSG_Tensor.py:42-44).
    """
    n = int(n)
    xmin = 0
    xmax = xmin + d * (n - 1 - 2 * star)
    lo = xmin + thick
    hi = xmax - thick
    d0 = -3.0 * vp_max * math.log(Rcoef) / (2.0 * thick)
    arr = {k: np.zeros(n, dtype=dtype) for k in PROFILE_NAMES}

    for half, (pn, an, kn) in enumerate((("pml", "alpha", "k"), ("pml_half", "alpha_half", "k_half"))):
        P, AL, K = arr[pn], arr[an], arr[kn]
        for i in range(n):
            x = (i - star) * d + d / 2 if half else (i - star) * d
            if x <= lo and use_lo:
                s = (lo - x) / thick
                p = d0 * s ** 2
                al = alpha_max * (1 - s)
                kk = 1 + (kmax - 1) * s ** 2
            elif x >= hi and use_hi:
                s = (x - hi) / thick
                p = d0 * s ** 2
                al = alpha_max * (1 - s)
                kk = 1 + (kmax - 1) * s ** 2
            else:
                p, al, kk = 0, 0, 1
            P[i] = p
            AL[i] = al
            K[i] = kk
            if AL[i] < 0:
                AL[i] = 0

    for pn, an, kn, bn, aan in (("pml", "alpha", "k", "b", "a"),
                                ("pml_half", "alpha_half", "k_half", "b_half", "a_half")):
        for i in range(n):
            p = float(arr[pn][i])
            al = float(arr[an][i])
            kk = float(arr[kn][i])
            arr[bn][i] = (1 - (1 - theta) * dt * (p / kk + al)) / (1 + theta * dt * (p / kk + al))
            if np.abs(p) > 1e-6:
                arr[aan][i] = -dt * p / (kk * kk) / (1 + theta * dt * (p / kk + al))
    return AxisProfile(arr, lo, hi, thick)


def axis_flags(n: int, star: int, d: float, pml_min: float, pml_max: float, dtype=np.float32) -> np.ndarray:
    """Per-index PML predicate of the Taichi kernels, in the field type.

    x = (i-star)*dx (integer point, bit 0) and (i-star)*dx + dx/2 (half point,
    bit 1) compared with xmin_pml / xmax_pml, as in e.g. Elastic2D_CPML.py:145-149.
    """
    T = np.dtype(dtype).type
    i = np.arange(int(n))
    dd = T(d)
    x_int = (i - star).astype(dtype) * dd
    x_half = (i - star).astype(dtype) * dd + dd / T(2)
    lo, hi = T(pml_min), T(pml_max)
    f_int = (x_int <= lo) | (x_int >= hi)
    f_half = (x_half <= lo) | (x_half >= hi)
    return (f_int.astype(np.uint8) | (f_half.astype(np.uint8) << 1)).astype(np.uint8)


def slab_extent(prof: AxisProfile) -> tuple[int, int]:
    """(lo, hi): leading and trailing index ranges where any CPML coefficient
    (integer or half point) departs from the identity (a != 0 or kappa != 1)."""
    a = prof.arrays
    active = (a["a"] != 0) | (a["k"] != 1) | (a["a_half"] != 0) | (a["k_half"] != 1)
    n = active.size
    if not active.any():
        return 0, 0
    idx = np.nonzero(active)[0]
    # leading run [0, lo) and trailing run [n-hi, n) must cover every active index
    lo = 0
    while lo < n and active[lo]:
        lo += 1
    hi = 0
    while hi < n - lo and active[n - 1 - hi]:
        hi += 1
    inner = idx[(idx >= lo) & (idx < n - hi)]
    if inner.size:
        # an active index in the middle: extend the slabs over it
        lo = max(lo, int(inner.max()) + 1)
    return lo, hi


def flag_extent(flags: np.ndarray) -> tuple[int, int]:
    """(lo, hi): leading and trailing index ranges that hold every index whose
    PML predicate flag (axis_flags, either bit) is set -- the slabs of the
    split-field PML's shell."""
    f = np.asarray(flags) != 0
    n = f.size
    if not f.any():
        return 0, 0
    lo = 0
    while lo < n and f[lo]:
        lo += 1
    hi = 0
    while hi < n - lo and f[n - 1 - hi]:
        hi += 1
    inner = np.nonzero(f[lo:n - hi])[0]
    if inner.size:
        lo = lo + int(inner.max()) + 1
    return lo, hi


def coef_table(prof: AxisProfile, dtype=np.float32) -> np.ndarray:
    """Rows b, a, k, b_half, a_half, k_half, concatenated (6*n values)."""
    a = prof.arrays
    return np.concatenate([a["b"], a["a"], a["k"], a["b_half"], a["a_half"], a["k_half"]]).astype(dtype)


def damp_table(prof: AxisProfile, dtype=np.float32) -> np.ndarray:
    """Rows d, d_half (2*n values), the split-PML damping profile."""
    a = prof.arrays
    return np.concatenate([a["pml"], a["pml_half"]]).astype(dtype)


def courant_check(vp_max: float, dt: float, spacings, c) -> float:
    """Stability number vp_max*dt*sqrt(sum 1/h^2)*sum|c| of the staggered scheme
    (the reference's drivers check vp_max*dt*sqrt(sum 1/h^2) <= 1 only, e.g.
    test2d_homegenous.py:32-36); stable when the returned value is <= 1."""
    s = math.sqrt(sum(1.0 / float(h) ** 2 for h in spacings))
    return float(vp_max) * float(dt) * s * float(np.sum(np.abs(np.asarray(c, dtype=np.float64))))
