"""Python side of the CPU oracle (test infrastructure only).

Loads oracle/libsworacle.so (built by oracle/Makefile from sw_oracle.cpp) and
sets up a reference-faithful CPU run entirely on its own: finite-difference
coefficients (oracle_diff_coff), PML profiles (oracle_pml_axis), mu/lam
(numpy, as Compute_mu/Compute_lam), full-grid memory variables and wavefields.
Nothing here is imported by the product; tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it as the checker.

Parity unpinned: the reference has no golden vectors and Taichi cannot run
here; the restatement is held by closed-form coefficients, the numpy twin and
the physics checks of tests/test_oracle.py (see sw_oracle.cpp's header).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libsworacle.so"


class OAxis(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("pml", "pml_half", "alpha", "alpha_half", "k", "k_half",
                                          "b", "b_half", "a", "a_half")] + \
               [("pml_min", C.c_double), ("pml_max", C.c_double)]


class O2Desc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nz", C.c_int32), ("N", C.c_int32), ("dtype", C.c_int32),
                ("dx", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("c", C.c_double * 16)] + \
               [(n, C.c_void_p) for n in ("vx", "vz", "sxx", "szz", "sxz", "rho", "lam", "mu")] + \
               [("mem", C.c_void_p * 10), ("ax", OAxis * 2),
                ("isx", C.c_int32), ("isz", C.c_int32), ("rsx", C.c_int32), ("rsz", C.c_int32),
                ("f0", C.c_double), ("wavelet", C.c_void_p), ("data", C.c_void_p),
                ("src_kind", C.c_int32), ("nrec", C.c_int32), ("mt", C.c_double * 3),
                ("rec_idx", C.c_void_p)]


class O3Desc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("N", C.c_int32),
                ("dtype", C.c_int32), ("scheme", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("c", C.c_double * 16)] + \
               [(n, C.c_void_p) for n in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz",
                                          "rho", "lam", "mu")] + \
               [("mem", C.c_void_p * 24), ("ax", OAxis * 3),
                ("isx", C.c_int32), ("isy", C.c_int32), ("isz", C.c_int32),
                ("f0", C.c_double), ("src_scale", C.c_double), ("t0", C.c_double),
                ("mt", C.c_double * 6), ("wavelet", C.c_void_p),
                ("nrec", C.c_int32), ("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p),
                ("data", C.c_void_p)]


_lib = None


def build() -> Path:
    """Compile the oracle library (make) if needed."""
    src = HERE / "sw_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        lib.oracle_diff_coff.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        lib.oracle_pml_axis.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        lib.oracle_wavelet.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_void_p]
        lib.oracle2d_run.argtypes = [C.POINTER(O2Desc), C.c_int, C.c_int, C.c_int, C.c_void_p]
        lib.oracle3d_run.argtypes = [C.POINTER(O3Desc), C.c_int, C.c_int]
        lib.oracle_set_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def set_threads(n: int) -> int:
    return load().oracle_set_threads(int(n))


def _p(a):
    return None if a is None else a.ctypes.data


def diff_coff(order: int):
    """(float64, float32) coefficients of the oracle's own solve."""
    d = np.zeros(order, np.float64)
    f = np.zeros(order, np.float32)
    if load().oracle_diff_coff(order, _p(d), _p(f)) != 0:
        raise ValueError("bad order")
    return d, f


def pml_axis(n, star, d, thick, use_lo, use_hi, vp_max, Rcoef, alpha_max, kmax, theta, dt,
             dtype=np.float32):
    """The oracle's restatement of one SetADEPML axis: dict of ten arrays + (lo, hi)."""
    names = ("pml", "pml_half", "alpha", "alpha_half", "k", "k_half", "b", "b_half", "a", "a_half")
    arrs = {k: np.zeros(n, dtype) for k in names}
    ptrs = (C.c_void_p * 10)(*[arrs[k].ctypes.data for k in names])
    mm = np.zeros(2, np.float64)
    load().oracle_pml_axis(n, star, float(d), float(thick), int(bool(use_lo)), int(bool(use_hi)),
                           float(vp_max), float(Rcoef), float(alpha_max), float(kmax), float(theta),
                           float(dt), 0 if dtype == np.float32 else 1, ptrs, _p(mm))
    return arrs, (float(mm[0]), float(mm[1]))


def wavelet(kind: str, nt: int, dt, freq, scale=1.0, t0=0.0) -> np.ndarray:
    out = np.zeros(nt, np.float32)
    k = {"ricker": 0, "ricker2": 1, "ricker3": 2}[kind]
    load().oracle_wavelet(k, nt, float(dt), float(t0), float(freq), float(scale), _p(out))
    return out


def _axis_struct(arrs, mm):
    ax = OAxis()
    for k, v in arrs.items():
        setattr(ax, k, v.ctypes.data)
    ax.pml_min, ax.pml_max = mm
    return ax


class Oracle2D:
    """CPU run of Elastic2D_CPML (schemes 'VS', 'SV', 'RSG')."""

    def __init__(self, vs, vp, rho, dx, dz, dt, isx, isz, rsx, rsz, nt, accuracy, freq,
                 pml_surface, pml_parameter, dtype=np.float32, wavelet=None, coef=None, MT=None,
                 rec_index=None):
        """MT (xx, zz, xz) selects the moment-tensor source (wavelet required);
        rec_index (linear cell indices) records (nt, nrec) traces instead of
        the single receiver (rsx, rsz)."""
        T = dtype
        self.T = T
        self.vs = np.ascontiguousarray(vs, dtype=T)
        self.vp = np.ascontiguousarray(vp, dtype=T)
        self.rho = np.ascontiguousarray(rho, dtype=T)
        self.mu = self.rho * self.vs ** 2
        self.lam = self.rho * (self.vp ** 2 - 2 * self.vs ** 2)
        nx, nz = self.vs.shape
        self.shape = (nx, nz)
        self.N = int(accuracy)
        z = lambda: np.zeros((nx, nz), T)
        self.vx, self.vz, self.sxx, self.szz, self.sxz = z(), z(), z(), z(), z()
        self.mem = [z() for _ in range(10)]
        self.rec_index = None if rec_index is None else np.ascontiguousarray(rec_index, np.int64).reshape(-1)
        self.data = np.zeros(nt, T) if self.rec_index is None else np.zeros((nt, self.rec_index.size), T)
        p = pml_parameter
        self.axes = []
        for a, (n, h, th) in enumerate(((nx, dx, p["pml_x_thick"]), (nz, dz, p["pml_z_thick"]))):
            self.axes.append(pml_axis(n, self.N, h, th, pml_surface[2 * a], pml_surface[2 * a + 1],
                                      p["vp_max"], p["Rcoef"], p["alpha_max_pml"], p["kmax_pml"],
                                      p["theta"], dt, T))
        if coef is None:
            coef = diff_coff(self.N)[1].astype(np.float64)
        self.wavelet = None if wavelet is None else np.ascontiguousarray(wavelet, np.float32)
        d = O2Desc()
        d.nx, d.nz, d.N, d.dtype = nx, nz, self.N, 0 if T == np.float32 else 1
        d.dx, d.dz, d.dt = dx, dz, dt
        for m in range(self.N):
            d.c[m] = float(coef[m])
        for nm in ("vx", "vz", "sxx", "szz", "sxz", "rho", "lam", "mu"):
            setattr(d, nm, getattr(self, nm).ctypes.data)
        for q in range(10):
            d.mem[q] = self.mem[q].ctypes.data
        for a in range(2):
            d.ax[a] = _axis_struct(*self.axes[a])
        d.isx, d.isz, d.rsx, d.rsz = isx, isz, rsx, rsz
        d.f0 = freq
        d.wavelet = _p(self.wavelet)
        d.data = self.data.ctypes.data
        if MT is not None:
            if self.wavelet is None:
                raise ValueError("the moment-tensor source needs its wavelet")
            d.src_kind = 1
            for q in range(3):
                d.mt[q] = float(MT[q])
        if self.rec_index is not None:
            d.nrec = int(self.rec_index.size)
            d.rec_idx = self.rec_index.ctypes.data
        self.desc = d

    def run(self, scheme: str, it0: int, n: int, rsg_sources=None):
        s = {"VS": 0, "SV": 1, "RSG": 2}[scheme]
        src = None
        if rsg_sources is not None:
            src = np.ascontiguousarray(rsg_sources, np.float64)
        load().oracle2d_run(C.byref(self.desc), s, it0, n, _p(src))
        return self

    # full-grid memory arrays by reference name
    MEM_NAMES = ("memory_sxx_dx", "memory_sxx_dz", "memory_sxz_dx", "memory_sxz_dz", "memory_szz_dx",
                 "memory_szz_dz", "memory_dvx_dx", "memory_dvx_dz", "memory_dvz_dx", "memory_dvz_dz")

    def memory(self, name):
        return self.mem[self.MEM_NAMES.index(name)]


class Oracle3D:
    """CPU run of the 3D solvers: scheme 'CPML' (point force), 'TENSOR', 'SPML'."""

    MEM_CPML = ("memory_sxx_dx", "memory_sxy_dy", "memory_sxz_dz", "memory_sxy_dx", "memory_syy_dy",
                "memory_syz_dz", "memory_sxz_dx", "memory_syz_dy", "memory_szz_dz", "memory_dvx_dx",
                "memory_dvy_dy", "memory_dvz_dz", "memory_dvy_dx", "memory_dvx_dy", "memory_dvz_dx",
                "memory_dvx_dz", "memory_dvz_dy", "memory_dvy_dz")
    SPLIT = ("vx_x", "vx_y", "vx_z", "vy_x", "vy_y", "vy_z", "vz_x", "vz_y", "vz_z",
             "sxx_x", "sxx_y", "sxx_z", "syy_x", "syy_y", "syy_z",
             "sxy_x", "sxy_y", "sxz_x", "sxz_z", "syz_y", "syz_z", "szz_x", "szz_y", "szz_z")

    def __init__(self, scheme, vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, rsx, rsy, rsz, nt,
                 accuracy, freq, pml_surface, pml_parameter, dtype=np.float32, MT=None,
                 src_scale=1.0, t0=0.03, wavelet=None, coef=None):
        T = dtype
        self.T = T
        self.scheme = {"CPML": 0, "TENSOR": 1, "SPML": 2}[scheme]
        self.vs = np.ascontiguousarray(vs, dtype=T)
        self.vp = np.ascontiguousarray(vp, dtype=T)
        self.rho = np.ascontiguousarray(rho, dtype=T)
        self.mu = self.rho * self.vs ** 2
        self.lam = self.rho * (self.vp ** 2 - 2 * self.vs ** 2)
        nx, ny, nz = self.vs.shape
        self.shape = (nx, ny, nz)
        self.N = int(accuracy)
        z = lambda: np.zeros((nx, ny, nz), T)
        for nm in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
            setattr(self, nm, z())
        nmem = 24 if self.scheme == 2 else 18
        self.mem = [z() for _ in range(nmem)]
        self.rx = np.ascontiguousarray(np.asarray(rsx).reshape(-1), np.int32)
        self.ry = np.ascontiguousarray(np.asarray(rsy).reshape(-1), np.int32)
        self.rz = np.ascontiguousarray(np.asarray(rsz).reshape(-1), np.int32)
        nrec = self.rx.size
        self.data = np.zeros((nt, nrec) if self.scheme == 1 else nt, np.float32)
        p = pml_parameter
        self.axes = []
        for a, (n, h, th) in enumerate(((nx, dx, p["pml_x_thick"]), (ny, dy, p["pml_y_thick"]),
                                        (nz, dz, p["pml_z_thick"]))):
            self.axes.append(pml_axis(n, self.N, h, th, pml_surface[2 * a], pml_surface[2 * a + 1],
                                      p["vp_max"], p["Rcoef"], p["alpha_max_pml"], p["kmax_pml"],
                                      p["theta"], dt, T))
        if coef is None:
            coef = diff_coff(self.N)[1].astype(np.float64)
        self.wavelet = None if wavelet is None else np.ascontiguousarray(wavelet, np.float32)
        d = O3Desc()
        d.nx, d.ny, d.nz, d.N = nx, ny, nz, self.N
        d.dtype = 0 if T == np.float32 else 1
        d.scheme = self.scheme
        d.dx, d.dy, d.dz, d.dt = dx, dy, dz, dt
        for m in range(self.N):
            d.c[m] = float(coef[m])
        for nm in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz", "rho", "lam", "mu"):
            setattr(d, nm, getattr(self, nm).ctypes.data)
        for q in range(nmem):
            d.mem[q] = self.mem[q].ctypes.data
        for a in range(3):
            d.ax[a] = _axis_struct(*self.axes[a])
        d.isx, d.isy, d.isz = isx, isy, isz
        d.f0, d.src_scale, d.t0 = freq, src_scale, t0
        if MT is not None:
            M = np.asarray(MT, np.float32).reshape(3, 3)
            for q, v in enumerate((M[0, 0], M[1, 1], M[2, 2], M[0, 1], M[0, 2], M[1, 2])):
                d.mt[q] = float(v)
        d.wavelet = _p(self.wavelet)
        d.nrec = nrec
        d.rx, d.ry, d.rz = self.rx.ctypes.data, self.ry.ctypes.data, self.rz.ctypes.data
        d.data = self.data.ctypes.data
        self.desc = d

    def run(self, it0: int, n: int):
        load().oracle3d_run(C.byref(self.desc), it0, n)
        return self

    def memory(self, name):
        names = self.SPLIT if self.scheme == 2 else self.MEM_CPML
        return self.mem[names.index(name)]


def rel_l2(a, b) -> float:
    """||a-b|| / ||b|| in float64 (0 when both are zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    na = np.linalg.norm(a - b)
    if nb == 0:
        return 0.0 if na == 0 else float("inf")
    return float(na / nb)
