"""Seeded synthetic earth models and the run set-ups of the benchmark
configurations (no external model files are needed: the reference's
overhustp.mat and SEG-Y models are not available, so seeded models of the
stated shapes and value ranges stand in for them).

All models are float32 (nx, ny, nz) / (nx, nz) arrays, last index = depth.
"""
from __future__ import annotations

import math

import numpy as np

from . import sources


def homogeneous(shape, vp=3000.0, vs=1732.0, rho=2000.0):
    return (np.full(shape, vp, np.float32), np.full(shape, vs, np.float32),
            np.full(shape, rho, np.float32))


def gardner(vp):
    """rho = 1741 (vp/1000)^0.25 kg/m^3 (as in test3d_homegenous_overhust.py:15)."""
    return (1741.0 * (np.asarray(vp, np.float64) / 1000.0) ** 0.25).astype(np.float32)


def correlated_noise(shape, corr_len_cells, seed):
    """Zero-mean unit-std Gaussian field with a Gaussian correlation of the
    given length (in cells), by FFT filtering of white noise."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    k = np.meshgrid(*[np.fft.fftfreq(n) for n in shape], indexing="ij")
    k2 = sum(kk ** 2 for kk in k)
    filt = np.exp(-0.5 * (2 * math.pi) ** 2 * k2 * (corr_len_cells ** 2) / 2.0)
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    f -= f.mean()
    s = f.std()
    return f / s if s > 0 else f


def thrust_belt(shape=(400, 400, 200), h=12.5, seed=0, nlayers=12, vp_min=2000.0, vp_max=6000.0,
                pert=0.03, corr_m=50.0):
    """Seeded thrust-belt model: `nlayers` dipping layers with vp from vp_min
    to vp_max, two planar faults offsetting the layers, vs = vp/1.73, Gardner
    density and a +/-`pert` Gaussian-correlated perturbation."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None, None] * h
    y = np.arange(ny)[None, :, None] * h
    z = np.arange(nz)[None, None, :] * h
    dip_x, dip_y = math.tan(math.radians(rng.uniform(8, 20))), math.tan(math.radians(rng.uniform(-8, 8)))
    depth = z - dip_x * (x - x.mean()) - dip_y * (y - y.mean())
    # two planar faults: points on the hanging-wall side are shifted up by a throw
    for _ in range(2):
        n = rng.normal(size=3)
        n[2] = abs(n[2]) + 0.5
        n /= np.linalg.norm(n)
        c = np.array([rng.uniform(0.3, 0.7) * nx * h, rng.uniform(0.3, 0.7) * ny * h, 0.5 * nz * h])
        side = (x - c[0]) * n[0] + (y - c[1]) * n[1] + (z - c[2]) * n[2] > 0
        depth = depth - side * rng.uniform(0.06, 0.12) * nz * h
    span = nz * h * (1 + dip_x) + 1e-9
    lay = np.clip(np.floor((depth - depth.min()) / (depth.max() - depth.min() + 1e-9) * nlayers), 0, nlayers - 1)
    vp = vp_min + (vp_max - vp_min) * lay / (nlayers - 1)
    vp = vp * (1.0 + pert * np.clip(correlated_noise(shape, corr_m / h, seed + 1), -1, 1))
    vp = vp.astype(np.float32)
    vs = (vp / np.float32(1.73)).astype(np.float32)
    del span
    return vp, vs, gardner(vp)


def layered(shape, vp_top, vp_bottom, nlayers=8, seed=0, anomaly=0.0, vs_ratio=1.73):
    """Flat layers with vp from vp_top to vp_bottom plus an optional Gaussian
    anomaly of relative amplitude `anomaly` in the model centre."""
    rng = np.random.default_rng(seed)
    nz = shape[-1]
    bounds = np.sort(rng.uniform(0.05, 0.95, nlayers - 1)) * nz
    zi = np.arange(nz)
    lay = np.searchsorted(bounds, zi)
    v1d = vp_top + (vp_bottom - vp_top) * lay / (nlayers - 1)
    vp = np.broadcast_to(v1d, shape).astype(np.float64).copy()
    if anomaly:
        grids = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
        r2 = sum(((g - n / 2.0) / (n / 8.0)) ** 2 for g, n in zip(grids, shape))
        vp *= 1.0 + anomaly * np.exp(-r2)
    vp = vp.astype(np.float32)
    vs = (vp / np.float32(vs_ratio)).astype(np.float32)
    return vp, vs, gardner(vp)


def pml_parameter(vp_max, vs_max, h, freq, npml=20, dims=3):
    """The drivers' canonical recipe (test2d_homegenous.py:40-51): Rcoef=1e-6,
    theta=1, alpha_max = pi*freq, kmax = vs_max/(5*h*freq)."""
    p = {"vp_max": float(vp_max), "Rcoef": 1e-6, "theta": 1, "alpha_max_pml": math.pi * freq,
         "kmax_pml": float(vs_max) / (5 * h * freq)}
    for ax in ("xyz" if dims == 3 else "xz"):
        p[f"pml_{ax}_thick"] = npml * h
    return p


def config2(n=200, nt=1000, accuracy=2):
    """3D homogeneous SSG-CPML, n^3, dx=10 m, vp=3000, vs=1732, rho=2000,
    dt=1 ms, 20-cell CPML, double couple (30/60/90) with a 15 Hz Ricker2 at
    the centre, 50x50 receiver grid at k = N+5."""
    shape = (n, n, n)
    vp, vs, rho = homogeneous(shape)
    h = 10.0
    nr = 50
    rx = np.linspace(accuracy + 21, n - accuracy - 22, nr).astype(np.int64)
    RX, RY = np.meshgrid(rx, rx, indexing="ij")
    return dict(
        name=f"3d-ssg-cpml-tensor-{n}^3-nt{nt}", shape=shape, vp=vp, vs=vs, rho=rho, dx=h, dy=h, dz=h,
        dt=1e-3, nt=nt, accuracy=accuracy, freq=15.0, isx=n // 2, isy=n // 2, isz=n // 2,
        rsx=RX.reshape(1, -1), rsy=RY.reshape(1, -1), rsz=np.full((1, nr * nr), accuracy + 5, np.int64),
        MT=sources.double_couple(30, 60, 90), src_scale=1.0,
        pml=pml_parameter(3000.0, 1732.0, h, 15.0, 20), surface=[True] * 6)


def config3(shape=(400, 400, 200), nt=2000, accuracy=2, seed=0):
    """3D heterogeneous thrust-belt SSG-CPML, dx=12.5 m, dt=0.8 ms, general
    moment tensor (six N(0,1) components), 10 Hz Ricker2."""
    vp, vs, rho = thrust_belt(shape, 12.5, seed)
    nx, ny, nz = shape
    h = 12.5
    nr = 50
    rx = np.linspace(accuracy + 21, nx - accuracy - 22, nr).astype(np.int64)
    ry = np.linspace(accuracy + 21, ny - accuracy - 22, nr).astype(np.int64)
    RX, RY = np.meshgrid(rx, ry, indexing="ij")
    return dict(
        name=f"3d-ssg-cpml-tensor-thrust-{nx}x{ny}x{nz}-nt{nt}", shape=shape, vp=vp, vs=vs, rho=rho,
        dx=h, dy=h, dz=h, dt=8e-4, nt=nt, accuracy=accuracy, freq=10.0, isx=nx // 2, isy=ny // 2,
        isz=nz // 2, rsx=RX.reshape(1, -1), rsy=RY.reshape(1, -1),
        rsz=np.full((1, nr * nr), accuracy + 5, np.int64), MT=sources.random_tensor(seed), src_scale=1.0,
        pml=pml_parameter(float(vp.max()), float(vs.max()), h, 10.0, 20), surface=[True] * 6)


def config1(n=400, nt=1000, accuracy=2):
    """2D homogeneous P-SV, n^2, dx=dz=10, vp=3000, vs=1732, rho=2000, dt=1 ms,
    20-cell CPML, explosive source (M = I) with the 25 Hz Ricker2 (t0 = 1.5/f)
    at the centre, 200 receivers at z = N+5."""
    shape = (n, n)
    vp, vs, rho = homogeneous(shape)
    nr = 200
    return dict(
        name=f"2d-ssg-vs-{n}^2-nt{nt}", shape=shape, vp=vp, vs=vs, rho=rho, dx=10.0, dz=10.0, dt=1e-3,
        nt=nt, accuracy=accuracy, freq=25.0, isx=n // 2, isz=n // 2,
        rsx=np.linspace(accuracy + 1, n - accuracy - 2, nr).astype(np.int64).reshape(1, nr),
        rsz=np.full((1, nr), accuracy + 5, np.int64), MT="explosive", src_scale=1.0,
        pml=pml_parameter(3000.0, 1732.0, 10.0, 25.0, 20, dims=2), surface=[True] * 4)


def config4(nshots=64, nt=1500, accuracy=2, seed=0, nx_range=(600, 1200), nz_range=(300, 500)):
    """Batched 2D workload: nshots seeded heterogeneous models of uneven sizes
    (nx ~ U[600, 1200], nz ~ U[300, 500], dx = dz = 10 m), layered vp
    1500-4500 m/s with a +10% Gaussian anomaly, explosive 15 Hz Ricker2 source
    below the surface at the model centre, receivers every 4 cells at
    z = N + 5, dt = 1 ms, 20-cell CPML.  Returns a list of per-shot dicts."""
    rng = np.random.default_rng(seed)
    shots = []
    for s in range(nshots):
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
        vp, vs, rho = layered((nx, nz), 1500.0, 4500.0, nlayers=8, seed=seed + 100 + s, anomaly=0.10)
        rx = np.arange(accuracy + 21, nx - accuracy - 21, 4, dtype=np.int64)
        shots.append(dict(
            name=f"2d-batch-{nshots}shots-nt{nt}", shape=(nx, nz), vp=vp, vs=vs, rho=rho, dx=10.0, dz=10.0,
            dt=1e-3, nt=nt, accuracy=accuracy, freq=15.0, isx=nx // 2, isz=accuracy + 25,
            rsx=rx.reshape(1, -1), rsz=np.full((1, rx.size), accuracy + 5, np.int64), MT="explosive",
            src_scale=1.0, pml=pml_parameter(float(vp.max()), float(vs.max()), 10.0, 15.0, 20, dims=2),
            surface=[True] * 4))
    return shots
