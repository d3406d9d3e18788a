"""Problem builders shared by the tests: one description drives both the
product (seiswave_taichi_b200 drop-in classes, GPU) and the oracle (CPU)."""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pml_param(vp_max, vs_max, h, freq, npml, dims=3):
    p = {"vp_max": vp_max, "Rcoef": 1e-6, "theta": 1, "alpha_max_pml": math.pi * freq,
         "kmax_pml": vs_max / (5 * h[0] * freq)}
    for ax, hh in zip("xyz" if dims == 3 else "xz", h):
        p[f"pml_{ax}_thick"] = npml * hh
    return p


def layered_model(shape, seed=0, vp0=2500.0, vp1=4200.0, dtype=np.float32):
    """Heterogeneous test model: dipping layers plus random perturbation, so that
    every material average and every stagger of the scheme matters."""
    rng = np.random.default_rng(seed)
    idx = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    depth = idx[-1] + 0.3 * idx[0]
    nlay = 5
    lay = np.floor(depth / (depth.max() + 1) * nlay)
    vp = vp0 + (vp1 - vp0) * lay / (nlay - 1)
    vp = vp * (1 + 0.03 * rng.standard_normal(shape))
    vs = vp / 1.73
    rho = 1741.0 * (vp / 1000.0) ** 0.25
    return vp.astype(dtype), vs.astype(dtype), rho.astype(dtype)


def case3d(shape=(40, 36, 44), N=2, scheme="TENSOR", hetero=True, npml=8, nt=120, dtype=np.float32,
           dx=10.0, dy=10.0, dz=10.0, dt=1e-3, freq=20.0, seed=0, surface=(True,) * 6):
    nx, ny, nz = shape
    if hetero:
        vp, vs, rho = layered_model(shape, seed, dtype=dtype)
    else:
        vp = np.full(shape, 3000.0, dtype)
        vs = np.full(shape, 1732.0, dtype)
        rho = np.full(shape, 2000.0, dtype)
    c = dict(scheme=scheme, shape=shape, N=N, vp=vp, vs=vs, rho=rho, dx=dx, dy=dy, dz=dz, dt=dt,
             freq=freq, nt=nt, dtype=dtype,
             isx=nx // 2, isy=ny // 2, isz=nz // 2,
             pml=pml_param(float(vp.max()), float(vs.max()), (dx, dy, dz), freq, npml),
             surface=list(surface))
    if scheme == "TENSOR":
        nr = 6
        c["rsx"] = np.full((1, nr), nx // 2 - 3, dtype=np.int64)
        c["rsy"] = np.linspace(N + 2, ny - N - 3, nr).astype(np.int64).reshape(1, nr)
        c["rsz"] = np.full((1, nr), N + 4, dtype=np.int64)
        c["MT"] = np.array([[0.3, 1.0, -0.4], [1.0, -0.7, 0.2], [-0.4, 0.2, 0.5]], np.float32)
        c["src_scale"] = 1.0e6
    else:
        c["rsx"], c["rsy"], c["rsz"] = nx // 2 - 4, ny // 2 - 3, nz // 2 - 5
        if scheme == "CPML":
            c["isx"], c["isy"], c["isz"] = nx // 2 - 5, ny // 2 - 5, nz // 2 - 5
        c["src_scale"] = 1.0e3
    return c


def product3d(c, **kw):
    """The drop-in solver for case c; exact numerics unless exact=False is passed."""
    import torch
    kw.setdefault("exact", True)
    if c["scheme"] == "TENSOR":
        from seiswave_taichi_b200.Elastic3D_SSG_Tensor import ElasticWAVE
        w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dy"], c["dz"], c["dt"], c["isx"], c["isy"],
                        c["isz"], c["rsx"], c["rsy"], c["rsz"], c["MT"], c["src_scale"], c["nt"], c["N"],
                        c["freq"], torch.float64 if c["dtype"] == np.float64 else torch.float32, **kw)
    elif c["scheme"] == "CPML":
        from seiswave_taichi_b200.Elastic3D_SSG_CPML import ElasticWAVE
        w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dy"], c["dz"], c["dt"], c["isx"], c["isy"],
                        c["isz"], c["rsx"], c["rsy"], c["rsz"], c["nt"], c["N"], c["freq"],
                        torch.float64 if c["dtype"] == np.float64 else torch.float32, **kw)
    else:
        from seiswave_taichi_b200.Elastic3D_SSG_SPML import ElasticWAVE
        w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dy"], c["dz"], c["dt"], c["isx"], c["isy"],
                        c["isz"], c["rsx"], c["rsy"], c["rsz"], c["nt"], c["N"], c["freq"], c["src_scale"],
                        torch.float64 if c["dtype"] == np.float64 else torch.float32, **kw)
    w.SetADEPML3D(c["surface"], c["pml"])
    return w


def oracle3d(c, wavelet=None):
    from oracle.oracle import Oracle3D
    return Oracle3D(c["scheme"], c["vs"], c["vp"], c["rho"], c["dx"], c["dy"], c["dz"], c["dt"],
                    c["isx"], c["isy"], c["isz"], c["rsx"], c["rsy"], c["rsz"], c["nt"], c["N"], c["freq"],
                    c["surface"], c["pml"], dtype=c["dtype"], MT=c.get("MT"),
                    src_scale=c.get("src_scale", 1.0), t0=0.03, wavelet=wavelet)


def case2d(shape=(80, 72), N=2, hetero=True, npml=10, nt=200, dtype=np.float32, dx=10.0, dz=10.0,
           dt=1e-3, freq=25.0, seed=1, surface=(True,) * 4, nrec=None, MT=None, src_scale=1.0):
    nx, nz = shape
    if hetero:
        vp, vs, rho = layered_model(shape, seed, dtype=dtype)
    else:
        vp = np.full(shape, 3000.0, dtype)
        vs = np.full(shape, 1732.0, dtype)
        rho = np.full(shape, 2000.0, dtype)
    c = dict(shape=shape, N=N, vp=vp, vs=vs, rho=rho, dx=dx, dz=dz, dt=dt, freq=freq, nt=nt, dtype=dtype,
             isx=nx // 2, isz=nz // 2, rsx=nx // 2 + 7, rsz=nz // 2 - 9,
             pml=pml_param(float(vp.max()), float(vs.max()), (dx, dz), freq, npml, dims=2),
             surface=list(surface))
    if nrec:
        c["rsx"] = np.linspace(N + 2, nx - N - 3, nrec).astype(np.int64).reshape(1, nrec)
        c["rsz"] = np.full((1, nrec), N + 5, dtype=np.int64)
    if MT is not None:
        c["MT"] = MT
        c["src_scale"] = src_scale
    return c


def product2d(c, **kw):
    import torch
    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    if "MT" in c:
        kw.setdefault("MT", c["MT"])
        kw.setdefault("src_scale", c["src_scale"])
    w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"], c["rsx"],
                    c["rsz"], c["nt"], c["N"], c["freq"],
                    torch.float64 if c["dtype"] == np.float64 else torch.float32, **kw)
    w.SetADEPML2D(c["surface"], c["pml"])
    return w


def oracle2d(c, wavelet=None):
    from oracle.oracle import Oracle2D
    rx = np.asarray(c["rsx"]).reshape(-1)
    rz = np.asarray(c["rsz"]).reshape(-1)
    table = None if rx.size == 1 and np.ndim(c["rsx"]) == 0 else rx * c["shape"][1] + rz
    mt = None
    if "MT" in c:
        from seiswave_taichi_b200.Elastic2D_CPML import moment_2d
        mt = moment_2d(c["MT"])
    return Oracle2D(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"], int(rx[0]),
                    int(rz[0]), c["nt"], c["N"], c["freq"], c["surface"], c["pml"], dtype=c["dtype"],
                    wavelet=wavelet, MT=mt, rec_index=table)


def to_np(t):
    return t.detach().cpu().numpy()
