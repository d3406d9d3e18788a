"""Write tests/golden/reference_small.npz: small runs of SeisWave_Taichi's OWN
solver source, executed unmodified through the numpy stand-in for Taichi
(tests/golden/ti_standin.py).  These fixtures pin the CPU oracle and the CUDA
kernels to the reference's code, not to a restatement of it.

    python tests/golden/make_reference_golden.py [REFERENCE_ROOT]

REFERENCE_ROOT is the SeisWave_Taichi checkout (the directory holding src/);
it defaults to /root/reference.  The reference is only read: bytecode
writing is switched off so nothing lands in its tree.  The fixture file
holds each case's inputs (vp, vs, rho), the reference's final wavefields and
receiver traces, and the PML profiles its SetADEPML2D/3D built, so the tests
need neither the reference nor this script.

Cases (every reference update function, orders 2 and 3):
  vs2d       Elastic2D_CPML.update_SSG_VS            40x36, N=2, 60 steps
  vs2d_aea   AEA_init(); then AEA() + update_SSG_VS  40x36, N=2, 60 steps
             (the driver loop of Relay_wave.py:55-59)
  sv2d       Elastic2D_CPML.update_SSG_SV            36x40, N=3, 50 steps
  rsg2d      Elastic2D_CPML.update_RSG(nt, source)   40x40, N=2, 60 steps
  tensor3d   Elastic3D_SSG_Tensor.update_SSG         18x16x20, N=2, 40 steps
  tensor3dn3 Elastic3D_SSG_Tensor.update_SSG         20x18x22, N=3, 30 steps
  cpml3d     Elastic3D_SSG_CPML.update_SSG           16x18x20, N=2, 40 steps
  spml3d     Elastic3D_SSG_SPML.update_SSG_SPML      16x18x20, N=2, 40 steps
The 3D CPML and SPML grids keep nx <= ny <= nz: those two kernels zero six
dead-border slabs with loop ranges that borrow another axis's extent
(Elastic3D_SSG_CPML.py:220,230 and Elastic3D_SSG_SPML.py:268,278), which
stay in bounds only then.
"""
from __future__ import annotations

import math
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

OUT = HERE / "reference_small.npz"

F2D = ("vx", "vz", "sxx", "szz", "sxz")
F3D = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
PROFILES = ("pml", "alpha", "k", "b", "a")


def model(shape, seed):
    from cases import layered_model
    return layered_model(shape, seed)


def specs():
    """Case definitions shared with the tests (inputs are stored as well)."""
    mt = np.array([[0.3, 1.0, -0.4], [1.0, -0.7, 0.2], [-0.4, 0.2, 0.5]], np.float32)
    return [
        dict(name="vs2d", kind="2d", scheme="VS", shape=(40, 36), N=2, npml=6, nt=60, seed=11,
             dx=10.0, dz=10.0, dt=1e-3, freq=25.0, isx=20, isz=18, rsx=27, rsz=9, aea=False),
        dict(name="vs2d_aea", kind="2d", scheme="VS", shape=(40, 36), N=2, npml=6, nt=60, seed=12,
             dx=10.0, dz=10.0, dt=1e-3, freq=25.0, isx=18, isz=17, rsx=25, rsz=10, aea=True,
             surface=[False, True, True, True]),
        dict(name="sv2d", kind="2d", scheme="SV", shape=(36, 40), N=3, npml=6, nt=50, seed=13,
             dx=10.0, dz=10.0, dt=1e-3, freq=25.0, isx=18, isz=20, rsx=12, rsz=27, aea=False),
        dict(name="rsg2d", kind="2d", scheme="RSG", shape=(40, 40), N=2, npml=6, nt=60, seed=14,
             dx=10.0, dz=10.0, dt=1e-3, freq=25.0, isx=20, isz=20, rsx=26, rsz=12, aea=False),
        dict(name="tensor3d", kind="TENSOR", shape=(18, 16, 20), N=2, npml=4, nt=40, seed=21,
             dx=10.0, dy=10.0, dz=10.0, dt=1e-3, freq=20.0, isx=9, isy=8, isz=10, MT=mt,
             src_scale=1.0e6, rsx=[[6, 6, 6, 6, 6]], rsy=[[4, 6, 8, 10, 11]], rsz=[[6, 6, 6, 6, 6]]),
        dict(name="tensor3dn3", kind="TENSOR", shape=(20, 18, 22), N=3, npml=4, nt=30, seed=22,
             dx=10.0, dy=10.0, dz=12.5, dt=1e-3, freq=20.0, isx=10, isy=9, isz=11, MT=mt,
             src_scale=1.0e6, rsx=[[7, 7, 7, 7]], rsy=[[5, 7, 9, 11]], rsz=[[7, 7, 7, 7]]),
        dict(name="cpml3d", kind="CPML", shape=(16, 18, 20), N=2, npml=4, nt=40, seed=23,
             dx=10.0, dy=10.0, dz=10.0, dt=1e-3, freq=20.0, isx=3, isy=4, isz=5, rsx=5, rsy=6, rsz=7),
        dict(name="spml3d", kind="SPML", shape=(16, 18, 20), N=2, npml=4, nt=40, seed=24,
             dx=10.0, dy=10.0, dz=10.0, dt=1e-3, freq=20.0, isx=8, isy=9, isz=10, rsx=5, rsy=6, rsz=7,
             src_scale=1.0e3),
    ]


def pml_params(s, vp, vs):
    from cases import pml_param
    h = (s["dx"], s["dz"]) if s["kind"] == "2d" else (s["dx"], s["dy"], s["dz"])
    return pml_param(float(vp.max()), float(vs.max()), h, s["freq"], s["npml"],
                     dims=2 if s["kind"] == "2d" else 3)


def ricker_series(s):
    """update_RSG's caller-given source per step: the reference's Ricker
    (BaseFun.py:4-11) as a driver would pass it, in float32."""
    from seiswave_taichi_b200 import BaseFun
    return BaseFun.series("ricker", s["nt"], s["dt"], s["freq"], 1.0)


def run_case(s, ti, mods):
    vp, vs, rho = model(s["shape"], s["seed"])

    def fld(a, dtype=ti.f32):
        f = ti.field(dtype=dtype, shape=a.shape)
        f.from_numpy(a)
        return f

    out = {f"{s['name']}__vp": vp, f"{s['name']}__vs": vs, f"{s['name']}__rho": rho}
    par = pml_params(s, vp, vs)
    if s["kind"] == "2d":
        w = mods["2d"].ElasticWAVE(fld(vs), fld(vp), fld(rho), s["dx"], s["dz"], s["dt"], s["isx"], s["isz"],
                                   s["rsx"], s["rsz"], s["nt"], s["N"], s["freq"], ti.f32)
        w.SetADEPML2D(list(s.get("surface", [True] * 4)), par)
        if s["aea"]:
            w.AEA_init()
        src = ricker_series(s) if s["scheme"] == "RSG" else None
        if src is not None:
            out[f"{s['name']}__source"] = src
        for it in range(s["nt"]):
            if s["aea"]:
                w.AEA()
            if s["scheme"] == "VS":
                w.update_SSG_VS(it)
            elif s["scheme"] == "SV":
                w.update_SSG_SV(it)
            else:
                w.update_RSG(it, float(src[it]))
        for f in F2D:
            out[f"{s['name']}_{f}"] = getattr(w, f).to_numpy()
        out[f"{s['name']}_data"] = w.data.to_numpy()
        axes = "xz"
    else:
        nx, ny, nz = s["shape"]
        if s["kind"] == "TENSOR":
            rs = [fld(np.asarray(s[k], np.int32), ti.i32) for k in ("rsx", "rsy", "rsz")]
            w = mods["TENSOR"].ElasticWAVE(fld(vs), fld(vp), fld(rho), s["dx"], s["dy"], s["dz"], s["dt"],
                                           s["isx"], s["isy"], s["isz"], rs[0], rs[1], rs[2], fld(s["MT"]),
                                           s["src_scale"], s["nt"], s["N"], s["freq"], ti.f32)
        elif s["kind"] == "CPML":
            w = mods["CPML"].ElasticWAVE(fld(vs), fld(vp), fld(rho), s["dx"], s["dy"], s["dz"], s["dt"],
                                         s["isx"], s["isy"], s["isz"], s["rsx"], s["rsy"], s["rsz"], s["nt"],
                                         s["N"], s["freq"], ti.f32)
        else:
            w = mods["SPML"].ElasticWAVE(fld(vs), fld(vp), fld(rho), s["dx"], s["dy"], s["dz"], s["dt"],
                                         s["isx"], s["isy"], s["isz"], s["rsx"], s["rsy"], s["rsz"], s["nt"],
                                         s["N"], s["freq"], s["src_scale"], ti.f32)
        w.SetADEPML3D([True] * 6, par)
        step = w.update_SSG_SPML if s["kind"] == "SPML" else w.update_SSG
        for it in range(s["nt"]):
            step(it)
        for f in F3D:
            out[f"{s['name']}_{f}"] = getattr(w, f).to_numpy()
        out[f"{s['name']}_data"] = w.data.to_numpy()
        axes = "xyz"
    for ax in axes:
        for pname in PROFILES:
            for suf in ("", "_half"):
                attr = f"{pname}_{ax}{suf}"
                if hasattr(w, attr):
                    out[f"{s['name']}__{attr}"] = getattr(w, attr).to_numpy()
    return out


def wavelet_specs():
    """(name, reference function, args after nt) of the wavelet series pinned:
    the reference's own @ti.func's evaluated at steps 0..NT_WAVELET-1, called
    as its kernels call them (dt, t0, freq, src_scale as f32 variables)."""
    return [
        ("ricker_f15", "Ricker", (1e-3, 15.0, 1.0)),
        ("ricker_f20_s1000", "Ricker", (1e-3, 20.0, 1000)),
        ("ricker2_t003_f15", "Ricker2", (1e-3, 0.03, 15.0, 1.0e6)),
        ("ricker2_t003_f12_dt08", "Ricker2", (8e-4, 0.03, 12.0, 1.0)),
        ("ricker2_t003_f10_dt08", "Ricker2", (8e-4, 0.03, 10.0, 1.0)),
        ("ricker2_vs_f25", "Ricker2", (1e-3, 1.5 / 25.0, 25.0, 1)),
        ("ricker3_f10", "Ricker3", (1e-3, 0.0, 10.0, 1.0)),
    ]


NT_WAVELET = 2000


def wavelets(ti):
    import importlib
    bf = importlib.import_module("src.BaseFun")
    out = {}
    ti._state["depth"] += 1          # kernel scope, as inside update_*
    try:
        for name, fn, args in wavelet_specs():
            f = getattr(bf, fn)
            out[f"wavelet__{name}"] = np.array([f(it, *args) for it in range(NT_WAVELET)], np.float32)
    finally:
        ti._state["depth"] -= 1
    return out


def main(argv):
    ref = Path(argv[1] if len(argv) > 1 else "/root/reference").resolve()
    if not (ref / "src" / "Elastic3D_SSG_Tensor.py").is_file():
        raise SystemExit(f"no SeisWave_Taichi source under {ref}")
    sys.dont_write_bytecode = True
    import ti_standin
    ti = ti_standin.install()
    sys.path.insert(0, str(ref))
    import importlib
    mods = {"2d": importlib.import_module("src.Elastic2D_CPML"),
            "TENSOR": importlib.import_module("src.Elastic3D_SSG_Tensor"),
            "CPML": importlib.import_module("src.Elastic3D_SSG_CPML"),
            "SPML": importlib.import_module("src.Elastic3D_SSG_SPML")}
    out = wavelets(ti)
    for s in specs():
        t = time.time()
        out.update(run_case(s, ti, mods))
        amp = float(np.abs(out[f"{s['name']}_vx"]).max())
        print(f"{s['name']:11s} {time.time() - t:6.1f} s   max|vx| {amp:.3e}", flush=True)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main(sys.argv)
