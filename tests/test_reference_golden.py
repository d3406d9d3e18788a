"""Parity against SeisWave_Taichi's OWN source.

tests/golden/reference_small.npz holds small runs of the reference's solver
modules (src/Elastic2D_CPML.py:128-353, src/Elastic3D_SSG_Tensor.py:166-345,
src/Elastic3D_SSG_CPML.py:144-309, src/Elastic3D_SSG_SPML.py:160-393), their
SetADEPML2D/3D profiles and their BaseFun wavelets, executed unmodified
through a numpy stand-in for Taichi (tests/golden/ti_standin.py; generator
tests/golden/make_reference_golden.py).  The fixture carries every input, so
neither the reference nor the generator is needed here.

CPU: the oracle (oracle/sw_oracle.cpp), the host PML builder (pml.py) and the
wavelet tables (BaseFun.py) reproduce the reference's output bit for bit.
GPU: the CUDA path meets the parity gate -- relative L2 <= 1e-5 for every
wavefield and seismogram -- and, in the default exact numeric mode, is
bit-identical to the reference's output.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from golden.make_reference_golden import F2D, F3D, NT_WAVELET, PROFILES, specs, wavelet_specs

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_small.npz")
SPECS = specs()
TOL = 1e-5  # relative L2 gate for seismograms and wavefields


def _ids(s):
    return s["name"]


def _inputs(s):
    n = s["name"]
    return GOLD[n + "__vp"], GOLD[n + "__vs"], GOLD[n + "__rho"]


def _pml(s, vp, vs):
    from golden.make_reference_golden import pml_params
    return pml_params(s, vp, vs)


def _fields(s):
    return F2D if s["kind"] == "2d" else F3D


def _wavelet(s):
    """The product's own wavelet table for the case's scheme."""
    from seiswave_taichi_b200 import BaseFun
    if s["kind"] == "2d":
        if s["scheme"] == "VS":
            return BaseFun.series("ricker2", s["nt"], s["dt"], s["freq"], 1.0, t0=np.float32(1.5 / s["freq"]))
        return BaseFun.series("ricker", s["nt"], s["dt"], s["freq"], 1.0)
    if s["kind"] == "TENSOR":
        return BaseFun.series("ricker2", s["nt"], s["dt"], s["freq"], s["src_scale"], t0=0.03)
    if s["kind"] == "CPML":
        return BaseFun.series("ricker", s["nt"], s["dt"], s["freq"], 1000.0)
    return BaseFun.series("ricker", s["nt"], s["dt"], s["freq"], s["src_scale"])


def _rel(a, b):
    from oracle.oracle import rel_l2
    return rel_l2(np.asarray(a, np.float64), np.asarray(b, np.float64))


# --------------------------------------------------------------------------
# CPU: oracle, PML profiles, wavelets
# --------------------------------------------------------------------------
def test_fixture_is_complete():
    for s in SPECS:
        n = s["name"]
        for f in _fields(s) + ("data",):
            assert GOLD[f"{n}_{f}"].dtype == np.float32
        assert np.abs(GOLD[f"{n}_vx"]).max() > 0, n
        if s.get("scheme") != "RSG":  # update_RSG records no receiver (Elastic2D_CPML.py:277-353)
            assert np.abs(GOLD[f"{n}_data"]).max() > 0, n


@pytest.mark.parametrize("w", wavelet_specs(), ids=lambda w: w[0])
def test_wavelets_equal_reference(w):
    """BaseFun tables and the oracle's wavelets equal the reference's
    @ti.func's (BaseFun.py:4-27) bit for bit."""
    from oracle import oracle as O
    from seiswave_taichi_b200 import BaseFun
    name, fn, args = w
    ref = GOLD[f"wavelet__{name}"]
    assert ref.shape == (NT_WAVELET,)
    if fn == "Ricker":
        dt, f, sc = args
        ours = BaseFun.series("ricker", NT_WAVELET, dt, f, sc)
        orc = O.wavelet("ricker", NT_WAVELET, np.float32(dt), np.float32(f), np.float32(sc))
    else:
        dt, t0, f, sc = args
        kind = "ricker2" if fn == "Ricker2" else "ricker3"
        ours = BaseFun.series(kind, NT_WAVELET, dt, f, sc, t0=np.float32(t0))
        orc = O.wavelet(kind, NT_WAVELET, np.float32(dt), np.float32(f), np.float32(sc), t0=np.float32(t0))
    np.testing.assert_array_equal(ours, ref)
    # the oracle's own C++ series call libm's expf, which differs from numpy's
    # float32 exp in the last bit for a few percent of the samples; the parity
    # cases feed the product's table (above) to the oracle instead
    np.testing.assert_allclose(orc, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("s", SPECS, ids=_ids)
def test_pml_profiles_equal_reference(s):
    """pml.axis_profile (the product's SetADEPML2D/3D) and the oracle's
    restatement equal the reference's ten arrays per axis bit for bit."""
    from oracle import oracle as O
    from seiswave_taichi_b200 import pml as P
    vp, vs, rho = _inputs(s)
    par = _pml(s, vp, vs)
    axes = "xz" if s["kind"] == "2d" else "xyz"
    surf = list(s.get("surface", [True] * (2 * len(axes))))
    for a, ax in enumerate(axes):
        h = s["d" + ax]
        n = s["shape"][a]
        args = (n, s["N"], h, par[f"pml_{ax}_thick"], surf[2 * a], surf[2 * a + 1], par["vp_max"], par["Rcoef"],
                par["alpha_max_pml"], par["kmax_pml"], par["theta"], s["dt"])
        prof = P.axis_profile(*args)
        orc, _ = O.pml_axis(*args)
        for pname in PROFILES:
            for suf in ("", "_half"):
                ref = GOLD[f"{s['name']}__{pname}_{ax}{suf}"]
                key = pname + suf
                np.testing.assert_array_equal(prof[key], ref, err_msg=f"pml.py {key} {ax}")
                np.testing.assert_array_equal(orc[key], ref, err_msg=f"oracle {key} {ax}")


def _oracle_run(s):
    from oracle.oracle import Oracle2D, Oracle3D
    vp, vs, rho = _inputs(s)
    par = _pml(s, vp, vs)
    if s["kind"] == "2d":
        wav = None if s["scheme"] == "RSG" else _wavelet(s)
        o = Oracle2D(vs, vp, rho, s["dx"], s["dz"], s["dt"], s["isx"], s["isz"], s["rsx"], s["rsz"], s["nt"],
                     s["N"], s["freq"], list(s.get("surface", [True] * 4)), par, dtype=np.float32, wavelet=wav)
        if s["aea"]:
            N = s["N"]
            o.lam[:N] = 0
            o.rho[:N] *= np.float32(0.5)
            for it in range(s["nt"]):
                o.sxx[N, :] = 0
                o.run(s["scheme"], it, 1)
        elif s["scheme"] == "RSG":
            o.run("RSG", 0, s["nt"], rsg_sources=GOLD[s["name"] + "__source"].astype(np.float64))
        else:
            o.run(s["scheme"], 0, s["nt"])
        return o
    o = Oracle3D(s["kind"], vs, vp, rho, s["dx"], s["dy"], s["dz"], s["dt"], s["isx"], s["isy"], s["isz"],
                 np.asarray(s["rsx"]), np.asarray(s["rsy"]), np.asarray(s["rsz"]), s["nt"], s["N"], s["freq"],
                 [True] * 6, par, dtype=np.float32, MT=s.get("MT"), src_scale=s.get("src_scale", 1.0), t0=0.03,
                 wavelet=_wavelet(s))
    return o.run(0, s["nt"])


@pytest.mark.parametrize("s", SPECS, ids=_ids)
def test_oracle_equals_reference(s):
    """The CPU oracle reproduces the reference's own run bit for bit."""
    o = _oracle_run(s)
    for f in _fields(s) + ("data",):
        np.testing.assert_array_equal(np.asarray(getattr(o, f)), GOLD[f"{s['name']}_{f}"], err_msg=f)


# --------------------------------------------------------------------------
# GPU: the CUDA path through the drop-in classes
# --------------------------------------------------------------------------
def _product_run(s, exact=True, per_step=False):
    import torch
    vp, vs, rho = _inputs(s)
    par = _pml(s, vp, vs)
    dtype = torch.float32
    if s["kind"] == "2d":
        from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
        w = ElasticWAVE(vs, vp, rho, s["dx"], s["dz"], s["dt"], s["isx"], s["isz"], s["rsx"], s["rsz"], s["nt"],
                        s["N"], s["freq"], dtype)
        w.SetADEPML2D(list(s.get("surface", [True] * 4)), par)
        if s["aea"]:
            w.AEA_init()
        if s["scheme"] == "RSG":
            src = GOLD[s["name"] + "__source"]
            for it in range(s["nt"]):
                w.update_RSG(it, float(src[it]))
        elif per_step:
            step = w.update_SSG_VS if s["scheme"] == "VS" else w.update_SSG_SV
            for it in range(s["nt"]):
                if s["aea"]:
                    w.AEA()
                step(it)
        else:
            w.run(s["nt"], scheme=s["scheme"], free_surface=bool(s["aea"]))
    else:
        if s["kind"] == "TENSOR":
            from seiswave_taichi_b200.Elastic3D_SSG_Tensor import ElasticWAVE
            w = ElasticWAVE(vs, vp, rho, s["dx"], s["dy"], s["dz"], s["dt"], s["isx"], s["isy"], s["isz"],
                            np.asarray(s["rsx"]), np.asarray(s["rsy"]), np.asarray(s["rsz"]), s["MT"],
                            s["src_scale"], s["nt"], s["N"], s["freq"], dtype, exact=exact)
        elif s["kind"] == "CPML":
            from seiswave_taichi_b200.Elastic3D_SSG_CPML import ElasticWAVE
            w = ElasticWAVE(vs, vp, rho, s["dx"], s["dy"], s["dz"], s["dt"], s["isx"], s["isy"], s["isz"],
                            s["rsx"], s["rsy"], s["rsz"], s["nt"], s["N"], s["freq"], dtype, exact=exact)
        else:
            from seiswave_taichi_b200.Elastic3D_SSG_SPML import ElasticWAVE
            w = ElasticWAVE(vs, vp, rho, s["dx"], s["dy"], s["dz"], s["dt"], s["isx"], s["isy"], s["isz"],
                            s["rsx"], s["rsy"], s["rsz"], s["nt"], s["N"], s["freq"], s["src_scale"], dtype,
                            exact=exact)
        w.SetADEPML3D([True] * 6, par)
        if per_step:
            step = w.update_SSG_SPML if s["kind"] == "SPML" else w.update_SSG
            for it in range(s["nt"]):
                step(it)
        else:
            w.run(s["nt"])
    torch.cuda.synchronize()
    return w


def _check(s, w, bitwise):
    from cases import to_np
    worst = 0.0
    for f in _fields(s) + ("data",):
        got = to_np(getattr(w, f))
        ref = GOLD[f"{s['name']}_{f}"]
        assert got.shape == ref.shape, f
        if bitwise:
            np.testing.assert_array_equal(got, ref, err_msg=f"{s['name']} {f}")
        err = _rel(got, ref)
        worst = max(worst, err)
        assert err <= TOL, f"{s['name']} {f}: relative L2 {err:.3e} > {TOL}"
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize("s", SPECS, ids=_ids)
def test_gpu_within_gate_of_reference(cuda, s):
    """North-star gate: seismograms and final wavefields within relative L2
    1e-5 of the reference's own run (exact and fast numeric modes)."""
    _check(s, _product_run(s), bitwise=False)
    if s["kind"] in ("TENSOR", "CPML"):
        fast = _product_run(s, exact=False)
        from cases import to_np
        assert _rel(to_np(fast.data), GOLD[s["name"] + "_data"]) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("s", SPECS, ids=_ids)
def test_gpu_bit_identical_to_reference(cuda, s):
    """The default exact numeric mode equals the reference's own run bit for
    bit: whole-loop run() (one CUDA graph) and the per-step reference API."""
    _check(s, _product_run(s), bitwise=True)
    _check(s, _product_run(s, per_step=True), bitwise=True)
