"""Parity at the benchmark workloads' full sizes.

* 2D homogeneous P-SV, 400^2, 1000 steps (explosive source, 200 receivers):
  the whole loop equals the oracle bit for bit.
* 3D double couple, 200^3, 1000 steps: the whole loop against the oracle
  bit for bit (about a minute on 16 host cores), fields and traces.
* 3D heterogeneous thrust belt, 400x400x200, 2000 steps: the oracle cannot
  run this loop in a test's time, so its first 160 steps on the full grid
  are compared with it bit for bit (all host cores).
* For both 3D workloads the whole loop is also checked by exact and by
  tolerance properties:
  - the TMA-staged kernels (the default path) equal the plain two-pass
    kernels, an independent implementation of the same IEEE operations that
    the small-grid tests check against the oracle, bit for bit over the whole
    loop, fields and traces; a second staged run with another work-unit size
    equals them too;
  - linearity in the source amplitude and the opt-in fast numeric mode, within
    1e-4 relative L2 of the traces: ten times the float32 run's own error
    against float64 at these sizes (1.3e-5 at 200^3, 1.0e-5 at 400x400x200).
    Doubling the source is not bit-exact over a long loop: the far-field tail
    ahead of the numerical front grows out of subnormal values, whose
    rounding does not commute with doubling, and those differences reach the
    normal range through the roundings of later sums;
  - the wavefield stays finite and the traces are not zero.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
F2 = ("vx", "vz", "sxx", "szz", "sxz")
TOL = 1e-4


def _np(t):
    return t.detach().cpu().numpy()


def _eq(name, a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (name, a.shape, b.shape)
    bad = int((a.view(np.uint32 if a.dtype == np.float32 else np.uint64) !=
               b.view(np.uint32 if b.dtype == np.float32 else np.uint64)).sum())
    assert bad == 0, (name, bad)


def _solver3d(cfg, exact=True, scale=1.0):
    from seiswave_taichi_b200.Elastic3D_SSG_Tensor import ElasticWAVE
    w = ElasticWAVE(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dy"], cfg["dz"], cfg["dt"], cfg["isx"],
                    cfg["isy"], cfg["isz"], cfg["rsx"], cfg["rsy"], cfg["rsz"], cfg["MT"],
                    cfg["src_scale"] * scale, cfg["nt"], cfg["accuracy"], cfg["freq"], torch.float32,
                    exact=exact)
    w.SetADEPML3D(cfg["surface"], cfg["pml"])
    return w


def _oracle3d(cfg, wavelet):
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    return O.Oracle3D("TENSOR", cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dy"], cfg["dz"], cfg["dt"],
                      cfg["isx"], cfg["isy"], cfg["isz"], cfg["rsx"], cfg["rsy"], cfg["rsz"], cfg["nt"],
                      cfg["accuracy"], cfg["freq"], cfg["surface"], cfg["pml"], MT=cfg["MT"],
                      src_scale=cfg["src_scale"], wavelet=wavelet)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_2d_full_loop_equals_oracle(cuda):
    """400^2, 1000 steps, the whole loop against the oracle bit for bit."""
    from oracle import oracle as O
    from seiswave_taichi_b200 import _native as N
    from seiswave_taichi_b200 import synthetic as S
    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE, moment_2d
    cfg = S.config1()
    w = ElasticWAVE(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dz"], cfg["dt"], cfg["isx"], cfg["isz"],
                    cfg["rsx"], cfg["rsz"], cfg["nt"], cfg["accuracy"], cfg["freq"], torch.float32, MT=cfg["MT"],
                    src_scale=cfg["src_scale"])
    w.SetADEPML2D(cfg["surface"], cfg["pml"])
    w.run(cfg["nt"])
    torch.cuda.synchronize()
    wav = _np(w._wavelets[N.SW2D_SSG_VS]).astype(np.float32)
    table = cfg["rsx"].reshape(-1) * cfg["shape"][1] + cfg["rsz"].reshape(-1)
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle2D(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dz"], cfg["dt"], cfg["isx"], cfg["isz"],
                   int(cfg["rsx"].reshape(-1)[0]), int(cfg["rsz"].reshape(-1)[0]), cfg["nt"], cfg["accuracy"],
                   cfg["freq"], cfg["surface"], cfg["pml"], wavelet=wav, MT=moment_2d(cfg["MT"]),
                   rec_index=table)
    o.run("VS", 0, cfg["nt"])
    for f in F2:
        _eq(f, _np(getattr(w, f)), getattr(o, f))
    _eq("data", _np(w.data), o.data)
    assert np.abs(o.data).max() > 0


@pytest.mark.parametrize("which,steps", [("config2", 1000), ("config3", 160)])
def test_3d_full_grid(cuda, which, steps):
    from seiswave_taichi_b200 import synthetic as S
    cfg = getattr(S, which)()
    nt = cfg["nt"]
    # the first steps on the full grid against the oracle, bit for bit
    w = _solver3d(cfg)
    plan = w._build_plan()
    assert plan.info()["path"] == "staged"
    wav = _np(w._wavelet).astype(np.float32)
    w.run(steps)
    torch.cuda.synchronize()
    o = _oracle3d(cfg, wav).run(0, steps)
    for f in F3:
        _eq(f, _np(getattr(w, f)), getattr(o, f))
    _eq("data", _np(w.data)[:steps], o.data[:steps])
    del o
    # the whole loop on the staged path
    if nt > steps:
        w.run(nt - steps, it0=steps)
    plan.status()
    ref = {f: _np(getattr(w, f)) for f in F3}
    ref["data"] = _np(w.data)
    for f in F3:
        assert np.isfinite(ref[f]).all(), f
    assert np.abs(ref["data"]).max() > 0
    # the plain two-pass kernels, and the staged kernels with another
    # work-unit size, over the same loop: identical bits
    chunk = plan.info()["staged_chunk"]
    for path, chunk_len in (("two_pass", 0), ("staged", 6 if chunk != 6 else 12)):
        w.reset()
        plan.set_path(path, chunk_len)
        w.run(nt)
        plan.status()
        for f in F3:
            _eq(f"{path} {f}", _np(getattr(w, f)), ref[f])
        _eq(f"{path} data", _np(w.data), ref["data"])
    del w
    # twice the source: twice the traces within the tolerance
    w2 = _solver3d(cfg, scale=2.0)
    w2.run(nt)
    w2._plan.status()
    e = _rel(_np(w2.data), 2.0 * ref["data"].astype(np.float64))
    assert e <= TOL, ("linearity", e)
    del w2
    # the fast numeric mode over the whole loop
    wf = _solver3d(cfg, exact=False)
    wf.run(nt)
    wf._plan.status()
    e = _rel(_np(wf.data), ref["data"])
    assert e <= TOL, ("fast mode", e)
