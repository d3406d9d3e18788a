"""The drop-in for src/Elastic2D_sparse.py: the dense solver with that file's
VS source (Ricker(nt, dt, f0, 1), Elastic2D_sparse.py:170) and the memory
variables as struct members; bit for bit against the oracle driven with that
wavelet, and SV / RSG unchanged from the dense class."""
import numpy as np
import pytest
import torch

from cases import case2d, oracle2d, product2d, to_np

pytestmark = pytest.mark.gpu

F2 = ("vx", "vz", "sxx", "szz", "sxz")
MEM = ("sxx_dx", "sxz_dx", "dvx_dx", "dvz_dx", "sxz_dz", "szz_dz", "dvz_dz", "dvx_dz")


def _sparse(c):
    from seiswave_taichi_b200.Elastic2D_sparse import ElasticWAVE
    w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"], c["rsx"], c["rsz"],
                    c["nt"], c["N"], c["freq"], torch.float64 if c["dtype"] == np.float64 else torch.float32)
    w.SetADEPML2D(c["surface"], c["pml"])
    return w


@pytest.mark.parametrize("kw", [dict(N=2), dict(N=3, dtype=np.float64)])
def test_sparse_vs_equals_oracle_with_ricker(cuda, kw):
    import seiswave_taichi_b200._native as N
    from seiswave_taichi_b200 import BaseFun
    nt = 150
    c = case2d(nt=nt, **kw)
    w = _sparse(c)
    for it in range(nt):
        w.update_SSG_VS(it)
    wav = to_np(w._wavelets[N.SW2D_SSG_VS])
    ref = BaseFun.series("ricker", nt, c["dt"], c["freq"], 1.0)
    assert np.array_equal(wav.astype(np.float32), np.asarray(ref, np.float32))
    o = oracle2d(c, wavelet=np.asarray(ref, np.float32))
    o.run("VS", 0, nt)
    for f in F2:
        assert np.array_equal(to_np(getattr(w, f)), getattr(o, f)), f
    assert np.array_equal(to_np(w.data), o.data)
    for m in MEM:
        assert np.array_equal(to_np(getattr(w.memory, m)), o.memory("memory_" + m)), m
    assert np.abs(o.vz).max() > 0


def test_sparse_sv_matches_dense(cuda):
    c = case2d(nt=100)
    a, b = _sparse(c), product2d(c)
    a.run(100, scheme="SV")
    b.run(100, scheme="SV")
    for f in F2:
        assert np.array_equal(to_np(getattr(a, f)), to_np(getattr(b, f))), f
