"""The 2D persistent path (sw_run as one cooperative launch for all its
steps, phases separated by a bounded grid barrier) against the two-launch
path and the oracle, bit for bit: VS and SV, orders 2 and 4, float32 and
float64, point-force and moment-tensor sources, runs split in pieces, and a
receiver table that records a stress (the gather after the stress phase)."""
import ctypes as C

import numpy as np
import pytest
import torch

from cases import case2d, oracle2d, product2d, to_np

pytestmark = pytest.mark.gpu

F2 = ("vx", "vz", "sxx", "szz", "sxz")
MEM = ("memory_sxx_dx", "memory_sxz_dx", "memory_dvx_dx", "memory_dvz_dx", "memory_sxz_dz", "memory_szz_dz",
       "memory_dvz_dz", "memory_dvx_dz")


def _pid(scheme):
    import seiswave_taichi_b200._native as N
    return {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]


def _state(w):
    out = {f: to_np(getattr(w, f)).copy() for f in F2 + MEM}
    out["data"] = to_np(w.data).copy()
    return out


def _same(a, b):
    for k in a:
        assert a[k].tobytes() == b[k].tobytes(), k


def _run(c, scheme, path, pieces):
    w = product2d(c)
    plan = w._plan(_pid(scheme))
    plan.set_path(path)
    assert plan.info()["path"] == path
    it = 0
    for n in pieces:
        w.run(n, it0=it, scheme=scheme)
        it += n
    plan.status(w._stream())
    return w


CASES = [dict(N=2), dict(N=4), dict(N=2, dtype=np.float64), dict(N=2, MT="explosive", src_scale=1e5),
         dict(N=4, MT=[[1.0, 0.4], [0.4, -0.7]], src_scale=1e5, dtype=np.float64)]


@pytest.mark.parametrize("kw", CASES)
@pytest.mark.parametrize("scheme", ["VS", "SV"])
def test_persistent_equals_two_launch_path(cuda, kw, scheme):
    nt = 140
    c = case2d(nt=nt, nrec=7, **kw)
    a = _run(c, scheme, "persistent", [nt])
    b = _run(c, scheme, "two_pass", [nt])
    sa, sb = _state(a), _state(b)
    _same(sa, sb)
    assert np.abs(sa["data"]).max() > 0


@pytest.mark.parametrize("scheme", ["VS", "SV"])
def test_persistent_split_runs_equal_oracle(cuda, scheme):
    nt = 150
    c = case2d(nt=nt, nrec=5, MT="explosive", src_scale=1e5)
    w = _run(c, scheme, "persistent", [1, 48, 60, 41])
    wav = to_np(w._wavelets[_pid(scheme)]).astype(np.float32)
    o = oracle2d(c, wavelet=wav)
    o.run(scheme, 0, nt)
    for f in F2:
        got, ref = to_np(getattr(w, f)), np.asarray(getattr(o, f))
        assert got.shape == ref.shape and np.array_equal(got, ref), f
    assert np.array_equal(to_np(w.data), np.asarray(o.data))


def test_persistent_path_is_opt_in(cuda):
    c = case2d(nt=20)
    w = product2d(c)
    plan = w._plan(_pid("VS"))
    assert plan.info()["path"] == "two_pass"
    plan.set_path("persistent")
    assert plan.info()["path"] == "persistent"


@pytest.mark.parametrize("mt", [None, "explosive"])
def test_persistent_stress_receivers(cuda, mt):
    """Receivers recording sxx: the gather runs after the stress phase, and
    a moment-tensor source is then injected at the start of every step."""
    import seiswave_taichi_b200._native as N
    nt = 120
    kw = dict(MT=mt, src_scale=1e5) if mt else {}
    c = case2d(nt=nt, nrec=6, **kw)
    w = product2d(c)
    base = w._plan(_pid("VS"))
    d = N.Desc2D()
    C.memmove(C.byref(d), C.byref(base._desc), C.sizeof(d))
    d.rec.field = 2  # sxx
    out = {}
    for path in ("persistent", "two_pass"):
        plan = N.Plan(d, base._keep, False)
        plan.set_path(path)
        w.reset()
        plan.run(0, nt, True, w._stream())
        plan.status(w._stream())
        out[path] = _state(w)
        plan.close()
    _same(out["persistent"], out["two_pass"])
    assert np.abs(out["persistent"]["data"]).max() > 0
    torch.cuda.synchronize()
