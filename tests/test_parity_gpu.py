"""Parity of the CUDA path against the CPU oracle (GPU tests).

Each case runs the drop-in class through the C ABI on the GPU and the oracle
on the CPU from the same inputs.  Two comparisons per case:

* shared wavelet: the oracle is handed the product's per-step source table,
  so both sides evaluate identical expressions in identical order (kernels are
  built with -fmad=false and IEEE division, the oracle with
  -ffp-contract=off).  The wavefields, memory variables and traces must agree
  BIT FOR BIT.
* independent wavelet: the oracle tabulates its own wavelet (its exp() may
  differ from numpy's by an ulp); traces and wavefields must agree to the
  north-star tolerance, relative L2 <= 1e-5.
"""
import numpy as np
import pytest

from cases import case2d, case3d, oracle2d, oracle3d, product2d, product3d, to_np
from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5
F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
F2 = ("vx", "vz", "sxx", "szz", "sxz")


def _assert_equal(name, got, ref):
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    bad = np.argwhere(got != ref)
    if bad.size:
        q = tuple(bad[0])
        raise AssertionError(f"{name}: {len(bad)} values differ, first at {q}: gpu={got[q]!r} "
                             f"oracle={ref[q]!r}; rel_l2={rel_l2(got, ref):.3e}")


def _run3d(c, steps, use_run):
    w = product3d(c)
    wav = to_np(w._build_plan() and w._wavelet).astype(np.float32)
    o = oracle3d(c, wavelet=wav)
    if use_run:
        w.run(steps)
    else:
        for it in range(steps):
            w._step(it)
    o.run(0, steps)
    return w, o


CASES3 = [
    dict(scheme="TENSOR", N=2),
    dict(scheme="TENSOR", N=5, shape=(44, 40, 46)),
    dict(scheme="TENSOR", N=3, hetero=False, surface=(True, True, True, True, False, True)),
    dict(scheme="CPML", N=2),
    dict(scheme="CPML", N=4, shape=(42, 40, 38)),
    # z extents whose staged tiles are 40 wide (nz=76: a partial last tile)
    dict(scheme="TENSOR", N=2, shape=(36, 34, 76)),
    dict(scheme="CPML", N=3, shape=(34, 38, 40)),
    dict(scheme="SPML", N=2, shape=(36, 34, 80)),
    dict(scheme="SPML", N=2),
    dict(scheme="SPML", N=3, shape=(38, 42, 40)),
    dict(scheme="TENSOR", N=2, dtype=np.float64),
    dict(scheme="CPML", N=2, dtype=np.float64),
]


@pytest.mark.parametrize("kw", CASES3, ids=lambda k: "-".join(f"{v}" for v in k.values()))
@pytest.mark.parametrize("use_run", [False, True], ids=["step", "run"])
def test_3d_bitwise(cuda, kw, use_run):
    c = case3d(nt=90, **kw)
    w, o = _run3d(c, 90, use_run)
    for f in F3:
        _assert_equal(f, to_np(getattr(w, f)), getattr(o, f))
    _assert_equal("data", to_np(w.data), o.data)
    if c["scheme"] == "SPML":
        for name in o.SPLIT:
            _assert_equal(name, to_np(getattr(w, name)), o.memory(name))
    else:
        for name in o.MEM_CPML:
            _assert_equal(name, to_np(getattr(w, name)), o.memory(name))
    assert np.abs(o.vx).max() > 0, "the wave never reached the grid"


@pytest.mark.parametrize("scheme", ["TENSOR", "CPML", "SPML"])
def test_3d_independent_wavelet(cuda, scheme):
    c = case3d(scheme=scheme, N=2, nt=120)
    w = product3d(c)
    w.run(120)
    o = oracle3d(c).run(0, 120)
    for f in F3:
        assert rel_l2(to_np(getattr(w, f)), getattr(o, f)) <= TOL_L2, f
    assert rel_l2(to_np(w.data), o.data) <= TOL_L2


CASES2 = [
    dict(N=2), dict(N=3, shape=(90, 64)), dict(N=5, shape=(70, 84)), dict(N=2, hetero=False),
    dict(N=2, surface=(True, True, False, True)), dict(N=2, dtype=np.float64),
]


@pytest.mark.parametrize("kw", CASES2, ids=lambda k: "-".join(f"{v}" for v in k.values()))
@pytest.mark.parametrize("scheme", ["VS", "SV", "RSG"])
def test_2d_bitwise(cuda, kw, scheme):
    nt = 150
    c = case2d(nt=nt, **kw)
    w = product2d(c)
    import seiswave_taichi_b200._native as N
    plan_id = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV, "RSG": N.SW2D_RSG}[scheme]
    w._plan(plan_id)
    wav = to_np(w._wavelets[plan_id]) if scheme != "RSG" else None
    o = oracle2d(c, wavelet=None if wav is None else wav.astype(np.float32))
    if scheme == "RSG":
        from seiswave_taichi_b200 import BaseFun
        src = BaseFun.series("ricker", nt, c["dt"], c["freq"], 1.0)
        for it in range(nt):
            w.update_RSG(it, float(src[it]))
        o.run("RSG", 0, nt, rsg_sources=src.astype(np.float64))
    else:
        for it in range(nt):
            (w.update_SSG_VS if scheme == "VS" else w.update_SSG_SV)(it)
        o.run(scheme, 0, nt)
    for f in F2:
        _assert_equal(f, to_np(getattr(w, f)), getattr(o, f))
    if scheme != "RSG":
        _assert_equal("data", to_np(w.data), o.data)
    for name in ("memory_sxx_dx", "memory_sxz_dx", "memory_dvx_dx", "memory_dvz_dx", "memory_sxz_dz",
                 "memory_szz_dz", "memory_dvz_dz", "memory_dvx_dz"):
        _assert_equal(name, to_np(getattr(w, name)), o.memory(name))


MT2 = [
    dict(MT="explosive", nrec=12, src_scale=1e5),
    dict(MT=[[0.4, -1.0], [-1.0, 0.7]], nrec=7, src_scale=1e5, N=3, shape=(90, 64)),
    dict(MT="explosive", nrec=5, src_scale=1e5, dtype=np.float64),
]


@pytest.mark.parametrize("kw", MT2, ids=lambda k: "-".join(f"{v}" for v in k.values())[:40])
@pytest.mark.parametrize("scheme", ["VS", "SV"])
@pytest.mark.parametrize("graph", [False, True])
def test_2d_moment_tensor_bitwise(cuda, kw, scheme, graph):
    """2D moment-tensor / explosive source with a receiver table: per-step
    calls (source injected before each velocity pass) and the graph-captured
    run (next step's source folded into the stress pass) both equal the
    oracle bit for bit."""
    nt = 160
    c = case2d(nt=nt, **kw)
    w = product2d(c)
    import seiswave_taichi_b200._native as N
    plan_id = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]
    w._plan(plan_id)
    wav = to_np(w._wavelets[plan_id]).astype(np.float32)
    o = oracle2d(c, wavelet=wav)
    if graph:
        w.run(nt, scheme=scheme)
    else:
        for it in range(nt):
            (w.update_SSG_VS if scheme == "VS" else w.update_SSG_SV)(it)
    o.run(scheme, 0, nt)
    for f in F2:
        _assert_equal(f, to_np(getattr(w, f)), getattr(o, f))
    assert w.data.shape == o.data.shape
    _assert_equal("data", to_np(w.data), o.data)
    assert np.abs(o.data).max() > 0


def test_2d_run_graph_matches_steps(cuda):
    c = case2d(nt=200)
    a = product2d(c)
    for it in range(200):
        a.update_SSG_VS(it)
    b = product2d(c)
    b.run(200)
    for f in F2:
        _assert_equal(f, to_np(getattr(b, f)), to_np(getattr(a, f)))
    _assert_equal("data", to_np(b.data), to_np(a.data))


def test_2d_independent_wavelet(cuda):
    c = case2d(nt=300, shape=(100, 90))
    w = product2d(c)
    w.run(300)
    o = oracle2d(c).run("VS", 0, 300)
    for f in F2:
        assert rel_l2(to_np(getattr(w, f)), getattr(o, f)) <= TOL_L2, f
    assert rel_l2(to_np(w.data), o.data) <= TOL_L2
