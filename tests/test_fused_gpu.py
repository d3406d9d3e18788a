"""The fused single-pass 3D kernel (TMA-fed, ping-pong buffers) against the
oracle, bit for bit.  sw_run takes the fused path for float 3D CPML plans with
N <= 3 and nz % 4 == 0; these cases cover chunk seams, tile edges that are
not multiples of the tile, odd step counts (last step on the two-pass path),
both source kinds, slabs on or off, and the constant-divisor fast path."""
import numpy as np
import pytest

from cases import case3d, oracle3d, product3d, to_np

pytestmark = pytest.mark.gpu

F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


def _check(w, o):
    for f in F3:
        g, r = to_np(getattr(w, f)), getattr(o, f)
        if not np.array_equal(g, r):
            bad = np.argwhere(g != r)
            q = tuple(bad[0])
            raise AssertionError(f"{f}: {len(bad)} cells differ, first {q}: gpu={g[q]!r} oracle={r[q]!r}")
    assert np.array_equal(to_np(w.data), o.data), "receiver traces differ"
    for name in o.MEM_CPML:
        assert np.array_equal(to_np(getattr(w, name)), o.memory(name)), name


CASES = [
    dict(scheme="TENSOR", N=2, shape=(40, 36, 44)),
    dict(scheme="TENSOR", N=2, shape=(37, 29, 52)),
    dict(scheme="CPML", N=2, shape=(41, 38, 40)),
    dict(scheme="TENSOR", N=3, shape=(34, 30, 48)),
    dict(scheme="CPML", N=3, shape=(36, 35, 36)),
    dict(scheme="TENSOR", N=1, shape=(30, 33, 40)),
    dict(scheme="TENSOR", N=2, shape=(40, 36, 44), surface=(True, False, True, True, False, True)),
    dict(scheme="TENSOR", N=2, shape=(36, 34, 72), hetero=False),
]


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(str(v) for v in k.values()))
@pytest.mark.parametrize("steps,chunk", [(70, 0), (71, 5), (64, 9)])
def test_fused_bitwise(cuda, kw, steps, chunk):
    c = case3d(nt=80, **kw)
    w = product3d(c)
    plan = w._build_plan()
    plan.set_path("fused", chunk)
    info = plan.info()
    assert info["fused"] and info["path"] == "fused", info
    wav = to_np(w._wavelet).astype(np.float32)
    o = oracle3d(c, wavelet=wav)
    w.run(steps)
    plan.status()
    o.run(0, steps)
    _check(w, o)


def test_fused_constant_divisor_verified(cuda):
    c = case3d(nt=10, dx=10.0, dy=12.5, dz=7.5)
    w = product3d(c)
    plan = w._build_plan()
    plan.set_path("fused")
    info = plan.info()
    assert info["fused"] and info["fast_div"], info


def test_fused_in_two_runs_equals_one(cuda):
    """Splitting the loop (run(30) then run(33, it0=30)) gives the same state."""
    c = case3d(nt=80, shape=(38, 34, 40))
    a = product3d(c)
    a._build_plan().set_path("fused")
    a.run(63)
    b = product3d(c)
    b._build_plan().set_path("fused")
    b.run(30)
    b.run(33, it0=30)
    for f in F3:
        assert np.array_equal(to_np(getattr(a, f)), to_np(getattr(b, f))), f
    assert np.array_equal(to_np(a.data), to_np(b.data))


def test_fused_matches_two_pass(cuda):
    c = case3d(nt=80, shape=(44, 40, 48), N=2)
    a = product3d(c)
    a._build_plan().set_path("fused")
    a.run(80)
    b = product3d(c)
    b._build_plan().set_path("two_pass")
    b.run(80)
    for f in F3:
        assert np.array_equal(to_np(getattr(a, f)), to_np(getattr(b, f))), f
    assert np.array_equal(to_np(a.data), to_np(b.data))


@pytest.mark.parametrize("kw", CASES, ids=lambda k: "-".join(str(v) for v in k.values()))
@pytest.mark.parametrize("steps,chunk", [(70, 0), (71, 7), (33, 13)])
def test_staged_bitwise(cuda, kw, steps, chunk):
    c = case3d(nt=80, **kw)
    w = product3d(c)
    plan = w._build_plan()
    plan.set_path("staged", chunk)
    assert plan.info()["path"] == "staged"
    wav = to_np(w._wavelet).astype(np.float32)
    o = oracle3d(c, wavelet=wav)
    w.run(steps)
    plan.status()
    o.run(0, steps)
    _check(w, o)


def test_staged_is_default_and_per_step(cuda):
    c = case3d(nt=40, shape=(40, 36, 44))
    w = product3d(c)
    assert w._build_plan().info()["path"] == "staged"
    wav = to_np(w._wavelet).astype(np.float32)
    o = oracle3d(c, wavelet=wav)
    for it in range(40):
        w.update_SSG(it)
    o.run(0, 40)
    _check(w, o)
