"""Run-level checkpoint/resume and checked runs (seiswave_taichi_b200.state):
the .npz format round trip and its refusals (truncated or corrupt file,
another configuration, a missing or reshaped array) on CPU tensors, the
segmenting of run_checked with a fake solver whose state turns non-finite,
and the stability number of the staggered scheme; on the GPU, a run saved
half way and resumed in a new solver equals the uninterrupted run bit for bit
(2D, 3D CPML, 3D split PML), a NaN in the density is caught within one
segment, and a state is never loaded into another configuration."""
import numpy as np
import pytest
import torch

from seiswave_taichi_b200 import pml as P
from seiswave_taichi_b200 import state

CFG = {"class": "T", "grid": [4, 5], "dtype": "torch.float32"}


def _arrays(seed=0):
    g = torch.Generator().manual_seed(seed)
    return {"vx": torch.randn(4, 5, generator=g), "mem0": torch.randn(2, 3, 5, generator=g), "mem1": None,
            "data": torch.randn(7, generator=g, dtype=torch.float64)}


def test_round_trip(tmp_path):
    p = tmp_path / "s.npz"
    a = _arrays(0)
    state.write(p, a, {"config": CFG, "it": 42})
    b = _arrays(1)
    meta = state.read(p, b, CFG)
    assert meta["it"] == 42
    for k in a:
        if a[k] is None:
            assert b[k] is None
        else:
            assert torch.equal(a[k], b[k]) and a[k].dtype == b[k].dtype
    assert not (tmp_path / "s.npz.tmp").exists()


def _refused(p, arrays, config, match):
    before = {k: None if v is None else v.clone() for k, v in arrays.items()}
    with pytest.raises(ValueError, match=match):
        state.read(p, arrays, config)
    for k, v in arrays.items():
        assert (v is None and before[k] is None) or torch.equal(v, before[k]), k


def test_refusals_leave_the_state_untouched(tmp_path):
    p = tmp_path / "s.npz"
    state.write(p, _arrays(0), {"config": CFG, "it": 3})
    raw = p.read_bytes()
    # truncated and corrupt files
    t = tmp_path / "trunc.npz"
    t.write_bytes(raw[: len(raw) // 2])
    _refused(t, _arrays(1), CFG, "unreadable")
    c = tmp_path / "junk.npz"
    c.write_bytes(b"\x00" * 100)
    _refused(c, _arrays(1), CFG, "unreadable")
    _refused(tmp_path / "absent.npz", _arrays(1), CFG, "unreadable")
    # another configuration
    _refused(p, _arrays(1), dict(CFG, grid=[4, 6]), "another configuration")
    a = _arrays(1)
    a["vx"] = torch.zeros(4, 6)
    _refused(p, a, dict(CFG, grid=[4, 6]), "another configuration")
    # a missing array, one the solver lacks, another shape, another dtype
    a = _arrays(1)
    a["extra"] = torch.zeros(2)
    _refused(p, a, CFG, "lacks extra")
    a = _arrays(1)
    a["mem1"] = torch.zeros(3)
    _refused(p, a, CFG, "lacks mem1")
    a = _arrays(1)
    a["mem0"] = None
    _refused(p, a, CFG, "does not have")
    a = _arrays(1)
    a["vx"] = torch.zeros(5, 4)
    _refused(p, a, CFG, "vx is")
    a = _arrays(1)
    a["data"] = torch.zeros(7, dtype=torch.float32)
    _refused(p, a, CFG, "data is")
    # not a checkpoint at all
    np.savez(tmp_path / "other.npz", x=np.zeros(3))
    _refused(tmp_path / "other.npz", _arrays(1), CFG, "not a solver checkpoint")


class _FakeSolver:
    """run() advances a step counter; the state turns non-finite at bad_at."""

    def __init__(self, bad_at=None):
        self.calls, self.next, self.bad_at = [], None, bad_at

    def run(self, n, it0=0, **kw):
        assert self.next is None or it0 == self.next
        self.calls.append((it0, n, kw))
        self.next = it0 + n

    def check_finite(self):
        return 7 if self.bad_at is not None and self.next > self.bad_at else 0


def test_run_checked_segments_and_stops():
    s = _FakeSolver()
    state.run_checked(s, 250, 10, 100, scheme="SV")
    assert [(a, b) for a, b, _ in s.calls] == [(10, 100), (110, 100), (210, 50)]
    assert all(kw == {"scheme": "SV"} for _, _, kw in s.calls)
    s = _FakeSolver(bad_at=130)
    with pytest.raises(state.NonFiniteError) as e:
        state.run_checked(s, 300, 0, 100)
    assert e.value.step == 199 and e.value.count == 7 and len(s.calls) == 2
    with pytest.raises(ValueError):
        state.run_checked(_FakeSolver(), 10, 0, 0)


def test_courant_number():
    c = [9 / 8, -1 / 24]
    # config 1: vp 3000, dt 1 ms, dx = dz = 10 m: 0.3 * sqrt(2) * 7/6
    assert P.courant_check(3000.0, 1e-3, (10.0, 10.0), c) == pytest.approx(0.3 * 2 ** 0.5 * 7 / 6, rel=1e-12)
    assert P.courant_check(3000.0, 1e-3, (10.0,) * 3, c) == pytest.approx(0.3 * 3 ** 0.5 * 7 / 6, rel=1e-12)


# ---- GPU ------------------------------------------------------------------------
def _fields(w):
    names = ("vx", "vz", "sxx", "szz", "sxz") if len(w.gridsize) == 2 else \
        ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
    return {f: getattr(w, f).cpu().numpy() for f in names}


def _resume_equals_uninterrupted(tmp_path, make, nt, cut, run_kw=None):
    run_kw = run_kw or {}
    a = make()
    a.run(nt, **run_kw)
    b = make()
    b.run(cut, **run_kw)
    b.save_state(tmp_path / "cut.npz", cut)
    del b
    c = make()
    it = c.load_state(tmp_path / "cut.npz")
    assert it == cut
    c.run(nt - it, it0=it, **run_kw)
    fa, fc = _fields(a), _fields(c)
    for f in fa:
        assert np.array_equal(fa[f].view(np.uint32), fc[f].view(np.uint32)), f
    assert np.array_equal(a.data.cpu().numpy(), c.data.cpu().numpy())
    return a


@pytest.mark.gpu
def test_2d_resume_bitwise(cuda, tmp_path):
    from cases import case2d, product2d
    c = case2d(nt=120, N=2, MT="explosive", src_scale=1e5, nrec=6)
    a = _resume_equals_uninterrupted(tmp_path, lambda: product2d(c), 120, 50, {"scheme": "VS"})
    assert 0 < a.courant() < 1


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["TENSOR", "SPML"])
def test_3d_resume_bitwise(cuda, tmp_path, scheme):
    from cases import case3d, product3d
    c = case3d(scheme=scheme, nt=80, N=2)
    a = _resume_equals_uninterrupted(tmp_path, lambda: product3d(c), 80, 37)
    assert 0 < a.courant() < 1


@pytest.mark.gpu
def test_state_refused_for_another_configuration(cuda, tmp_path):
    from cases import case3d, product3d
    a = product3d(case3d(scheme="TENSOR", nt=30, N=2))
    a.run(10)
    a.save_state(tmp_path / "a.npz", 10)
    b = product3d(case3d(scheme="TENSOR", nt=30, N=3))
    b.run(5)
    before = b.vx.clone()
    with pytest.raises(ValueError, match="another configuration"):
        b.load_state(tmp_path / "a.npz")
    assert torch.equal(before, b.vx)


@pytest.mark.gpu
def test_run_checked_catches_a_nan_in_the_model(cuda):
    from cases import case3d, product3d
    c = case3d(scheme="TENSOR", nt=90, N=2)
    w = product3d(c)
    w._build_plan()
    w.rho[c["isx"] + 2, c["isy"], c["isz"]] = float("nan")
    with pytest.raises(state.NonFiniteError) as e:
        w.run_checked(every=30)
    assert e.value.step in (29, 59, 89) and e.value.count > 0
    ok = product3d(c)
    ok.run_checked(every=30)
    assert ok.check_finite() == 0
