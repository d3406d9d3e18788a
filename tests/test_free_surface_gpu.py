"""The 2D free-surface mode: after AEA_init (lambda = 0 and rho halved on the
first N x layers), every step first zeroes sxx on the x layer N (AEA), as the
reference's driver loop `AEA(); update_SSG_VS(i)` does.  The mode folds the
hooks into the stress passes of run(); it must equal the per-step loop with
the host hook and the oracle driven the same way, bit for bit."""
import numpy as np
import pytest

from cases import case2d, oracle2d, product2d, to_np

pytestmark = pytest.mark.gpu

F2 = ("vx", "vz", "sxx", "szz", "sxz")


def _sid(scheme):
    import seiswave_taichi_b200._native as N
    return {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]


def _eq(name, a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and np.array_equal(a, b), (name, int((a != b).sum()))


@pytest.mark.parametrize("scheme", ["VS", "SV"])
@pytest.mark.parametrize("kw", [dict(), dict(MT="explosive", src_scale=1e5, nrec=6)],
                         ids=["force", "moment"])
def test_free_surface_run_equals_hooked_loop_and_oracle(cuda, scheme, kw):
    nt, N = 120, 2
    c = case2d(nt=nt, N=N, surface=(False, True, True, True), **kw)
    step = {"VS": "update_SSG_VS", "SV": "update_SSG_SV"}[scheme]
    a = product2d(c)
    a.AEA_init()
    a.set_free_surface(True)
    a.run(50, scheme=scheme)
    a.run(nt - 50, it0=50, scheme=scheme)
    b = product2d(c)
    b.AEA_init()
    for it in range(nt):
        b.AEA()
        getattr(b, step)(it)
    for f in F2:
        _eq(f, to_np(getattr(a, f)), to_np(getattr(b, f)))
    _eq("data", to_np(a.data), to_np(b.data))
    # per-step calls in free-surface mode apply the hook themselves
    d = product2d(c)
    d.AEA_init()
    d.set_free_surface(True)
    for it in range(nt):
        getattr(d, step)(it)
    for f in F2:
        _eq(f, to_np(getattr(d, f)), to_np(getattr(b, f)))
    # the oracle, hooked by hand
    o = oracle2d(c, wavelet=to_np(a._wavelets[_sid(scheme)]).astype(np.float32))
    o.lam[:N] = 0
    o.rho[:N] *= 0.5
    for it in range(nt):
        o.sxx[N, :] = 0
        o.run(scheme, it, 1)
    for f in F2:
        _eq(f, to_np(getattr(a, f)), getattr(o, f))
    _eq("data", to_np(a.data), o.data)
    assert np.abs(o.vx).max() > 0


def test_free_surface_mode_off_again(cuda):
    c = case2d(nt=60, N=2)
    a = product2d(c)
    a.run(60, free_surface=True)
    a.reset()
    a.run(60, free_surface=False)
    b = product2d(c)
    b.run(60)
    for f in F2:
        _eq(f, to_np(getattr(a, f)), to_np(getattr(b, f)))


F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


@pytest.mark.parametrize("kw", [dict(scheme="TENSOR"), dict(scheme="TENSOR", src_on_surface=True),
                                dict(scheme="CPML"), dict(scheme="SPML"), dict(scheme="TENSOR", path="fused"),
                                dict(scheme="TENSOR", dtype=np.float64)],
                         ids=["tensor", "tensor-src-k=N", "cpml", "spml", "tensor-fused", "tensor-f64"])
def test_free_surface_3d_equals_hooked_loop_and_oracle(cuda, kw):
    """3D: szz = 0 on the z layer N before every step (Elastic3D_SSG_Tensor.py:
    160-163) as one kernel of the captured step; a moment source on that layer
    is injected after the zeroing, and the fused path steps aside."""
    from cases import case3d, oracle3d, product3d
    kw = dict(kw)
    on_surface = kw.pop("src_on_surface", False)
    path = kw.pop("path", None)
    nt = 70
    c = case3d(nt=nt, N=2, **kw)
    if on_surface:
        c["isz"] = c["N"]
    N = c["N"]
    a = product3d(c)
    a.AEA_init()
    if path:
        a._build_plan().set_path(path)
    a.set_free_surface(True)
    a.run(30)
    a.run(nt - 30, it0=30)
    b = product3d(c)
    b.AEA_init()
    for it in range(nt):
        b.AEA()
        b._step(it)
    for f in F3:
        _eq(f, to_np(getattr(a, f)), to_np(getattr(b, f)))
    _eq("data", to_np(a.data), to_np(b.data))
    o = oracle3d(c, wavelet=to_np(a._wavelet).astype(np.float32))
    o.lam[:, :, :N] = 0
    o.rho[:, :, :N] *= 0.5
    for it in range(nt):
        o.szz[:, :, N] = 0
        o.run(it, 1)
    for f in F3:
        _eq(f, to_np(getattr(a, f)), getattr(o, f))
    _eq("data", to_np(a.data), o.data)
    assert np.abs(o.vx).max() > 0


def test_free_surface_3d_refused_by_the_adjoint(cuda):
    import torch
    from cases import case3d, product3d
    c = case3d(scheme="TENSOR", nt=20, N=2)
    w = product3d(c)
    w.set_free_surface(True)
    vp, vs, rho = (torch.as_tensor(c[k], device="cuda") for k in ("vp", "vs", "rho"))
    with pytest.raises(RuntimeError, match="free-surface"):
        w.forward_op(vp, vs, rho, checkpoint_every=10)
