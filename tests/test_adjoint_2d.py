"""Adjoint of the 2D SSG_VS and SSG_SV time loops (moment-tensor source).

Gradient oracle: oracle/torch_twin2d.py, a float64 PyTorch restatement of the
step differentiated by torch.autograd, itself pinned to the C++ oracle's
forward.  Tolerances: float64 adjoint vs twin relative L2 <= 1e-9 (both are
exact discrete gradients, up to float64 rounding of different operation
orders); central finite differences (float64) agree with the adjoint's
directional derivative within 1e-5; the float32 adjoint is within 2e-3 of the
float64 one."""
import numpy as np
import pytest
import torch

from cases import case2d, oracle2d, product2d, to_np
from oracle.oracle import rel_l2


def _case(dtype=np.float64, nt=120, **kw):
    kw.setdefault("MT", [[0.6, -0.8], [-0.8, 1.0]])
    return case2d(shape=(48, 40), N=2, npml=8, nt=nt, dtype=dtype, nrec=6, src_scale=1e5, seed=3, **kw)


SCHEMES = ["VS", "SV"]


def _twin(c, wav, scheme="VS"):
    from oracle.torch_twin2d import TwinSV2D, TwinVS2D
    from seiswave_taichi_b200.Elastic2D_CPML import moment_2d
    o = oracle2d(c, wavelet=wav)
    rec = np.asarray(c["rsx"]).reshape(-1) * c["shape"][1] + np.asarray(c["rsz"]).reshape(-1)
    return o, (TwinSV2D if scheme == "SV" else TwinVS2D)(o, moment_2d(c["MT"]), wav, rec)


def _sid(scheme):
    import seiswave_taichi_b200._native as N
    return {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]


def _wavelet(c):
    from seiswave_taichi_b200 import BaseFun
    return BaseFun.series("ricker2", c["nt"], c["dt"], c["freq"], c["src_scale"],
                          t0=np.float32(1.5 / float(c["freq"])))


@pytest.mark.parametrize("scheme", SCHEMES)
def test_twin_forward_matches_oracle(scheme):
    c = _case(nt=60)
    wav = _wavelet(c)
    o, tw = _twin(c, wav, scheme)
    rho = torch.as_tensor(o.rho)
    d = tw.traces(rho, torch.as_tensor(o.lam), torch.as_tensor(o.mu), 60)
    o.run(scheme, 0, 60)
    assert rel_l2(d.numpy(), o.data) <= 1e-13
    for f, t in zip(("vx", "vz", "sxx", "szz", "sxz"), tw.final):
        assert rel_l2(t.numpy(), getattr(o, f)) <= 1e-13, f
    assert np.abs(o.data).max() > 0


def _gpu_grads(c, weights, K, scheme="VS"):
    from seiswave_taichi_b200.adjoint import Adjoint2D
    w = product2d(c)
    drv = Adjoint2D(w, K, scheme)
    d = drv.forward()
    g = drv.backward(torch.as_tensor(weights, device="cuda", dtype=w.rho.dtype))
    return w, d, g


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("K", [50, 120])
def test_adjoint_matches_twin_autograd(cuda, K, scheme):
    c = _case()
    rng = np.random.default_rng(0)
    W = rng.standard_normal((c["nt"], 6))
    w, d, (g_rho, g_lam, g_mu) = _gpu_grads(c, W, K, scheme)
    wav = to_np(w._wavelets[_sid(scheme)]).astype(np.float32)
    o, tw = _twin(c, wav, scheme)
    rho = torch.tensor(o.rho, requires_grad=True)
    lam = torch.tensor(o.lam, requires_grad=True)
    mu = torch.tensor(o.mu, requires_grad=True)
    dt = tw.traces(rho, lam, mu, c["nt"])
    assert rel_l2(to_np(d), dt.detach().numpy()) <= 1e-12
    (dt * torch.as_tensor(W)).sum().backward()
    for name, mine, ref in (("rho", g_rho, rho.grad), ("lam", g_lam, lam.grad), ("mu", g_mu, mu.grad)):
        e = rel_l2(to_np(mine), ref.numpy())
        assert e <= 1e-9, (name, e)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES)
def test_forward_op_finite_differences(cuda, scheme):
    """Central differences of 0.5*||d(m) - d_obs||^2 along a random smooth
    direction in (vp, vs, rho), float64, against the autograd gradient."""
    c = _case(nt=150, hetero=True)
    w = product2d(c)
    dev = "cuda"
    vp0 = torch.as_tensor(c["vp"], dtype=torch.float64, device=dev)
    vs0 = torch.as_tensor(c["vs"], dtype=torch.float64, device=dev)
    rh0 = torch.as_tensor(c["rho"], dtype=torch.float64, device=dev)
    d_obs = w.forward_op(vp0 * 1.02, vs0 * 0.99, rh0, scheme=scheme).detach()
    vp = vp0.clone().requires_grad_(True)
    vs = vs0.clone().requires_grad_(True)
    rh = rh0.clone().requires_grad_(True)
    loss = 0.5 * ((w.forward_op(vp, vs, rh, checkpoint_every=40, scheme=scheme) - d_obs) ** 2).sum()
    loss.backward()
    rng = np.random.default_rng(1)
    x = np.linspace(0, 1, c["shape"][0])[:, None]
    z = np.linspace(0, 1, c["shape"][1])[None, :]
    dirs = []
    for _ in range(3):
        a, b = rng.uniform(1, 3, 2)
        dirs.append(torch.as_tensor(np.sin(a * np.pi * x) * np.cos(b * np.pi * z), device=dev))
    dvp, dvs, drh = 30.0 * dirs[0], 20.0 * dirs[1], 15.0 * dirs[2]
    pred = float((vp.grad * dvp).sum() + (vs.grad * dvs).sum() + (rh.grad * drh).sum())
    eps = 1e-3
    f = lambda s: float(0.5 * ((w.forward_op(vp0 + s * dvp, vs0 + s * dvs, rh0 + s * drh, scheme=scheme)
                                - d_obs) ** 2).sum())
    fd = (f(eps) - f(-eps)) / (2 * eps)
    assert abs(pred) > 0
    assert abs(fd - pred) <= 1e-5 * abs(pred), (fd, pred)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES)
def test_float32_adjoint_close_to_float64(cuda, scheme):
    W = np.random.default_rng(2).standard_normal((120, 6))
    _, _, g64 = _gpu_grads(_case(np.float64), W, 60, scheme)
    _, _, g32 = _gpu_grads(_case(np.float32), W, 60, scheme)
    for a, b in zip(g32, g64):
        assert rel_l2(to_np(a).astype(np.float64), to_np(b)) <= 2e-3
