"""Adjoint of the 3D SSG-CPML moment-tensor loop.

Gradient oracle: oracle/torch_twin3d.py, a float64 PyTorch restatement of the
step differentiated by torch.autograd, pinned to the C++ oracle's forward.
Tolerances: float64 adjoint vs twin relative L2 <= 1e-9; central finite
differences of the forward_op misfit within 2e-3 (the 3D traces are stored in
float32, as in the reference, which limits the differences' accuracy)."""
import numpy as np
import pytest
import torch

from cases import case3d, oracle3d, product3d, to_np
from oracle.oracle import rel_l2


def _case(nt=60):
    return case3d(shape=(20, 18, 22), N=2, scheme="TENSOR", nt=nt, npml=5, dtype=np.float64, seed=4)


def _wavelet(c):
    from seiswave_taichi_b200 import BaseFun
    return BaseFun.series("ricker2", c["nt"], c["dt"], c["freq"], c["src_scale"], t0=0.03)


def _twin(c, wav):
    from oracle.torch_twin3d import TwinTensor3D
    o = oracle3d(c, wavelet=wav)
    nx, ny, nz = c["shape"]
    rec = (np.asarray(c["rsx"]).reshape(-1) * ny + np.asarray(c["rsy"]).reshape(-1)) * nz + \
        np.asarray(c["rsz"]).reshape(-1)
    return o, TwinTensor3D(o, wav, rec)


def _force_case(nt=60):
    return case3d(shape=(20, 18, 22), N=2, scheme="CPML", nt=nt, npml=5, dtype=np.float64, seed=7)


def _force_twin(c, wav):
    from oracle.torch_twin3d import TwinForce3D
    o = oracle3d(c, wavelet=wav)
    nx, ny, nz = c["shape"]
    rec = (np.asarray(c["rsx"]).reshape(-1) * ny + np.asarray(c["rsy"]).reshape(-1)) * nz + \
        np.asarray(c["rsz"]).reshape(-1)
    return o, TwinForce3D(o, wav, rec)


def test_force_twin3d_forward_matches_oracle():
    from seiswave_taichi_b200 import BaseFun
    c = _force_case(nt=40)
    wav = BaseFun.series("ricker", 40, c["dt"], c["freq"], 1000)
    o, tw = _force_twin(c, wav)
    d = tw.traces(torch.as_tensor(o.rho), torch.as_tensor(o.lam), torch.as_tensor(o.mu), 40)
    o.run(0, 40)
    assert rel_l2(d.numpy().astype(np.float32), np.asarray(o.data).reshape(d.shape)) <= 1e-6
    for f, t in zip(("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"), tw.final):
        assert rel_l2(t.numpy(), getattr(o, f)) <= 1e-13, f
    assert np.abs(o.data).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("K", [25, 60])
def test_force_adjoint3d_matches_twin_autograd(cuda, K):
    """The point-force (Elastic3D_SSG_CPML) scheme: the same adjoint kernels
    plus the force's dt/rho term at the source cell."""
    from seiswave_taichi_b200.adjoint import Adjoint3D
    c = _force_case()
    w = product3d(c)
    drv = Adjoint3D(w, K)
    d = drv.forward()
    nrec = d.shape[1] if d.dim() > 1 else 1
    W = np.random.default_rng(1).standard_normal(tuple(d.shape))
    g_rho, g_lam, g_mu = drv.backward(torch.as_tensor(W, device="cuda"))
    wav = to_np(w._wavelet).astype(np.float32)
    o, tw = _force_twin(c, wav)
    rho = torch.tensor(o.rho, requires_grad=True)
    lam = torch.tensor(o.lam, requires_grad=True)
    mu = torch.tensor(o.mu, requires_grad=True)
    dt = tw.traces(rho, lam, mu, c["nt"]).reshape(tuple(d.shape))
    assert rel_l2(to_np(d).astype(np.float64), dt.detach().numpy()) <= 1e-6
    (dt * torch.as_tensor(W)).sum().backward()
    for name, mine, ref in (("rho", g_rho, rho.grad), ("lam", g_lam, lam.grad), ("mu", g_mu, mu.grad)):
        e = rel_l2(to_np(mine), ref.numpy())
        assert e <= 1e-9, (name, e, nrec)
    # the source cell's rho gradient carries the force term
    s = tw.src
    assert abs(float(g_rho[s])) > 0


def test_twin3d_forward_matches_oracle():
    c = _case(nt=40)
    wav = _wavelet(c)
    o, tw = _twin(c, wav)
    d = tw.traces(torch.as_tensor(o.rho), torch.as_tensor(o.lam), torch.as_tensor(o.mu), 40)
    o.run(0, 40)
    assert rel_l2(d.numpy().astype(np.float32), o.data) <= 1e-6
    for f, t in zip(("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"), tw.final):
        assert rel_l2(t.numpy(), getattr(o, f)) <= 1e-13, f
    assert np.abs(o.data).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("K", [25, 60])
def test_adjoint3d_matches_twin_autograd(cuda, K):
    from seiswave_taichi_b200.adjoint import Adjoint3D
    c = _case()
    w = product3d(c)
    drv = Adjoint3D(w, K)
    d = drv.forward()
    nrec = d.shape[1]
    W = np.random.default_rng(0).standard_normal((c["nt"], nrec))
    g_rho, g_lam, g_mu = drv.backward(torch.as_tensor(W, device="cuda"))
    wav = to_np(w._wavelet).astype(np.float32)
    np.testing.assert_array_equal(wav, _wavelet(c))
    o, tw = _twin(c, wav)
    rho = torch.tensor(o.rho, requires_grad=True)
    lam = torch.tensor(o.lam, requires_grad=True)
    mu = torch.tensor(o.mu, requires_grad=True)
    dt = tw.traces(rho, lam, mu, c["nt"])
    assert rel_l2(to_np(d).astype(np.float64), dt.detach().numpy()) <= 1e-6
    (dt * torch.as_tensor(W)).sum().backward()
    for name, mine, ref in (("rho", g_rho, rho.grad), ("lam", g_lam, lam.grad), ("mu", g_mu, mu.grad)):
        e = rel_l2(to_np(mine), ref.numpy())
        assert e <= 1e-9, (name, e)


@pytest.mark.gpu
def test_forward_op3d_finite_differences(cuda):
    c = _case(nt=70)
    w = product3d(c)
    dev = "cuda"
    vp0 = torch.as_tensor(c["vp"], dtype=torch.float64, device=dev)
    vs0 = torch.as_tensor(c["vs"], dtype=torch.float64, device=dev)
    rh0 = torch.as_tensor(c["rho"], dtype=torch.float64, device=dev)
    d_obs = w.forward_op(vp0 * 1.02, vs0 * 0.99, rh0).detach().double()
    vp = vp0.clone().requires_grad_(True)
    vs = vs0.clone().requires_grad_(True)
    rh = rh0.clone().requires_grad_(True)
    loss = 0.5 * ((w.forward_op(vp, vs, rh, checkpoint_every=30).double() - d_obs) ** 2).sum()
    loss.backward()
    x = np.linspace(0, 1, c["shape"][0])[:, None, None]
    y = np.linspace(0, 1, c["shape"][1])[None, :, None]
    z = np.linspace(0, 1, c["shape"][2])[None, None, :]
    sm = torch.as_tensor(np.sin(2 * np.pi * x) * np.cos(np.pi * y) * np.sin(np.pi * z), device=dev)
    dvp, dvs, drh = 40.0 * sm, 25.0 * sm.flip(0), 15.0 * sm.flip(1)
    pred = float((vp.grad * dvp).sum() + (vs.grad * dvs).sum() + (rh.grad * drh).sum())
    eps = 2e-2
    f = lambda s: float(0.5 * ((w.forward_op(vp0 + s * dvp, vs0 + s * dvs, rh0 + s * drh).double() - d_obs)
                               ** 2).sum())
    fd = (f(eps) - f(-eps)) / (2 * eps)
    assert abs(pred) > 0
    assert abs(fd - pred) <= 2e-3 * abs(pred), (fd, pred)
