"""Learned thin absorbing layer (2D).

* The GPU training kernels' loss and gradient equal the float64 numpy
  reference (oracle/mlp_ref.py) within 2e-4 relative (float32 sums), and the
  forward kernel its outputs within 1e-5.
* Layer tables: every cell within 6 of an edge, once, with its nearest face.
* An untrained network (zero output layer) leaves the thin CPML run unchanged
  bit for bit.
* The gradient of the trace misfit through the whole time loop (correction
  adjoints + time-step adjoints + sw_mlp_backward) equals central finite
  differences within 1%.
* Trained through the time loop on two models and sources, the network lowers
  the trace error of the thin 6-cell CPML against a large-domain run on a
  model and source it was not trained on (by at least 5%)."""
import numpy as np
import pytest
import torch

from oracle import mlp_ref

NI, NH = 51, 32


def test_layer_cells_cover_the_edge_once():
    from seiswave_taichi_b200.learned_abc import layer_cells
    cell, face, dep = layer_cells(20, 17)
    assert len(set(cell.tolist())) == cell.size
    i, j = cell // 17, cell % 17
    d = np.minimum.reduce([i, 19 - i, j, 16 - j])
    np.testing.assert_array_equal(d, dep)
    assert cell.size == 20 * 17 - 8 * 5
    assert set(face.tolist()) == {0, 1, 2, 3}


def test_mlp_reference_gradient_by_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(NH * NI + NH + NH * NH + NH + 5 * NH + 5) * 0.2
    X = rng.standard_normal((7, NI))
    Y = rng.standard_normal((7, 5))
    _, g = mlp_ref.loss_and_grad(p, X, Y, NI, NH)
    for q in rng.integers(0, p.size, 12):
        e = np.zeros_like(p)
        e[q] = 1e-6
        fd = (mlp_ref.loss_and_grad(p + e, X, Y, NI, NH)[0] - mlp_ref.loss_and_grad(p - e, X, Y, NI, NH)[0]) / 2e-6
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q]))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 300, 5000])
def test_mlp_kernels_match_reference(cuda, n):
    from seiswave_taichi_b200.learned_abc import mlp_forward, mlp_grad, NP
    rng = np.random.default_rng(n)
    p = (rng.standard_normal(NP) * 0.3).astype(np.float32)
    X = rng.standard_normal((n, NI)).astype(np.float32)
    Y = rng.standard_normal((n, 5)).astype(np.float32)
    loss, grad = mlp_grad(torch.as_tensor(p, device="cuda"), torch.as_tensor(X, device="cuda"),
                          torch.as_tensor(Y, device="cuda"))
    l_ref, g_ref = mlp_ref.loss_and_grad(p, X, Y, NI, NH)
    assert abs(float(loss) - l_ref) <= 2e-4 * abs(l_ref)
    g = grad.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - g_ref) <= 2e-4 * np.linalg.norm(g_ref)
    y = mlp_forward(torch.as_tensor(p, device="cuda"), torch.as_tensor(X, device="cuda")).cpu().numpy()
    y_ref = mlp_ref.forward(p, X, NI, NH)[0]
    assert np.abs(y - y_ref).max() <= 1e-5 * max(1.0, np.abs(y_ref).max())


def _model(n, seed):
    from seiswave_taichi_b200.synthetic import layered
    return layered((n, n), 2500.0, 4000.0, nlayers=5, seed=seed, anomaly=0.05)


@pytest.mark.gpu
def test_untrained_network_is_plain_thin_cpml(cuda):
    from seiswave_taichi_b200.learned_abc import LearnedABC2D, _solver
    vp, vs, rho = _model(96, 1)
    abc = LearnedABC2D(scale=(1e-3, 1e-3, 1e3, 1e3, 1e3))
    a = _solver(vp, vs, rho, 10.0, 1e-3, 40, 50, 150, 2, 15.0, 6, "explosive", 1e5)
    b = _solver(vp, vs, rho, 10.0, 1e-3, 40, 50, 150, 2, 15.0, 6, "explosive", 1e5)
    abc.run(a, 150, net=True)
    abc.run(b, 150, net=False)
    for f in ("vx", "vz", "sxx", "szz", "sxz"):
        np.testing.assert_array_equal(getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy())


def test_band_receivers():
    from seiswave_taichi_b200.learned_abc import band_receivers
    i, j = band_receivers(40, 30, 8, 12)
    d = np.minimum.reduce([i, 39 - i, j, 29 - j])
    assert d.min() == 8 and d.max() == 11
    assert i.size == (40 - 16) * (30 - 16) - (40 - 24) * (30 - 24)


@pytest.mark.gpu
def test_rollout_gradient_matches_finite_differences(cuda):
    from seiswave_taichi_b200 import learned_abc as LA
    vp, vs, rho = _model(72, 5)
    _, _, rolls = LA.train_rollout([(vp, vs, rho, 30, 40)], nt=160, iters=0, pad=120)
    r = rolls[0]
    gen = torch.Generator(device="cuda").manual_seed(0)
    r.abc.params.add_(torch.randn(r.abc.params.shape, generator=gen, device="cuda") * 0.05)
    _, g = r.loss_and_grad()
    flat = g.reshape(-1)
    for q in torch.topk(flat.abs(), 3).indices.tolist():
        f, k = divmod(q, LA.NP)
        old = float(r.abc.params[f, k])
        eps = 1e-2 * max(1e-3, abs(old))
        r.abc.params[f, k] = old + eps
        lp = r.forward(True)
        r.abc.params[f, k] = old - eps
        lm = r.forward(True)
        r.abc.params[f, k] = old
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - float(flat[q])) <= 1e-2 * abs(float(flat[q])), (q, fd, float(flat[q]))


@pytest.mark.gpu
def test_trained_layer_reduces_trace_error(cuda):
    from seiswave_taichi_b200 import learned_abc as LA
    n, nt = 96, 300
    cases = []
    for seed, (sx, sz) in ((11, (34, 52)), (12, (60, 40))):
        vp, vs, rho = _model(n, seed)
        cases.append((vp, vs, rho, sx, sz))
    abc, hist, _ = LA.train_rollout(cases, nt=nt, iters=150, lr=2e-3, pad=150)
    assert hist[-1] < hist[0]
    vp, vs, rho = _model(n, 99)
    r = LA.evaluate(abc, vp, vs, rho, 47, 45, nt, pad=150)
    assert r["net_traces"] < 0.95 * r["plain_traces"], r
