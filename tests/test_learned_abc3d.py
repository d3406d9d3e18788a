"""Learned thin absorbing layer (3D moment-tensor solver).

* sw3d_mlp_grad / sw3d_mlp_forward equal the float64 numpy reference
  (oracle/mlp_ref.py, 33 inputs, 9 outputs) within 2e-4 / 1e-5 relative.
* Layer tables: every cell within 6 of a face, once, with its nearest face.
* The correction kernel (sw3d_abc_correct) gives every layer
  cell's nine corrections within 1e-5 relative of the float64 numpy network
  on that cell's inputs (sw3d_abc_features), for cells of all six faces.
* An untrained network leaves the thin CPML run unchanged bit for bit.
* The through-the-loop gradient (correction adjoints + 3D step adjoints +
  sw3d_mlp_backward) equals central finite differences of the float32
  rollout's loss along its own direction within 2%.
* Trained through the time loop on two models and sources, the network lowers
  the receiver-band trace error of the thin 6-cell CPML on an unseen model
  and source by at least 2%."""
import numpy as np
import pytest
import torch

from oracle import mlp_ref

NI, NH, NO = 33, 32, 9


def test_layer_cells3_cover_the_faces_once():
    from seiswave_taichi_b200.learned_abc3d import layer_cells3
    cell, face, dep = layer_cells3(16, 15, 17)
    assert len(set(cell.tolist())) == cell.size
    assert cell.size == 16 * 15 * 17 - 4 * 3 * 5
    k = cell % 17
    j = (cell // 17) % 15
    i = cell // (15 * 17)
    np.testing.assert_array_equal(np.minimum.reduce([i, 15 - i, j, 14 - j, k, 16 - k]), dep)
    assert set(face.tolist()) == set(range(6))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 700])
def test_mlp3_kernels_match_reference(cuda, n):
    import ctypes as C
    from seiswave_taichi_b200 import _native as N
    P = N.SW_ABC3_PARAMS
    rng = np.random.default_rng(n)
    p = (rng.standard_normal(P) * 0.3).astype(np.float32)
    X = rng.standard_normal((n, NI)).astype(np.float32)
    Y = rng.standard_normal((n, NO)).astype(np.float32)
    tp, tx, ty = (torch.as_tensor(a, device="cuda") for a in (p, X, Y))
    grad = torch.zeros(P, device="cuda")
    loss = torch.zeros(1, device="cuda")
    out = torch.empty((n, NO), device="cuda")
    lib = N.load()
    N.check(lib.sw3d_mlp_grad(C.c_void_p(tp.data_ptr()), C.c_void_p(tx.data_ptr()), C.c_void_p(ty.data_ptr()), n,
                              C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()), None))
    N.check(lib.sw3d_mlp_forward(C.c_void_p(tp.data_ptr()), C.c_void_p(tx.data_ptr()), n,
                                 C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    l_ref, g_ref = mlp_ref.loss_and_grad(p, X, Y, NI, NH, NO)
    assert abs(float(loss) - l_ref) <= 2e-4 * abs(l_ref)
    g = grad.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - g_ref) <= 2e-4 * np.linalg.norm(g_ref)
    y_ref = mlp_ref.forward(p, X, NI, NH, NO)[0]
    assert np.abs(out.cpu().numpy() - y_ref).max() <= 1e-5 * max(1.0, np.abs(y_ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(20, 18, 22), (17, 16, 19)])
def test_correction_equals_reference_network(cuda, shape):
    from seiswave_taichi_b200.learned_abc3d import FIELDS, LearnedABC3D, solver3d
    vp, vs, rho = _model(max(shape), 3)
    vp, vs, rho = (m[: shape[0], : shape[1], : shape[2]].copy() for m in (vp, vs, rho))
    rng = np.random.default_rng(sum(shape))
    p = (rng.standard_normal((6, mlp_ref_params())) * 0.3).astype(np.float32)
    scale = (1e-3,) * 3 + (1e3,) * 6
    oscale = tuple(float(v) for v in rng.uniform(0.5, 2.0, 9))
    abc = LearnedABC3D(p, scale=scale, oscale=oscale)
    w = solver3d(vp, vs, rho, 10.0, 1e-3, shape[0] // 2, shape[1] // 2, shape[2] // 2, 10)
    w._build_plan()
    for f, s_ in zip(FIELDS, scale):
        getattr(w, f).copy_(torch.as_tensor(rng.standard_normal(shape).astype(np.float32) * s_, device="cuda"))
    X = abc.features(w).cpu().numpy().astype(np.float64)
    before = [getattr(w, f).clone() for f in FIELDS]
    abc.correct(w)
    torch.cuda.synchronize()
    _, delta = abc._cache[w.gridsize]
    got = delta.cpu().numpy().astype(np.float64)
    from seiswave_taichi_b200.learned_abc3d import layer_cells3
    cell, face, _ = layer_cells3(*shape)
    want = np.zeros_like(got)
    for f in range(6):
        m = face == f
        want[m] = mlp_ref.forward(p[f].astype(np.float64), X[m], NI, NH, NO)[0] * np.asarray(oscale)
    assert set(face.tolist()) == set(range(6))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-5, err
    # the correction is added to the fields of the layer cells
    for q, f in enumerate(FIELDS):
        d = (getattr(w, f) - before[q]).reshape(-1).cpu().numpy().astype(np.float64)
        tol = 1e-6 * float(before[q].abs().max()) + 1e-5 * np.abs(want[:, q]).max()
        assert np.abs(d[cell] - want[:, q]).max() <= tol, f


def mlp_ref_params():
    from seiswave_taichi_b200 import _native as N
    return N.SW_ABC3_PARAMS


def _model(n, seed):
    from seiswave_taichi_b200.synthetic import layered
    return layered((n, n, n), 2500.0, 4000.0, nlayers=4, seed=seed, anomaly=0.05)


@pytest.mark.gpu
def test_untrained_network_is_plain_thin_cpml_3d(cuda):
    from seiswave_taichi_b200.learned_abc3d import LearnedABC3D, solver3d
    vp, vs, rho = _model(28, 1)
    abc = LearnedABC3D(scale=(1e-3,) * 3 + (1e3,) * 6)
    a = solver3d(vp, vs, rho, 10.0, 1e-3, 12, 14, 15, 60)
    b = solver3d(vp, vs, rho, 10.0, 1e-3, 12, 14, 15, 60)
    abc.run(a, 60, net=True)
    abc.run(b, 60, net=False)
    for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
        np.testing.assert_array_equal(getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy())


@pytest.mark.gpu
def test_rollout3d_gradient_matches_finite_differences(cuda):
    """Directional derivative along the normalised gradient: central
    differences of the float32 rollout's loss against |grad|."""
    from seiswave_taichi_b200 import learned_abc3d as LA
    vp, vs, rho = _model(30, 5)
    _, _, rolls = LA.train_rollout3d([(vp, vs, rho, 13, 16, 15)], nt=90, iters=0, pad=50)
    r = rolls[0]
    gen = torch.Generator(device="cuda").manual_seed(0)
    r.abc.params.add_(torch.randn(r.abc.params.shape, generator=gen, device="cuda") * 0.05)
    _, g = r.loss_and_grad()
    gn = float(torch.linalg.norm(g))
    u = g / gn
    base = r.abc.params.clone()
    eps = 2e-2
    r.abc.params.copy_(base + eps * u)
    lp = r.forward(True)
    r.abc.params.copy_(base - eps * u)
    lm = r.forward(True)
    r.abc.params.copy_(base)
    fd = (lp - lm) / (2 * eps)
    assert gn > 0
    assert abs(fd - gn) <= 2e-2 * gn, (fd, gn)


@pytest.mark.gpu
def test_trained_3d_layer_reduces_trace_error(cuda):
    from seiswave_taichi_b200 import learned_abc3d as LA
    n, nt = 36, 120
    cases = []
    for seed, s in ((11, (14, 20, 18)), (12, (22, 15, 20))):
        vp, vs, rho = _model(n, seed)
        cases.append((vp, vs, rho) + s)
    abc, hist, _ = LA.train_rollout3d(cases, nt=nt, iters=60, lr=2e-3)
    assert hist[-1] < hist[0]
    vp, vs, rho = _model(n, 99)
    r = LA.evaluate3d(abc, vp, vs, rho, n // 2, n // 2 - 3, n // 2 + 2, nt)
    assert r["net_traces"] < 0.98 * r["plain_traces"], r
