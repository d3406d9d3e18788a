"""The adjoints' last step on the host: the per-cell sums of the gradient with
respect to each update's material coefficient (dt/rho averages, lam + 2 mu,
lam, the averaged mu) are chained to (rho, lam, mu) by
adjoint.coefficient_chain (2D VS), coefficient_chain_sv (2D SV) and
coefficient_chain3 (3D).  Each must equal torch autograd's vector-Jacobian
product of sum_k G_k * coef_k(rho, lam, mu) in float64 on the CPU, with the
coefficients built from the reference's averages
(Elastic2D_CPML.py:154,159,174-176,190 for VS, :225,238,252-253,266 for SV,
Elastic3D_SSG_Tensor.py:178-310 for 3D)."""
import pytest
import torch

from seiswave_taichi_b200 import adjoint as A


def _model(shape, seed):
    g = torch.Generator().manual_seed(seed)
    rho = 1800 + 600 * torch.rand(shape, generator=g, dtype=torch.float64)
    lam = 4e9 + 4e9 * torch.rand(shape, generator=g, dtype=torch.float64)
    mu = 2e9 + 2e9 * torch.rand(shape, generator=g, dtype=torch.float64)
    return rho, lam, mu


def _sums(shape, n, seed):
    g = torch.Generator().manual_seed(seed)
    return [torch.randn(shape, generator=g, dtype=torch.float64) for _ in range(n)]


def _vjp(coefs, G, rho, lam, mu):
    r, l, m = (t.clone().requires_grad_(True) for t in (rho, lam, mu))
    loss = sum((gk * ck).sum() for gk, ck in zip(G, coefs(r, l, m)))
    return torch.autograd.grad(loss, (r, l, m), allow_unused=True)


def _check(got, want):
    for name, a, b in zip(("rho", "lam", "mu"), got, want):
        b = torch.zeros_like(a) if b is None else b
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-12 * float(b.abs().max() + 1e-300)), name


def test_chain_2d_vs():
    rho, lam, mu = _model((9, 11), 0)
    G = _sums((9, 11), 5, 1)

    def coefs(r, l, m):
        r4 = 0.25 * (r[:-1, :-1] + r[:-1, 1:] + r[1:, 1:] + r[1:, :-1])
        lhx = 0.5 * (l[:-1] + l[1:])
        mhx = 0.5 * (m[:-1] + m[1:])
        mhz = 0.5 * (m[:, :-1] + m[:, 1:])
        return 1 / r, 1 / r4, lhx + 2 * mhx, lhx, mhz

    Gc = [G[0], G[1][:-1, :-1], G[2][:-1], G[3][:-1], G[4][:, :-1]]
    _check(A.coefficient_chain(rho, G), _vjp(coefs, Gc, rho, lam, mu))


def test_chain_2d_sv():
    rho, lam, mu = _model((10, 8), 2)
    G = _sums((10, 8), 5, 3)

    def coefs(r, l, m):
        r2 = (r[:-1] + r[1:]) / 2
        rz = 0.5 * (r[:, :-1] + r[:, 1:])
        m4 = 0.25 * (m[:-1, :-1] + m[:-1, 1:] + m[1:, 1:] + m[1:, :-1])
        return 1 / r2, 1 / rz, l + 2 * m, l, m4

    Gc = [G[0][:-1], G[1][:, :-1], G[2], G[3], G[4][:-1, :-1]]
    _check(A.coefficient_chain_sv(rho, G), _vjp(coefs, Gc, rho, lam, mu))


@pytest.mark.parametrize("shape", [(6, 7, 5), (4, 4, 4)])
def test_chain_3d(shape):
    rho, lam, mu = _model(shape, 4)
    G = _sums(shape, 8, 5)
    # the averaged-mu sums vanish where their stencil would leave the grid,
    # as the kernels' sums do (the update ranges lie inside)
    G[5][-1], G[5][:, -1], G[6][-1], G[6][:, -1] = 0, 0, 0, 0
    G[7][:, -1], G[7][:, :, -1] = 0, 0

    def coefs(r, l, m):
        ry = 0.5 * (r[:, :-1] + r[:, 1:])
        r4 = 0.25 * (r[:-1, :-1] + r[:-1, 1:] + r[1:, 1:] + r[1:, :-1])
        lhx = 0.5 * (l[:-1] + l[1:])
        mhx = 0.5 * (m[:-1] + m[1:])
        mxy = 0.25 * (m[:-1, 1:] + 2 * m[:-1, :-1] + m[1:, :-1])
        mxz = 0.25 * (2 * m[:-1, :-1] + m[1:, :-1] + m[:-1, 1:])
        myz = 0.25 * (m[:, 1:, :-1] + 2 * m[:, :-1, :-1] + m[:, :-1, 1:])
        return 1 / r, 1 / ry, 1 / r4, lhx + 2 * mhx, lhx, mxy, mxz, myz

    Gc = [G[0], G[1][:, :-1], G[2][:-1, :-1], G[3][:-1], G[4][:-1], G[5][:-1, :-1], G[6][:-1, :-1],
          G[7][:, :-1, :-1]]
    _check(A.coefficient_chain3(rho, G), _vjp(coefs, Gc, rho, lam, mu))
