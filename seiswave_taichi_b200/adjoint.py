"""Gradients of a 2D seismogram misfit with respect to vp, vs and rho
(no reference counterpart; the forward is Elastic2D_CPML.py:128-200).

    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    w = ElasticWAVE(vs, vp, rho, dx, dz, dt, isx, isz, rsx, rsz, nt, N, f0, MT="explosive")
    w.SetADEPML2D(surface, pml)
    d = w.forward_op(vp_t, vs_t, rho_t)            # (nt, nrec), differentiable
    loss = 0.5 * ((d - d_obs) ** 2).sum()
    loss.backward()                                # vp_t.grad, vs_t.grad, rho_t.grad

The forward run keeps the state every `checkpoint_every` steps.  The backward
pass walks the segments from last to first: it restores the segment's
checkpoint, re-runs the segment with snapshots (sw2d_record) and steps the
hand-written adjoint back over it (sw2d_adjoint_run), accumulating per-cell
gradients of the step's material coefficients, which are chained here to
rho, lambda, mu and then to vp, vs, rho (mu = rho vs^2,
lambda = rho (vp^2 - 2 vs^2)).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


class Adjoint2D:
    """Checkpointed forward + adjoint driver for one 2D solver, scheme "VS"
    (update_SSG_VS, vz traces) or "SV" (update_SSG_SV, vx traces)."""

    SCHEMES = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}

    def __init__(self, wave, checkpoint_every: int = 100, scheme: str = "VS"):
        if wave.MT is None:
            raise ValueError("the 2D adjoint needs the moment-tensor source (MT=...)")
        if scheme not in self.SCHEMES:
            raise ValueError(f"scheme must be 'VS' or 'SV', not {scheme!r}")
        self.w = wave
        self.scheme = scheme
        self.K = int(checkpoint_every)
        if self.K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.plan = wave._plan(self.SCHEMES[scheme])
        n = C.c_int64(0)
        N.check(N.load().sw2d_snapshot_elems(self.plan.handle, C.byref(n)))
        self.snap_elems = int(n.value)
        self.checkpoints = []

    # -- state copies --------------------------------------------------------
    def _state(self):
        w = self.w
        return [getattr(w, f) for f in ("vx", "vz", "sxx", "szz", "sxz")] + [m for m in w._mem if m is not None]

    def forward(self, nt: int | None = None) -> torch.Tensor:
        """Zero the state, run nt steps keeping checkpoints; returns a copy of
        the traces."""
        w = self.w
        nt = w.nt if nt is None else int(nt)
        self.nt = nt
        w.reset()
        st = w._stream()
        self.checkpoints = []
        for it0 in range(0, nt, self.K):
            n = min(self.K, nt - it0)
            self.checkpoints.append((it0, n, [t.clone() for t in self._state()]))
            self.plan.run(it0, n, False, st)
        return w.data[:nt].clone()

    def backward(self, residual: torch.Tensor):
        """Per-cell gradients (g_rho, g_lam, g_mu) of the misfit whose
        derivative with respect to the traces is `residual` (nt, nrec)."""
        w = self.w
        dev, dt_ = w.rho.device, w.rho.dtype
        nx, nz = w.gridsize
        res = torch.zeros(w.data.shape, dtype=dt_, device=dev)
        res[: residual.shape[0]] = residual.to(dt_)
        z = lambda: torch.zeros((nx, nz), dtype=dt_, device=dev)
        adj_f = [z() for _ in range(5)]
        adj_m = [torch.zeros_like(m) if m is not None else None for m in w._mem]
        tmp = [z() for _ in range(4)]
        grad = [z() for _ in range(5)]
        snap = torch.empty((self.K + 1) * self.snap_elems, dtype=dt_, device=dev)
        d = N.Adjoint2D()
        for q in range(5):
            d.field[q] = adj_f[q].data_ptr()
            d.grad[q] = grad[q].data_ptr()
        for q in range(4):
            d.tmp[q] = tmp[q].data_ptr()
        for q in range(2):
            d.mem[q] = adj_m[q].data_ptr() if adj_m[q] is not None else None
        d.residual = res.data_ptr()
        st = w._stream()
        lib = N.load()
        for it0, n, saved in reversed(self.checkpoints):
            for dst, src in zip(self._state(), saved):
                dst.copy_(src)
            N.check(lib.sw2d_record(self.plan.handle, it0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
            N.check(lib.sw2d_adjoint_run(self.plan.handle, C.byref(d), it0, n, C.c_void_p(snap.data_ptr()),
                                         C.c_void_p(st)))
        return (coefficient_chain_sv if self.scheme == "SV" else coefficient_chain)(w.rho, grad)


def coefficient_chain_sv(rho, grad):
    """The SV scheme's per-cell sums to (g_rho, g_lam, g_mu).

    grad[0]: vx += dt/rho2 * s, rho2 = (rho[i,j] + rho[i+1,j])/2
    grad[1]: vz += dt/rhoz * s, rhoz = (rho[i,j] + rho[i,j+1])/2
    grad[2]: lpm = lam + 2 mu at sxx (i, j);  grad[3]: lam at sxx
    grad[4]: m4 = mean of mu over (i,j) (i,j+1) (i+1,j+1) (i+1,j) at sxz
    (Elastic2D_CPML.py:225,238,252-253,266).
    """
    g0, g1, g2, g3, g4 = grad
    g_rho = torch.zeros_like(rho)
    r2 = (rho[:-1] + rho[1:]) / 2
    q = 0.5 * (-g0[:-1] / (r2 * r2))
    g_rho[:-1] += q
    g_rho[1:] += q
    rz = 0.5 * (rho[:, :-1] + rho[:, 1:])
    q = 0.5 * (-g1[:, :-1] / (rz * rz))
    g_rho[:, :-1] += q
    g_rho[:, 1:] += q
    g_lam = g2 + g3
    g_mu = 2 * g2
    q = 0.25 * g4[:-1, :-1]
    g_mu[:-1, :-1] += q
    g_mu[:-1, 1:] += q
    g_mu[1:, 1:] += q
    g_mu[1:, :-1] += q
    return g_rho, g_lam, g_mu


def coefficient_chain(rho, grad):
    """Map the per-cell coefficient sums of the adjoint to (g_rho, g_lam, g_mu).

    grad[0]: vx += dt/rho * s            -> d/drho[i,j] = -G/rho^2
    grad[1]: vz += dt/rho4 * s, rho4 = (rho[i,j]+rho[i,j+1]+rho[i+1,j+1]+rho[i+1,j])/4
    grad[2]: lpm = lhx + 2 mhx at sxx (i+1/2, j), lhx, mhx averaged over i, i+1
    grad[3]: lhx at sxx
    grad[4]: mhz = (mu[i,j] + mu[i,j+1])/2 at sxz
    (Elastic2D_CPML.py:154,159,174-176,190).
    """
    g0, g1, g2, g3, g4 = grad
    g_rho = -g0 / (rho * rho)
    r4 = 0.25 * (rho[:-1, :-1] + rho[:-1, 1:] + rho[1:, 1:] + rho[1:, :-1])
    q = 0.25 * (-g1[:-1, :-1] / (r4 * r4))
    g_rho = g_rho.clone()
    g_rho[:-1, :-1] += q
    g_rho[:-1, 1:] += q
    g_rho[1:, 1:] += q
    g_rho[1:, :-1] += q
    g_lam = torch.zeros_like(rho)
    g_mu = torch.zeros_like(rho)
    hl = 0.5 * (g3 + g2)[:-1]
    g_lam[:-1] += hl
    g_lam[1:] += hl
    hm = g2[:-1]
    g_mu[:-1] += hm
    g_mu[1:] += hm
    hz = 0.5 * g4[:, :-1]
    g_mu[:, :-1] += hz
    g_mu[:, 1:] += hz
    return g_rho, g_lam, g_mu


class ForwardOp2D(torch.autograd.Function):
    """traces = F(vp, vs, rho) through the B200 kernels, with the adjoint as
    its backward."""

    @staticmethod
    def forward(ctx, vp, vs, rho, wave, checkpoint_every, scheme="VS"):
        wave.set_model(vp.detach(), vs.detach(), rho.detach())
        drv = Adjoint2D(wave, checkpoint_every, scheme)
        out = drv.forward()
        ctx.drv = drv
        ctx.save_for_backward(vp.detach(), vs.detach(), rho.detach())
        return out

    @staticmethod
    def backward(ctx, grad_out):
        vp, vs, rho = ctx.saved_tensors
        g_rho, g_lam, g_mu = ctx.drv.backward(grad_out.contiguous())
        g_vp = g_lam * 2 * rho * vp
        g_vs = g_mu * 2 * rho * vs - g_lam * 4 * rho * vs
        g_rh = g_rho + g_mu * vs * vs + g_lam * (vp * vp - 2 * vs * vs)
        return g_vp.to(vp.dtype), g_vs.to(vs.dtype), g_rh.to(rho.dtype), None, None, None


# ---- 3D (CPML moment-tensor scheme) ---------------------------------------------
F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


class Adjoint3D:
    """Checkpointed forward + adjoint driver for one 3D CPML solver, moment
    tensor (Elastic3D_SSG_Tensor) or point force (Elastic3D_SSG_CPML); exact
    numerics, orders 1..4."""

    def __init__(self, wave, checkpoint_every: int = 100):
        if not getattr(wave, "exact", True):
            raise ValueError("the 3D adjoint transposes the exact step: build the solver with exact=True")
        self.w = wave
        self.K = int(checkpoint_every)
        if self.K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.plan = wave._plan or wave._build_plan()
        n = C.c_int64(0)
        N.check(N.load().sw3d_snapshot_elems(self.plan.handle, C.byref(n)))
        self.snap_elems = int(n.value)
        self.checkpoints = []

    def _state(self):
        w = self.w
        return [getattr(w, f) for f in F3] + [m for m in w._mem if m is not None]

    def forward(self, nt: int | None = None) -> torch.Tensor:
        w = self.w
        nt = w.nt if nt is None else int(nt)
        self.nt = nt
        w.reset()
        st = w._stream()
        self.checkpoints = []
        for it0 in range(0, nt, self.K):
            n = min(self.K, nt - it0)
            self.checkpoints.append((it0, n, [t.clone() for t in self._state()]))
            self.plan.run(it0, n, False, st)
        return w.data[:nt].clone()

    def backward(self, residual: torch.Tensor):
        w = self.w
        dev, dt_ = w.rho.device, w.rho.dtype
        shape = w.gridsize
        res = torch.zeros(w.data.shape, dtype=dt_, device=dev)
        res[: residual.shape[0]] = residual.to(dt_)
        z = lambda: torch.zeros(shape, dtype=dt_, device=dev)
        adj_f = [z() for _ in range(9)]
        adj_m = [torch.zeros_like(m) if m is not None else None for m in w._mem]
        tmp = [z() for _ in range(9)]
        grad = [z() for _ in range(8)]
        snap = torch.empty((self.K + 1) * self.snap_elems, dtype=dt_, device=dev)
        d = N.Adjoint3D()
        for q in range(9):
            d.field[q] = adj_f[q].data_ptr()
            d.tmp[q] = tmp[q].data_ptr()
        for q in range(8):
            d.grad[q] = grad[q].data_ptr()
        for q in range(3):
            d.mem[q] = adj_m[q].data_ptr() if adj_m[q] is not None else None
        d.residual = res.data_ptr()
        st = w._stream()
        lib = N.load()
        for it0, n, saved in reversed(self.checkpoints):
            for dst, src in zip(self._state(), saved):
                dst.copy_(src)
            N.check(lib.sw3d_record(self.plan.handle, it0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
            N.check(lib.sw3d_adjoint_run(self.plan.handle, C.byref(d), it0, n, C.c_void_p(snap.data_ptr()),
                                         C.c_void_p(st)))
        return coefficient_chain3(w.rho, grad)


def coefficient_chain3(rho, grad):
    """(g_rho, g_lam, g_mu) from the 3D per-cell coefficient sums
    (Elastic3D_SSG_Tensor.py's averages: vx unaveraged rho, vy the y pair,
    vz the x-y quad; normal stresses lam/mu over i, i+1; mu_xy = (mu[j+1] +
    2 mu + mu[i+1])/4, mu_xz = (2 mu + mu[i+1] + mu[j+1])/4,
    mu_yz = (mu[j+1] + 2 mu + mu[k+1])/4)."""
    g0, g1, g2, g3, g4, g5, g6, g7 = grad
    g_rho = (-g0 / (rho * rho)).clone()
    ry = 0.5 * (rho[:, :-1] + rho[:, 1:])
    q = 0.5 * (-g1[:, :-1] / (ry * ry))
    g_rho[:, :-1] += q
    g_rho[:, 1:] += q
    r4 = 0.25 * (rho[:-1, :-1] + rho[:-1, 1:] + rho[1:, 1:] + rho[1:, :-1])
    q = 0.25 * (-g2[:-1, :-1] / (r4 * r4))
    g_rho[:-1, :-1] += q
    g_rho[:-1, 1:] += q
    g_rho[1:, 1:] += q
    g_rho[1:, :-1] += q
    g_lam = torch.zeros_like(rho)
    g_mu = torch.zeros_like(rho)
    hl = 0.5 * (g4 + g3)[:-1]
    g_lam[:-1] += hl
    g_lam[1:] += hl
    g_mu[:-1] += g3[:-1]
    g_mu[1:] += g3[:-1]
    g_mu += 0.5 * (g5 + g6 + g7)
    g_mu[:, 1:] += 0.25 * (g5 + g6 + g7)[:, :-1]
    g_mu[1:] += 0.25 * (g5 + g6)[:-1]
    g_mu[:, :, 1:] += 0.25 * g7[:, :, :-1]
    return g_rho, g_lam, g_mu


class ForwardOp3D(torch.autograd.Function):
    """3D traces = F(vp, vs, rho) through the B200 kernels, with the 3D
    adjoint as its backward."""

    @staticmethod
    def forward(ctx, vp, vs, rho, wave, checkpoint_every):
        wave.set_model(vp.detach(), vs.detach(), rho.detach())
        drv = Adjoint3D(wave, checkpoint_every)
        out = drv.forward()
        ctx.drv = drv
        ctx.save_for_backward(vp.detach(), vs.detach(), rho.detach())
        return out

    @staticmethod
    def backward(ctx, grad_out):
        vp, vs, rho = ctx.saved_tensors
        g_rho, g_lam, g_mu = ctx.drv.backward(grad_out.contiguous())
        g_vp = g_lam * 2 * rho * vp
        g_vs = g_mu * 2 * rho * vs - g_lam * 4 * rho * vs
        g_rh = g_rho + g_mu * vs * vs + g_lam * (vp * vp - 2 * vs * vs)
        return g_vp.to(vp.dtype), g_vs.to(vs.dtype), g_rh.to(rho.dtype), None, None
