"""Learned thin absorbing layer for the 2D VS solver (no reference
counterpart).

The solver grid ends in a thin CPML of SW_ABC_DEPTH (6) cells built by the
reference's SetADEPML2D (Elastic2D_CPML.py:392-528); after every time step a
small network per face corrects the five fields of the outer 6 cells from
their 3x3 stencils (sw2d_abc_correct).  Plain thin CPML is the fallback (run
without the network) and a 20-cell CPML is the yardstick for reflected energy.

Training runs through the time loop with this library's own kernels: the
thin solver with the network runs forward with per-step snapshots
(sw2d_record) and stored network inputs; the loss is the misfit of vz traces
on a band of interior receivers against a large-domain run of the same model
and source (the solver on a grid padded by 200 cells, whose own CPML is too
far away to matter); the reverse sweep alternates the adjoint of each
correction (sw2d_abc_adjoint, back-propagation through the network into the
stencil) and of each time step (sw2d_adjoint_run), and sw_mlp_backward turns
the adjoints of the network outputs into parameter gradients for Adam.

A first formulation, one-step supervision on states forced to the reference
(the network predicting each step's residual), fitted the residuals poorly
from local stencils and was unstable once run in closed loop; the through-
the-loop training is what is kept.

    abc, losses, _ = train_rollout(cases)             # or LearnedABC2D.load(path)
    w = ElasticWAVE(...); w.SetADEPML2D(surface, pml_parameter(..., npml=6))
    abc.run(w, nt)                                    # steps + corrections
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _native as N

L = N.SW_ABC_DEPTH
NP = N.SW_ABC_PARAMS
NI, NH = N.SW_ABC_INPUTS, N.SW_ABC_HIDDEN
FIELDS = ("vx", "vz", "sxx", "szz", "sxz")


def layer_cells(nx: int, nz: int, depth: int = L):
    """Cells within `depth` of an edge, with the face whose distance is
    smallest (0 x-low, 1 x-high, 2 z-low, 3 z-high; ties in that order) and
    that distance."""
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    dist = np.stack([i, nx - 1 - i, j, nz - 1 - j])
    face = np.argmin(dist, axis=0)
    dep = np.min(dist, axis=0)
    sel = dep < depth
    return ((i * nz + j)[sel].astype(np.int32), face[sel].astype(np.int8), dep[sel].astype(np.int8))


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform hidden layers and a zero output layer: the untrained
    network adds nothing (plain thin CPML)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((4, NP), np.float32)
    for f in range(4):
        w1 = rng.uniform(-1, 1, (NH, NI)) * math.sqrt(6.0 / (NI + NH))
        w2 = rng.uniform(-1, 1, (NH, NH)) * math.sqrt(6.0 / (2 * NH))
        out[f, : NH * NI] = w1.reshape(-1)
        o = NH * NI + NH
        out[f, o: o + NH * NH] = w2.reshape(-1)
    return out


class LearnedABC2D:
    def __init__(self, params=None, scale=(1.0,) * 5, oscale=(0.0,) * 5):
        p = init_params() if params is None else np.asarray(params, np.float32).reshape(4, NP)
        self.params = torch.as_tensor(p, device="cuda").contiguous()
        self.scale = [float(s) for s in scale]
        self.oscale = [float(s) for s in oscale]
        self._cache = {}

    # -- persistence -----------------------------------------------------------
    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), scale=np.asarray(self.scale, np.float64),
                 oscale=np.asarray(self.oscale, np.float64))

    @classmethod
    def load(cls, path):
        d = np.load(path)
        return cls(d["params"], d["scale"], d["oscale"])

    # -- kernels ----------------------------------------------------------------
    def _desc(self, wave):
        key = wave.gridsize
        if key not in self._cache:
            cell, face, dep = layer_cells(*key)
            t = [torch.as_tensor(a, device="cuda") for a in (cell, face, dep)]
            delta = torch.empty((cell.size, 5), dtype=torch.float32, device="cuda")
            self._cache[key] = (t, delta)
        (cell, face, dep), delta = self._cache[key]
        d = N.AbcDesc()
        d.ncell = int(cell.numel())
        d.cell, d.face, d.depth = cell.data_ptr(), face.data_ptr(), dep.data_ptr()
        d.params = self.params.data_ptr()
        for q in range(5):
            d.scale[q] = self.scale[q]
            d.oscale[q] = self.oscale[q]
        d.delta = delta.data_ptr()
        return d, cell

    def correct(self, wave):
        """Add the network's corrections to the layer cells of `wave`."""
        d, _ = self._desc(wave)
        plan = wave._plan(N.SW2D_SSG_VS)
        N.check(N.load().sw2d_abc_correct(plan.handle, C.byref(d), C.c_void_p(wave._stream())))

    def features(self, wave) -> torch.Tensor:
        d, cell = self._desc(wave)
        x = torch.empty((cell.numel(), NI), dtype=torch.float32, device="cuda")
        plan = wave._plan(N.SW2D_SSG_VS)
        N.check(N.load().sw2d_abc_features(plan.handle, C.byref(d), C.c_void_p(x.data_ptr()),
                                           C.c_void_p(wave._stream())))
        return x

    def run(self, wave, nt: int, it0: int = 0, net: bool = True):
        """Steps it0 .. it0+nt-1 of update_SSG_VS, each followed by the
        network's correction (net=False: plain thin CPML)."""
        for it in range(it0, it0 + nt):
            wave.update_SSG_VS(it)
            if net:
                self.correct(wave)
        return wave


def mlp_grad(params_face: torch.Tensor, X: torch.Tensor, Y: torch.Tensor):
    """(loss, grad) of mean |net(X) - Y|^2 for one face, by sw_mlp_grad."""
    grad = torch.zeros(NP, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    N.check(N.load().sw_mlp_grad(C.c_void_p(params_face.data_ptr()), C.c_void_p(X.data_ptr()),
                                 C.c_void_p(Y.data_ptr()), int(X.shape[0]), C.c_void_p(grad.data_ptr()),
                                 C.c_void_p(loss.data_ptr()), C.c_void_p(st)))
    return loss, grad


def mlp_forward(params_face: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
    y = torch.empty((X.shape[0], 5), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    N.check(N.load().sw_mlp_forward(C.c_void_p(params_face.data_ptr()), C.c_void_p(X.data_ptr()),
                                    int(X.shape[0]), C.c_void_p(y.data_ptr()), C.c_void_p(st)))
    return y


# ---- data generation -----------------------------------------------------------
def _solver(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, npml, MT, src_scale, rec=None):
    from .Elastic2D_CPML import ElasticWAVE
    from .synthetic import pml_parameter
    nx, nz = vp.shape
    rx, rz = (nx // 2, nz // 2) if rec is None else rec
    w = ElasticWAVE(vs, vp, rho, h, h, dt, isx, isz, rx, rz, nt, N_, freq, torch.float32, MT=MT,
                    src_scale=src_scale)
    w.SetADEPML2D([True] * 4, pml_parameter(float(vp.max()), float(vs.max()), h, freq, npml, dims=2))
    return w


def truth_run(vp, vs, rho, h, dt, isx, isz, nt, N_=2, freq=15.0, pad=200, MT="explosive", src_scale=1e5,
              rec=None):
    """Large-domain run: the model padded by `pad` edge-replicated cells per
    side with a 20-cell CPML at the far edges; returns the truncated region's
    five fields before every step (nt+1 states) and its traces."""
    P = int(pad)
    big = [np.pad(a, P, mode="edge") for a in (vp, vs, rho)]
    nx, nz = vp.shape
    recb = None if rec is None else (np.asarray(rec[0]) + P, np.asarray(rec[1]) + P)
    w = _solver(*big, h, dt, isx + P, isz + P, nt, N_, freq, 20, MT, src_scale, recb)
    states = torch.empty((nt + 1, 5, nx, nz), dtype=torch.float32, device="cuda")
    for it in range(nt + 1):
        for q, f in enumerate(FIELDS):
            states[it, q].copy_(getattr(w, f)[P:P + nx, P:P + nz])
        if it < nt:
            w.update_SSG_VS(it)
    return states, w.data.clone()


def field_scales(states, nx, nz) -> list:
    cell, _, _ = layer_cells(nx, nz)
    c = torch.as_tensor(cell, device="cuda").long()
    out = []
    for q in range(5):
        v = states[:, q].reshape(states.shape[0], -1)[:, c]
        out.append(max(float(v.pow(2).mean().sqrt()), 1e-30))
    return out


def evaluate(abc: LearnedABC2D, vp, vs, rho, isx, isz, nt, h=10.0, dt=1e-3, N_=2, freq=15.0, pad=200,
             margin=10):
    """Relative L2 errors against a large-domain run (`pad` cells of model
    and a far 20-cell CPML on every side), over the cells more than `margin`
    from the grid edge, of the final (vx, vz) and of the vz traces of a
    receiver line at z = margin: the thin 6-cell CPML with the network
    ("net") and without it ("plain"), and the same interior with a 20-cell
    CPML ("cpml20", the yardstick)."""
    nx, nz = vp.shape
    rx = np.arange(margin, nx - margin, 2, dtype=np.int64)
    rz = np.full(rx.size, margin, np.int64)
    truth, d_true = truth_run(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, pad, rec=(rx, rz))
    thick, d_thick = truth_run(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, 20 - L, rec=(rx, rz))
    sl = (slice(margin, nx - margin), slice(margin, nz - margin))
    ref = truth[nt][:2][(slice(None),) + sl]

    def err(fields, data):
        return (float(torch.linalg.norm(fields - ref) / torch.linalg.norm(ref)),
                float(torch.linalg.norm(data - d_true) / torch.linalg.norm(d_true)))

    out = {}
    for tag in ("net", "plain"):
        w = _solver(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, L, "explosive", 1e5, rec=(rx, rz))
        abc.run(w, nt, net=tag == "net")
        out[tag], out[tag + "_traces"] = err(torch.stack([w.vx[sl], w.vz[sl]]), w.data)
    out["cpml20"], out["cpml20_traces"] = err(thick[nt][:2][(slice(None),) + sl], d_thick)
    return out


# ---- training through the time loop ----------------------------------------------
def band_receivers(nx, nz, lo=8, hi=20):
    """Cells whose distance to the grid edge is in [lo, hi): the interior
    band where the boundary's reflections are first seen."""
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    d = np.minimum.reduce([i, nx - 1 - i, j, nz - 1 - j])
    sel = (d >= lo) & (d < hi)
    return i[sel].astype(np.int64), j[sel].astype(np.int64)


class Rollout:
    """One training case: the thin solver with the network, run forward with
    snapshots, and the gradient of its trace misfit on the receiver band
    against given reference traces with respect to the network parameters:
    the reverse sweep alternates the adjoint of each correction
    (sw2d_abc_adjoint) and of each time step (sw2d_adjoint_run)."""

    def __init__(self, abc: LearnedABC2D, vp, vs, rho, isx, isz, nt, d_ref, rec, h=10.0, dt=1e-3, N_=2,
                 freq=15.0):
        self.abc, self.nt = abc, int(nt)
        self.w = _solver(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, L, "explosive", 1e5, rec=rec)
        w = self.w
        self.plan = w._plan(N.SW2D_SSG_VS)
        n = C.c_int64(0)
        N.check(N.load().sw2d_snapshot_elems(self.plan.handle, C.byref(n)))
        self.elems = int(n.value)
        self.snap = torch.empty((self.nt, 2, self.elems), dtype=torch.float32, device="cuda")
        _, cell = abc._desc(w)
        self.ncell = int(cell.numel())
        self.xs = torch.empty((self.nt, self.ncell, NI), dtype=torch.float32, device="cuda")
        self.ybar = torch.empty((self.nt, self.ncell, 5), dtype=torch.float32, device="cuda")
        face = torch.as_tensor(layer_cells(*w.gridsize)[1], device="cuda").long()
        self.face_idx = [torch.nonzero(face == f).reshape(-1) for f in range(4)]
        self.d_ref = d_ref.to(torch.float32)
        self.norm = float((self.d_ref ** 2).sum())
        nx, nz = w.gridsize
        z = lambda: torch.zeros((nx, nz), dtype=torch.float32, device="cuda")
        self.adj = [z() for _ in range(5)]
        self.adj_mem = [torch.zeros_like(m) if m is not None else None for m in w._mem]
        self.tmp = [z() for _ in range(4)]
        self.gmat = [z() for _ in range(5)]
        self.res = torch.zeros_like(w.data)
        d = N.Adjoint2D()
        for q in range(5):
            d.field[q] = self.adj[q].data_ptr()
            d.grad[q] = self.gmat[q].data_ptr()
        for q in range(4):
            d.tmp[q] = self.tmp[q].data_ptr()
        for q in range(2):
            d.mem[q] = self.adj_mem[q].data_ptr() if self.adj_mem[q] is not None else None
        d.residual = self.res.data_ptr()
        self.adesc = d
        self.adj_ptrs = (C.c_void_p * 5)(*[t.data_ptr() for t in self.adj])

    def forward(self, net: bool = True):
        w, lib, st = self.w, N.load(), C.c_void_p(self.w._stream())
        w.reset()
        for t in range(self.nt):
            N.check(lib.sw2d_record(self.plan.handle, t, 1, C.c_void_p(self.snap[t].data_ptr()), st))
            if net:
                self.xs[t].copy_(self.abc.features(w))
                self.abc.correct(w)
        r = w.data - self.d_ref
        return 0.5 * float((r ** 2).sum()) / self.norm

    def loss_and_grad(self):
        loss = self.forward(True)
        lib, st = N.load(), C.c_void_p(self.w._stream())
        self.res.copy_((self.w.data - self.d_ref) / self.norm)
        for t in self.adj + [m for m in self.adj_mem if m is not None] + self.gmat:
            t.zero_()
        d, _ = self.abc._desc(self.w)
        for t in reversed(range(self.nt)):
            N.check(lib.sw2d_abc_adjoint(self.plan.handle, C.byref(d), C.c_void_p(self.snap[t, 1].data_ptr()),
                                         self.adj_ptrs, C.c_void_p(self.ybar[t].data_ptr()), st))
            N.check(lib.sw2d_adjoint_run(self.plan.handle, C.byref(self.adesc), t, 1,
                                         C.c_void_p(self.snap[t].data_ptr()), st))
        grad = torch.zeros((4, NP), dtype=torch.float32, device="cuda")
        for f in range(4):
            idx = self.face_idx[f]
            x = self.xs[:, idx].reshape(-1, NI).contiguous()
            yb = self.ybar[:, idx].reshape(-1, 5).contiguous()
            N.check(lib.sw_mlp_backward(C.c_void_p(self.abc.params[f].data_ptr()), C.c_void_p(x.data_ptr()),
                                        C.c_void_p(yb.data_ptr()), int(x.shape[0]),
                                        C.c_void_p(grad[f].data_ptr()), st))
        return loss, grad


def train_rollout(cases, nt=400, h=10.0, dt=1e-3, N_=2, freq=15.0, pad=200, iters=200, lr=1e-3, band=(8, 20),
                  abc: LearnedABC2D | None = None, log=None):
    """Fit the network through the time loop: minimise, over the training
    cases, the band-receiver trace misfit of the thin 6-cell CPML solver with
    the network against large-domain runs.  cases: (vp, vs, rho, isx, isz)."""
    nx, nz = cases[0][0].shape
    rec = band_receivers(nx, nz, *band)
    refs, scs = [], []
    for vp, vs, rho, isx, isz in cases:
        st, d = truth_run(vp, vs, rho, h, dt, isx, isz, nt, N_, freq, pad, rec=rec)
        refs.append(d)
        scs.append(field_scales(st, nx, nz))
    if abc is None:
        abc = LearnedABC2D(scale=np.mean(scs, axis=0), oscale=np.mean(scs, axis=0) * 1e-2)
    rolls = [Rollout(abc, vp, vs, rho, isx, isz, nt, d, rec, h, dt, N_, freq)
             for (vp, vs, rho, isx, isz), d in zip(cases, refs)]
    p = torch.nn.Parameter(abc.params.clone())
    opt = torch.optim.Adam([p], lr=lr)
    hist = []
    for k in range(iters):
        tot, g = 0.0, torch.zeros_like(p)
        for r in rolls:
            loss, grad = r.loss_and_grad()
            tot += loss
            g += grad
        hist.append(tot / len(rolls))
        if log:
            log(k, hist[-1])
        p.grad = g / len(rolls)
        opt.step()
        abc.params.copy_(p.data)
    return abc, hist, rolls
