"""Learned thin absorbing layer for the 3D moment-tensor solver (no reference
counterpart): the 3D form of learned_abc.

The solver grid ends in a 6-cell CPML built by the reference's SetADEPML3D
(Elastic3D_SSG_Tensor.py:361-568); after every time step a small network per
face (six faces) corrects the nine fields of the outer 6 cells from the
fields at the cell and its two neighbours along the face's inward normal
(sw3d_abc_correct).  Plain thin CPML is the fallback (run without the
network); a 20-cell CPML is the yardstick.

Training runs through the time loop with this library's kernels: forward
steps with snapshots (sw3d_record) and stored network inputs, a vx-trace
misfit on a band of interior receivers against a large-domain run, and a
reverse sweep alternating the adjoint of each correction (sw3d_abc_adjoint)
and of each time step (sw3d_adjoint_run); sw3d_mlp_backward turns the output
adjoints into parameter gradients for Adam.

    abc, losses, _ = train_rollout3d(cases, nt=120)
    w = solver3d(vp, vs, rho, h, dt, isx, isy, isz, nt)     # thin 6-cell CPML
    abc.run(w, nt)
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _native as N

L = N.SW_ABC_DEPTH
NP = N.SW_ABC3_PARAMS
NI, NH = N.SW_ABC3_INPUTS, N.SW_ABC_HIDDEN
FIELDS = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


def layer_cells3(nx: int, ny: int, nz: int, depth: int = L):
    """Cells within `depth` of a face, with the nearest face (0 x-low,
    1 x-high, 2 y-low, 3 y-high, 4 z-low, 5 z-high; ties in that order) and
    the distance to it."""
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    dist = np.stack([i, nx - 1 - i, j, ny - 1 - j, k, nz - 1 - k])
    face = np.argmin(dist, axis=0)
    dep = np.min(dist, axis=0)
    sel = dep < depth
    lin = (i * ny + j) * nz + k
    return lin[sel].astype(np.int32), face[sel].astype(np.int8), dep[sel].astype(np.int8)


def init_params3(seed: int = 0) -> np.ndarray:
    """Glorot-uniform hidden layers, zero output layer (plain thin CPML)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((6, NP), np.float32)
    for f in range(6):
        out[f, : NH * NI] = (rng.uniform(-1, 1, (NH, NI)) * math.sqrt(6.0 / (NI + NH))).reshape(-1)
        o = NH * NI + NH
        out[f, o: o + NH * NH] = (rng.uniform(-1, 1, (NH, NH)) * math.sqrt(6.0 / (2 * NH))).reshape(-1)
    return out


class LearnedABC3D:
    def __init__(self, params=None, scale=(1.0,) * 9, oscale=(0.0,) * 9):
        p = init_params3() if params is None else np.asarray(params, np.float32).reshape(6, NP)
        self.params = torch.as_tensor(p, device="cuda").contiguous()
        self.scale = [float(s) for s in scale]
        self.oscale = [float(s) for s in oscale]
        self._cache = {}

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), scale=np.asarray(self.scale),
                 oscale=np.asarray(self.oscale))

    @classmethod
    def load(cls, path):
        d = np.load(path)
        return cls(d["params"], d["scale"], d["oscale"])

    def _desc(self, wave):
        key = wave.gridsize
        if key not in self._cache:
            cell, face, dep = layer_cells3(*key)
            t = [torch.as_tensor(a, device="cuda") for a in (cell, face, dep)]
            delta = torch.empty((cell.size, 9), dtype=torch.float32, device="cuda")
            self._cache[key] = (t, delta)
        (cell, face, dep), delta = self._cache[key]
        d = N.Abc3Desc()
        d.ncell = int(cell.numel())
        d.cell, d.face, d.depth = cell.data_ptr(), face.data_ptr(), dep.data_ptr()
        d.params = self.params.data_ptr()
        for q in range(9):
            d.scale[q] = self.scale[q]
            d.oscale[q] = self.oscale[q]
        d.delta = delta.data_ptr()
        return d, cell

    def correct(self, wave):
        d, _ = self._desc(wave)
        N.check(N.load().sw3d_abc_correct(wave._plan.handle, C.byref(d), C.c_void_p(wave._stream())))

    def features(self, wave) -> torch.Tensor:
        d, cell = self._desc(wave)
        x = torch.empty((cell.numel(), NI), dtype=torch.float32, device="cuda")
        N.check(N.load().sw3d_abc_features(wave._plan.handle, C.byref(d), C.c_void_p(x.data_ptr()),
                                           C.c_void_p(wave._stream())))
        return x

    def run(self, wave, nt: int, it0: int = 0, net: bool = True):
        wave._plan or wave._build_plan()
        for it in range(it0, it0 + nt):
            wave.update_SSG(it)
            if net:
                self.correct(wave)
        return wave


def solver3d(vp, vs, rho, h, dt, isx, isy, isz, nt, npml=L, N_=2, freq=15.0, MT=None, src_scale=1e6, rec=None,
             dtype=None):
    """3D moment-tensor solver (exact numerics) with an npml-cell CPML
    (float32 unless dtype is given)."""
    from .Elastic3D_SSG_Tensor import ElasticWAVE
    from .synthetic import pml_parameter
    nx, ny, nz = vp.shape
    if rec is None:
        rec = (np.array([nx // 2]), np.array([ny // 2]), np.array([nz // 2]))
    M = np.eye(3, dtype=np.float32) if MT is None else np.asarray(MT, np.float32)
    rx, ry, rz = (np.asarray(r, np.int64).reshape(1, -1) for r in rec)
    w = ElasticWAVE(vs, vp, rho, h, h, h, dt, isx, isy, isz, rx, ry, rz, M, src_scale, nt, N_, freq,
                    dtype or torch.float32, exact=True)
    w.SetADEPML3D([True] * 6, pml_parameter(float(vp.max()), float(vs.max()), h, freq, npml, dims=3))
    w._build_plan()
    return w


def truth_run3d(vp, vs, rho, h, dt, isx, isy, isz, nt, pad, rec, N_=2, freq=15.0, MT=None, src_scale=1e6,
                npml=20):
    """The model padded by `pad` edge-replicated cells per side, with an
    npml-cell CPML at the far edges: traces at `rec` (coordinates of the
    unpadded grid), the unpadded region's final (vx, vy, vz), and the RMS of
    each field over the unpadded grid's layer cells at every 10th step."""
    P = int(pad)
    big = [np.pad(a, P, mode="edge") for a in (vp, vs, rho)]
    nx, ny, nz = vp.shape
    recb = tuple(np.asarray(r) + P for r in rec)
    w = solver3d(*big, h, dt, isx + P, isy + P, isz + P, nt, npml, N_, freq, MT, src_scale, recb)
    cell, _, _ = layer_cells3(nx, ny, nz)
    ii, rr = np.divmod(cell, ny * nz)
    jj, kk = np.divmod(rr, nz)
    sel = torch.as_tensor(((ii + P) * (ny + 2 * P) + jj + P) * (nz + 2 * P) + kk + P, device="cuda").long()
    sq = torch.zeros(9, dtype=torch.float64, device="cuda")
    cnt = 0
    for it in range(nt):
        w.update_SSG(it)
        if it % 10 == 9:
            for q, f in enumerate(FIELDS):
                sq[q] += getattr(w, f).reshape(-1)[sel].double().pow(2).mean()
            cnt += 1
    fin = torch.stack([getattr(w, f)[P:P + nx, P:P + ny, P:P + nz].clone() for f in FIELDS[:3]])
    rms = (sq / max(cnt, 1)).sqrt().clamp_min(1e-30).cpu().numpy()
    return w.data.clone(), fin, rms


def band_receivers3(nx, ny, nz, lo=6, hi=10):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    d = np.minimum.reduce([i, nx - 1 - i, j, ny - 1 - j, k, nz - 1 - k])
    sel = (d >= lo) & (d < hi)
    return i[sel].astype(np.int64), j[sel].astype(np.int64), k[sel].astype(np.int64)


class Rollout3D:
    """One training case: the thin solver with the network, forward with
    per-step snapshots, and the gradient of its band-receiver trace misfit
    against reference traces with respect to the six faces' parameters."""

    def __init__(self, abc: LearnedABC3D, vp, vs, rho, isx, isy, isz, nt, d_ref, rec, h=10.0, dt=1e-3, N_=2,
                 freq=15.0):
        self.abc, self.nt = abc, int(nt)
        self.w = solver3d(vp, vs, rho, h, dt, isx, isy, isz, nt, L, N_, freq, rec=rec)
        w = self.w
        self.plan = w._plan
        n = C.c_int64(0)
        N.check(N.load().sw3d_snapshot_elems(self.plan.handle, C.byref(n)))
        self.elems = int(n.value)
        self.snap = torch.empty((self.nt, 2, self.elems), dtype=torch.float32, device="cuda")
        _, cell = abc._desc(w)
        self.ncell = int(cell.numel())
        self.xs = torch.empty((self.nt, self.ncell, NI), dtype=torch.float32, device="cuda")
        self.ybar = torch.empty((self.nt, self.ncell, 9), dtype=torch.float32, device="cuda")
        face = torch.as_tensor(layer_cells3(*w.gridsize)[1], device="cuda").long()
        self.face_idx = [torch.nonzero(face == f).reshape(-1) for f in range(6)]
        self.d_ref = d_ref.to(torch.float32)
        self.norm = float((self.d_ref.double() ** 2).sum())
        z = lambda: torch.zeros(w.gridsize, dtype=torch.float32, device="cuda")
        self.adj = [z() for _ in range(9)]
        self.adj_mem = [torch.zeros_like(m) if m is not None else None for m in w._mem]
        self.tmp = [z() for _ in range(9)]
        self.gmat = [z() for _ in range(8)]
        self.res = torch.zeros(w.data.shape, dtype=torch.float32, device="cuda")
        d = N.Adjoint3D()
        for q in range(9):
            d.field[q] = self.adj[q].data_ptr()
            d.tmp[q] = self.tmp[q].data_ptr()
        for q in range(8):
            d.grad[q] = self.gmat[q].data_ptr()
        for q in range(3):
            d.mem[q] = self.adj_mem[q].data_ptr() if self.adj_mem[q] is not None else None
        d.residual = self.res.data_ptr()
        self.adesc = d
        self.adj_ptrs = (C.c_void_p * 9)(*[t.data_ptr() for t in self.adj])

    def forward(self, net: bool = True):
        w, lib, st = self.w, N.load(), C.c_void_p(self.w._stream())
        w.reset()
        for t in range(self.nt):
            N.check(lib.sw3d_record(self.plan.handle, t, 1, C.c_void_p(self.snap[t].data_ptr()), st))
            if net:
                self.xs[t].copy_(self.abc.features(w))
                self.abc.correct(w)
        r = w.data.double() - self.d_ref.double()
        return 0.5 * float((r ** 2).sum()) / self.norm

    def loss_and_grad(self):
        loss = self.forward(True)
        lib, st = N.load(), C.c_void_p(self.w._stream())
        self.res.copy_((self.w.data - self.d_ref) / self.norm)
        for t in self.adj + [m for m in self.adj_mem if m is not None] + self.gmat:
            t.zero_()
        d, _ = self.abc._desc(self.w)
        for t in reversed(range(self.nt)):
            N.check(lib.sw3d_abc_adjoint(self.plan.handle, C.byref(d), C.c_void_p(self.snap[t, 1].data_ptr()),
                                         self.adj_ptrs, C.c_void_p(self.ybar[t].data_ptr()), st))
            N.check(lib.sw3d_adjoint_run(self.plan.handle, C.byref(self.adesc), t, 1,
                                         C.c_void_p(self.snap[t].data_ptr()), st))
        grad = torch.zeros((6, NP), dtype=torch.float32, device="cuda")
        for f in range(6):
            idx = self.face_idx[f]
            x = self.xs[:, idx].reshape(-1, NI).contiguous()
            yb = self.ybar[:, idx].reshape(-1, 9).contiguous()
            N.check(lib.sw3d_mlp_backward(C.c_void_p(self.abc.params[f].data_ptr()), C.c_void_p(x.data_ptr()),
                                          C.c_void_p(yb.data_ptr()), int(x.shape[0]),
                                          C.c_void_p(grad[f].data_ptr()), st))
        return loss, grad


def train_rollout3d(cases, nt=120, h=10.0, dt=1e-3, N_=2, freq=15.0, pad=60, iters=100, lr=2e-3, band=(6, 10),
                    abc: LearnedABC3D | None = None, log=None):
    """cases: (vp, vs, rho, isx, isy, isz) on the thin grid.  Adam on the
    band-trace misfit against large-domain runs, through the time loop."""
    nx, ny, nz = cases[0][0].shape
    rec = band_receivers3(nx, ny, nz, *band)
    refs, scs = [], []
    for vp, vs, rho, sx, sy, sz in cases:
        d, _, rms = truth_run3d(vp, vs, rho, h, dt, sx, sy, sz, nt, pad, rec, N_, freq)
        refs.append(d)
        scs.append(rms)
    if abc is None:
        sc = np.mean(scs, axis=0)
        abc = LearnedABC3D(scale=sc, oscale=sc * 1e-2)
    rolls = [Rollout3D(abc, vp, vs, rho, sx, sy, sz, nt, d, rec, h, dt, N_, freq)
             for (vp, vs, rho, sx, sy, sz), d in zip(cases, refs)]
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


def evaluate3d(abc: LearnedABC3D, vp, vs, rho, isx, isy, isz, nt, h=10.0, dt=1e-3, N_=2, freq=15.0, pad=60,
               band=(6, 10)):
    """Relative L2 errors against a large-domain run: vx traces on the
    receiver band and the final (vx, vy, vz) more than band[0] cells from the
    edge, for the thin 6-cell CPML with the network ("net") and without it
    ("plain") and for the same interior inside a 20-cell CPML ("cpml20")."""
    nx, ny, nz = vp.shape
    rec = band_receivers3(nx, ny, nz, *band)
    d_true, f_true, _ = truth_run3d(vp, vs, rho, h, dt, isx, isy, isz, nt, pad, rec, N_, freq)
    d_j, f_j, _ = truth_run3d(vp, vs, rho, h, dt, isx, isy, isz, nt, 20 - L, rec, N_, freq)
    m = band[0]
    sl = (slice(None), slice(m, nx - m), slice(m, ny - m), slice(m, nz - m))
    ref = f_true[sl]

    def err(f, d):
        return (float(torch.linalg.norm(f[sl] - ref) / torch.linalg.norm(ref)),
                float(torch.linalg.norm(d - d_true) / torch.linalg.norm(d_true)))

    out = {}
    for tag in ("net", "plain"):
        w = solver3d(vp, vs, rho, h, dt, isx, isy, isz, nt, L, N_, freq, rec=rec)
        abc.run(w, nt, net=tag == "net")
        out[tag], out[tag + "_traces"] = err(torch.stack([w.vx, w.vy, w.vz]), w.data)
    out["cpml20"], out["cpml20_traces"] = err(f_j, d_j)
    return out
