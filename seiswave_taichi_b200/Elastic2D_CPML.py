"""Drop-in for src/Elastic2D_CPML.py: 2D P-SV velocity-stress with ADE-CPML.

    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    w = ElasticWAVE(vs, vp, rho, dx, dz, dt, isx, isz, rsx, rsz, nt, accuracy, freq)
    w.SetADEPML2D(pml_surface, pml_parameter)
    for i in range(nt): w.update_SSG_VS(i)     # or w.run(nt)

Schemes (Elastic2D_CPML.py):
* update_SSG_VS(nt)  :128-200  vz point source Ricker2(t0=1.5/freq), records vz
* update_SSG_SV(nt)  :203-274  vx point source Ricker, records vx
* update_RSG(nt, source) :277-353  rotated grid, source spread over 2x2 cells,
  no receiver write
Receivers may be single ints (data is (nt,)) or (1, nrec) / (nrec,) integer
arrays (data is (nt, nrec)).

Keyword MT (no reference counterpart) replaces the point force of the VS and
SV schemes by a moment-tensor source in the convention of
Elastic3D_SSG_Tensor.py:186-193, sigma_ab[isx, isz] += w(t) * (-M_ab) at the
start of the step, with the scheme's own wavelet times src_scale: a 2x2
[[xx, xz], [xz, zz]] or 3x3 tensor (its x-z block), or "explosive" (M = I).

State on the device: vx vz sxx szz sxz (nx, nz); memory variables
slab-compact, _mem[0] (4, Lx+Rx, nz) = sxx_dx sxz_dx dvx_dx dvz_dx and
_mem[1] (4, nx, Lz+Rz) = sxz_dz szz_dz dvz_dz dvx_dz, shared by the three
schemes as in the reference; the full-grid names (memory_sxx_dx, ...) are
readable attributes expanded from the slabs.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from . import BaseFun
from . import pml as P
from ._common import (as_device, as_numpy, compute_lam, compute_mu, device, receiver_table,
                      sw_dtype, torch_dtype)

FIELDS2 = ("vx", "vz", "sxx", "szz", "sxz")
MEM2 = {
    "memory_sxx_dx": (0, 0), "memory_sxz_dx": (0, 1), "memory_dvx_dx": (0, 2), "memory_dvz_dx": (0, 3),
    "memory_sxz_dz": (1, 0), "memory_szz_dz": (1, 1), "memory_dvz_dz": (1, 2), "memory_dvx_dz": (1, 3),
    # allocated but never used by the reference (Elastic2D_CPML.py:83,86)
    "memory_sxx_dz": None, "memory_szz_dx": None,
}


def moment_2d(MT) -> np.ndarray:
    """(xx, zz, xz) of a 2D moment tensor given as "explosive", a 2x2
    [[xx, xz], [xz, zz]] array or a 3x3 tensor (its x-z block)."""
    if isinstance(MT, str):
        if MT != "explosive":
            raise ValueError("MT must be an array or 'explosive'")
        return np.array([1.0, 1.0, 0.0], np.float32)
    M = np.asarray(MT, np.float32)
    if M.shape == (2, 2):
        return np.array([M[0, 0], M[1, 1], M[0, 1]], np.float32)
    if M.shape == (3, 3):
        return np.array([M[0, 0], M[2, 2], M[0, 2]], np.float32)
    raise ValueError("MT must be 2x2, 3x3 or 'explosive'")


class ElasticWAVE:
    def __init__(self, vs, vp, rho, dx, dz, dt, isx, isz, rsx, rsz, nt, accuracy=3, freq=100.,
                 fieldtype=torch.float32, *, coef64=False, MT=None, src_scale=1.0, rec_component=None):
        self._dt_torch = torch_dtype(fieldtype)
        self._np_dtype = np.float64 if self._dt_torch == torch.float64 else np.float32
        self._dev = device()
        self.vs = as_device(vs, self._dt_torch, self._dev)
        self.vp = as_device(vp, self._dt_torch, self._dev)
        self.rho = as_device(rho, self._dt_torch, self._dev)
        if self.vs.dim() != 2 or self.vp.shape != self.vs.shape or self.rho.shape != self.vs.shape:
            raise ValueError("vs, vp and rho must be 2D arrays of one shape (nx, nz)")
        self.gridsize = tuple(int(s) for s in self.vs.shape)
        self.dx, self.dz = dx, dz
        self.xmin = self.zmin = 0
        self.star = int(accuracy)
        if not 1 <= self.star <= N.SW_MAX_ORDER:
            raise ValueError(f"accuracy must be in 1..{N.SW_MAX_ORDER}")
        if min(self.gridsize) < 2 * self.star + 3:
            raise ValueError("grid too small for the stencil order")
        self._coef64 = bool(coef64)
        self.c = torch.as_tensor(self._coefs(self.star), device=self._dev)
        nx, nz = self.gridsize
        self.xmax = self.xmin + dx * (nx - 1 - 2 * accuracy)
        self.zmax = self.zmin + dz * (nz - 1 - 2 * accuracy)
        self.mu = self.Compute_mu(fieldtype)
        self.lam = self.Compute_lam(fieldtype)
        self.f0 = freq
        self.dt = dt
        self.isx, self.isz = int(isx), int(isz)
        self.rsx, self.rsz = rsx, rsz
        self.nt = int(nt)
        self._rec_lin, single = receiver_table(self.gridsize, rsx, rsz)
        shape = (self.nt,) if single else (self.nt, int(self._rec_lin.size))
        self.data = torch.zeros(shape, dtype=self._dt_torch, device=self._dev)
        z = lambda: torch.zeros(self.gridsize, dtype=self._dt_torch, device=self._dev)
        for f in FIELDS2:
            setattr(self, f, z())
        for ax, n in zip(("x", "z"), self.gridsize):
            for name in P.PROFILE_NAMES:
                base, _, half = name.partition("_")
                setattr(self, f"{base}_{ax}_half" if half else f"{base}_{ax}",
                        torch.zeros(n, dtype=self._dt_torch, device=self._dev))
        self.xmin_pml, self.xmax_pml = self.xmin, self.xmax
        self.zmin_pml, self.zmax_pml = self.zmin, self.zmax
        self._prof = None
        self._plans = {}
        self._free_surface = False
        self._wavelets = {}
        self._mem = [None, None]
        self.MT = None if MT is None else moment_2d(MT)
        self.src_scale = float(src_scale)
        # receivers of update_SSG_VS / update_SSG_SV: the scheme's component
        # (vz, vx) unless a field is named
        if rec_component is not None and rec_component not in FIELDS2:
            raise ValueError(f"rec_component must be one of {FIELDS2}")
        self._rec_component = rec_component

    # ---- reference helpers ------------------------------------------------
    def Compute_mu(self, fieldtype=None):
        """mu = rho*vs**2 (Elastic2D_CPML.py:93-100)."""
        return compute_mu(self.vs, self.rho)

    def Compute_lam(self, fieldtype=None):
        """lam = rho*(vp**2-2*vs**2) (Elastic2D_CPML.py:102-110)."""
        return compute_lam(self.vs, self.vp, self.rho)

    def _coefs(self, order):
        if self._coef64:
            b = np.zeros(order)
            b[0] = 1
            A = np.array([[(2 * j + 1) ** (2 * i + 1) for j in range(order)] for i in range(order)], float)
            return np.linalg.solve(A, b)
        return P.diff_coff(order)

    @staticmethod
    def diff_coff(order):
        """Elastic2D_CPML.py:355-366 (float32)."""
        return P.diff_coff(order)

    @staticmethod
    def diff_coff_op(order):
        """Elastic2D_CPML.py:368-390."""
        return P.diff_coff_op(order)

    # ---- free surface hooks (Elastic2D_CPML.py:113-125) ----------------------
    def AEA_init(self):
        """lam = 0 and rho halved on the first `star` x layers."""
        o = self.star
        self.lam[:o, :] = 0
        self.rho[:o, :] = 0.5 * self.rho[:o, :]

    def AEA(self):
        """sxx = 0 on the x layer `star`."""
        self.sxx[self.star, :] = 0

    # ---- PML -------------------------------------------------------------
    def SetADEPML2D(self, pml_surface, parameter: dict):
        """Elastic2D_CPML.py:392-528."""
        pml_surface = list(pml_surface)
        if len(pml_surface) != 4:
            raise ValueError("pml_surface is [xLeft, xRight, zTop, zBottom]")
        thick = (parameter["pml_x_thick"], parameter["pml_z_thick"])
        h = (self.dx, self.dz)
        self._prof = []
        self._tables = []
        for a, ax in enumerate(("x", "z")):
            pr = P.axis_profile(self.gridsize[a], self.star, h[a], thick[a], bool(pml_surface[2 * a]),
                                bool(pml_surface[2 * a + 1]), parameter["vp_max"], parameter["Rcoef"],
                                parameter["alpha_max_pml"], parameter["kmax_pml"], parameter["theta"],
                                self.dt, self._np_dtype)
            self._prof.append(pr)
            for name in P.PROFILE_NAMES:
                base, _, half = name.partition("_")
                setattr(self, f"{base}_{ax}_half" if half else f"{base}_{ax}",
                        torch.as_tensor(pr[name], device=self._dev))
            setattr(self, f"{ax}min_pml", pr.pml_min)
            setattr(self, f"{ax}max_pml", pr.pml_max)
            lo, hi = P.slab_extent(pr)
            self._tables.append(dict(
                lo=lo, hi=hi,
                coef=torch.as_tensor(P.coef_table(pr, self._np_dtype), device=self._dev),
                flag=torch.as_tensor(P.axis_flags(self.gridsize[a], self.star, h[a], pr.pml_min,
                                                  pr.pml_max, self._np_dtype), device=self._dev),
            ))
        nx, nz = self.gridsize
        sx = self._tables[0]["lo"] + self._tables[0]["hi"]
        sz = self._tables[1]["lo"] + self._tables[1]["hi"]
        self._mem = [torch.zeros((4, sx, nz), dtype=self._dt_torch, device=self._dev) if sx else None,
                     torch.zeros((4, nx, sz), dtype=self._dt_torch, device=self._dev) if sz else None]
        self._plans = {}

    def __getattr__(self, name):
        if name in MEM2:
            return self._mem_full(name)
        raise AttributeError(name)

    def _mem_full(self, name):
        out = torch.zeros(self.gridsize, dtype=self._dt_torch, device=self._dev)
        key = MEM2[name]
        if key is None or self.__dict__.get("_prof") is None:
            return out
        d, comp = key
        m = self._mem[d]
        if m is None:
            return out
        lo, hi = self._tables[d]["lo"], self._tables[d]["hi"]
        n = self.gridsize[d]
        sel = lambda a, b: (slice(a, b), slice(None)) if d == 0 else (slice(None), slice(a, b))
        if lo:
            out[sel(0, lo)] = m[comp][sel(0, lo)]
        if hi:
            out[sel(n - hi, n)] = m[comp][sel(lo, lo + hi)]
        return out

    # ---- plans -------------------------------------------------------------
    def _plan(self, scheme):
        if scheme in self._plans:
            return self._plans[scheme]
        if self._prof is None:
            raise RuntimeError("call SetADEPML2D(pml_surface, parameter) before stepping")
        nx, nz = self.gridsize
        d = N.Desc2D()
        d.scheme = scheme
        d.dtype = sw_dtype(self._dt_torch)
        d.nx, d.nz = nx, nz
        d.order = self.star
        d.nt_max = self.nt
        d.dx, d.dz, d.dt = float(self.dx), float(self.dz), float(self.dt)
        cv = as_numpy(self.c).astype(np.float64)
        for m in range(self.star):
            d.coef[m] = float(cv[m])
        keep = []
        for q, f in enumerate(FIELDS2):
            t = getattr(self, f)
            keep.append(t)
            d.field[q] = t.data_ptr()
        for nm in ("rho", "lam", "mu"):
            t = getattr(self, nm)
            keep.append(t)
            setattr(d, nm, t.data_ptr())
        for a in range(2):
            tb = self._tables[a]
            d.pml[a].lo, d.pml[a].hi = tb["lo"], tb["hi"]
            d.pml[a].coef = tb["coef"].data_ptr()
            d.pml[a].flag = tb["flag"].data_ptr()
            keep += [tb["coef"], tb["flag"]]
            m = self._mem[a]
            d.mem[a] = m.data_ptr() if m is not None else None
            keep.append(m)
        if scheme == N.SW2D_SSG_VS:
            wav = self._vs_wavelet()
            d.src.kind = N.SW_SRC_FORCE
            rec_field = 1  # vz (Elastic2D_CPML.py:200)
        elif scheme == N.SW2D_SSG_SV:
            wav = BaseFun.series("ricker", self.nt, self.dt, self.f0, self.src_scale)
            d.src.kind = N.SW_SRC_FORCE
            rec_field = 0  # vx (Elastic2D_CPML.py:274)
        else:
            wav = np.zeros(self.nt, dtype=np.float32)
            d.src.kind = N.SW_SRC_RSG4
            rec_field = -1  # update_RSG records nothing
        if rec_field >= 0 and self._rec_component is not None:
            rec_field = FIELDS2.index(self._rec_component)
        wt = torch.as_tensor(wav, device=self._dev).to(self._dt_torch).contiguous()
        keep.append(wt)
        self._wavelets[scheme] = wt
        d.src.i, d.src.j = self.isx, self.isz
        d.src.wavelet = wt.data_ptr()
        if self.MT is not None and scheme != N.SW2D_RSG:
            d.src.kind = N.SW_SRC_MOMENT
            d.src.mt[0], d.src.mt[2], d.src.mt[4] = (float(v) for v in self.MT)
        if rec_field >= 0:
            ri = torch.as_tensor(self._rec_lin, dtype=torch.int64, device=self._dev)
            keep += [ri, self.data]
            d.rec.nrec = int(self._rec_lin.size)
            d.rec.field = rec_field
            d.rec.index = ri.data_ptr()
            d.rec.data = self.data.data_ptr()
            d.rec.dtype = N.SW_F64 if self.data.dtype == torch.float64 else N.SW_F32
        plan = N.Plan(d, keep, three_d=False)
        if self._free_surface:
            plan.set_free_surface(True)
        self._plans[scheme] = plan
        return plan

    def _vs_wavelet(self):
        """update_SSG_VS's source series: Ricker2 with t0 = 1.5/f0 (:142, :170).
        `1.5/self.f0` is folded in Python (double) by Taichi's frontend and
        rounded once to float32 when assigned to t0."""
        t0 = np.float32(1.5 / float(self.f0))
        return BaseFun.series("ricker2", self.nt, self.dt, self.f0, self.src_scale, t0=t0)

    def _stream(self) -> int:
        return torch.cuda.current_stream(self._dev).cuda_stream

    def _check_it(self, nt):
        if not 0 <= int(nt) < self.nt:
            raise IndexError(f"time step {nt} outside 0..{self.nt - 1}")

    def update_SSG_VS(self, nt: int):
        """One step of Elastic2D_CPML.py:128-200."""
        self._check_it(nt)
        self._plan(N.SW2D_SSG_VS).step(int(nt), self._stream())

    def update_SSG_SV(self, nt: int):
        """One step of Elastic2D_CPML.py:203-274."""
        self._check_it(nt)
        self._plan(N.SW2D_SSG_SV).step(int(nt), self._stream())

    def update_RSG(self, nt: int, source: float):
        """One step of Elastic2D_CPML.py:277-353 with the caller's source value."""
        self._plan(N.SW2D_RSG).step_amp(int(nt), float(np.float32(source)), self._stream())

    def set_free_surface(self, on: bool = True):
        """Free-surface mode (no reference counterpart as a mode): every
        update_SSG_VS / update_SSG_SV / update_RSG step and every run() step
        first applies AEA (sxx = 0 on the x layer `star`), as the reference's
        driver loop `AEA(); update_SSG_VS(i)` does (Relay_wave.py:55-59); in
        run() the hooks are folded into the kernels.  Call AEA_init() once
        for the material part of the condition."""
        self._free_surface = bool(on)
        for plan in self._plans.values():
            plan.set_free_surface(self._free_surface)
        return self

    def run(self, nt=None, it0: int = 0, scheme: str = "VS", use_graph: bool = True, free_surface=None):
        """Steps it0 .. it0+nt-1 of update_SSG_VS ("VS") or update_SSG_SV ("SV")
        in one enqueue (CUDA graph); free_surface=True/False sets the
        free-surface mode first (set_free_surface)."""
        if free_surface is not None:
            self.set_free_surface(free_surface)
        nt = self.nt - it0 if nt is None else int(nt)
        s = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]
        self._plan(s).run(int(it0), nt, use_graph, self._stream())
        return self

    def forward_op(self, vp, vs, rho, checkpoint_every: int = 100, scheme: str = "VS"):
        """Differentiable seismogram: the (nt, nrec) traces of the VS scheme
        (vz) or the SV scheme (vx) as a function of the vp, vs, rho tensors
        (device, the solver's dtype), with the hand-written adjoint as
        backward (no reference counterpart)."""
        from .adjoint import ForwardOp2D
        return ForwardOp2D.apply(vp, vs, rho, self, int(checkpoint_every), scheme)

    def check_finite(self) -> int:
        return self._plan(N.SW2D_SSG_VS).check_finite(self._stream())

    # ---- stability, checked runs, checkpoint/resume (no reference counterpart)
    def courant(self) -> float:
        """Stability number vp_max*dt*sqrt(1/dx^2 + 1/dz^2)*sum|c| of the
        staggered scheme; the run is stable when it is <= 1."""
        return P.courant_check(float(self.vp.max()), self.dt, (self.dx, self.dz), as_numpy(self.c))

    def run_checked(self, nt=None, it0: int = 0, every: int = 100, **run_kw):
        """run() in segments of `every` steps with a NaN/Inf scan of the
        wavefields after each; raises state.NonFiniteError (with the step)
        instead of running on with a blown-up state."""
        from . import state
        state.run_checked(self, self.nt - it0 if nt is None else int(nt), it0, every, **run_kw)
        return self

    def _state_arrays(self):
        d = {f: getattr(self, f) for f in FIELDS2}
        d.update({f"mem{a}": m for a, m in enumerate(self._mem)})
        d["data"] = self.data
        return d

    def _fingerprint(self):
        if self._prof is None:
            raise RuntimeError("call SetADEPML2D(pml_surface, parameter) before saving or loading a state")
        return {"class": "Elastic2D_CPML", "grid": list(self.gridsize), "dtype": str(self._dt_torch),
                "order": self.star, "h": [float(self.dx), float(self.dz)], "dt": float(self.dt), "nt": self.nt,
                "slabs": [[t["lo"], t["hi"]] for t in self._tables], "data": list(self.data.shape)}

    def save_state(self, path, it: int):
        """Write the state after steps 0..it-1 (it = the next step) to an
        .npz file (state.write)."""
        from . import state
        torch.cuda.current_stream(self._dev).synchronize()
        state.write(path, self._state_arrays(), {"config": self._fingerprint(), "it": int(it)})

    def load_state(self, path) -> int:
        """Load a state written by save_state for this configuration; returns
        the next step index (resume with run(nt - it, it0=it))."""
        from . import state
        torch.cuda.current_stream(self._dev).synchronize()
        return int(state.read(path, self._state_arrays(), self._fingerprint())["it"])

    def set_model(self, vp, vs, rho, non_blocking: bool = True):
        """Load a new model of the same shape into the solver's own arrays
        (host->device copy for host inputs) and recompute mu and lam."""
        for name, src in (("vp", vp), ("vs", vs), ("rho", rho)):
            t = getattr(self, name)
            s = src if isinstance(src, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(as_numpy(src)))
            if tuple(s.shape) != self.gridsize:
                raise ValueError(f"{name} has shape {tuple(s.shape)}, the solver grid is {self.gridsize}")
            t.copy_(s, non_blocking=non_blocking)
        self.mu.copy_(compute_mu(self.vs, self.rho))
        self.lam.copy_(compute_lam(self.vs, self.vp, self.rho))

    def reset(self):
        """Zero every wavefield, memory variable and trace (new shot, same model)."""
        for f in FIELDS2:
            getattr(self, f).zero_()
        for m in self._mem:
            if m is not None:
                m.zero_()
        self.data.zero_()
