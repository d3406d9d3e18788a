"""Shared implementation of the three 3D ElasticWAVE drop-ins.

State layout on the device (C-contiguous, last index fastest, as a Taichi
dense field):
  vx vy vz sxx syy szz sxy sxz syz   (nx, ny, nz) each, field type
  rho lam mu                          (nx, ny, nz) each
  CPML memory variables               slab-compact, 6 per direction:
      _mem[0] (6, Lx+Rx, ny, nz), _mem[1] (6, nx, Ly+Ry, nz), _mem[2] (6, nx, ny, Lz+Rz)
  split-PML fields                    (24, S) on the PML shell (shell_size)
  data                                (nt, nrec) float32 receiver traces
The reference's full-grid memory arrays (memory_sxx_dx, ...) and split fields
(vx_x, ...) are still readable as attributes; they are expanded from the slabs
or the shell on access.

The split-PML shell is the union of the axes' slabs [0, lo) and [n-hi, n)
(pml.flag_extent of the predicate flags): the x slabs (sx, ny, nz) first, then
the y slabs of the x interior (nx-sx, sy, nz), then the z slabs of the x-y
interior (nx-sx, ny-sy, sz), s_d = lo_d + hi_d.  The split kernels index it the
same way (shell_index in csrc/sw_device.cuh).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from . import pml as P
from ._common import as_device, as_numpy, compute_lam, compute_mu, device, sw_dtype, torch_dtype

FIELDS3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")

# slab-compact memory variables: name -> (direction, component)
MEM3 = {
    "memory_sxx_dx": (0, 0), "memory_sxy_dx": (0, 1), "memory_sxz_dx": (0, 2),
    "memory_dvx_dx": (0, 3), "memory_dvy_dx": (0, 4), "memory_dvz_dx": (0, 5),
    "memory_sxy_dy": (1, 0), "memory_syy_dy": (1, 1), "memory_syz_dy": (1, 2),
    "memory_dvy_dy": (1, 3), "memory_dvx_dy": (1, 4), "memory_dvz_dy": (1, 5),
    "memory_sxz_dz": (2, 0), "memory_syz_dz": (2, 1), "memory_szz_dz": (2, 2),
    "memory_dvz_dz": (2, 3), "memory_dvx_dz": (2, 4), "memory_dvy_dz": (2, 5),
}

SPLIT3 = ("vx_x", "vx_y", "vx_z", "vy_x", "vy_y", "vy_z", "vz_x", "vz_y", "vz_z",
          "sxx_x", "sxx_y", "sxx_z", "syy_x", "syy_y", "syy_z",
          "sxy_x", "sxy_y", "sxz_x", "sxz_z", "syz_y", "syz_z",
          "szz_x", "szz_y", "szz_z")

AXES = ("x", "y", "z")


def shell_size(grid, lohi) -> int:
    """Cells in the split-PML shell of a grid whose axes have slabs lohi[d] = (lo, hi)."""
    (nx, ny, nz), s = grid, [lo + hi for lo, hi in lohi]
    return s[0] * ny * nz + (nx - s[0]) * s[1] * nz + (nx - s[0]) * (ny - s[1]) * s[2]


def _slab_indices(n, lo, hi, dev):
    return torch.cat([torch.arange(lo, device=dev), torch.arange(n - hi, n, device=dev)])


def shell_to_full(src: torch.Tensor, grid, lohi) -> torch.Tensor:
    """One split component (S,) on the shell as a full (nx, ny, nz) grid, zero
    outside the shell."""
    nx, ny, nz = grid
    (l0, h0), (l1, h1), (l2, h2) = lohi
    s0, s1, s2 = l0 + h0, l1 + h1, l2 + h2
    dev = src.device
    out = torch.zeros(grid, dtype=src.dtype, device=dev)
    a = s0 * ny * nz
    b = (nx - s0) * s1 * nz
    out[_slab_indices(nx, l0, h0, dev)] = src[:a].view(s0, ny, nz)
    xi = torch.arange(l0, nx - h0, device=dev)
    yi = torch.arange(l1, ny - h1, device=dev)
    out[xi[:, None], _slab_indices(ny, l1, h1, dev)[None, :]] = src[a:a + b].view(nx - s0, s1, nz)
    out[xi[:, None, None], yi[None, :, None], _slab_indices(nz, l2, h2, dev)[None, None, :]] = \
        src[a + b:].view(nx - s0, ny - s1, s2)
    return out


class Elastic3DBase:
    """Common state, PML set-up and stepping of the 3D staggered-grid solvers."""

    _scheme = N.SW3D_CPML_TENSOR

    def _init_common(self, vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, nt, accuracy, freq,
                     fieldtype, coef64=False, exact=True):
        self._dt_torch = torch_dtype(fieldtype)
        self._np_dtype = np.float64 if self._dt_torch == torch.float64 else np.float32
        self._dev = device()
        self.vs = as_device(vs, self._dt_torch, self._dev)
        self.vp = as_device(vp, self._dt_torch, self._dev)
        self.rho = as_device(rho, self._dt_torch, self._dev)
        if self.vs.dim() != 3 or self.vp.shape != self.vs.shape or self.rho.shape != self.vs.shape:
            raise ValueError("vs, vp and rho must be 3D arrays of one shape (nx, ny, nz)")
        self.gridsize = tuple(int(s) for s in self.vs.shape)
        self.dx, self.dy, self.dz = dx, dy, dz
        self.xmin = self.ymin = self.zmin = 0
        self.star = int(accuracy)
        if not 1 <= self.star <= N.SW_MAX_ORDER:
            raise ValueError(f"accuracy must be in 1..{N.SW_MAX_ORDER}")
        nx, ny, nz = self.gridsize
        if min(self.gridsize) < 2 * self.star + 3:
            raise ValueError("grid too small for the stencil order")
        self._coef64 = bool(coef64)
        # exact=True (default): IEEE-exact reference operation order everywhere,
        # bit for bit the CPU oracle.  exact=False: the staged kernels fold the
        # spacings into the coefficients, fuse multiply-adds and divide by the
        # material approximately -- faster, with traces within relative L2 1e-5
        # of the exact run and final wavefields within 1e-4.
        self.exact = bool(exact)
        self.c = torch.as_tensor(self.diff_coff(self.star), device=self._dev)
        self.xmax = self.xmin + dx * (nx - 1 - 2 * accuracy)
        self.ymax = self.zmin + dy * (ny - 1 - 2 * accuracy)
        self.zmax = self.zmin + dz * (nz - 1 - 2 * accuracy)
        self.mu = self.Compute_mu(fieldtype)
        self.lam = self.Compute_lam(fieldtype)
        self.f0 = freq
        self.dt = dt
        self.isx, self.isy, self.isz = int(isx), int(isy), int(isz)
        self.nt = int(nt)
        z = lambda: torch.zeros(self.gridsize, dtype=self._dt_torch, device=self._dev)
        for f in FIELDS3:
            setattr(self, f, z())
        for ax, n in zip(AXES, self.gridsize):
            for name in P.PROFILE_NAMES:
                base, _, half = name.partition("_")
                attr = f"{base}_{ax}_half" if half else f"{base}_{ax}"
                setattr(self, attr, torch.zeros(n, dtype=self._dt_torch, device=self._dev))
        self.xmin_pml, self.xmax_pml = self.xmin, self.xmax
        self.zmin_pml, self.zmax_pml = self.zmin, self.zmax
        self._prof = None
        self._plan = None
        self._free_surface = False
        self._mem = [None, None, None]
        self._split = None

    # ---- reference helpers ------------------------------------------------
    def Compute_mu(self, fieldtype=None):
        """mu = rho*vs**2 (Elastic3D_SSG_Tensor.py:132-139)."""
        return compute_mu(self.vs, self.rho)

    def Compute_lam(self, fieldtype=None):
        """lam = rho*(vp**2-2*vs**2) (Elastic3D_SSG_Tensor.py:141-149)."""
        return compute_lam(self.vs, self.vp, self.rho)

    def diff_coff(self, order):
        """Elastic3D_SSG_Tensor.py:348-359 (float32 coefficients; float64 ones
        when the solver was built with coef64=True)."""
        c32 = P.diff_coff(order)
        if getattr(self, "_coef64", False):
            b = np.zeros(order)
            b[0] = 1
            A = np.array([[(2 * j + 1) ** (2 * i + 1) for j in range(order)] for i in range(order)], float)
            return np.linalg.solve(A, b)
        return c32

    @staticmethod
    def diff_coff_op(order):
        return P.diff_coff_op(order)

    # ---- PML set-up -------------------------------------------------------
    def SetADEPML3D(self, pml_surface, parameter: dict):
        """Elastic3D_SSG_Tensor.py:361-568 (identical in the CPML/SPML classes)."""
        pml_surface = list(pml_surface)
        if len(pml_surface) != 6:
            raise ValueError("pml_surface is [xL, xR, yL, yR, zTop, zBottom]")
        thick = (parameter["pml_x_thick"], parameter["pml_y_thick"], parameter["pml_z_thick"])
        h = (self.dx, self.dy, self.dz)
        profs = []
        for a, ax in enumerate(AXES):
            pr = P.axis_profile(self.gridsize[a], self.star, h[a], thick[a], bool(pml_surface[2 * a]),
                                bool(pml_surface[2 * a + 1]), parameter["vp_max"], parameter["Rcoef"],
                                parameter["alpha_max_pml"], parameter["kmax_pml"], parameter["theta"],
                                self.dt, self._np_dtype)
            profs.append(pr)
            for name in P.PROFILE_NAMES:
                base, _, half = name.partition("_")
                attr = f"{base}_{ax}_half" if half else f"{base}_{ax}"
                setattr(self, attr, torch.as_tensor(pr[name], device=self._dev))
            setattr(self, f"{ax}min_pml", pr.pml_min)
            setattr(self, f"{ax}max_pml", pr.pml_max)
        self._prof = profs
        self._pml_param = dict(parameter)
        self._pml_surface = pml_surface
        self._tables = []
        for a in range(3):
            pr = profs[a]
            flag = P.axis_flags(self.gridsize[a], self.star, h[a], pr.pml_min, pr.pml_max, self._np_dtype)
            # CPML: slabs where the correction departs from the identity;
            # split PML: slabs that hold every flagged index (the shell)
            lo, hi = P.flag_extent(flag) if self._scheme == N.SW3D_SPML else P.slab_extent(pr)
            self._tables.append(dict(
                lo=lo, hi=hi,
                coef=torch.as_tensor(P.coef_table(pr, self._np_dtype), device=self._dev),
                damp=torch.as_tensor(P.damp_table(pr, self._np_dtype), device=self._dev),
                flag=torch.as_tensor(flag, device=self._dev),
            ))
        self._alloc_boundary_state()
        self._plan = None

    def _alloc_boundary_state(self):
        nx, ny, nz = self.gridsize
        if self._scheme == N.SW3D_SPML:
            self._split = torch.zeros((24, shell_size(self.gridsize, self._lohi())), dtype=self._dt_torch,
                                      device=self._dev)
            return
        s = [t["lo"] + t["hi"] for t in self._tables]
        shapes = [(6, s[0], ny, nz), (6, nx, s[1], nz), (6, nx, ny, s[2])]
        self._mem = [torch.zeros(sh, dtype=self._dt_torch, device=self._dev) if min(sh) > 0 else None
                     for sh in shapes]

    def _lohi(self):
        return [(t["lo"], t["hi"]) for t in self._tables]

    # ---- reference attribute access to the boundary state ------------------
    def _mem_full(self, name):
        nx, ny, nz = self.gridsize
        out = torch.zeros(self.gridsize, dtype=self._dt_torch, device=self._dev)
        if self._prof is None:
            return out
        d, comp = MEM3[name]
        m = self._mem[d]
        if m is None:
            return out
        lo, hi = self._tables[d]["lo"], self._tables[d]["hi"]
        n = self.gridsize[d]
        sl = [slice(None)] * 3
        src = m[comp]
        sel = lambda a, b: tuple(slice(a, b) if q == d else slice(None) for q in range(3))
        if lo:
            out[sel(0, lo)] = src[sel(0, lo)]
        if hi:
            out[sel(n - hi, n)] = src[sel(lo, lo + hi)]
        return out

    def __getattr__(self, name):
        if name in MEM3:
            if self._scheme == N.SW3D_SPML:
                raise AttributeError(name)
            return self._mem_full(name)
        if name in SPLIT3 and self._scheme == N.SW3D_SPML:
            if self.__dict__.get("_split") is None:
                return torch.zeros(self.gridsize, dtype=self._dt_torch, device=self._dev)
            return shell_to_full(self._split[SPLIT3.index(name)], self.gridsize, self._lohi())
        raise AttributeError(name)

    # ---- free surface hooks (Elastic3D_SSG_Tensor.py:151-163) ---------------
    def AEA_init(self):
        """lam = 0 and rho halved on the first `star` z layers."""
        o = self.star
        self.lam[:, :, :o] = 0
        self.rho[:, :, :o] = 0.5 * self.rho[:, :, :o]

    def AEA(self):
        """szz = 0 on the z layer `star`."""
        self.szz[:, :, self.star] = 0

    # ---- plan --------------------------------------------------------------
    def _source(self):
        raise NotImplementedError

    def _receivers(self):
        raise NotImplementedError

    def _build_plan(self):
        if self._prof is None:
            raise RuntimeError("call SetADEPML3D(pml_surface, parameter) before stepping")
        nx, ny, nz = self.gridsize
        d = N.Desc3D()
        d.scheme = self._scheme
        d.dtype = sw_dtype(self._dt_torch)
        d.nx, d.ny, d.nz = nx, ny, nz
        d.order = self.star
        d.nt_max = self.nt
        d.dx, d.dy, d.dz, d.dt = float(self.dx), float(self.dy), float(self.dz), float(self.dt)
        cvals = as_numpy(self.c).astype(np.float64)
        for m in range(self.star):
            d.coef[m] = float(cvals[m])
        keep = []
        for q, f in enumerate(FIELDS3):
            t = getattr(self, f)
            keep.append(t)
            d.field[q] = t.data_ptr()
        for nm in ("rho", "lam", "mu"):
            t = getattr(self, nm)
            keep.append(t)
            setattr(d, nm, t.data_ptr())
        for a in range(3):
            tb = self._tables[a]
            d.pml[a].lo, d.pml[a].hi = tb["lo"], tb["hi"]
            d.pml[a].coef = tb["coef"].data_ptr()
            d.pml[a].damp = tb["damp"].data_ptr()
            d.pml[a].flag = tb["flag"].data_ptr()
            keep += [tb["coef"], tb["damp"], tb["flag"]]
            m = self._mem[a]
            d.mem[a] = m.data_ptr() if m is not None else None
            keep.append(m)
        if self._split is not None:
            d.split = self._split.data_ptr()
            keep.append(self._split)
        kind, (si, sj, sk), wav, mt = self._source()
        d.src.kind = kind
        d.src.i, d.src.j, d.src.k = si, sj, sk
        self._wavelet = torch.as_tensor(wav, device=self._dev).to(self._dt_torch).contiguous()
        d.src.wavelet = self._wavelet.data_ptr()
        keep.append(self._wavelet)
        for q in range(6):
            d.src.mt[q] = float(mt[q])
        field, lin = self._receivers()
        self._rec_index = torch.as_tensor(lin, dtype=torch.int64, device=self._dev)
        d.rec.nrec = int(lin.size)
        d.rec.field = field
        d.rec.index = self._rec_index.data_ptr()
        d.rec.data = self.data.data_ptr()
        d.rec.dtype = N.SW_F64 if self.data.dtype == torch.float64 else N.SW_F32
        keep += [self._rec_index, self.data]
        self._plan = N.Plan(d, keep, three_d=True)
        self._plan.set_exact(self.exact)
        if self._free_surface:
            self._plan.set_free_surface(True)
        return self._plan

    def _stream(self) -> int:
        return torch.cuda.current_stream(self._dev).cuda_stream

    def _step(self, nt):
        if not 0 <= int(nt) < self.nt:
            raise IndexError(f"time step {nt} outside 0..{self.nt - 1}")
        plan = self._plan or self._build_plan()
        plan.step(int(nt), self._stream())

    def set_free_surface(self, on: bool = True):
        """Free-surface mode (no reference counterpart as a mode): every
        update_SSG / update_SSG_SPML step and every run() step first applies
        AEA (szz = 0 on the z layer `star`), as a driver loop
        `AEA(); update_SSG(i)` would; in run() the hook is one kernel of the
        captured step.  Call AEA_init() once for the material part of the
        condition.  The adjoint (forward_op) does not cover this mode."""
        self._free_surface = bool(on)
        if self._plan is not None:
            self._plan.set_free_surface(self._free_surface)
        return self

    def run(self, nt=None, it0: int = 0, use_graph: bool = True, free_surface=None):
        """Steps it0 .. it0+nt-1 in one enqueue (CUDA graph), the drivers'
        `for i in range(nt): test.update_SSG(i)` loop; free_surface=True/False
        sets the free-surface mode first (set_free_surface)."""
        if free_surface is not None:
            self.set_free_surface(free_surface)
        nt = self.nt - it0 if nt is None else int(nt)
        plan = self._plan or self._build_plan()
        plan.run(int(it0), nt, use_graph, self._stream())
        return self

    def set_tile(self, x_chunk: int):
        (self._plan or self._build_plan()).set_tile(int(x_chunk))

    # -- autotuner (no reference counterpart) ------------------------------------
    AUTOTUNE_CHUNKS = (6, 8, 12, 16, 25, 50)

    def autotune(self, steps: int = 6, force: bool = False) -> int:
        """Choose the x planes per work unit of the plan's current path (the
        staged or fused chunk, or the two-pass kernels' x_chunk) by timing
        `steps` steps of each candidate on this solver's own grid, with its
        state replaced by random values for the trials and restored
        afterwards (results do not depend on the choice).  The winner is
        cached per (GPU, solver class, order, dtype, numeric mode, path, log2
        shape bucket) in the batch autotuner's JSON file
        (SEISWAVE_AUTOTUNE_CACHE).  Returns the chosen chunk length."""
        import math
        from .batch import cache_load, cache_store
        plan = self._plan or self._build_plan()
        info = plan.info()
        path_name = info["path"]
        nx, ny, nz = self.gridsize
        dev = torch.cuda.get_device_name(self._dev).replace(" ", "_")
        bucket = "-".join(str(round(math.log2(max(n, 1)))) for n in (nx, ny, nz))
        key = (f"3d|{dev}|{type(self).__module__}|{self.star}|{self._dt_torch}|{int(info['exact'])}|"
               f"{path_name}|{bucket}")

        def apply(chunk):
            if path_name in ("staged", "fused"):
                plan.set_path(path_name, int(chunk))
            else:
                plan.set_tile(int(chunk))

        v = cache_load().get(key)
        if not force and isinstance(v, int) and v in self.AUTOTUNE_CHUNKS and v <= nx:
            apply(v)
            return v
        # every array a trial step writes is saved and restored
        state = [getattr(self, f) for f in FIELDS3] + [m for m in self._mem if m is not None] + [self.data]
        if self._split is not None:
            state.append(self._split)
        saved = [t.clone() for t in state]
        gen = torch.Generator(device=state[0].device).manual_seed(0)
        for t in state:
            t.copy_(torch.randn(t.shape, generator=gen, device=t.device, dtype=t.dtype) * 1e-3)
        st = torch.cuda.current_stream(self._dev)
        steps = max(1, min(int(steps), self.nt - 1))
        best, best_ms = None, float("inf")
        for chunk in [c for c in self.AUTOTUNE_CHUNKS if c <= nx]:
            apply(chunk)
            self.run(1, 0, use_graph=False)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            self.run(steps, 1, use_graph=False)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if ms < best_ms:
                best, best_ms = chunk, ms
        for t, v in zip(state, saved):
            t.copy_(v)
        apply(best)
        cache_store(key, best)
        return best

    def check_finite(self) -> int:
        """Number of non-finite wavefield values (0 when the state is finite)."""
        return (self._plan or self._build_plan()).check_finite(self._stream())

    # ---- stability, checked runs, checkpoint/resume (no reference counterpart)
    def courant(self) -> float:
        """Stability number vp_max*dt*sqrt(1/dx^2 + 1/dy^2 + 1/dz^2)*sum|c| of
        the staggered scheme; the run is stable when it is <= 1."""
        return P.courant_check(float(self.vp.max()), self.dt, (self.dx, self.dy, self.dz), as_numpy(self.c))

    def run_checked(self, nt=None, it0: int = 0, every: int = 100, **run_kw):
        """run() in segments of `every` steps with a NaN/Inf scan of the
        wavefields after each; raises state.NonFiniteError (with the step)
        instead of running on with a blown-up state."""
        from . import state
        state.run_checked(self, self.nt - it0 if nt is None else int(nt), it0, every, **run_kw)
        return self

    def _state_arrays(self):
        d = {f: getattr(self, f) for f in FIELDS3}
        d.update({f"mem{a}": m for a, m in enumerate(self._mem)})
        d["split"] = self._split
        d["data"] = self.data
        return d

    def _fingerprint(self):
        if self._prof is None:
            raise RuntimeError("call SetADEPML3D(pml_surface, parameter) before saving or loading a state")
        return {"class": type(self).__module__.rsplit(".", 1)[-1], "grid": list(self.gridsize),
                "dtype": str(self._dt_torch), "order": self.star,
                "h": [float(self.dx), float(self.dy), float(self.dz)], "dt": float(self.dt), "nt": self.nt,
                "slabs": [list(lh) for lh in self._lohi()], "data": list(self.data.shape)}

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
        for f in FIELDS3:
            getattr(self, f).zero_()
        for m in self._mem:
            if m is not None:
                m.zero_()
        if self._split is not None:
            self._split.zero_()
        self.data.zero_()
