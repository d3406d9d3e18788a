"""Drop-in for src/Elastic3D_SSG_CPML.py: 3D SSG with ADE-CPML and a vertical
point force, one receiver.

Per step (Elastic3D_SSG_CPML.py:144-309): velocity phase; the six Dirichlet
loops (:215-243), which only touch cells no phase writes and so change nothing
on a valid grid; the point force vz[isx+5, isy+5, isz+5] +=
dt*Ricker(it, dt, freq, 1000)/rho[...] (the +5 offset and the amplitude 1000
are the reference's); stress phase; data[it] = vx[rsx, rsy, rsz].
"""
from __future__ import annotations

import torch

from . import _native as N
from . import BaseFun
from ._common import receiver_table
from ._elastic3d import Elastic3DBase


class ElasticWAVE(Elastic3DBase):
    _scheme = N.SW3D_CPML_FORCE

    def __init__(self, vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, rsx, rsy, rsz, nt, accuracy,
                 freq=100, fieldtype=torch.float32, *, coef64=False, exact=True):
        self._init_common(vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, nt, accuracy, freq, fieldtype,
                          coef64, exact)
        self.rsx, self.rsy, self.rsz = rsx, rsy, rsz
        self._rec_lin, _ = receiver_table(self.gridsize, rsx, rsy, rsz)
        self.data = torch.zeros(self.nt, dtype=torch.float32, device=self._dev)

    def _source(self):
        wav = BaseFun.series("ricker", self.nt, self.dt, self.f0, 1000)
        return N.SW_SRC_FORCE, (self.isx + 5, self.isy + 5, self.isz + 5), wav, (0,) * 6

    def _receivers(self):
        return 0, self._rec_lin

    def forward_op(self, vp, vs, rho, checkpoint_every: int = 100):
        """Differentiable seismogram: the (nt, nrec) vx traces as a function of
        the vp, vs, rho tensors (device, the solver's dtype), with the
        hand-written 3D adjoint as backward, the point force's dt/rho term
        included (no reference counterpart; exact numerics, orders 1..4)."""
        from .adjoint import ForwardOp3D
        return ForwardOp3D.apply(vp, vs, rho, self, int(checkpoint_every))

    def update_SSG(self, nt: int):
        """One time step (Elastic3D_SSG_CPML.py:144-309)."""
        self._step(nt)
