"""Drop-in for src/Elastic3D_SSG_Tensor.py: 3D SSG with ADE-CPML and a
moment-tensor source recorded by a receiver array.

    from seiswave_taichi_b200.Elastic3D_SSG_Tensor import ElasticWAVE
    w = ElasticWAVE(vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, rsx, rsy, rsz,
                    MT, src_scale, nt, accuracy, freq)
    w.SetADEPML3D(pml_surface, pml_parameter)
    for i in range(nt): w.update_SSG(i)        # or w.run(nt)

Per step (Elastic3D_SSG_Tensor.py:166-345): sigma_ab[isx,isy,isz] +=
Ricker2(it, dt, t0=0.03, freq, src_scale) * (-MT[a,b]) for the upper
triangle, then the velocity and stress phases, then data[it, r] =
vx[rsx[0,r], rsy[0,r], rsz[0,r]].
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from . import BaseFun
from ._common import as_numpy, receiver_table
from ._elastic3d import FIELDS3, Elastic3DBase


class ElasticWAVE(Elastic3DBase):
    _scheme = N.SW3D_CPML_TENSOR

    def __init__(self, vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, rsx, rsy, rsz, MT, src_scale,
                 nt, accuracy, freq=100., fieldtype=torch.float32, *, t0=0.03, coef64=False, exact=True,
                 rec_component="vx"):
        self._init_common(vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, nt, accuracy, freq, fieldtype,
                          coef64, exact)
        self.rsx, self.rsy, self.rsz = rsx, rsy, rsz
        self.MT = np.asarray(as_numpy(MT), dtype=np.float32).reshape(3, 3)
        self.src_scale = src_scale
        self.t0 = t0
        self._rec_lin, _ = receiver_table(self.gridsize, rsx, rsy, rsz)
        self.datasize = int(self._rec_lin.size)
        self._rec_component = FIELDS3.index(rec_component)
        self.data = torch.zeros((self.nt, self.datasize), dtype=torch.float32, device=self._dev)
        self.src = torch.zeros(self.nt, dtype=torch.float32, device=self._dev)

    def _source(self):
        wav = BaseFun.series("ricker2", self.nt, self.dt, self.f0, self.src_scale, t0=self.t0)
        M = self.MT
        mt = (M[0, 0], M[1, 1], M[2, 2], M[0, 1], M[0, 2], M[1, 2])
        return N.SW_SRC_MOMENT, (self.isx, self.isy, self.isz), wav, mt

    def _receivers(self):
        return self._rec_component, self._rec_lin

    def update_SSG(self, nt: int):
        """One time step (Elastic3D_SSG_Tensor.py:166-345)."""
        self._step(nt)

    def forward_op(self, vp, vs, rho, checkpoint_every: int = 100):
        """Differentiable seismogram: the (nt, nrec) traces as a function of
        the vp, vs, rho tensors (device, the solver's dtype), with the
        hand-written 3D adjoint as backward (no reference counterpart;
        exact numerics, orders 1..4)."""
        from .adjoint import ForwardOp3D
        return ForwardOp3D.apply(vp, vs, rho, self, int(checkpoint_every))
