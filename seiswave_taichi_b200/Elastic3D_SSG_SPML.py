"""Drop-in for src/Elastic3D_SSG_SPML.py: 3D SSG with the classic split-field
PML (damping d only), a vertical point force and one receiver.

Per step (Elastic3D_SSG_SPML.py:160-393): velocity phase (inside the PML each
component is the sum of its split parts), the point force vz[isx,isy,isz] +=
dt*Ricker(it, dt, freq, src_scale)/rho, stress phase, data[it] = vx[rsx,rsy,rsz].
"""
from __future__ import annotations

import torch

from . import _native as N
from . import BaseFun
from ._common import receiver_table
from ._elastic3d import Elastic3DBase


class ElasticWAVE(Elastic3DBase):
    _scheme = N.SW3D_SPML

    def __init__(self, vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, rsx, rsy, rsz, nt, accuracy,
                 freq=100., src_scale=1., fieldtype=torch.float32, *, coef64=False, exact=True):
        self._init_common(vs, vp, rho, dx, dy, dz, dt, isx, isy, isz, nt, accuracy, freq, fieldtype,
                          coef64, exact)
        self.src_scale = src_scale
        self.rsx, self.rsy, self.rsz = rsx, rsy, rsz
        self._rec_lin, _ = receiver_table(self.gridsize, rsx, rsy, rsz)
        self.data = torch.zeros(self.nt, dtype=torch.float32, device=self._dev)

    def _source(self):
        wav = BaseFun.series("ricker", self.nt, self.dt, self.f0, self.src_scale)
        return N.SW_SRC_FORCE, (self.isx, self.isy, self.isz), wav, (0,) * 6

    def _receivers(self):
        return 0, self._rec_lin

    def update_SSG_SPML(self, nt: int):
        """One time step (Elastic3D_SSG_SPML.py:160-393)."""
        self._step(nt)
