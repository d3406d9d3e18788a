"""Drop-in for src/Elastic2D_sparse.py: the 2D P-SV solver whose CPML memory
variables live in a bitmasked (sparse) Taichi field (Elastic2D_sparse.py:51-64)
instead of dense arrays.  This library's 2D solver already keeps them only on
the PML slabs, so the class is Elastic2D_CPML.ElasticWAVE with that file's one
difference in the physics: update_SSG_VS's source is Ricker(nt, dt, f0, 1)
(the first-derivative wavelet with t0 = 1.5/f0, Elastic2D_sparse.py:170)
instead of Ricker2.  The memory variables are reachable as the reference's
struct members, w.memory.sxx_dx and so on, full-grid like the dense names.
"""
from __future__ import annotations

from . import BaseFun
from .Elastic2D_CPML import ElasticWAVE as _DenseWAVE


class _MemoryStruct:
    """w.memory.<name>: the full-grid view of memory variable <name>."""

    def __init__(self, wave):
        self._w = wave

    def __getattr__(self, name):
        return getattr(self._w, "memory_" + name)


class ElasticWAVE(_DenseWAVE):
    def _vs_wavelet(self):
        return BaseFun.series("ricker", self.nt, self.dt, self.f0, self.src_scale)

    @property
    def memory(self):
        return _MemoryStruct(self)
