"""One full-waveform-inversion gradient step over a batch of 2D shots of
uneven sizes (no reference counterpart; the forward is Elastic2D_CPML.py's
update_SSG_VS loop, :128-200).

    step = FWIStep(waves, checkpoint_every=100)    # ElasticWAVE objects, MT source
    misfit, grads = step(d_obs)                    # grads[s] = (g_vp, g_vs, g_rho)

The forward runs all shots together (ShotBatch2D: per step one velocity and
one stress launch over every shot's tiles), one checkpoint interval at a time,
copying every shot's state at the start of each interval.  The misfit is
J = sum_s 0.5 * |d_s - d_obs_s|^2.  Each shot's backward pass then restores
its checkpoints from last to first, re-runs the interval with snapshots and
steps the hand-written adjoint back over it (adjoint.Adjoint2D), and chains
the coefficient gradients to vp, vs and rho.  The batched forward is
bit-identical to each shot's own run, so the gradients equal the per-shot
ones (ElasticWAVE.forward_op) exactly.
"""
from __future__ import annotations

import torch

from .adjoint import Adjoint2D
from .batch import ShotBatch2D


class FWIStep:
    def __init__(self, waves, checkpoint_every: int = 100, autotune: bool = True):
        self.waves = list(waves)
        self.K = int(checkpoint_every)
        self.batch = ShotBatch2D(self.waves, "VS", autotune=autotune)
        self.drivers = [Adjoint2D(w, self.K) for w in self.waves]
        self.nt = self.waves[0].nt

    def forward(self):
        """All shots' traces, keeping each shot's checkpoints."""
        for d in self.drivers:
            d.checkpoints = []
            d.nt = self.nt
        self.batch.reset()
        for it0 in range(0, self.nt, self.K):
            n = min(self.K, self.nt - it0)
            for d in self.drivers:
                d.checkpoints.append((it0, n, [t.clone() for t in d._state()]))
            self.batch.run(n, it0)
        return [w.data.clone() for w in self.waves]

    def __call__(self, d_obs):
        traces = self.forward()
        misfit = 0.0
        grads = []
        for w, d, tr, ob in zip(self.waves, self.drivers, traces, d_obs):
            r = tr - ob.to(tr.dtype)
            misfit += 0.5 * float((r.double() ** 2).sum())
            g_rho, g_lam, g_mu = d.backward(r)
            vp, vs, rho = w.vp, w.vs, w.rho
            g_vp = g_lam * 2 * rho * vp
            g_vs = g_mu * 2 * rho * vs - g_lam * 4 * rho * vs
            g_rh = g_rho + g_mu * vs * vs + g_lam * (vp * vp - 2 * vs * vs)
            grads.append((g_vp, g_vs, g_rh))
        return misfit, grads
