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
the coefficient gradients to vp, vs and rho.  The backward passes of
different shots share nothing, so they run concurrently: `streams` CUDA
streams, each fed by its own host thread (the native calls release the
interpreter lock), take the shots round robin after waiting for the forward,
and the caller's stream waits for all of them before the misfit is read.
The batched forward is bit-identical to each shot's own run, so the
gradients equal the per-shot ones (ElasticWAVE.forward_op) exactly.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import torch

from .adjoint import Adjoint2D
from .batch import ShotBatch2D


class FWIStep:
    def __init__(self, waves, checkpoint_every: int = 100, autotune: bool = True, streams: int = 8):
        self.waves = list(waves)
        self.K = int(checkpoint_every)
        self.batch = ShotBatch2D(self.waves, "VS", autotune=autotune)
        self.drivers = [Adjoint2D(w, self.K) for w in self.waves]
        self.nt = self.waves[0].nt
        self.nstreams = max(1, min(int(streams), len(self.waves)))
        self._streams = None

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

    @staticmethod
    def _shot_grad(w, d, r):
        g_rho, g_lam, g_mu = d.backward(r)
        vp, vs, rho = w.vp, w.vs, w.rho
        g_vp = g_lam * 2 * rho * vp
        g_vs = g_mu * 2 * rho * vs - g_lam * 4 * rho * vs
        g_rh = g_rho + g_mu * vs * vs + g_lam * (vp * vp - 2 * vs * vs)
        return g_vp, g_vs, g_rh

    def __call__(self, d_obs):
        traces = self.forward()
        res = [tr - ob.to(tr.dtype) for tr, ob in zip(traces, d_obs)]
        main = torch.cuda.current_stream(self.waves[0]._dev)
        if self._streams is None:
            self._streams = [torch.cuda.Stream(device=main.device) for _ in range(self.nstreams)]
        for s in self._streams:
            s.wait_stream(main)
        grads = [None] * len(self.waves)

        def lane(k):
            with torch.cuda.device(main.device), torch.cuda.stream(self._streams[k]):
                for q in range(k, len(self.waves), self.nstreams):
                    grads[q] = self._shot_grad(self.waves[q], self.drivers[q], res[q])

        if self.nstreams == 1:
            lane(0)
        else:
            with ThreadPoolExecutor(max_workers=self.nstreams) as ex:
                for f in [ex.submit(lane, k) for k in range(self.nstreams)]:
                    f.result()
        for s in self._streams:
            main.wait_stream(s)
        misfit = sum(0.5 * float((r.double() ** 2).sum()) for r in res)
        return misfit, grads
