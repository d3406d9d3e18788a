"""FWIStep: batched ragged forward with checkpoints + per-shot adjoints.  The
batched forward is bit-identical to single-shot runs, so its misfit and
gradients must equal those of each shot's own forward_op / autograd backward
exactly (float64 here, so the comparison is free of accumulated float32
rounding differences in the host-side chain)."""
import numpy as np
import pytest

from cases import case2d, product2d

pytestmark = pytest.mark.gpu

SHAPES = [(64, 48), (70, 57), (52, 66)]


def _cases():
    return [case2d(shape=s, N=2, nt=130, npml=8, dtype=np.float64, seed=20 + q, nrec=6 + q, MT="explosive",
                   src_scale=1e5) for q, s in enumerate(SHAPES)]


@pytest.mark.parametrize("streams", [1, 3])
def test_fwi_step_equals_per_shot_autograd(cuda, streams):
    from seiswave_taichi_b200.fwi import FWIStep
    cs = _cases()
    # observed data from perturbed models
    d_obs = []
    for c in cs:
        w = product2d(c)
        d_obs.append(w.forward_op(w.vp * 1.03, w.vs * 0.98, w.rho).detach())
    waves = [product2d(c) for c in cs]
    step = FWIStep(waves, checkpoint_every=40, autotune=False, streams=streams)
    misfit, grads = step(d_obs)
    tot = 0.0
    for c, ob, (gvp, gvs, grh) in zip(cs, d_obs, grads):
        w = product2d(c)
        vp = w.vp.clone().requires_grad_(True)
        vs = w.vs.clone().requires_grad_(True)
        rh = w.rho.clone().requires_grad_(True)
        loss = 0.5 * ((w.forward_op(vp, vs, rh, checkpoint_every=40) - ob) ** 2).sum()
        loss.backward()
        tot += float(loss.detach())
        for a, b in ((gvp, vp.grad), (gvs, vs.grad), (grh, rh.grad)):
            np.testing.assert_allclose(a.cpu().numpy(), b.cpu().numpy(), rtol=1e-12, atol=1e-12 * float(b.abs().max()))
    assert misfit == pytest.approx(tot, rel=1e-12)
    assert misfit > 0
