"""Batched ragged 2D shots (ShotBatch2D, one CUDA graph for all shots and
steps) against each shot's own single-shot run: the kernels evaluate every
cell with the same expressions, so wavefields and traces must be equal bit for
bit, for every tile shape the autotuner can choose."""
import numpy as np
import pytest

from cases import case2d, product2d, to_np

pytestmark = pytest.mark.gpu

F2 = ("vx", "vz", "sxx", "szz", "sxz")
SHAPES = [(64, 48), (90, 57), (41, 120), (77, 77), (50, 66)]


def _shots(dtype=np.float32, nt=120, N=2, mt="explosive"):
    cs = []
    for q, shape in enumerate(SHAPES):
        c = case2d(shape=shape, N=N, nt=nt, dtype=dtype, seed=10 + q, nrec=5 + q, MT=mt, src_scale=1e5, npml=8)
        cs.append(c)
    return cs


@pytest.mark.parametrize("scheme", ["VS", "SV"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_batch_equals_single_shots(cuda, scheme, dtype):
    from seiswave_taichi_b200.batch import ShotBatch2D, TILES
    cs = _shots(dtype)
    ref = []
    for c in cs:
        w = product2d(c)
        w.run(c["nt"], scheme=scheme)
        ref.append(w)
    waves = [product2d(c) for c in cs]
    b = ShotBatch2D(waves, scheme=scheme, autotune=False)
    for k in range(len(TILES)):
        b.reset()
        b.set_tile(k)
        assert b.info()["tile"] == k
        b.run()
        for w, r in zip(waves, ref):
            for f in F2:
                np.testing.assert_array_equal(to_np(getattr(w, f)), to_np(getattr(r, f)), err_msg=f"{f} tile {k}")
            np.testing.assert_array_equal(to_np(w.data), to_np(r.data))
    assert np.abs(to_np(ref[0].data)).max() > 0


def test_batch_per_step_and_graph_agree(cuda):
    from seiswave_taichi_b200.batch import ShotBatch2D
    cs = _shots(N=3)
    a = [product2d(c) for c in cs]
    ba = ShotBatch2D(a, autotune=False)
    ba.run(40)
    ba.run(80, it0=40)
    b = [product2d(c) for c in cs]
    ShotBatch2D(b, autotune=False).run(use_graph=False)
    for x, y in zip(a, b):
        for f in F2:
            np.testing.assert_array_equal(to_np(getattr(x, f)), to_np(getattr(y, f)))


def test_autotune_restores_state_and_caches(cuda, tmp_path, monkeypatch):
    from seiswave_taichi_b200.batch import ShotBatch2D, TILES
    monkeypatch.setenv("SEISWAVE_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    cs = _shots()
    waves = [product2d(c) for c in cs]
    b = ShotBatch2D(waves, autotune=False)
    b.run(30)
    before = [to_np(w.vx).copy() for w in waves]
    k = b.autotune(steps=3)
    assert 0 <= k < len(TILES) and b.info()["tile"] == k
    for w, v in zip(waves, before):
        np.testing.assert_array_equal(to_np(w.vx), v)
    assert (tmp_path / "tune.json").exists()
    b2 = ShotBatch2D([product2d(c) for c in cs])  # cached choice
    assert b2.info()["tile"] == k


def test_batch_rejects_mixed_orders(cuda):
    import seiswave_taichi_b200._native as N
    from seiswave_taichi_b200.batch import ShotBatch2D
    w1 = product2d(case2d(N=2, nt=50))
    w2 = product2d(case2d(N=3, nt=50))
    with pytest.raises(N.SeisWaveError, match="differs from shot 0"):
        ShotBatch2D([w1, w2], autotune=False)
