"""The 3D solver's autotuner: it picks an x chunk from its candidates for the
current path, leaves the state as it found it (bit for bit), reuses its
cached choice, and runs after tuning equal untuned runs bit for bit."""
import numpy as np
import pytest
import torch

from cases import case3d, product3d, to_np

pytestmark = pytest.mark.gpu

F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


@pytest.mark.parametrize("exact", [True, False])
def test_autotune_keeps_state_and_results(cuda, tmp_path, monkeypatch, exact):
    monkeypatch.setenv("SEISWAVE_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    c = case3d(shape=(40, 36, 44), N=2, scheme="TENSOR", nt=60, npml=8, seed=2)
    a = product3d(c, exact=exact)
    a.run(20)
    before = {f: to_np(getattr(a, f)).copy() for f in F3}
    chunk = a.autotune(steps=3)
    assert chunk in a.AUTOTUNE_CHUNKS
    for f in F3:
        assert to_np(getattr(a, f)).tobytes() == before[f].tobytes(), f
    a.run(40, it0=20)
    b = product3d(c, exact=exact)
    b.run(60)
    for f in F3:
        assert to_np(getattr(a, f)).tobytes() == to_np(getattr(b, f)).tobytes(), f
    assert to_np(a.data).tobytes() == to_np(b.data).tobytes()
    # a second solver of the same bucket takes the cached choice
    c2 = product3d(c, exact=exact)
    assert c2.autotune(steps=3) == chunk
    torch.cuda.synchronize()


def test_autotune_keeps_split_pml_state(cuda, tmp_path, monkeypatch):
    """The split-PML solver's shell of split fields is saved and restored
    around the trial steps like the wavefields."""
    monkeypatch.setenv("SEISWAVE_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    c = case3d(shape=(40, 36, 44), N=2, scheme="SPML", nt=60, npml=8, seed=3)
    a = product3d(c)
    a.run(20)
    split = a._split.clone()
    a.autotune(steps=3)
    assert torch.equal(a._split, split)
    a.run(40, it0=20)
    b = product3d(c)
    b.run(60)
    for f in F3:
        assert to_np(getattr(a, f)).tobytes() == to_np(getattr(b, f)).tobytes(), f
    assert torch.equal(a._split, b._split)
