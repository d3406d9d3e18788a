"""Golden fixtures (tests/golden/oracle_small.npz, written by
tests/golden/make_golden.py from the CPU oracle): the oracle must keep
reproducing them (CPU, relative 1e-6 to allow another compiler's rounding of
the host build), and the GPU kernels must equal them bit for bit (the exact
numeric mode)."""
from pathlib import Path

import numpy as np
import pytest

from golden.make_golden import cases, rsg_sources, run, wavelet_of

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "oracle_small.npz")


def test_diff_coff_fixture():
    from seiswave_taichi_b200.pml import diff_coff
    for n in range(1, 9):
        np.testing.assert_array_equal(diff_coff(n), GOLD[f"diff_coff_{n}"])
    np.testing.assert_allclose(GOLD["diff_coff_2"], [1.125, -1 / 24], rtol=1e-6)


@pytest.mark.parametrize("item", cases(), ids=lambda t: t[0])
def test_oracle_reproduces_fixture(item):
    out = run(*item)
    for k, v in out.items():
        np.testing.assert_allclose(v, GOLD[k], rtol=1e-6, atol=1e-6 * np.abs(GOLD[k]).max(), err_msg=k)
        assert np.abs(GOLD[k]).max() > 0, k


@pytest.mark.gpu
@pytest.mark.parametrize("item", cases(), ids=lambda t: t[0])
def test_gpu_equals_fixture(cuda, item):
    import torch
    from cases import product2d, product3d, to_np
    name, c, scheme, steps = item
    if scheme == "RSG":
        w = product2d(c)
        src = rsg_sources(c)
        for it in range(steps):
            w.update_RSG(it, float(src[it]))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_np(w.vx), GOLD[f"{name}_vx"])
        np.testing.assert_array_equal(to_np(w.vz), GOLD[f"{name}_vz"])
        return
    if scheme in ("VS", "SV"):
        w = product2d(c)
        w.run(steps, scheme=scheme)
    else:
        w = product3d(c)
        w._build_plan()
        wav = to_np(w._wavelet).astype(np.float32)
        np.testing.assert_array_equal(wav[:steps], wavelet_of(c, scheme)[:steps])
        w.run(steps)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_np(w.data), GOLD[f"{name}_data"])
    np.testing.assert_array_equal(to_np(w.vx), GOLD[f"{name}_vx"])
