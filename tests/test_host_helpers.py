"""Host-side input handling of the drop-in classes (CPU): the reference's
fieldtype spellings, array conversion of torch / numpy / ti.field-like
inputs, receiver tables (a single receiver, the tensor variant's (1, nrec)
arrays, broadcasting, bounds), and mu / lam computed in the reference's
float32 operation order (Elastic2D_CPML.py:93-110)."""
import numpy as np
import pytest
import torch

from seiswave_taichi_b200._common import as_numpy, compute_lam, compute_mu, receiver_table, torch_dtype


class _Field:
    """Stand-in for a ti.field: only to_numpy()."""

    def __init__(self, a):
        self.a = a

    def to_numpy(self):
        return self.a


@pytest.mark.parametrize("spelling,want", [
    (None, torch.float32), (torch.float32, torch.float32), (torch.float64, torch.float64),
    (np.float32, torch.float32), (np.float64, torch.float64), ("f32", torch.float32), ("ti.f64", torch.float64),
    ("float64", torch.float64),
])
def test_fieldtype_spellings(spelling, want):
    assert torch_dtype(spelling) == want


@pytest.mark.parametrize("bad", [torch.int32, torch.float16, "f16", np.int64])
def test_fieldtype_refused(bad):
    with pytest.raises(TypeError):
        torch_dtype(bad)


def test_as_numpy_inputs():
    a = np.arange(6.0).reshape(2, 3)
    for x in (a, torch.as_tensor(a), _Field(a), a.tolist()):
        assert np.array_equal(as_numpy(x), a)


def test_receiver_tables():
    shape = (10, 12, 14)
    lin, single = receiver_table(shape, 3, 4, 5)
    assert single and lin.tolist() == [(3 * 12 + 4) * 14 + 5]
    rx = np.array([[1, 2, 9]])
    lin, single = receiver_table(shape, rx, np.array([[0, 11, 5]]), 7)  # a scalar broadcasts
    assert not single and lin.tolist() == [(1 * 12 + 0) * 14 + 7, (2 * 12 + 11) * 14 + 7, (9 * 12 + 5) * 14 + 7]
    lin2, _ = receiver_table((10, 12), torch.tensor([0, 9]), 11)
    assert lin2.tolist() == [11, 9 * 12 + 11]
    for bad in ((10, 0, 0), (0, -1, 0), (0, 0, 14)):
        with pytest.raises(IndexError):
            receiver_table(shape, *bad)


def test_mu_lam_in_reference_order():
    g = np.random.default_rng(0)
    vp = g.uniform(2000, 6000, 50).astype(np.float32)
    vs = (vp / np.float32(1.73)).astype(np.float32)
    rho = g.uniform(1800, 2600, 50).astype(np.float32)
    mu = compute_mu(torch.as_tensor(vs), torch.as_tensor(rho)).numpy()
    lam = compute_lam(torch.as_tensor(vs), torch.as_tensor(vp), torch.as_tensor(rho)).numpy()
    assert np.array_equal(mu, rho * vs ** 2)
    assert np.array_equal(lam, rho * (vp ** 2 - np.float32(2) * vs ** 2))
