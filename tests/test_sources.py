"""Moment-tensor helpers (sources.py) on the CPU: a double couple is
deviatoric with eigenvalues (+m0, 0, -m0) for any strike/dip/rake, and two
textbook cases come out as expected in the x = north, y = east, z = down
frame; the explosive and random tensors are symmetric and reproducible."""
import numpy as np
import pytest

from seiswave_taichi_b200 import sources as S


@pytest.mark.parametrize("sdr", [(30, 60, 90), (0, 90, 0), (117, 23, -45), (250, 80, 170), (45, 45, 90)])
def test_double_couple_is_a_pure_double_couple(sdr):
    M = S.double_couple(*sdr, m0=2.5).astype(np.float64)
    assert np.allclose(M, M.T)
    assert abs(np.trace(M)) < 1e-5
    ev = np.sort(np.linalg.eigvalsh(M))
    assert np.allclose(ev, [-2.5, 0.0, 2.5], atol=1e-5)


def test_double_couple_textbook_cases():
    # vertical strike-slip fault striking north, left-lateral slip: Mxy only
    assert np.allclose(S.double_couple(0, 90, 0), [[0, 1, 0], [1, 0, 0], [0, 0, 0]], atol=1e-7)
    # 45-degree thrust striking north: horizontal east-west compression,
    # vertical extension
    assert np.allclose(S.double_couple(0, 45, 90), np.diag([0.0, -1.0, 1.0]), atol=1e-7)


def test_explosive_and_random_tensors():
    assert np.array_equal(S.explosive(3.0), 3.0 * np.eye(3, dtype=np.float32))
    a, b = S.random_tensor(7), S.random_tensor(7)
    assert np.array_equal(a, b) and np.array_equal(a, a.T) and a.dtype == np.float32
    assert not np.array_equal(a, S.random_tensor(8))


def test_moment_2d_forms():
    """2D moment tensors as (xx, zz, xz): 'explosive', a 2x2 [[xx, xz], [xz, zz]]
    array, or a 3x3 tensor's x-z block (x first axis, z last)."""
    from seiswave_taichi_b200.Elastic2D_CPML import moment_2d
    assert moment_2d("explosive").tolist() == [1.0, 1.0, 0.0]
    assert moment_2d([[0.5, -2.0], [-2.0, 3.0]]).tolist() == [0.5, 3.0, -2.0]
    M = S.double_couple(30, 60, 90)
    assert np.array_equal(moment_2d(M), np.array([M[0, 0], M[2, 2], M[0, 2]], np.float32))
    for bad in ("implosive", np.zeros(3), np.zeros((2, 3))):
        with pytest.raises(ValueError):
            moment_2d(bad)
