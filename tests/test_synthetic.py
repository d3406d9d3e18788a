"""The seeded synthetic models that stand in for the benchmark workloads'
data (CPU): the thrust belt has 12 layer velocities from 2000 to 6000 m/s,
a +/-3% Gaussian-correlated perturbation, vs = vp / 1.73 and Gardner
density; the correlated noise is zero-mean, unit-std with a Gaussian
correlation of the requested length; the batched 2D workload's 64 models
have the stated size ranges and keep sources and receivers on the grid."""
import numpy as np

from seiswave_taichi_b200 import synthetic as S


def test_correlated_noise_statistics():
    f = S.correlated_noise((64, 64, 64), 4.0, 3)
    assert abs(f.mean()) < 1e-9 and abs(f.std() - 1.0) < 1e-9
    # Gaussian correlation exp(-r^2 / (2 L^2)): exp(-1/2) at one length, exp(-2) at two
    for axis in (0, 2):
        c1 = np.mean(f * np.roll(f, 4, axis=axis))
        c2 = np.mean(f * np.roll(f, 8, axis=axis))
        assert abs(c1 - np.exp(-0.5)) < 0.08 and c2 < 0.3, (axis, c1, c2)


def test_thrust_belt_model():
    shape = (60, 50, 40)
    base, _, _ = S.thrust_belt(shape, 12.5, seed=0, pert=0.0)
    levels = (2000.0 + np.arange(12) * 4000.0 / 11).astype(np.float32)
    assert set(np.unique(base).tolist()) == set(levels.tolist())
    vp, vs, rho = S.thrust_belt(shape, 12.5, seed=0)
    ratio = vp.astype(np.float64) / base
    assert ratio.min() >= 0.97 - 1e-6 and ratio.max() <= 1.03 + 1e-6 and np.std(ratio - 1) > 0.01
    assert np.array_equal(vs, (vp / np.float32(1.73)).astype(np.float32))
    assert np.array_equal(rho, S.gardner(vp))
    np.testing.assert_allclose(S.gardner(np.float32(2000.0)), 1741.0 * 2.0 ** 0.25, rtol=1e-6)
    again = S.thrust_belt(shape, 12.5, seed=0)
    assert all(np.array_equal(a, b) for a, b in zip((vp, vs, rho), again))
    assert not np.array_equal(vp, S.thrust_belt(shape, 12.5, seed=1)[0])


def test_batched_2d_workload():
    shots = S.config4(nshots=64, nt=10)
    assert len(shots) == 64
    sizes = {s["shape"] for s in shots}
    assert len(sizes) > 50
    for s in shots:
        nx, nz = s["shape"]
        assert 600 <= nx <= 1200 and 300 <= nz <= 500
        assert s["vp"].min() >= 1500 - 1e-3 and s["vp"].max() <= 4500 * 1.10 + 1e-3
        assert 0 <= s["isx"] < nx and 0 <= s["isz"] < nz
        assert s["rsx"].min() >= 0 and s["rsx"].max() < nx and (s["rsz"] < nz).all()
