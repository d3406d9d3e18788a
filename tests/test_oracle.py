"""CPU tests of the oracle and of the product's host-side set-up.

The reference ships no tests and no golden vectors (its test*.py are plotting
scripts), and Taichi cannot run here, so the oracle is pinned by:
  * known answers of diff_coff (closed-form Taylor coefficients),
  * a second independent transcription (oracle/np_twin.py) that must agree
    with the C++ oracle bit for bit,
  * the committed golden fixtures of tests/golden/ (made by
    tests/golden/make_golden.py from the oracle and checked by the twin),
  * physics: P- and S-wave arrival times, source-receiver reciprocity,
    mirror symmetry (2D force, 3D explosion), CPML absorption and reflection against a large domain,
    and a higher-order stencil converging towards a refined reference.
"""
from fractions import Fraction

import numpy as np
import pytest

from cases import case2d, case3d, oracle2d, oracle3d
from oracle import np_twin
from oracle import oracle as O
from seiswave_taichi_b200 import BaseFun, pml as P


def _taylor_exact(order):
    # exact rational solve of A c = e1, A[i][j] = (2j+1)^(2i+1)
    n = order
    A = [[Fraction((2 * j + 1) ** (2 * i + 1)) for j in range(n)] for i in range(n)]
    b = [Fraction(1 if i == 0 else 0) for i in range(n)]
    for col in range(n):
        piv = next(r for r in range(col, n) if A[r][col] != 0)
        A[col], A[piv] = A[piv], A[col]
        b[col], b[piv] = b[piv], b[col]
        for r in range(n):
            if r != col and A[r][col] != 0:
                f = A[r][col] / A[col][col]
                A[r] = [x - f * y for x, y in zip(A[r], A[col])]
                b[r] -= f * b[col]
    return [b[i] / A[i][i] for i in range(n)]


def test_diff_coff_known_answers():
    assert _taylor_exact(2) == [Fraction(9, 8), Fraction(-1, 24)]
    assert _taylor_exact(3) == [Fraction(75, 64), Fraction(-25, 384), Fraction(3, 640)]
    for n in range(1, 9):
        exact = np.array([float(x) for x in _taylor_exact(n)], np.float32)
        assert np.array_equal(P.diff_coff(n), exact), n
        d, f = O.diff_coff(n)
        assert np.array_equal(f, exact), n
        np.testing.assert_allclose(d, [float(x) for x in _taylor_exact(n)], rtol=1e-9)


def test_diff_coff_op_table():
    assert np.allclose(P.diff_coff_op(2), [1.129042, -0.0430142])
    assert P.diff_coff_op(5).shape == (5,)
    assert not P.diff_coff_op(7).any()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n,star,d,thick,lo,hi", [
    (400, 2, 10.0, 200.0, True, True), (200, 2, 10.0, 200.0, True, True),
    (171, 2, 1.0, 15.0, True, True), (251, 5, 2.5, 37.5, True, True),
    (80, 3, 12.5, 100.0, False, True), (96, 2, 7.3, 73.0, True, False),
])
def test_pml_profiles_match_oracle(dtype, n, star, d, thick, lo, hi):
    freq = 15.0
    args = (n, star, d, thick, lo, hi, 3000.0, 1e-6, np.pi * freq, 1732.0 / (5 * d * freq), 1, 1e-3)
    ours = P.axis_profile(*args, dtype=dtype)
    ref, (pmin, pmax) = O.pml_axis(*args, dtype=dtype)
    for k in P.PROFILE_NAMES:
        assert np.array_equal(ours[k], ref[k]), k
    assert (ours.pml_min, ours.pml_max) == (pmin, pmax)


def test_slab_extent_covers_every_active_index():
    pr = P.axis_profile(200, 2, 10.0, 200.0, True, True, 3000.0, 1e-6, np.pi * 15, 1732 / (5 * 10 * 15), 1, 1e-3)
    lo, hi = P.slab_extent(pr)
    a = pr.arrays
    active = (a["a"] != 0) | (a["k"] != 1) | (a["a_half"] != 0) | (a["k_half"] != 1)
    inside = np.zeros(200, bool)
    inside[:lo] = True
    inside[200 - hi:] = True
    assert not (active & ~inside).any()
    assert (lo, hi) == (22, 23)
    # no PML on one side: that slab is empty
    pr = P.axis_profile(200, 2, 10.0, 200.0, False, True, 3000.0, 1e-6, np.pi * 15, 1732 / 750, 1, 1e-3)
    assert P.slab_extent(pr)[0] == 0


def test_axis_flags_reference_predicate():
    f = P.axis_flags(200, 2, 10.0, 200.0, 3750.0)
    x_int = (np.arange(200) - 2) * 10.0
    assert np.array_equal(f & 1, ((x_int <= 200) | (x_int >= 3750)).astype(np.uint8))
    x_half = x_int + 5.0
    assert np.array_equal((f >> 1) & 1, ((x_half <= 200) | (x_half >= 3750)).astype(np.uint8))


def test_identity_outside_slabs():
    """Outside the slabs the reference's CPML update is an exact no-op:
    a = 0 and kappa = 1, so psi stays 0 and the derivative is unchanged."""
    pr = P.axis_profile(120, 3, 10.0, 150.0, True, True, 3500.0, 1e-6, np.pi * 20, 2000 / 1000, 1, 8e-4)
    lo, hi = P.slab_extent(pr)
    mid = slice(lo, 120 - hi)
    for s in ("", "_half"):
        assert not pr["a" + s][mid].any()
        assert (pr["k" + s][mid] == 1).all()


@pytest.mark.parametrize("kind", ["ricker", "ricker2", "ricker3"])
def test_wavelets_match_oracle(kind):
    nt, dt, f = 1500, 8e-4, 12.0
    t0 = np.float32(1.5) / np.float32(f)
    ours = BaseFun.series(kind, nt, dt, f, 3.0, t0=t0)
    ref = O.wavelet(kind, nt, dt, f, 3.0, t0=float(t0))
    # the two exp() implementations may differ by an ulp
    assert np.max(np.abs(ours - ref)) <= 4 * np.finfo(np.float32).eps * np.max(np.abs(ref))
    assert np.argmax(np.abs(ours)) == np.argmax(np.abs(ref))


def test_ricker2_shape():
    w = BaseFun.series("ricker2", 400, 1e-3, 25.0, 1.0, t0=0.06)
    assert np.argmax(w) == 60 and abs(w[60] - 1.0) < 1e-6


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_twin_2d_vs_bitwise(dtype):
    c = case2d(shape=(48, 40), N=2, npml=6, nt=80, dtype=dtype)
    o = oracle2d(c)
    wav = O.wavelet("ricker2", 80, c["dt"], c["freq"], 1.0, t0=float(np.float32(1.5) / np.float32(c["freq"])))
    o = oracle2d(c, wavelet=wav)
    t = np_twin.Twin2D(o)
    o.run("VS", 0, 80)
    for it in range(80):
        t.step(it, wav[it])
    for f in ("vx", "vz", "sxx", "szz", "sxz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    assert np.array_equal(t.data, o.data)
    for k, v in t.mem.items():
        assert np.array_equal(v, o.memory("memory_" + k)), k
    assert np.abs(o.vz).max() > 0


@pytest.mark.parametrize("N", [2, 3])
def test_twin_3d_tensor_bitwise(N):
    c = case3d(shape=(26, 24, 28), N=N, npml=5, nt=40)
    wav = O.wavelet("ricker2", 40, c["dt"], c["freq"], c["src_scale"], t0=0.03)
    o = oracle3d(c, wavelet=wav)
    t = np_twin.Twin3DTensor(o)
    o.run(0, 40)
    for it in range(40):
        t.step(it, wav[it])
    for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    assert np.array_equal(t.data, o.data)
    for k, v in t.mem.items():
        assert np.array_equal(v, o.memory("memory_" + k)), k


@pytest.mark.parametrize("N,dtype", [(2, np.float32), (3, np.float32), (2, np.float64)])
def test_twin_2d_sv_bitwise(N, dtype):
    """The SV step (Elastic2D_CPML.py:203-274): oracle and numpy
    transcription bit for bit, wavefields, vx trace and memory variables."""
    nt = 80
    c = case2d(shape=(48, 40), N=N, npml=6, nt=nt, dtype=dtype)
    wav = O.wavelet("ricker", nt, c["dt"], c["freq"], 1.0)
    o = oracle2d(c, wavelet=wav)
    t = np_twin.Twin2DSV(o)
    o.run("SV", 0, nt)
    for it in range(nt):
        t.step(it, wav[it])
    for f in ("vx", "vz", "sxx", "szz", "sxz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    assert np.array_equal(t.data, o.data)
    for k, v in t.mem.items():
        assert np.array_equal(v, o.memory("memory_" + k)), k
    assert np.abs(o.vx).max() > 0 and np.abs(o.data).max() > 0


@pytest.mark.parametrize("N,dtype", [(2, np.float32), (3, np.float32), (2, np.float64)])
def test_twin_2d_rsg_bitwise(N, dtype):
    """The rotated-grid step (Elastic2D_CPML.py:277-353) with a caller-given
    source value per step: oracle and numpy transcription bit for bit,
    wavefields and the eight memory variables."""
    from seiswave_taichi_b200 import BaseFun
    nt = 80
    c = case2d(shape=(48, 40), N=N, npml=6, nt=nt, dtype=dtype)
    src = BaseFun.series("ricker", nt, c["dt"], c["freq"], 1.0)
    o = oracle2d(c)
    t = np_twin.Twin2DRSG(o)
    o.run("RSG", 0, nt, rsg_sources=src.astype(np.float64))
    for it in range(nt):
        t.step(it, src[it])
    for f in ("vx", "vz", "sxx", "szz", "sxz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    for k, v in t.mem.items():
        assert np.array_equal(v, o.memory("memory_" + k)), k
    assert np.abs(o.vz).max() > 0 and np.abs(o.memory("memory_dvx_dx")).max() > 0


@pytest.mark.parametrize("N,dtype", [(2, np.float32), (4, np.float32), (2, np.float64)])
def test_twin_3d_cpml_force_bitwise(N, dtype):
    """The point-force CPML step (Elastic3D_SSG_CPML.py:144-309): oracle and
    numpy transcription bit for bit, wavefields, vx trace and the 18 memory
    variables."""
    c = case3d(scheme="CPML", shape=(28, 26, 30), N=N, npml=5, nt=40, dtype=dtype)
    wav = O.wavelet("ricker", 40, c["dt"], c["freq"], 1000.0)
    o = oracle3d(c, wavelet=wav)
    t = np_twin.Twin3DCPML(o)
    o.run(0, 40)
    for it in range(40):
        t.step(it, wav[it])
    for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    assert np.array_equal(t.data, o.data)
    for k, v in t.mem.items():
        assert np.array_equal(v, o.memory("memory_" + k)), k
    assert len(t.mem) == 18 and np.abs(o.vz).max() > 0


@pytest.mark.parametrize("N,dtype", [(2, np.float32), (3, np.float32), (2, np.float64)])
def test_twin_3d_spml_bitwise(N, dtype):
    """The split-field PML step (Elastic3D_SSG_SPML.py:160-393): the C++ oracle
    and the independent numpy transcription agree bit for bit, wavefields,
    trace and all 24 split fields."""
    c = case3d(scheme="SPML", shape=(26, 24, 28), N=N, npml=5, nt=40, dtype=dtype)
    wav = O.wavelet("ricker", 40, c["dt"], c["freq"], c["src_scale"])
    o = oracle3d(c, wavelet=wav)
    t = np_twin.Twin3DSPML(o)
    o.run(0, 40)
    for it in range(40):
        t.step(it, wav[it])
    for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
        assert np.array_equal(getattr(t, f), getattr(o, f)), f
    assert np.array_equal(t.data, o.data)
    for name in t.SPLIT:
        assert np.array_equal(t.split[name], o.memory(name)), name
    assert np.abs(o.vx).max() > 0 and np.abs(o.memory("sxx_x")).max() > 0


def test_oracle_p_arrival_time():
    """Homogeneous 2D medium: the first arrival at a receiver r metres from an
    explosive-like vz source comes at about r / vp."""
    nx = 220
    c = case2d(shape=(nx, nx), N=2, hetero=False, npml=20, nt=420, freq=25.0)
    c["isx"], c["isz"] = 110, 110
    c["rsx"], c["rsz"] = 110, 110 + 100  # 1000 m straight down
    o = oracle2d(c).run("VS", 0, 420)
    tr = np.abs(o.data)
    t_peak = np.argmax(tr) * c["dt"]
    # Ricker2 peaks at t0 = 1.5/f = 0.06 s, then travels 1000 m at 3000 m/s
    assert abs(t_peak - (0.06 + 1000.0 / 3000.0)) < 0.02


def test_oracle_s_arrival_time():
    """A vertical point force radiates S waves, not P, along the horizontal:
    the vz peak 1000 m away along x comes at about t0 + r / vs (0.637 s;
    numerical dispersion of the S wave, ~3 cells per wavelength at the top of
    the band, delays it by ~20 ms), far from the P time t0 + r / vp (0.393 s)."""
    c = case2d(shape=(240, 140), N=2, hetero=False, npml=20, nt=760, freq=25.0)
    c["isx"], c["isz"] = 60, 70
    c["rsx"], c["rsz"] = 160, 70
    o = oracle2d(c).run("VS", 0, 760)
    t_peak = np.argmax(np.abs(o.data)) * c["dt"]
    assert abs(t_peak - (0.06 + 1000.0 / 1732.0)) < 0.03, t_peak


def test_oracle_source_receiver_reciprocity():
    """Constant density, varying vp and vs: the vz trace at B from a vertical
    force at A equals the vz trace at A from the force at B (the staggered
    operators are transposes of each other; the window ends before the waves
    reach the CPML).  Measured: 1.9e-7 relative."""
    c = case2d(shape=(160, 160), N=2, hetero=True, npml=20, nt=130, freq=25.0)
    c["rho"] = np.full(c["shape"], 2000.0, np.float32)

    def trace(src, rec):
        cc = dict(c)
        cc["isx"], cc["isz"] = src
        cc["rsx"], cc["rsz"] = rec
        return oracle2d(cc).run("VS", 0, 130).data.astype(np.float64)

    ab, ba = trace((70, 80), (86, 74)), trace((86, 74), (70, 80))
    assert np.abs(ab).max() > 0
    assert np.linalg.norm(ab - ba) / np.linalg.norm(ab) < 1e-5


def test_oracle_cpml_reflection_against_large_domain():
    """A receiver 8 cells inside the 20-cell CPML's inner edge, 0.5 s: its
    trace differs from the same point in a domain so large that no boundary
    echo returns by 3.7e-5 relative L2 (measured); a 5-cell CPML on the same
    grid reflects about 60 times more."""
    nt = 500

    def trace(n, npml, src, rec):
        c = case2d(shape=(n, n), N=2, hetero=False, npml=npml, nt=nt, freq=25.0)
        c["isx"], c["isz"] = src
        c["rsx"], c["rsz"] = rec
        return oracle2d(c).run("VS", 0, nt).data.astype(np.float64)

    big = trace(320, 20, (160, 160), (160, 190))
    rel = lambda a: np.linalg.norm(a - big) / np.linalg.norm(big)
    e20 = rel(trace(120, 20, (60, 60), (60, 90)))
    e5 = rel(trace(120, 5, (60, 60), (60, 90)))
    assert e20 < 2e-4 and e5 > 10 * e20, (e20, e5)


def test_oracle_higher_order_converges():
    """Grid refinement and stencil order: on a 10 m grid the 4th-order-pair
    (N=4) stencil reproduces a 5 m, N=4 reference trace (500 m offset, 0.45 s)
    better than N=2 (measured 2.3% against 6.5% relative L2 after a
    least-squares amplitude fit), and the fitted amplitude is the cell-area
    ratio 1/4 of a point force."""

    def trace(n, N, h, dt, nt, npml, src, rec):
        c = case2d(shape=(n, n), N=N, hetero=False, npml=npml, nt=nt, freq=25.0, dx=h, dz=h, dt=dt)
        c["isx"], c["isz"] = src
        c["rsx"], c["rsz"] = rec
        return oracle2d(c).run("VS", 0, nt).data.astype(np.float64)

    ref = trace(400, 4, 5.0, 5e-4, 900, 40, (200, 200), (200, 300))[1::2]

    def err(N):
        a = trace(200, N, 10.0, 1e-3, 450, 20, (100, 100), (100, 150))
        al = np.dot(a, ref) / np.dot(a, a)
        return np.linalg.norm(al * a - ref) / np.linalg.norm(ref), al

    (e2, a2), (e4, a4) = err(2), err(4)
    assert e4 < 0.5 * e2 and e4 < 0.04, (e2, e4)
    assert abs(a4 - 0.25) < 0.01 and abs(a2 - 0.25) < 0.01, (a2, a4)


def test_oracle_mirror_symmetry():
    """A vz point force at the centre of a homogeneous box gives a vz field
    that is even under x -> -x.  vz lives at x = (i - N + 1/2) dx; with
    nx = 100 and N = 2 the box centre is x = 47.5 dx, the vz point of i = 49,
    and the mirror maps i -> 98 - i (the PML profiles are symmetric too)."""
    c = case2d(shape=(100, 90), N=2, hetero=False, npml=10, nt=150)
    c["isx"] = 49
    o = oracle2d(c).run("VS", 0, 150)
    vz = o.vz.astype(np.float64)
    lhs = vz[3:49, :]
    rhs = vz[95:49:-1, :]
    assert np.abs(vz).max() > 0
    # equal up to the rounding of the unsymmetric summation order
    assert np.max(np.abs(lhs - rhs)) <= 1e-4 * np.max(np.abs(vz))


def test_oracle_3d_explosion_mirror_symmetry():
    """3D tensor scheme, explosive source (M = I) at the centre of an odd
    homogeneous box: the grid and its PML profiles are symmetric about the
    source, so the normal stresses (integer points) are even and vx (at
    i + 1/2, mirror i -> 59 - i) is odd under x -> -x, and the stresses even
    in y and z, up to the rounding of the unsymmetric summation orders
    (measured below 1e-6 of the maxima)."""
    c = case3d(shape=(61, 57, 63), N=2, scheme="TENSOR", hetero=False, npml=8, nt=80)
    c["isx"], c["isy"], c["isz"] = 30, 28, 31
    c["MT"] = np.eye(3, dtype=np.float32)
    o = oracle3d(c).run(0, 80)
    sxx, szz, vx = (getattr(o, f).astype(np.float64) for f in ("sxx", "szz", "vx"))
    rel = lambda d, f: np.abs(d).max() / np.abs(f).max()
    assert np.abs(sxx).max() > 0 and np.abs(vx).max() > 0
    assert rel(sxx - sxx[::-1], sxx) < 1e-5
    assert rel(szz - szz[::-1], szz) < 1e-5
    assert rel(vx[:60] + vx[59::-1], vx) < 1e-5
    assert rel(sxx - sxx[:, ::-1], sxx) < 1e-5 and rel(sxx - sxx[:, :, ::-1], sxx) < 1e-5


def test_oracle_cpml_absorbs():
    """After the wave has crossed the boundary, energy left in a CPML-bounded
    box is a small fraction of its peak (the reflections are weak)."""
    c = case2d(shape=(120, 120), N=2, hetero=False, npml=20, nt=700, freq=25.0)
    o = oracle2d(c)
    energies = []
    for k in range(14):
        o.run("VS", k * 50, 50)
        energies.append(float(np.sum(o.vx.astype(np.float64) ** 2 + o.vz.astype(np.float64) ** 2)))
    assert energies[-1] < 1e-3 * max(energies)


def test_oracle_2d_moment_source_and_receiver_table():
    """The 2D moment-tensor source injects -w*M into the stresses at the start
    of each step; the receiver table samples the scheme's component after the
    stress phase (the last row equals the final field at those cells)."""
    from cases import case2d, oracle2d
    from seiswave_taichi_b200 import BaseFun
    c = case2d(nt=60, hetero=False, MT=[[1.0, 0.0], [0.0, 1.0]], nrec=9, src_scale=1e5)
    wav = BaseFun.series("ricker2", 60, c["dt"], c["freq"], 1e5, t0=np.float32(1.5) / np.float32(c["freq"]))
    o = oracle2d(c, wavelet=wav).run("VS", 0, 60)
    # linear in the source: twice the wavelet gives twice the traces
    o2 = oracle2d(c, wavelet=(2 * wav).astype(np.float32)).run("VS", 0, 60)
    np.testing.assert_allclose(o2.data, 2 * o.data, rtol=1e-6, atol=1e-30)
    assert np.abs(o.data).max() > 0
    idx = np.asarray(c["rsx"]).reshape(-1) * c["shape"][1] + np.asarray(c["rsz"]).reshape(-1)
    assert o.data.shape == (60, 9)
    np.testing.assert_array_equal(o.data[59], o.vz.reshape(-1)[idx])
    # an explosive source in a homogeneous medium is mirror-symmetric in x
    # about the source's sxx/szz position (x half point, i + 1/2): vx(i+1/2+d) = -vx(i+1/2-d)
    i0 = c["isx"]
    np.testing.assert_allclose(o.szz[i0 + 5, :], o.szz[i0 - 5, :], rtol=0, atol=1e-6 * np.abs(o.szz).max())
