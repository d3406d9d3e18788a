"""The split-field PML's shell storage: the 24 split fields are kept only on
the union of the axes' slabs [0, lo) and [n-hi, n), with lo and hi taken from
the predicate flags (pml.flag_extent).  These CPU tests check that the slabs
cover every flagged index for the reference's PML set-ups, and that the shell
ordering used by the kernels (x slabs, then the y slabs of the x interior, then
the z slabs of the x-y interior) is a bijection onto the shell that
shell_to_full inverts."""
import numpy as np
import pytest
import torch

from seiswave_taichi_b200 import pml as P
from seiswave_taichi_b200._elastic3d import shell_size, shell_to_full


def _slab(i, n, lo, hi):
    return i if i < lo else (i - (n - hi) + lo if i >= n - hi else -1)


def _shell_index(i, j, k, grid, lohi):
    """Restatement of shell_index (csrc/sw_device.cuh) for one cell."""
    nx, ny, nz = grid
    (l0, h0), (l1, h1), (l2, h2) = lohi
    s0, s1, s2 = l0 + h0, l1 + h1, l2 + h2
    ix = _slab(i, nx, l0, h0)
    if ix >= 0:
        return (ix * ny + j) * nz + k
    a = s0 * ny * nz
    iy = _slab(j, ny, l1, h1)
    if iy >= 0:
        return a + ((i - l0) * s1 + iy) * nz + k
    b = (nx - s0) * s1 * nz
    iz = _slab(k, nz, l2, h2)
    return a + b + ((i - l0) * (ny - s1) + (j - l1)) * s2 + iz if iz >= 0 else -1


def _flags(n, star, h, thick_cells):
    xmax = h * (n - 1 - 2 * star)
    return P.axis_flags(n, star, h, thick_cells * h, xmax - thick_cells * h)


@pytest.mark.parametrize("n,star,thick", [(40, 2, 10), (38, 3, 8), (31, 5, 6), (200, 2, 20), (12, 2, 10)])
def test_flag_extent_covers_flags(n, star, thick):
    f = _flags(n, star, 10.0, thick)
    lo, hi = P.flag_extent(f)
    assert lo + hi <= n
    inside = np.zeros(n, bool)
    inside[:lo] = True
    inside[n - hi:] = True
    assert not (f.astype(bool) & ~inside).any()
    # tight: the slab edges are flagged
    if lo:
        assert f[lo - 1]
    if hi:
        assert f[n - hi]


def test_flag_extent_interior_flag_widens_slab():
    f = np.zeros(20, np.uint8)
    f[:3] = 1
    f[7] = 2
    f[-2:] = 1
    assert P.flag_extent(f) == (8, 2)
    assert P.flag_extent(np.zeros(5, np.uint8)) == (0, 0)
    assert P.flag_extent(np.ones(5, np.uint8)) == (5, 0)


@pytest.mark.parametrize("grid,lohi", [
    ((9, 8, 10), [(2, 3), (1, 2), (3, 1)]),
    ((7, 6, 5), [(0, 0), (2, 1), (1, 1)]),
    ((6, 7, 8), [(6, 0), (1, 1), (1, 1)]),
    ((8, 5, 6), [(1, 1), (0, 0), (0, 0)]),
    ((5, 5, 5), [(0, 0), (0, 0), (2, 2)]),
])
def test_shell_order_is_a_bijection_and_inverted(grid, lohi):
    nx, ny, nz = grid
    S = shell_size(grid, lohi)
    seen = np.full(S, -1)
    want = np.zeros(grid)
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                in_shell = any(_slab(q, n, lo, hi) >= 0 for q, n, (lo, hi) in zip((i, j, k), grid, lohi))
                s = _shell_index(i, j, k, grid, lohi)
                assert (s >= 0) == in_shell
                if s >= 0:
                    assert 0 <= s < S and seen[s] < 0
                    seen[s] = i * ny * nz + j * nz + k
                    want[i, j, k] = s + 1
    assert (seen >= 0).all()
    got = shell_to_full(torch.arange(1, S + 1, dtype=torch.float64), grid, lohi).numpy()
    assert np.array_equal(got, want)


def test_shell_saves_memory_at_the_benchmark_grids():
    for grid in ((200, 200, 200), (400, 400, 200)):
        lohi = [P.flag_extent(_flags(n, 2, 10.0, 20)) for n in grid]
        frac = shell_size(grid, lohi) / float(np.prod(grid))
        assert frac < 0.6, (grid, frac)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(N=2, shape=(44, 38, 41)), dict(N=4, shape=(40, 46, 37), npml=7),
                                dict(N=2, surface=(True, False, True, True, False, True))],
                         ids=["N2", "N4-npml7", "open-sides"])
def test_shell_storage_runs_equal_oracle(cuda, kw):
    from cases import case3d, oracle3d, product3d, to_np
    c = case3d(scheme="SPML", nt=80, **kw)
    w = product3d(c)
    w._build_plan()
    wav = to_np(w._wavelet).astype(np.float32)
    full = int(np.prod(c["shape"]))
    S = shell_size(c["shape"], w._lohi())
    assert tuple(w._split.shape) == (24, S) and S < full
    w.run(80)
    o = oracle3d(c, wavelet=wav).run(0, 80)
    for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
        assert np.array_equal(to_np(getattr(w, f)), getattr(o, f)), f
    assert np.array_equal(to_np(w.data), o.data)
    for name in o.SPLIT:
        assert np.array_equal(to_np(getattr(w, name)), o.memory(name)), name
    assert np.abs(o.memory("vx_x")).max() > 0


@pytest.mark.gpu
def test_plan_rejects_slabs_that_miss_a_flagged_index(cuda):
    from cases import case3d, product3d
    c = case3d(scheme="SPML", nt=10, N=2)
    w = product3d(c)
    w._tables[1]["lo"] -= 1
    with pytest.raises(RuntimeError, match="outside the slabs"):
        w._build_plan()
