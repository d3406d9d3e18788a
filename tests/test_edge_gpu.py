"""Edge cases against the oracle, bit for bit: the smallest grids the plans
accept, grids smaller than one kernel tile (the tensor-map loads then read
mostly out-of-range, zero-filled boxes), one-cell CPML layers, a point force
on a cell the update passes do not cover, and receivers on dead boundary
cells (never updated, so their traces stay zero) beside receivers on live
cells."""
import numpy as np
import pytest

from cases import case2d, case3d, oracle2d, oracle3d, product2d, product3d, to_np

pytestmark = pytest.mark.gpu

F2 = ("vx", "vz", "sxx", "szz", "sxz")
F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


def _eq(name, got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    assert np.array_equal(got, ref), (name, int((got != ref).sum()))


@pytest.mark.parametrize("scheme", ["VS", "SV"])
@pytest.mark.parametrize("N", [1, 2])
def test_2d_smallest_grid(cuda, scheme, N):
    import seiswave_taichi_b200._native as N_
    n = 2 * N + 3
    c = case2d(shape=(n, n), N=N, npml=1, nt=40, MT="explosive", src_scale=1e5)
    c["rsx"] = np.array([[0, n // 2, n - 1]], np.int64)
    c["rsz"] = np.array([[0, n // 2, n - 1]], np.int64)
    w = product2d(c)
    sid = {"VS": N_.SW2D_SSG_VS, "SV": N_.SW2D_SSG_SV}[scheme]
    w._plan(sid)
    o = oracle2d(c, wavelet=to_np(w._wavelets[sid]).astype(np.float32))
    w.run(40, scheme=scheme)
    o.run(scheme, 0, 40)
    for f in F2:
        _eq(f, to_np(getattr(w, f)), getattr(o, f))
    _eq("data", to_np(w.data), o.data)
    assert np.all(to_np(w.data)[:, 0] == 0) and np.all(to_np(w.data)[:, 2] == 0)


@pytest.mark.parametrize("scheme", ["TENSOR", "CPML"])
@pytest.mark.parametrize("shape", [(12, 12, 8), (9, 10, 12)])
def test_3d_grid_smaller_than_a_tile(cuda, scheme, shape):
    nx, ny, nz = shape
    c = case3d(shape=shape, N=2, scheme=scheme, npml=2, nt=50, seed=3)
    if scheme == "TENSOR":
        c["rsx"] = np.array([[0, nx // 2, nx - 1]], np.int64)
        c["rsy"] = np.array([[0, ny // 2, ny - 1]], np.int64)
        c["rsz"] = np.array([[0, nz // 2, nz - 1]], np.int64)
    else:
        c["isx"], c["isy"], c["isz"] = 1, 1, 1  # the point force lands at (6, 6, 6)
        c["rsx"], c["rsy"], c["rsz"] = 3, 4, nz // 2
    w = product3d(c)
    plan = w._build_plan()
    # the staged kernels carry the source when it lies in [N, n-N) on every
    # axis; otherwise (the point force at z = 6 of 8 here) the plan injects it
    # with its own kernel on the two-pass path
    off = 5 if scheme == "CPML" else 0
    src = (c["isx"] + off, c["isy"] + off, c["isz"] + off)
    inside = all(2 <= s_ < n - 2 for s_, n in zip(src, shape))
    assert plan.info()["path"] == ("staged" if nz % 4 == 0 and inside else "two_pass")
    o = oracle3d(c, wavelet=to_np(w._wavelet).astype(np.float32))
    w.run(50)
    o.run(0, 50)
    for f in F3:
        _eq(f, to_np(getattr(w, f)), getattr(o, f))
    _eq("data", to_np(w.data), o.data)
    for name in o.MEM_CPML:
        _eq(name, to_np(getattr(w, name)), o.memory(name))
    assert np.abs(o.vx).max() > 0
    if scheme == "TENSOR":
        d = to_np(w.data)
        assert np.all(d[:, 0] == 0) and np.all(d[:, 2] == 0)


@pytest.mark.parametrize("comp", ["sxx", "szz", "sxz", "vx"])
@pytest.mark.parametrize("mt", [None, "explosive"])
def test_2d_receiver_component_selector(cuda, comp, mt):
    """2D receivers of a named field: each step's sample is that field at the
    receiver cells after the step, with run() and per-step calls alike (the
    stress fields are gathered after the stress pass, and a moment source is
    then not folded into it); the adjoint refuses such plans."""
    import numpy as np
    import torch
    from cases import case2d
    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    kw = dict(MT=mt, src_scale=1e5) if mt else {}
    c = case2d(nt=70, N=2, nrec=9, **kw)

    def make():
        w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"], c["rsx"],
                        c["rsz"], c["nt"], c["N"], c["freq"], torch.float32, rec_component=comp, **kw)
        w.SetADEPML2D(c["surface"], c["pml"])
        return w

    a = make()
    lin = torch.as_tensor((c["rsx"].reshape(-1) * c["shape"][1] + c["rsz"].reshape(-1)).astype(np.int64),
                          device="cuda")
    want = []
    for it in range(c["nt"]):
        a.update_SSG_VS(it)
        want.append(getattr(a, comp).reshape(-1)[lin].clone())
    want = torch.stack(want).cpu().numpy()
    got = a.data.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.abs(want).max() > 0
    b = make()
    b.run(c["nt"])
    assert np.array_equal(b.data.cpu().numpy().view(np.uint32), got.view(np.uint32))
    for f in ("vx", "vz", "sxx", "szz", "sxz"):
        assert torch.equal(getattr(a, f), getattr(b, f)), f
    if comp != "vz" and mt:
        vp, vs, rho = (torch.as_tensor(c[k], device="cuda") for k in ("vp", "vs", "rho"))
        with pytest.raises(RuntimeError, match="own component"):
            make().forward_op(vp, vs, rho, checkpoint_every=10)


@pytest.mark.parametrize("h", [10.0, 12.5, 2.5])
def test_constant_divisor_path_verified(cuda, h):
    """The plan enables the corrected quotient by the grid spacing (Markstein's
    correction, and its scaled form for numerators below 2^-100) only after
    an exhaustive check against IEEE division over every float numerator;
    the spacings of the workloads pass that check."""
    c = case3d(shape=(24, 22, 20), N=2, scheme="TENSOR", nt=4, dx=h, dy=h, dz=h, dt=2e-4)
    w = product3d(c)
    assert w._build_plan().info()["fast_div"] is True


@pytest.mark.parametrize("d", [2000.0, 1741.3, 2155.25, 1.0, 1.7319, 3.3, 0.62])
def test_per_cell_quotient_equals_ieee_for_every_numerator(cuda, d):
    """The per-cell quotient (density averages, CPML kappa, split-PML
    denominators), including its scaled route for numerators below 2^-100,
    equals IEEE division for all 2^32 float numerators."""
    from seiswave_taichi_b200 import _native as N
    assert N.check_division(d, 1) == 0
    assert N.check_division(d, 3) == 0


@pytest.mark.parametrize("h", [10.0, 12.5, 2.5])
def test_spacing_quotient_equals_ieee_for_every_numerator(cuda, h):
    from seiswave_taichi_b200 import _native as N
    assert N.check_division(h, 0) == 0
    assert N.check_division(h, 2) == 0
