"""Dot-product tests of the hand-written adjoints, independent of the torch
twins: with the source switched off and the model fixed, n time steps are a
linear map A of the whole state (wavefields and CPML memory variables).
sw2d_record / sw3d_record apply A to a random state x; sw2d_adjoint_run /
sw3d_adjoint_run with a zero residual apply A^T to a random adjoint state y.
In float64, <A x, y> and <x, A^T y> agree to rounding (relative 1e-10)."""
import ctypes as C

import numpy as np
import pytest
import torch

from cases import case2d, case3d, product2d, product3d

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _dot(a, b):
    return sum(float((p.double() * q.double()).sum()) for p, q in zip(a, b))


def _rand_like(ts, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return [torch.randn(t.shape, dtype=t.dtype, device=t.device, generator=g) for t in ts]


@pytest.mark.parametrize("scheme", ["VS", "SV"])
@pytest.mark.parametrize("n", [1, 37])
def test_2d_adjoint_dot_product(cuda, scheme, n):
    import seiswave_taichi_b200._native as N
    c = case2d(shape=(40, 36), N=2, npml=8, nt=60, dtype=np.float64, nrec=4, src_scale=1e5, seed=5,
               MT="explosive")
    w = product2d(c)
    sid = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]
    plan = w._plan(sid)
    w._wavelets[sid].zero_()
    mems = [m for m in w._mem if m is not None]
    state = [w.vx, w.vz, w.sxx, w.szz, w.sxz] + mems
    x = _rand_like(state, 1)
    y = _rand_like(state, 2)
    for t, v in zip(state, x):
        t.copy_(v)
    lib, st = N.load(), w._stream()
    elems = C.c_int64(0)
    N.check(lib.sw2d_snapshot_elems(plan.handle, C.byref(elems)))
    snap = torch.empty((n + 1) * elems.value, dtype=torch.float64, device="cuda")
    N.check(lib.sw2d_record(plan.handle, 0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
    ax = [t.clone() for t in state]
    adj = [v.clone() for v in y]
    nx, nz = w.gridsize
    tmp = [torch.zeros((nx, nz), dtype=torch.float64, device="cuda") for _ in range(4)]
    grad = [torch.zeros((nx, nz), dtype=torch.float64, device="cuda") for _ in range(5)]
    res = torch.zeros(w.data.shape, dtype=torch.float64, device="cuda")
    d = N.Adjoint2D()
    for q in range(5):
        d.field[q] = adj[q].data_ptr()
        d.grad[q] = grad[q].data_ptr()
    for q in range(4):
        d.tmp[q] = tmp[q].data_ptr()
    k = 5
    for q in range(2):
        if w._mem[q] is not None:
            d.mem[q] = adj[k].data_ptr()
            k += 1
        else:
            d.mem[q] = None
    d.residual = res.data_ptr()
    N.check(lib.sw2d_adjoint_run(plan.handle, C.byref(d), 0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
    torch.cuda.synchronize()
    lhs, rhs = _dot(ax, y), _dot(x, adj)
    assert abs(lhs) > 0
    assert abs(lhs - rhs) <= TOL * max(abs(lhs), abs(rhs)), (lhs, rhs)


@pytest.mark.parametrize("scheme", ["TENSOR", "CPML"])
@pytest.mark.parametrize("n", [1, 23])
def test_3d_adjoint_dot_product(cuda, n, scheme):
    import seiswave_taichi_b200._native as N
    c = case3d(shape=(20, 18, 22), N=2, scheme=scheme, nt=40, npml=5, dtype=np.float64, seed=6)
    w = product3d(c)
    plan = w._plan or w._build_plan()
    w._wavelet.zero_()
    f3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
    mems = [m for m in w._mem if m is not None]
    state = [getattr(w, f) for f in f3] + mems
    x = _rand_like(state, 3)
    y = _rand_like(state, 4)
    for t, v in zip(state, x):
        t.copy_(v)
    lib, st = N.load(), w._stream()
    elems = C.c_int64(0)
    N.check(lib.sw3d_snapshot_elems(plan.handle, C.byref(elems)))
    snap = torch.empty((n + 1) * elems.value, dtype=torch.float64, device="cuda")
    N.check(lib.sw3d_record(plan.handle, 0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
    ax = [t.clone() for t in state]
    adj = [v.clone() for v in y]
    shape = w.gridsize
    tmp = [torch.zeros(shape, dtype=torch.float64, device="cuda") for _ in range(9)]
    grad = [torch.zeros(shape, dtype=torch.float64, device="cuda") for _ in range(8)]
    res = torch.zeros(w.data.shape, dtype=torch.float64, device="cuda")
    d = N.Adjoint3D()
    for q in range(9):
        d.field[q] = adj[q].data_ptr()
        d.tmp[q] = tmp[q].data_ptr()
    for q in range(8):
        d.grad[q] = grad[q].data_ptr()
    k = 9
    for q in range(3):
        if w._mem[q] is not None:
            d.mem[q] = adj[k].data_ptr()
            k += 1
        else:
            d.mem[q] = None
    d.residual = res.data_ptr()
    N.check(lib.sw3d_adjoint_run(plan.handle, C.byref(d), 0, n, C.c_void_p(snap.data_ptr()), C.c_void_p(st)))
    torch.cuda.synchronize()
    lhs, rhs = _dot(ax, y), _dot(x, adj)
    assert abs(lhs) > 0
    assert abs(lhs - rhs) <= TOL * max(abs(lhs), abs(rhs)), (lhs, rhs)
