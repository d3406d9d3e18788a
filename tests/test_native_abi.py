"""The C ABI library loads and matches include/seiswave.h (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from seiswave_taichi_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "seiswave.h").read_text()
    return sorted(set(re.findall(r"^SW_API\s+[\w\s\*]+?\b(sw\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_binding_exports():
    assert header_symbols() == sorted(N.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_struct_layouts_match():
    for name, (ours, theirs) in N.struct_sizes().items():
        assert ours == theirs, name


def test_version_and_empty_error():
    lib = N.load()
    assert lib.sw_version() == 1
    assert lib.sw_last_error() in (b"",) or isinstance(lib.sw_last_error(), bytes)


def test_bad_descriptors_fail_before_any_device_call():
    lib = N.load()
    h = C.c_void_p()
    assert lib.sw3d_plan_create(None, C.byref(h)) == N.SW_ERR_ARG
    d = N.Desc3D()
    d.scheme = N.SW3D_CPML_TENSOR
    d.order = 9
    assert lib.sw3d_plan_create(C.byref(d), C.byref(h)) == N.SW_ERR_ARG
    assert b"order" in lib.sw_last_error()
    d.order = 2
    d.nx = d.ny = d.nz = 5
    assert lib.sw3d_plan_create(C.byref(d), C.byref(h)) == N.SW_ERR_ARG
    assert b"too small" in lib.sw_last_error()
    d2 = N.Desc2D()
    d2.scheme = 7
    assert lib.sw2d_plan_create(C.byref(d2), C.byref(h)) == N.SW_ERR_ARG
    assert lib.sw_step(None, 0, None) == N.SW_ERR_ARG
    assert lib.sw_run(None, 0, 1, 1, None) == N.SW_ERR_ARG
    assert lib.sw_plan_destroy(None) == N.SW_OK


def test_division_check_arguments_fail_before_any_device_call():
    lib = N.load()
    out = C.c_uint64(7)
    for divisor, mode, what in ((10.0, 4, b"mode"), (10.0, -1, b"mode"), (0.0, 0, b"positive"),
                                (float("inf"), 1, b"positive"), (2.0 ** 70, 3, b"2^60")):
        assert lib.sw_check_division(C.c_float(divisor), mode, C.byref(out), None) == N.SW_ERR_ARG
        assert what in lib.sw_last_error()
    assert lib.sw_check_division(C.c_float(10.0), 0, None, None) == N.SW_ERR_ARG
    assert out.value == 7


def test_check_raises_with_message():
    lib = N.load()
    lib.sw3d_plan_create(None, C.byref(C.c_void_p()))
    with pytest.raises(N.SeisWaveError, match="null descriptor"):
        N.check(N.SW_ERR_ARG)


def test_product_fails_loudly_without_cuda(monkeypatch):
    import torch
    from seiswave_taichi_b200 import _common
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="CUDA device"):
        _common.device()
