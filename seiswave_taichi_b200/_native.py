"""ctypes binding of libseiswave.so (include/seiswave.h).

The structures below mirror the C declarations field for field; struct_sizes()
checks them against the library's own sizeof.  The library is loaded from the
package's lib/ folder (built in-tree by build_native.py).  There is no CPU
fallback: if the library is missing, load() raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libseiswave.so"

SW_MAX_ORDER = 8
SW_OK = 0
SW_ERR_ARG = -1
SW_ERR_CUDA = -2
SW_ERR_NONFINITE = -3
SW_ERR_UNSUPPORTED = -4
SW_ERR_TIMEOUT = -5

SW_F32, SW_F64 = 0, 1
SW2D_SSG_VS, SW2D_SSG_SV, SW2D_RSG = 0, 1, 2
SW3D_CPML_FORCE, SW3D_CPML_TENSOR, SW3D_SPML = 0, 1, 2
SW_SRC_NONE, SW_SRC_FORCE, SW_SRC_MOMENT, SW_SRC_RSG4 = 0, 1, 2, 3

# every symbol include/seiswave.h declares
EXPORTS = (
    "sw_version", "sw_last_error", "sw2d_plan_create", "sw3d_plan_create",
    "sw_plan_set_tile", "sw_abi_sizeof", "sw_plan_destroy", "sw_step", "sw_step_amp",
    "sw_run", "sw_check_finite", "sw_check_division", "sw_plan_status", "sw_plan_info", "sw_plan_set_path",
    "sw_plan_set_exact", "sw_count_nonfinite_noalloc", "sw2d_snapshot_elems", "sw2d_record",
    "sw2d_adjoint_run", "sw2d_batch_create", "sw_batch_set_tile", "sw_batch_info", "sw_batch_run",
    "sw_batch_destroy", "sw2d_abc_correct", "sw2d_abc_features", "sw_mlp_grad", "sw_mlp_forward",
    "sw_mlp_backward", "sw2d_abc_adjoint", "sw3d_snapshot_elems", "sw3d_record", "sw3d_adjoint_run",
    "sw3d_abc_correct", "sw3d_abc_features", "sw3d_abc_adjoint", "sw3d_mlp_grad", "sw3d_mlp_forward",
    "sw3d_mlp_backward", "sw_segy_decode", "sw_plan_set_free_surface",
)

SW_ABC_DEPTH = 6
SW_ABC_INPUTS = 45 + SW_ABC_DEPTH
SW_ABC_HIDDEN = 32
SW_ABC_PARAMS = (SW_ABC_HIDDEN * SW_ABC_INPUTS + SW_ABC_HIDDEN + SW_ABC_HIDDEN * SW_ABC_HIDDEN + SW_ABC_HIDDEN
                 + 5 * SW_ABC_HIDDEN + 5)

SW_ABC3_INPUTS = 27 + SW_ABC_DEPTH
SW_ABC3_PARAMS = (SW_ABC_HIDDEN * SW_ABC3_INPUTS + SW_ABC_HIDDEN + SW_ABC_HIDDEN * SW_ABC_HIDDEN + SW_ABC_HIDDEN
                  + 9 * SW_ABC_HIDDEN + 9)


class AbcDesc(C.Structure):
    _fields_ = [("ncell", C.c_int32), ("cell", C.c_void_p), ("face", C.c_void_p), ("depth", C.c_void_p),
                ("params", C.c_void_p), ("scale", C.c_float * 5), ("oscale", C.c_float * 5),
                ("delta", C.c_void_p)]


class Abc3Desc(C.Structure):
    _fields_ = [("ncell", C.c_int32), ("cell", C.c_void_p), ("face", C.c_void_p), ("depth", C.c_void_p),
                ("params", C.c_void_p), ("scale", C.c_float * 9), ("oscale", C.c_float * 9),
                ("delta", C.c_void_p)]


class Adjoint3D(C.Structure):
    _fields_ = [("field", C.c_void_p * 9), ("mem", C.c_void_p * 3), ("tmp", C.c_void_p * 9),
                ("grad", C.c_void_p * 8), ("residual", C.c_void_p)]


class Adjoint2D(C.Structure):
    _fields_ = [("field", C.c_void_p * 5), ("mem", C.c_void_p * 2), ("tmp", C.c_void_p * 4),
                ("grad", C.c_void_p * 5), ("residual", C.c_void_p)]


class PmlAxis(C.Structure):
    _fields_ = [
        ("lo", C.c_int32), ("hi", C.c_int32),
        ("coef", C.c_void_p), ("damp", C.c_void_p), ("flag", C.c_void_p),
    ]


class Receivers(C.Structure):
    _fields_ = [
        ("nrec", C.c_int32), ("field", C.c_int32),
        ("index", C.c_void_p), ("data", C.c_void_p), ("dtype", C.c_int32),
    ]


class Source(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("i", C.c_int32), ("j", C.c_int32), ("k", C.c_int32),
        ("wavelet", C.c_void_p), ("mt", C.c_double * 6),
    ]


class Desc2D(C.Structure):
    _fields_ = [
        ("scheme", C.c_int32), ("dtype", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32),
        ("order", C.c_int32), ("nt_max", C.c_int32),
        ("dx", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("coef", C.c_double * SW_MAX_ORDER),
        ("field", C.c_void_p * 5),
        ("rho", C.c_void_p), ("lam", C.c_void_p), ("mu", C.c_void_p),
        ("pml", PmlAxis * 2),
        ("mem", C.c_void_p * 2),
        ("src", Source),
        ("rec", Receivers),
    ]


class Desc3D(C.Structure):
    _fields_ = [
        ("scheme", C.c_int32), ("dtype", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
        ("nz", C.c_int32), ("order", C.c_int32), ("nt_max", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("coef", C.c_double * SW_MAX_ORDER),
        ("field", C.c_void_p * 9),
        ("rho", C.c_void_p), ("lam", C.c_void_p), ("mu", C.c_void_p),
        ("pml", PmlAxis * 3),
        ("mem", C.c_void_p * 3),
        ("split", C.c_void_p),
        ("src", Source),
        ("rec", Receivers),
    ]


_lib = None


def load() -> C.CDLL:
    """Load libseiswave.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the sm_100a kernels with "
            "`python -m seiswave_taichi_b200.build_native` (there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "sw_version": (C.c_int, []),
        "sw_last_error": (C.c_char_p, []),
        "sw2d_plan_create": (C.c_int, [C.POINTER(Desc2D), C.POINTER(vp)]),
        "sw3d_plan_create": (C.c_int, [C.POINTER(Desc3D), C.POINTER(vp)]),
        "sw_plan_set_tile": (C.c_int, [vp, C.c_int32]),
        "sw_abi_sizeof": (C.c_int, [C.c_int32]),
        "sw_plan_destroy": (C.c_int, [vp]),
        "sw_step": (C.c_int, [vp, C.c_int32, vp]),
        "sw_step_amp": (C.c_int, [vp, C.c_int32, C.c_double, vp]),
        "sw_run": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, vp]),
        "sw_check_finite": (C.c_int, [vp, vp, C.POINTER(C.c_int64)]),
        "sw_check_division": (C.c_int, [C.c_float, C.c_int32, C.POINTER(C.c_uint64), vp]),
        "sw_plan_status": (C.c_int, [vp, vp]),
        "sw_plan_info": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "sw_plan_set_path": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "sw_plan_set_exact": (C.c_int, [vp, C.c_int32]),
        "sw_count_nonfinite_noalloc": (C.c_int, [C.POINTER(vp), C.POINTER(C.c_int64), C.c_int32, C.c_int32, vp,
                                                 C.POINTER(C.c_int64)]),
        "sw2d_snapshot_elems": (C.c_int, [vp, C.POINTER(C.c_int64)]),
        "sw_segy_decode": (C.c_int, [vp, C.c_int64, C.c_int32, C.c_int32, vp, vp, vp]),
        "sw_plan_set_free_surface": (C.c_int, [vp, C.c_int32]),
        "sw2d_record": (C.c_int, [vp, C.c_int32, C.c_int32, vp, vp]),
        "sw2d_adjoint_run": (C.c_int, [vp, C.POINTER(Adjoint2D), C.c_int32, C.c_int32, vp, vp]),
        "sw2d_batch_create": (C.c_int, [C.POINTER(Desc2D), C.c_int32, C.POINTER(vp)]),
        "sw_batch_set_tile": (C.c_int, [vp, C.c_int32]),
        "sw_batch_info": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "sw_batch_run": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, vp]),
        "sw_batch_destroy": (C.c_int, [vp]),
        "sw2d_abc_correct": (C.c_int, [vp, C.POINTER(AbcDesc), vp]),
        "sw2d_abc_features": (C.c_int, [vp, C.POINTER(AbcDesc), vp, vp]),
        "sw_mlp_grad": (C.c_int, [vp, vp, vp, C.c_int64, vp, vp, vp]),
        "sw_mlp_forward": (C.c_int, [vp, vp, C.c_int64, vp, vp]),
        "sw_mlp_backward": (C.c_int, [vp, vp, vp, C.c_int64, vp, vp]),
        "sw2d_abc_adjoint": (C.c_int, [vp, C.POINTER(AbcDesc), vp, C.POINTER(vp), vp, vp]),
        "sw3d_snapshot_elems": (C.c_int, [vp, C.POINTER(C.c_int64)]),
        "sw3d_record": (C.c_int, [vp, C.c_int32, C.c_int32, vp, vp]),
        "sw3d_adjoint_run": (C.c_int, [vp, C.POINTER(Adjoint3D), C.c_int32, C.c_int32, vp, vp]),
        "sw3d_abc_correct": (C.c_int, [vp, C.POINTER(Abc3Desc), vp]),
        "sw3d_abc_features": (C.c_int, [vp, C.POINTER(Abc3Desc), vp, vp]),
        "sw3d_abc_adjoint": (C.c_int, [vp, C.POINTER(Abc3Desc), vp, C.POINTER(vp), vp, vp]),
        "sw3d_mlp_grad": (C.c_int, [vp, vp, vp, C.c_int64, vp, vp, vp]),
        "sw3d_mlp_forward": (C.c_int, [vp, vp, C.c_int64, vp, vp]),
        "sw3d_mlp_backward": (C.c_int, [vp, vp, vp, C.c_int64, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def struct_sizes() -> dict:
    """(python sizeof, library sizeof) of each ABI struct."""
    lib = load()
    ours = [PmlAxis, Receivers, Source, Desc2D, Desc3D]
    return {t.__name__: (C.sizeof(t), lib.sw_abi_sizeof(q)) for q, t in enumerate(ours)}


NOALLOC_MAX_ARRAYS = 64


def validate_noalloc_inputs(tensors) -> None:
    """Refuse, before any pointer reaches the library, every tensor that the
    scan could not read within bounds on the current device: not a torch
    tensor, not float32/float64 (the kernel reads 4 or 8 bytes per element),
    mixed dtypes, not contiguous, not on the current CUDA device."""
    import torch
    if not tensors:
        return
    cur = torch.cuda.current_device() if torch.cuda.is_available() else None
    for t in tensors:
        if not isinstance(t, torch.Tensor):
            raise TypeError("count_nonfinite_noalloc takes torch tensors")
        if t.dtype not in (torch.float32, torch.float64):
            raise ValueError(f"tensors must be float32 or float64, not {t.dtype}")
    if any(t.dtype != tensors[0].dtype for t in tensors):
        raise ValueError("tensors must share one dtype")
    if any(not t.is_contiguous() for t in tensors):
        raise ValueError("tensors must be contiguous")
    for t in tensors:
        if not t.is_cuda or t.device.index != cur:
            raise ValueError(f"tensors must be on the current CUDA device (cuda:{cur}), not {t.device}")


def count_nonfinite_noalloc(tensors, stream: int | None = None) -> list[int]:
    """Per-tensor NaN/Inf counts through sw_count_nonfinite_noalloc, which
    allocates no device memory (at most NOALLOC_MAX_ARRAYS contiguous tensors
    of one dtype, float32 or float64, on the current CUDA device; stream
    defaults to torch's current stream)."""
    import torch
    tensors = list(tensors)
    n = len(tensors)
    validate_noalloc_inputs(tensors)
    dt = SW_F64 if n and tensors[0].dtype == torch.float64 else SW_F32
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream if n else 0
    arr = (C.c_void_p * max(n, 1))(*[ptr(t) for t in tensors])
    lens = (C.c_int64 * max(n, 1))(*[t.numel() for t in tensors])
    out = (C.c_int64 * max(n, 1))()
    rc = load().sw_count_nonfinite_noalloc(arr, lens, n, dt, C.c_void_p(stream), out)
    if rc not in (SW_OK, SW_ERR_NONFINITE):
        check(rc)
    return [int(out[a]) for a in range(n)]


def check_division(divisor: float, mode: int, stream: int = 0) -> int:
    """Numerators (of all 2^32 floats) where the kernels' quotient by divisor
    differs from IEEE division: mode 0 the constant-spacing path, mode 1 the
    per-cell path, modes 2 and 3 their branch-free group forms over the
    numerators below 2^100 (sw_check_division)."""
    out = C.c_uint64(0)
    check(load().sw_check_division(C.c_float(divisor), int(mode), C.byref(out), C.c_void_p(stream)))
    return int(out.value)


class SeisWaveError(RuntimeError):
    """A libseiswave call returned an error status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libseiswave error {code}: {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != SW_OK:
        msg = load().sw_last_error()
        raise SeisWaveError(rc, msg.decode() if msg else "")


def ptr(t) -> int | None:
    """Raw device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


class Plan:
    """Owns one sw_plan; keeps every tensor it borrows alive."""

    def __init__(self, desc, keep, three_d: bool):
        lib = load()
        h = C.c_void_p()
        if three_d:
            check(lib.sw3d_plan_create(C.byref(desc), C.byref(h)))
        else:
            check(lib.sw2d_plan_create(C.byref(desc), C.byref(h)))
        self._h = h
        self._desc = desc
        self._keep = keep

    @property
    def handle(self):
        return self._h

    def step(self, it: int, stream: int = 0) -> None:
        check(load().sw_step(self._h, int(it), C.c_void_p(stream)))

    def step_amp(self, it: int, amp: float, stream: int = 0) -> None:
        check(load().sw_step_amp(self._h, int(it), float(amp), C.c_void_p(stream)))

    def run(self, it0: int, nsteps: int, use_graph: bool = True, stream: int = 0) -> None:
        check(load().sw_run(self._h, int(it0), int(nsteps), 1 if use_graph else 0, C.c_void_p(stream)))

    def set_tile(self, x_chunk: int) -> None:
        check(load().sw_plan_set_tile(self._h, int(x_chunk)))

    def check_finite(self, stream: int = 0) -> int:
        n = C.c_int64(0)
        rc = load().sw_check_finite(self._h, C.c_void_p(stream), C.byref(n))
        if rc not in (SW_OK, SW_ERR_NONFINITE):
            check(rc)
        return int(n.value)

    def status(self, stream: int = 0) -> None:
        """Synchronize and raise if a kernel recorded a device-side failure."""
        check(load().sw_plan_status(self._h, C.c_void_p(stream)))

    PATHS = {"two_pass": 0, "staged": 1, "fused": 2, "persistent": 3}

    def info(self) -> dict:
        a = (C.c_int32 * 9)()
        check(load().sw_plan_info(self._h, a))
        names = {v: k for k, v in self.PATHS.items()}
        return {"path": names[a[0]], "fast_div": bool(a[1]), "staged": bool(a[2]), "staged_grid": a[3],
                "staged_chunk": a[4], "fused": bool(a[5]), "fused_grid": a[6], "fused_chunk": a[7],
                "exact": bool(a[8])}

    def set_free_surface(self, on: bool = True) -> None:
        """2D: apply the free-surface hook AEA before every step (sticky)."""
        check(load().sw_plan_set_free_surface(self._h, 1 if on else 0))

    def set_exact(self, exact: bool) -> None:
        """Numeric mode of the staged path (the other paths are always exact)."""
        check(load().sw_plan_set_exact(self._h, 1 if exact else 0))

    def set_path(self, path: str = "staged", chunk_len: int = 0) -> None:
        """Execution path of step/run: "two_pass", "staged" or "fused"."""
        check(load().sw_plan_set_path(self._h, self.PATHS[path], int(chunk_len)))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load().sw_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
