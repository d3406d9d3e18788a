"""Shared host helpers of the drop-in ElasticWAVE classes.

Inputs follow the reference's conventions: models are (nx, nz) or (nx, ny, nz)
arrays with the last index fastest (a Taichi dense field, a C-contiguous numpy
array or torch tensor); anything with ``to_numpy()`` (a ti.field) or the array
protocol is accepted.  All state lives on one CUDA device; there is no CPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("seiswave_taichi_b200 runs on a CUDA device (sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device())


def torch_dtype(fieldtype) -> torch.dtype:
    """Map the reference's ``fieldtype`` (ti.f32 / ti.f64, or numpy / torch /
    string spellings of them) to a torch dtype."""
    if fieldtype is None:
        return torch.float32
    if isinstance(fieldtype, torch.dtype):
        if fieldtype in (torch.float32, torch.float64):
            return fieldtype
        raise TypeError(f"fieldtype {fieldtype} is not float32/float64")
    try:
        npd = np.dtype(fieldtype)
    except TypeError:
        npd = None  # not a numpy type (e.g. ti.f32): go by its name below
    if npd is not None:
        if npd == np.float32:
            return torch.float32
        if npd == np.float64:
            return torch.float64
        raise TypeError(f"fieldtype {fieldtype!r} is not float32/float64")
    s = str(fieldtype).lower()
    if "64" in s:
        return torch.float64
    if "32" in s:
        return torch.float32
    raise TypeError(f"unsupported fieldtype {fieldtype!r}")


def sw_dtype(t: torch.dtype) -> int:
    return N.SW_F64 if t == torch.float64 else N.SW_F32


def as_numpy(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    if hasattr(x, "to_numpy"):
        return np.asarray(x.to_numpy())
    return np.asarray(x)


def as_device(x, dtype: torch.dtype, dev=None) -> torch.Tensor:
    """A C-contiguous device tensor of `dtype`; a tensor already in that form
    is used as is (shared, like the reference shares its ti.field inputs)."""
    dev = dev or device()
    if isinstance(x, torch.Tensor):
        t = x.detach()
        if t.device != dev or t.dtype != dtype or not t.is_contiguous():
            t = t.to(device=dev, dtype=dtype).contiguous()
        return t
    return torch.as_tensor(np.ascontiguousarray(as_numpy(x)), device=dev).to(dtype).contiguous()


def compute_mu(vs: torch.Tensor, rho: torch.Tensor) -> torch.Tensor:
    """mu = rho*vs**2, elementwise in the field type (Elastic2D_CPML.py:93-100)."""
    return rho * (vs * vs)


def compute_lam(vs: torch.Tensor, vp: torch.Tensor, rho: torch.Tensor) -> torch.Tensor:
    """lam = rho*(vp**2-2*vs**2), elementwise in the field type (Elastic2D_CPML.py:102-110)."""
    return rho * ((vp * vp) - 2 * (vs * vs))


def receiver_table(shape, *coords) -> tuple[np.ndarray, bool]:
    """Linear cell indices of receivers given as ints (one receiver) or
    (1, nrec) / (nrec,) integer arrays (the tensor variant's rsx/rsy/rsz)."""
    single = all(np.ndim(as_numpy(c)) == 0 for c in coords)
    cs = [as_numpy(c).astype(np.int64).reshape(-1) for c in coords]
    n = max(c.size for c in cs)
    cs = [np.broadcast_to(c, (n,)) for c in cs]
    for ax, (c, lim) in enumerate(zip(cs, shape)):
        if (c < 0).any() or (c >= lim).any():
            raise IndexError(f"receiver coordinate on axis {ax} outside 0..{lim - 1}")
    lin = np.ravel_multi_index(tuple(cs), tuple(shape)).astype(np.int64)
    return lin, single
