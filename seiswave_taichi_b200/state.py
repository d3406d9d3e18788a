"""Run-level checkpoint/resume and checked runs (no reference counterpart: the
reference keeps its state only in ti.fields, and its drivers only print a
Courant number and the elapsed time).

write / read store one solver's whole time-stepping state -- wavefields,
CPML memory variables (slab layout) or split fields (shell layout), the
traces so far -- plus the next step index in an .npz file, with a
fingerprint of the configuration it belongs to (solver class, grid, dtype,
order, spacings, dt, steps, PML slabs, trace shape).  The solver classes use
them as save_state(path, it) and load_state(path) -> it; a run resumes with
run(nt - it, it0=it) and continues bit for bit as if never interrupted.

read validates the whole file before it touches the solver: a truncated or
corrupt file, another format, a configuration that differs, or an array that
is missing or has another shape or dtype raises ValueError and leaves the
solver's state as it was.  write goes through a temporary file and a rename,
so an interrupted write never leaves a half-written checkpoint under the
final name.

NonFiniteError is what run_checked raises when the NaN/Inf scan of the
wavefields (sw_check_finite) finds values after a segment; it carries the
index of the last step run.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

FORMAT = 1


class NonFiniteError(RuntimeError):
    def __init__(self, count: int, step: int):
        super().__init__(f"{count} non-finite wavefield values after time step {step}")
        self.count = int(count)
        self.step = int(step)


class _Invalid(Exception):
    """A readable file that is not a valid state for this solver."""


def _np_dtype(t: torch.Tensor) -> np.dtype:
    return torch.empty(0, dtype=t.dtype).numpy().dtype


def write(path, arrays: dict, meta: dict) -> None:
    """Save `arrays` (name -> tensor or None) and `meta` (JSON-able) to path."""
    path = os.fspath(path)
    payload = {f"a_{k}": v.detach().cpu().numpy() for k, v in arrays.items() if v is not None}
    payload["meta"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), dtype=np.uint8)
    payload["format"] = np.array([FORMAT], np.int64)
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        np.savez(fh, **payload)
    os.replace(tmp, path)


def read(path, arrays: dict, config: dict) -> dict:
    """Validate the file at path against `config` and the tensors in `arrays`
    (name -> tensor or None), then copy its arrays into them; returns the
    saved meta."""
    path = os.fspath(path)
    loaded = {}
    try:
        with np.load(path, allow_pickle=False) as z:
            files = set(z.files)
            if "format" not in files or "meta" not in files:
                raise _Invalid("not a solver checkpoint")
            fmt = int(z["format"][0])
            if fmt != FORMAT:
                raise _Invalid(f"format {fmt}, this library reads format {FORMAT}")
            meta = json.loads(bytes(z["meta"]).decode())
            if meta.get("config") != config:
                raise _Invalid(f"belongs to another configuration: {meta.get('config')} (this solver: {config})")
            for k, t in arrays.items():
                key = f"a_{k}"
                if t is None:
                    if key in files:
                        raise _Invalid(f"holds {k}, which this solver does not have")
                    continue
                if key not in files:
                    raise _Invalid(f"lacks {k}")
                a = z[key]
                if a.shape != tuple(t.shape) or a.dtype != _np_dtype(t):
                    raise _Invalid(f"{k} is {a.dtype}{list(a.shape)}, the solver's is "
                                     f"{_np_dtype(t)}{list(t.shape)}")
                loaded[k] = a
    except _Invalid as e:
        raise ValueError(f"checkpoint {path}: {e}") from e
    except Exception as e:  # truncated or corrupt archive, unreadable file
        raise ValueError(f"checkpoint {path}: unreadable ({type(e).__name__}: {e})") from e
    it = meta.get("it")
    if not isinstance(it, int) or it < 0:
        raise ValueError(f"checkpoint {path}: no valid step index")
    for k, a in loaded.items():
        arrays[k].copy_(torch.from_numpy(a))
    return meta


def run_checked(solver, nt, it0: int, every: int, **run_kw) -> None:
    """solver.run() over steps it0 .. it0+nt-1 in segments of `every` steps,
    scanning the wavefields for NaN/Inf after each segment."""
    if every < 1:
        raise ValueError("every must be >= 1")
    it = int(it0)
    end = it + int(nt)
    while it < end:
        n = min(int(every), end - it)
        solver.run(n, it0=it, **run_kw)
        it += n
        bad = solver.check_finite()
        if bad:
            raise NonFiniteError(bad, it - 1)
