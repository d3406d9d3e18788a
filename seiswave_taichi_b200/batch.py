"""Many 2D shots of uneven grid sizes in one CUDA graph (no reference
counterpart; it replaces a Python loop over Elastic2D_CPML.ElasticWAVE objects,
each running `for i in range(nt): update_SSG_VS(i)`, Elastic2D_CPML.py:128-200).

    from seiswave_taichi_b200.batch import ShotBatch2D
    shots = [ElasticWAVE(...) for each shot]        # any sizes, same N/nt/dtype
    for w in shots: w.SetADEPML2D(surface, pml)
    b = ShotBatch2D(shots)                         # autotunes the tile shape
    b.run()                                        # all shots, all steps
    traces = [w.data for w in shots]

Per time step the batch launches one velocity and one stress kernel whose
blocks cover every tile of every shot (a block finds its shot by binary search
over the prefix sum of tile counts); the whole step sequence is captured once
and replayed as a single CUDA graph.  Every shot's state and traces equal what
its own run() gives, bit for bit.

Autotuner: the tile shape (x rows x z columns: 8x32, 4x32, 16x32, 4x64) is
chosen by timing a few steps of each candidate on the batch itself, with the
state replaced by random values for the trial and restored afterwards, and
cached per (GPU, scheme, order, dtype, shape bucket) in a JSON file
(SEISWAVE_AUTOTUNE_CACHE, default ~/.cache/seiswave_taichi_b200/autotune.json).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from pathlib import Path

import torch

from . import _native as N

TILES = ((8, 32), (4, 32), (16, 32), (4, 64))


def _cache_path() -> Path:
    p = os.environ.get("SEISWAVE_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "seiswave_taichi_b200" / "autotune.json"


def cache_load() -> dict:
    """The autotuners' cache {key: choice}; a missing, unreadable or
    malformed file reads as empty."""
    try:
        d = json.loads(_cache_path().read_text())
    except (OSError, ValueError):
        return {}
    return d if isinstance(d, dict) else {}


def cache_store(key: str, value) -> None:
    """Add key -> value to the cache file, merged with its current entries
    and written through a temporary file and a rename, so tuners in several
    processes never leave a torn file; a cache that cannot be written is
    skipped."""
    p = _cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        d = cache_load()
        d[key] = value
        tmp = p.with_name(f"{p.name}.{os.getpid()}.tmp")
        tmp.write_text(json.dumps(d, indent=1, sort_keys=True))
        os.replace(tmp, p)
    except OSError:
        pass


class ShotBatch2D:
    def __init__(self, waves, scheme: str = "VS", autotune: bool = True):
        if not waves:
            raise ValueError("empty batch")
        if any(getattr(w, "_free_surface", False) for w in waves):
            raise ValueError("the batch runner does not apply the free-surface hook: run shots in free-surface "
                             "mode one by one (ElasticWAVE.run)")
        self.waves = list(waves)
        self.scheme = {"VS": N.SW2D_SSG_VS, "SV": N.SW2D_SSG_SV}[scheme]
        plans = [w._plan(self.scheme) for w in self.waves]
        arr = (N.Desc2D * len(plans))(*[p._desc for p in plans])
        self._plans = plans
        h = C.c_void_p()
        N.check(N.load().sw2d_batch_create(arr, len(plans), C.byref(h)))
        self._h = h
        self.nt = self.waves[0].nt
        self.cells = sum(w.gridsize[0] * w.gridsize[1] for w in self.waves)
        if autotune:
            self.autotune()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                N.load().sw_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.waves[0]._dev).cuda_stream

    def info(self) -> dict:
        a = (C.c_int32 * 6)()
        N.check(N.load().sw_batch_info(self._h, a))
        return {"tile": int(a[0]), "tiles": int(a[1]), "blocks": int(a[2]), "rows": int(a[3]), "cols": int(a[4]),
                "shots": int(a[5])}

    def set_tile(self, k: int) -> None:
        N.check(N.load().sw_batch_set_tile(self._h, int(k)))

    def run(self, nt: int | None = None, it0: int = 0, use_graph: bool = True) -> "ShotBatch2D":
        nt = self.nt - it0 if nt is None else int(nt)
        N.check(N.load().sw_batch_run(self._h, int(it0), nt, 1 if use_graph else 0, C.c_void_p(self._stream())))
        return self

    def reset(self) -> None:
        for w in self.waves:
            w.reset()

    # -- autotuner -------------------------------------------------------------
    def _key(self) -> str:
        w = self.waves[0]
        dev = torch.cuda.get_device_name(w._dev).replace(" ", "_")
        mean = self.cells / len(self.waves)
        bucket = f"{round(math.log2(max(mean, 1)))}-{round(math.log2(len(self.waves)))}"
        return f"{dev}|{self.scheme}|{w.star}|{w._dt_torch}|{bucket}"

    def _state(self):
        out = []
        for w in self.waves:
            out += [getattr(w, f) for f in ("vx", "vz", "sxx", "szz", "sxz")]
            out += [m for m in w._mem if m is not None]
            out.append(w.data)
        return out

    def autotune(self, steps: int = 6, force: bool = False) -> int:
        key = self._key()
        v = cache_load().get(key)
        if not force and isinstance(v, int) and 0 <= v < len(TILES):
            self.set_tile(v)
            return v
        state = self._state()
        saved = [t.clone() for t in state]
        gen = torch.Generator(device=state[0].device).manual_seed(0)
        for t in state:
            t.copy_(torch.randn(t.shape, generator=gen, device=t.device, dtype=t.dtype) * 1e-3)
        st = torch.cuda.current_stream(self.waves[0]._dev)
        steps = max(1, min(steps, self.nt - 1))
        best, best_ms = 0, float("inf")
        for k in range(len(TILES)):
            self.set_tile(k)
            self.run(1, 0, use_graph=False)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            self.run(steps, 1, use_graph=False)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if ms < best_ms:
                best, best_ms = k, ms
        for t, s in zip(state, saved):
            t.copy_(s)
        self.set_tile(best)
        cache_store(key, best)
        return best


def run_shots(waves, nt: int | None = None, scheme: str = "VS") -> ShotBatch2D:
    """Build a batch of the given solvers and run them all."""
    return ShotBatch2D(waves, scheme).run(nt)
