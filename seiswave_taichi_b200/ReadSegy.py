"""Model and shot-record ingestion without segyio: a drop-in for the
reference's ReadSegy.read_segy (ReadSegy.py:3-18) that decodes the traces on
the GPU (sw_segy_decode), and the .mat model loading of the reference's 3D
drivers (test3d_homegenous_overhust.py:9-22).

    from seiswave_taichi_b200.ReadSegy import read_segy, load_mat_model
    data = read_segy("shots.sgy")            # float64 numpy (shot, time, trace), squeezed
    data = read_segy("shots.sgy", as_numpy=False)  # float32 torch tensor left on the GPU
    vp, vs, rho = load_mat_model("overhustp.mat")

read_segy reads the SEG-Y rev 1 binary header (big-endian: sample interval
bytes 3217-3218, samples per trace 3221-3222, sample format 3225-3226,
extended textual headers 3505-3506), copies the trace records to the device
once, decodes every sample (formats 1 IBM float, 2 int32, 3 int16, 5 IEEE
float, 8 int8) and each trace's SourceX there, and groups the traces as the
reference does: shot_num = the number of distinct SourceX values unless
shotnum is given, trace_num // shot_num traces per shot, each shot as
(time, trace).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N

BYTES = {1: 4, 2: 4, 3: 2, 5: 4, 8: 1}


def segy_layout(raw: np.ndarray) -> dict:
    """Sample interval (us), samples per trace, format, byte offset of the
    first trace header, record length and trace count of a SEG-Y file's bytes."""
    b = np.asarray(raw, np.uint8)
    if b.size < 3600:
        raise ValueError("shorter than the 3600-byte SEG-Y file header")
    be = lambda lo, hi, signed=False: int.from_bytes(b[lo:hi].tobytes(), "big", signed=signed)
    dt_us, ns, fmt, next_ = be(3216, 3218), be(3220, 3222), be(3224, 3226, True), be(3504, 3506, True)
    if fmt not in BYTES:
        raise ValueError(f"sample format {fmt} not supported (1 IBM float, 2 int32, 3 int16, 5 IEEE float, 8 int8)")
    if next_ < 0:
        raise ValueError("a variable number of extended textual headers is not supported")
    first = 3600 + 3200 * next_
    rec = 240 + BYTES[fmt] * ns
    body = b.size - first
    if body < 0 or (ns > 0 and body % rec):
        raise ValueError("the file is not a whole number of traces")
    return dict(dt_us=dt_us, ns=ns, fmt=fmt, first=first, rec=rec, ntraces=body // rec if ns > 0 else 0)


def check_body(body, ntraces: int, ns: int, fmt: int) -> None:
    """Refuse a decode that would read past the end of `body`: the format must
    be known, ntraces and ns non-negative, and body a contiguous uint8 CUDA
    tensor of at least ntraces * (240 + bytes per sample * ns) bytes (the
    library takes no byte length, so this is its bounds check)."""
    if not isinstance(body, torch.Tensor) or body.dtype != torch.uint8:
        raise ValueError("decode_traces takes a uint8 tensor")
    if int(fmt) not in BYTES:
        raise ValueError(f"sample format {fmt} not supported (1 IBM float, 2 int32, 3 int16, 5 IEEE float, 8 int8)")
    if int(ntraces) < 0 or int(ns) < 0:
        raise ValueError("ntraces and ns must be non-negative")
    need = int(ntraces) * (240 + BYTES[int(fmt)] * int(ns))
    if body.numel() < need:
        raise ValueError(f"body holds {body.numel()} bytes, {ntraces} traces of {ns} samples need {need}")
    if not body.is_contiguous():
        raise ValueError("body must be contiguous")
    if body.device.type != "cuda":
        raise ValueError("decode_traces takes a CUDA tensor")


def decode_traces(body: torch.Tensor, ntraces: int, ns: int, fmt: int):
    """Decode trace records already in device memory (uint8, the bytes from the
    first trace header on): (ntraces, ns) float32 samples, (ntraces,) int32
    SourceX."""
    check_body(body, ntraces, ns, fmt)
    out = torch.empty((ntraces, ns), dtype=torch.float32, device=body.device)
    srcx = torch.empty(ntraces, dtype=torch.int32, device=body.device)
    st = torch.cuda.current_stream(body.device).cuda_stream
    N.check(N.load().sw_segy_decode(C.c_void_p(body.data_ptr()), int(ntraces), int(ns), int(fmt),
                                    C.c_void_p(out.data_ptr()), C.c_void_p(srcx.data_ptr()), C.c_void_p(st)))
    return out, srcx


def read_segy(data_dir, shotnum=0, as_numpy: bool = True, device="cuda"):
    """The reference's read_segy: all traces grouped into shots, (shot, time,
    trace) squeezed; float64 numpy like the reference, or (as_numpy=False)
    the float32 tensor on the GPU."""
    raw = np.fromfile(data_dir, dtype=np.uint8)
    lay = segy_layout(raw)
    ntr, ns = lay["ntraces"], lay["ns"]
    host = torch.from_numpy(raw[lay["first"]:lay["first"] + ntr * lay["rec"]].copy())
    body = host.pin_memory().to(device, non_blocking=True)
    traces, srcx = decode_traces(body, ntr, ns, lay["fmt"])
    shot_num = int(shotnum) if shotnum else int(torch.unique(srcx).numel())
    len_shot = ntr // shot_num
    data = traces[: shot_num * len_shot].reshape(shot_num, len_shot, ns).transpose(1, 2).squeeze()
    if as_numpy:
        return data.double().cpu().numpy()
    return data.contiguous()


def load_mat_model(path, key: str = "Vp", vs_ratio: float = 1.7):
    """vp from a MATLAB .mat file (scipy.io.loadmat), vs = vp / vs_ratio and the
    Gardner density 1.741 (vp/1000)^0.25 * 1000, as float32 arrays, the way the
    reference's overthrust driver builds its model (test3d_homegenous_overhust.py:13-18)."""
    import scipy.io as sio
    vp = np.asarray(sio.loadmat(path)[key], dtype=np.float64)
    vs = vp / vs_ratio
    rho = 1.741 * (vp / 1000.0) ** 0.25 * 1000.0
    return vp.astype(np.float32), vs.astype(np.float32), rho.astype(np.float32)
