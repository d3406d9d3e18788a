"""Test infrastructure, not product code: a numpy restatement of SEG-Y trace
decoding (the checker of sw_segy_decode) and a writer of synthetic SEG-Y
files, because segyio and the reference's data files are absent here.

read_segy_ref restates the reference's read_segy (ReadSegy.py:3-18): traces
are grouped into shot_num = number of distinct SourceX values (or the given
shotnum) shots of trace_num // shot_num traces, each shot transposed to
(time, trace), the (shot, time, trace) float64 array squeezed.

File layout (SEG-Y rev 1): 3200-byte textual header; 400-byte binary header,
big-endian, with the sample interval (bytes 3217-3218, microseconds), samples
per trace (3221-3222), sample format (3225-3226) and the number of extended
textual headers (3505-3506); then per trace a 240-byte header (SourceX at
bytes 73-76) and the samples.  Formats: 1 IBM float, 2 int32, 3 int16,
5 IEEE float, 8 int8, all big-endian.  IBM float: (-1)^s * f * 2^(4(e-64)-24)
for the 7-bit exponent e and 24-bit fraction f, evaluated exactly in float64
and rounded once to float32.
"""
from __future__ import annotations

import numpy as np

BYTES = {1: 4, 2: 4, 3: 2, 5: 4, 8: 1}


def layout(raw: np.ndarray) -> dict:
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


def ibm_to_float32(words: np.ndarray) -> np.ndarray:
    w = np.asarray(words, np.uint32)
    f = (w & np.uint32(0x00FFFFFF)).astype(np.float64)
    e = ((w >> np.uint32(24)) & np.uint32(0x7F)).astype(np.int64)
    neg = (w >> np.uint32(31)) != 0
    v = np.ldexp(f, 4 * (e - 64) - 24)
    v = np.where(neg, -v, v)
    with np.errstate(over="ignore"):
        out = v.astype(np.float32)
    return np.where(f == 0, np.where(neg, np.float32(-0.0), np.float32(0.0)), out).astype(np.float32)


def float_to_ibm(values) -> np.ndarray:
    """IBM words of float64 values (truncating fraction; exact for values with
    at most 21 significant bits and exponents in range)."""
    x = np.asarray(values, np.float64).reshape(-1)
    out = np.zeros(x.size, np.uint32)
    for n, v in enumerate(x):
        s = np.uint32(0x80000000) if np.signbit(v) else np.uint32(0)
        a = abs(float(v))
        if a == 0.0:
            out[n] = s
            continue
        m, p = np.frexp(a)
        q = -((-p) // 4)  # ceil(p / 4): 16^(q-1) <= a < 16^q
        f = int(np.ldexp(m, p - 4 * q + 24))
        if f >= 1 << 24:
            f >>= 4
            q += 1
        if not 0 <= q + 64 <= 127:
            raise ValueError(f"{v} outside the IBM exponent range")
        out[n] = s | np.uint32((q + 64) << 24) | np.uint32(f)
    return out


def decode(body: np.ndarray, ntraces: int, ns: int, fmt: int):
    """(ntraces, ns) float32 samples and (ntraces,) int32 SourceX of the trace
    records in body (the bytes from the first trace header on)."""
    bps = BYTES[fmt]
    rec = 240 + bps * ns
    b = np.asarray(body, np.uint8)[: ntraces * rec].reshape(ntraces, rec)
    srcx = b[:, 72:76].copy().view(">i4").reshape(ntraces).astype(np.int32)
    s = b[:, 240:].copy()
    if fmt == 1:
        vals = ibm_to_float32(s.view(">u4").astype(np.uint32))
    elif fmt == 5:
        vals = s.view(">f4").astype(np.float32)
    elif fmt == 2:
        vals = s.view(">i4").astype(np.float32)
    elif fmt == 3:
        vals = s.view(">i2").astype(np.float32)
    else:
        vals = s.view("i1").astype(np.float32)
    return vals.reshape(ntraces, ns), srcx


def read_segy_ref(path, shotnum=0):
    raw = np.fromfile(path, dtype=np.uint8)
    lay = layout(raw)
    traces, srcx = decode(raw[lay["first"]:], lay["ntraces"], lay["ns"], lay["fmt"])
    trace_num = traces.shape[0]
    shot_num = shotnum if shotnum else len(set(srcx.tolist()))
    len_shot = trace_num // shot_num
    data = np.zeros((shot_num, lay["ns"], len_shot))
    for j in range(shot_num):
        data[j] = traces[j * len_shot:(j + 1) * len_shot].T
    return np.squeeze(data)


def write_segy(path, traces, source_x, fmt=5, dt_us=1000, extended=0):
    """A minimal SEG-Y rev 1 file: blank textual header(s), the binary header
    fields above, trace headers with SourceX and the trace sample count."""
    t = np.asarray(traces)
    ntr, ns = t.shape
    head = bytearray(b" " * 3200) + bytearray(400)
    head[3216:3218] = int(dt_us).to_bytes(2, "big")
    head[3220:3222] = int(ns).to_bytes(2, "big")
    head[3224:3226] = int(fmt).to_bytes(2, "big", signed=True)
    head[3504:3506] = int(extended).to_bytes(2, "big", signed=True)
    parts = [bytes(head), b" " * (3200 * extended)]
    if fmt == 1:
        body = float_to_ibm(t).astype(">u4").reshape(ntr, ns)
    elif fmt == 5:
        body = t.astype(">f4")
    elif fmt == 2:
        body = t.astype(">i4")
    elif fmt == 3:
        body = t.astype(">i2")
    elif fmt == 8:
        body = t.astype("i1")
    else:
        raise ValueError(f"format {fmt}")
    sx = np.asarray(source_x, np.int64).reshape(ntr)
    for n in range(ntr):
        th = bytearray(240)
        th[72:76] = int(sx[n]).to_bytes(4, "big", signed=True)
        th[114:116] = int(ns).to_bytes(2, "big")
        parts.append(bytes(th))
        parts.append(body[n].tobytes())
    with open(path, "wb") as fh:
        fh.write(b"".join(parts))
