"""SEG-Y ingestion: the numpy decoder (oracle/segy_ref.py) pinned by IBM float
known answers and writer round trips on the CPU; the device decoder
(sw_segy_decode, read_segy) against it bit for bit on the GPU, every format,
random IBM words of every exponent, shot grouping as the reference's
read_segy does it; the .mat model loader."""
import numpy as np
import pytest
import torch

from oracle import segy_ref as R

# IBM hexadecimal float words and their values: 1.0, 100.0, -118.625 (the
# classic example of the format), 1/256, zeros of both signs, the largest
# word (overflows float32 to infinity) and a word below float32's range
KNOWN = [
    (0x41100000, 1.0), (0x42640000, 100.0), (0xC276A000, -118.625), (0x3F100000, 0.00390625),
    (0x00000000, 0.0), (0x80000000, -0.0), (0x7FFFFFFF, np.inf), (0x00100000, 0.0),
]


def test_ibm_known_answers():
    got = R.ibm_to_float32(np.array([w for w, _ in KNOWN], np.uint32))
    for (w, v), g in zip(KNOWN, got):
        assert g == np.float32(v) and np.signbit(g) == np.signbit(v), (hex(w), v, g)


def test_ibm_encoder_round_trip():
    rng = np.random.default_rng(0)
    # values with at most 21 significant bits survive IBM's hexadecimal normalisation
    v = np.ldexp(rng.integers(-(1 << 20), 1 << 20, 500).astype(np.float64), rng.integers(-60, 60, 500))
    w = R.float_to_ibm(v)
    assert np.array_equal(R.ibm_to_float32(w).astype(np.float64), v.astype(np.float32).astype(np.float64))
    assert R.float_to_ibm([1.0, 100.0, -118.625])[2] == 0xC276A000


@pytest.mark.parametrize("fmt", [1, 2, 3, 5, 8])
def test_writer_decoder_round_trip(tmp_path, fmt):
    rng = np.random.default_rng(fmt)
    t = rng.integers(-100, 100, (7, 13)).astype(np.float64) * (0.5 if fmt in (1, 5) else 1)
    p = tmp_path / "a.sgy"
    R.write_segy(p, t, source_x=np.arange(7) * 10, fmt=fmt, extended=1 if fmt == 3 else 0)
    raw = np.fromfile(p, np.uint8)
    lay = R.layout(raw)
    assert (lay["ns"], lay["fmt"], lay["ntraces"]) == (13, fmt, 7)
    vals, sx = R.decode(raw[lay["first"]:], 7, 13, fmt)
    assert np.array_equal(vals, t.astype(np.float32))
    assert np.array_equal(sx, np.arange(7) * 10)


def test_reference_grouping(tmp_path):
    t = np.arange(12 * 5, dtype=np.float64).reshape(12, 5)
    p = tmp_path / "g.sgy"
    R.write_segy(p, t, source_x=np.repeat([100, 200, 300], 4), fmt=5)
    d = R.read_segy_ref(p)
    assert d.shape == (3, 5, 4) and d.dtype == np.float64
    assert np.array_equal(d[1], t[4:8].T)
    assert R.read_segy_ref(p, shotnum=2).shape == (2, 5, 6)
    R.write_segy(p, t[:4], source_x=[7] * 4, fmt=5)
    assert R.read_segy_ref(p).shape == (5, 4)


def test_layout_errors(tmp_path):
    p = tmp_path / "bad.sgy"
    R.write_segy(p, np.zeros((2, 3)), source_x=[0, 0], fmt=5)
    raw = np.fromfile(p, np.uint8)
    from seiswave_taichi_b200.ReadSegy import segy_layout
    with pytest.raises(ValueError, match="whole number of traces"):
        segy_layout(raw[:-1])
    bad = raw.copy()
    bad[3224:3226] = [0, 4]
    with pytest.raises(ValueError, match="format 4"):
        segy_layout(bad)
    assert segy_layout(raw) == R.layout(raw)


def test_load_mat_model(tmp_path):
    import scipy.io as sio
    from seiswave_taichi_b200.ReadSegy import load_mat_model
    vp = np.linspace(2000, 6000, 4 * 5 * 6).reshape(4, 5, 6)
    sio.savemat(tmp_path / "m.mat", {"Vp": vp})
    a, b, c = load_mat_model(tmp_path / "m.mat")
    assert a.dtype == np.float32 and a.shape == (4, 5, 6)
    np.testing.assert_allclose(b, vp / 1.7, rtol=1e-6)
    np.testing.assert_allclose(c, 1.741 * (vp / 1000) ** 0.25 * 1000, rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("ns", [1, 7, 250])
def test_device_decoder_equals_oracle(cuda, fmt, ns):
    from seiswave_taichi_b200.ReadSegy import decode_traces
    rng = np.random.default_rng(ns * 10 + fmt)
    ntr = 37
    rec = 240 + R.BYTES[fmt] * ns
    body = rng.integers(0, 256, ntr * rec, dtype=np.uint8)  # every bit pattern, IBM exponents included
    ref, sx = R.decode(body, ntr, ns, fmt)
    out, srcx = decode_traces(torch.from_numpy(body).cuda(), ntr, ns, fmt)
    got = out.cpu().numpy()
    assert got.view(np.uint32).tobytes() == ref.view(np.uint32).tobytes()
    assert np.array_equal(srcx.cpu().numpy(), sx)


@pytest.mark.gpu
@pytest.mark.parametrize("shotnum", [0, 2])
@pytest.mark.parametrize("fmt", [1, 5])
def test_read_segy_equals_reference_logic(cuda, tmp_path, shotnum, fmt):
    from seiswave_taichi_b200.ReadSegy import read_segy
    rng = np.random.default_rng(3)
    t = rng.integers(-1000, 1000, (13, 40)).astype(np.float64) / 8
    p = tmp_path / "s.sgy"
    R.write_segy(p, t, source_x=np.repeat([5, 9, 11], [4, 4, 5]), fmt=fmt)
    ref = R.read_segy_ref(p, shotnum)
    got = read_segy(p, shotnum)
    assert got.dtype == np.float64 and got.shape == ref.shape
    assert np.array_equal(got, ref)
    g32 = read_segy(p, shotnum, as_numpy=False)
    assert g32.device.type == "cuda" and g32.dtype == torch.float32
