"""Host-side refusals that keep bad inputs away from the device (CPU only):
count_nonfinite_noalloc refuses tensors its scan could not read within
bounds, and decode_traces refuses a SEG-Y body shorter than the traces it is
asked to decode.  The library is never reached: its loader is replaced by
one that fails the test if called."""
import pytest
import torch

from seiswave_taichi_b200 import _native as N


@pytest.fixture
def no_library(monkeypatch):
    def boom():
        raise AssertionError("the native library was reached")
    monkeypatch.setattr(N, "load", boom)


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.int16, torch.int32, torch.uint8])
def test_noalloc_refuses_other_dtypes(no_library, dtype):
    with pytest.raises(ValueError, match="float32 or float64"):
        N.count_nonfinite_noalloc([torch.zeros(8, dtype=dtype)])


def test_noalloc_refuses_mixed_noncontiguous_and_host_tensors(no_library):
    a = torch.zeros(16, dtype=torch.float32)
    with pytest.raises(ValueError, match="one dtype"):
        N.count_nonfinite_noalloc([a, torch.zeros(16, dtype=torch.float64)])
    with pytest.raises(ValueError, match="contiguous"):
        N.count_nonfinite_noalloc([torch.zeros(4, 4)[:, 1]])
    with pytest.raises(ValueError, match="current CUDA device"):
        N.count_nonfinite_noalloc([a])
    with pytest.raises(TypeError):
        N.count_nonfinite_noalloc([a.numpy()])


def test_noalloc_empty_list_needs_no_device(monkeypatch):
    calls = []

    class Lib:
        def sw_count_nonfinite_noalloc(self, arr, lens, n, dt, st, out):
            calls.append(n)
            return 0
    monkeypatch.setattr(N, "load", lambda: Lib())
    assert N.count_nonfinite_noalloc([]) == []
    assert calls == [0]


def test_segy_decode_refuses_short_or_malformed_body(no_library):
    from seiswave_taichi_b200 import ReadSegy as R
    ns, ntr = 100, 3
    rec = 240 + 4 * ns
    short = torch.zeros(ntr * rec - 1, dtype=torch.uint8)
    with pytest.raises(ValueError, match="need"):
        R.decode_traces(short, ntr, ns, 1)
    with pytest.raises(ValueError, match="format"):
        R.decode_traces(torch.zeros(ntr * rec, dtype=torch.uint8), ntr, ns, 4)
    with pytest.raises(ValueError, match="non-negative"):
        R.decode_traces(torch.zeros(ntr * rec, dtype=torch.uint8), -1, ns, 1)
    with pytest.raises(ValueError, match="uint8"):
        R.decode_traces(torch.zeros(ntr * rec, dtype=torch.int32), ntr, ns, 1)
    with pytest.raises(ValueError, match="contiguous"):
        R.decode_traces(torch.zeros(2 * ntr * rec, dtype=torch.uint8)[::2], ntr, ns, 1)
    # a full-length host body passes every size check and stops at the device check
    with pytest.raises(ValueError, match="CUDA"):
        R.decode_traces(torch.zeros(ntr * rec, dtype=torch.uint8), ntr, ns, 1)
