"""sw_count_nonfinite_noalloc (counters in a static device array, no device
allocation) against sw_check_finite (plan-owned counter) on the same
wavefields: equal counts, on two calls in a row, for a finite state and for a
state with planted NaN/Inf values.  Counts are integers, so the tolerance is
exact equality."""
import math

import pytest

from cases import case3d, product3d

pytestmark = pytest.mark.gpu

F3 = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


def _state():
    c = case3d(shape=(40, 36, 44), N=2, scheme="TENSOR", nt=60)
    w = product3d(c)
    w.run(60)
    return w


def test_noalloc_matches_check_finite(cuda):
    import torch
    from seiswave_taichi_b200 import _native as N
    w = _state()
    plan = w._plan
    fields = [getattr(w, f) for f in F3]
    torch.cuda.synchronize()
    for _ in range(2):
        assert plan.check_finite() == 0
        assert N.count_nonfinite_noalloc(fields) == [0] * 9
    # plant non-finite values in three wavefields
    fields[0].view(-1)[[5, 17, 9000]] = float("nan")
    fields[4].view(-1)[123] = float("inf")
    fields[8].view(-1)[[0, 1]] = -float("inf")
    torch.cuda.synchronize()
    want = [3, 0, 0, 0, 1, 0, 0, 0, 2]
    for _ in range(2):
        total = plan.check_finite()
        got = N.count_nonfinite_noalloc(fields)
        assert got == want
        assert sum(got) == total == 6
    assert math.isnan(float(fields[0].view(-1)[5]))


def test_noalloc_allocates_nothing(cuda):
    """After a first call on the device (which resolves the counters' address
    and may load the module), a loop of calls changes neither the device's
    free memory nor torch's allocator state."""
    import torch
    from seiswave_taichi_b200 import _native as N
    fields = [torch.zeros(100_000, device="cuda") for _ in range(9)]
    fields[3][7] = float("nan")
    assert N.count_nonfinite_noalloc(fields) == [0, 0, 0, 1, 0, 0, 0, 0, 0]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(50):
        assert N.count_nonfinite_noalloc(fields) == [0, 0, 0, 1, 0, 0, 0, 0, 0]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0


def test_noalloc_float64_and_limits(cuda):
    import torch
    from seiswave_taichi_b200 import _native as N
    a = torch.zeros(1000, dtype=torch.float64, device="cuda")
    b = torch.ones(777, dtype=torch.float64, device="cuda")
    b[776] = float("nan")
    assert N.count_nonfinite_noalloc([a, b]) == [0, 1]
    assert N.count_nonfinite_noalloc([a, b]) == [0, 1]
    assert N.count_nonfinite_noalloc([]) == []
    many = [a] * (N.NOALLOC_MAX_ARRAYS + 1)
    with pytest.raises(N.SeisWaveError, match="at most 64"):
        N.count_nonfinite_noalloc(many)
    assert N.count_nonfinite_noalloc([a] * N.NOALLOC_MAX_ARRAYS) == [0] * N.NOALLOC_MAX_ARRAYS
