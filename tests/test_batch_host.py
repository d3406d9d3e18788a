"""Host-side checks of the 2D batch runner (no GPU)."""
from types import SimpleNamespace

import pytest


@pytest.mark.parametrize("flags", [(True,), (False, True)])
def test_batch_refuses_free_surface_solvers(flags):
    """The batch's launches carry no free-surface hook, so a solver in that
    mode is refused before any plan is made."""
    from seiswave_taichi_b200.batch import ShotBatch2D
    with pytest.raises(ValueError, match="free-surface"):
        ShotBatch2D([SimpleNamespace(_free_surface=f) for f in flags])


def test_batch_refuses_an_empty_list():
    from seiswave_taichi_b200.batch import ShotBatch2D
    with pytest.raises(ValueError, match="empty"):
        ShotBatch2D([])
