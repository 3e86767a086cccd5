"""Device memory shared by engines: samples created and dropped one after another reuse the
same pooled blocks (device memory in use stays flat), give the same results as the first
one, and samples alive at the same time never share a block (their results match the
same samples relaxed alone)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch

    free, _ = torch.cuda.mem_get_info(0)
    return free


def _relaxed(engine, group, count, seed, neighbourhood, calls=(3,)):
    with engine.haar(group, count, seed) as grid:
        for steps in calls:
            grid.relax(steps, neighbourhood=neighbourhood)
        return grid.quaternions.copy(), grid.stats["quey_energy"]


@pytest.mark.parametrize("neighbourhood", [0, 20])
def test_samples_reuse_pooled_memory(engine, neighbourhood):
    count = 3000 if neighbourhood == 0 else 30000
    first_q, first_e = _relaxed(engine, "O", count, 11, neighbourhood)
    free_after_first = _free_bytes()
    for _ in range(8):
        q, e = _relaxed(engine, "O", count, 11, neighbourhood)
        assert np.array_equal(q, first_q)
        assert e == first_e
    # Nothing leaks and nothing new is reserved for samples of the same size.
    assert abs(_free_bytes() - free_after_first) <= 64 << 20


def test_live_samples_do_not_share_blocks(engine):
    alone = [_relaxed(engine, g, n, 5, 20 if n > 5000 else 0, calls=(2, 2)) for g, n in
             [("O", 20000), ("I", 2000), ("D6", 12000)]]
    grids = [engine.haar(g, n, 5) for g, n in [("O", 20000), ("I", 2000), ("D6", 12000)]]
    try:
        for grid, n in zip(grids, (20000, 2000, 12000)):
            grid.relax(2, neighbourhood=20 if n > 5000 else 0)
        # Drop one while the others hold their buffers, then go on with the rest.
        grids[1].close()
        extra = engine.haar("T", 4000, 9)
        extra.relax(2, neighbourhood=0)
        for k in (0, 2):
            grids[k].relax(2)
            q = grids[k].quaternions
            assert np.array_equal(q, alone[k][0])
            assert grids[k].stats["quey_energy"] == alone[k][1]
        extra.close()
    finally:
        for grid in grids:
            grid.close()
