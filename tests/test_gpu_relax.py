"""BB relaxation on the GPU against the oracle's FP64 relaxation (shaders/relax.wgsl).

FP64 mode follows the oracle step for step: after 10 all-pairs steps the float32 copies of
the positions agree to one float32 rounding and the energy to 1e-12. FP32 mode (FP32 pair
arithmetic, FP64 BB products and renormalisation, float32 state) stays within 5e-6 in
position and 1e-6 relative in energy and separation of the FP64 trajectory.
"""
import numpy as np
import pytest

from conftest import GROUPS
from oracle import qvm

pytestmark = pytest.mark.gpu


def chord(a, b):
    return np.minimum(np.linalg.norm(a - b, axis=1), np.linalg.norm(a + b, axis=1))


@pytest.mark.parametrize("group,count", [("O", 300), ("I", 150), ("D6", 200)])
def test_fp64_relax_follows_oracle(engine, ops64, group, count):
    gid = GROUPS.index(group)
    ops = ops64[group]
    start = qvm.fold(qvm.haar(count, 7), gid, ops, f32=False)
    relax = qvm.Relax(start, gid, ops)
    with engine.haar(group, count, 7, precision="fp64") as grid:
        grid.relax(10)
        stats = grid.stats
        q = grid.quaternions.astype(np.float64)
    relax.run(10)
    assert chord(q, relax.q.astype(np.float32).astype(np.float64)).max() <= 1.2e-7
    expected = qvm.quick_measures(qvm.pair_rows(relax.q, ops), len(ops))
    assert stats["quey_energy"] == pytest.approx(expected["quey_energy"], rel=1e-12)
    assert stats["separation_deg"] == pytest.approx(expected["separation_deg"], rel=1e-10)
    assert stats["iteration"] == 10


@pytest.mark.parametrize("group,count", [("O", 300), ("I", 150)])
def test_fp32_relax_error_vs_fp64(engine, ops64, group, count):
    gid = GROUPS.index(group)
    ops = ops64[group]
    relax = qvm.Relax(qvm.fold(qvm.haar(count, 7), gid, ops, f32=False), gid, ops)
    with engine.haar(group, count, 7, precision="fp32") as grid:
        grid.relax(10)
        stats = grid.stats
        q = grid.quaternions.astype(np.float64)
    relax.run(10)
    assert chord(q, relax.q).max() < 5e-6
    expected = qvm.quick_measures(qvm.pair_rows(relax.q, ops), len(ops))
    assert stats["quey_energy"] == pytest.approx(expected["quey_energy"], rel=1e-6)
    assert stats["separation_deg"] == pytest.approx(expected["separation_deg"], rel=1e-6)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group", GROUPS)
def test_descent_three_steps(engine, group, precision):
    """test_measures.py:235-247: energy non-increasing over 3 steps, unit norms, quick
    energy equal to the full measure's."""
    with engine.haar(group, 256, 3, precision=precision) as grid:
        initial = grid.measure()["quey_energy"]
        grid.relax(3)
        quick = grid.stats
        assert quick["energy_ratios_current"] is False
        assert quick["riesz_1"] is None and quick["log_ratio"] is None
        final = grid.measure()["quey_energy"]
        assert quick["quey_energy"] == pytest.approx(final, rel=2e-6, abs=2e-6)
        assert final <= initial + 1e-6
        np.testing.assert_allclose(np.linalg.norm(grid.quaternions, axis=-1), 1, rtol=3e-7, atol=3e-7)
        assert grid.stats["iteration"] == 3
        assert grid.stats["point_separation_iteration"] == 3


def test_fixed_identity(engine):
    with engine.haar("O", 200, 9) as grid:
        grid.identity(add=True, fixed=True)
        n = len(grid)
        stats = grid.stats
        assert stats["fixed_identity"] is True and stats["identity_index"] == n - 1
        grid.relax(5)
        np.testing.assert_array_equal(grid.quaternions[n - 1], [1, 0, 0, 0])


def test_relax_history_and_batches(engine):
    with engine.haar("C4", 300, 2) as grid:
        grid.relax(7)
        assert len(grid.history) == 1 and grid.history[0]["iteration"] == 7
        seen = []
        grid.relax(3, callback=lambda g, s: seen.append(s["iteration"]))
        assert seen == [8, 9, 10]
        assert grid.stats["step_deg"] > 0
