"""Spacing pass: per-point nearest orbit neighbour (SO(3) degrees) and its source index.

Indices are compared exactly with the FP64 oracle (documented exception: exact-distance
ties, which seeded Haar samples do not produce); degrees to 1e-6 relative. Above 20,000
orientations the pass uses the near field of 4 mean radii, compared with the FP64 C oracle.
"""
import numpy as np
import pytest

from conftest import GROUPS
from oracle import cref, qvm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group,count", [("O", 2000), ("I", 1500), ("C6", 1000)])
def test_spacing_all_pairs(engine, ops32, ops64, group, count, precision):
    gid = GROUPS.index(group)
    ops = ops32[group] if precision == "fp32" else ops64[group]
    with engine.haar(group, count, 3, precision=precision) as grid:
        stats = grid.spacing()
        degrees = grid.point_values("separation")
        neighbours = grid.point_neighbours()
        q = grid.quaternions.astype(np.float64) if precision == "fp32" else qvm.fold(qvm.haar(count, 3), gid, ops,
                                                                                     f32=False)
    rows = cref.pair_rows(q, ops)
    assert np.array_equal(neighbours, rows["nearest_source"])
    np.testing.assert_allclose(degrees, qvm.nearest_degrees(rows), rtol=1e-6)
    assert stats["separation_deg"] == pytest.approx(degrees.min(), rel=1e-7)
    assert stats["quey_energy"] is None and "energy not measured" in stats["precision"]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_spacing_near_field(engine, ops32, ops64, precision):
    group, count, gid = "I", 40000, 10
    ops = ops32[group] if precision == "fp32" else ops64[group]
    with engine.haar(group, count, 7, precision=precision) as grid:
        grid.spacing()
        degrees = grid.point_values("separation")
        neighbours = grid.point_neighbours()
        q = grid.quaternions.astype(np.float64) if precision == "fp32" else qvm.fold(qvm.haar(count, 7), gid, ops,
                                                                                     f32=False)
    rows = cref.near_rows(q, ops, 4)
    assert np.array_equal(neighbours, rows["nearest_source"])
    np.testing.assert_allclose(degrees, qvm.nearest_degrees(rows), rtol=1e-6)


def test_point_values_track_runs(engine):
    with engine.haar("O", 1000, 9) as grid:
        assert grid.point_values("separation") is None
        assert grid.point_values("covering") is None
        grid.relax(10)
        assert grid.point_values("separation") is not None
        assert grid.stats["point_separation_iteration"] == grid.stats["iteration"]
