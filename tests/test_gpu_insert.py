"""Exact-count generation (zo_generate_exact, the reference's generate(..., exact=True)):
the largest inverse-Hopf grid within the target, then orientations at the centres of the
largest empty Delaunay caps (src/insert.zig), until the count is exact. Checked: the counts
and the stats, zone membership and unit norms, distinct orbits, the first inserted point at
the centre of the base grid's largest empty cap (its nearest orbit points at exactly the
base grid's covering radius, by the Qhull oracle), and the covering radius going down."""
import math

import numpy as np
import pytest
from scipy.spatial import cKDTree

from conftest import GROUPS
from oracle import covering as cov

pytestmark = pytest.mark.gpu


def in_zone(q, ops):
    return np.max(np.abs(q @ ops.T) - q[:, :1]) < 1e-6


@pytest.mark.parametrize("group,target", [("O", 400), ("D4", 300), ("I", 250), ("C2", 150), ("T", 1000)])
def test_exact_count_generation(engine, group, target):
    with engine.generate(group, count=target, exact=True) as grid:
        stats = grid.stats
        q = grid.quaternions.astype(np.float64)
        ops = grid.operations.astype(np.float64)
    assert len(q) == target and stats["count"] == target
    base = stats["base_count"]
    assert 0 < base <= target and stats["inserted_count"] == target - base and stats["grid"] == "hopf"
    with engine.generate(group, h=stats["h"]) as base_grid:
        assert len(base_grid) == base
        base_q = base_grid.quaternions.astype(np.float64)
    # The largest grid that fits: no frequency's count lies between the base and the target.
    counts = [len(engine.hopf_points(group, f)) for f in range(1, 25)]
    assert base == max(c for c in counts if c <= target)
    assert np.max(np.abs(np.linalg.norm(q, axis=1) - 1)) < 1e-6 and in_zone(q, ops)
    points, _ = cov.orbit(q, ops)
    distance, _ = cKDTree(points).query(points[:target], k=2)
    assert distance[:, 1].min() > 1e-4  # no two orbit points coincide
    if base < target:
        hull = cov.covering(base_q, ops)
        inserted = q[base:]
        base_points, _ = cov.orbit(base_q, ops)
        nearest = np.degrees(2 * np.arccos(np.clip((inserted @ base_points.T).max(axis=1), -1, 1)))
        assert nearest[0] == pytest.approx(hull["radius_deg"], abs=1e-3)
        assert nearest.max() <= hull["radius_deg"] + 1e-3
        assert cov.covering(q, ops)["radius_deg"] <= hull["radius_deg"] + 1e-6


def test_exact_count_with_fixed_identity(engine):
    with engine.generate("O", count=400, exact=True, fixed_identity=True) as grid:
        stats = grid.stats
        assert len(grid) == 400 and stats["fixed_identity"]
        index = stats["identity_index"]
        np.testing.assert_array_equal(grid.quaternions[index], [1, 0, 0, 0])
        grid.relax(3)
        np.testing.assert_array_equal(grid.quaternions[index], [1, 0, 0, 0])


def test_exact_count_errors(engine):
    with pytest.raises(RuntimeError, match="Exact-count generation: ExactCountRange32To1000000"):
        engine.generate("O", count=20, exact=True)
    with pytest.raises(RuntimeError, match="Exact-count generation: TransportNotAvailable"):
        engine.generate("O", count=400, exact=True, kind="transport")


@pytest.mark.parametrize("group", GROUPS)
def test_exact_count_identity_and_zone_after_relaxation(engine, group):
    """The reference's tests/test_workbench.py:7-30, mirrored: 1,000 orientations with a fixed
    identity; inserted centres do not cluster (every orbit point at least 0.01 in chord from
    the next); after relaxing, the zone holds, the identity stays and the sample has moved."""
    with engine.generate(group, count=1000, exact=True, fixed_identity=True) as grid:
        assert len(grid) == 1000
        assert grid.stats["base_count"] + grid.stats["inserted_count"] == 1000
        before = grid.quaternions.copy()
        ops = grid.operations.astype(np.float64)
        points, _ = cov.orbit(before.astype(np.float64), ops)
        assert cKDTree(points).query(before.astype(np.float64), k=2)[0][:, 1].min() > 0.01
        identity = grid.stats["identity_index"]
        assert identity is not None
        grid.relax(12)
        q = grid.quaternions.astype(np.float64)
        assert np.max(np.abs(q @ ops.T) - q[:, :1]) < 1e-6
        np.testing.assert_array_equal(q[identity], [1, 0, 0, 0])
        assert np.max(np.abs(q - before)) > 1e-5
        assert grid.stats["separation_deg"] > 0


@pytest.mark.parametrize("group,count", [("C6", 84), ("D3", 62), ("D3", 84), ("D4", 84)])
def test_exact_count_thin_shell(engine, group, count):
    with engine.generate(group, count=count, exact=True, identity=True) as grid:
        assert len(grid) == count
