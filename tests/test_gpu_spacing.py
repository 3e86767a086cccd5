"""Spacing pass: per-point nearest orbit neighbour (SO(3) degrees) and its source index.

Indices are compared exactly with the FP64 oracle (documented exception: exact-distance
ties, which seeded Haar samples do not produce; the engine counts them); degrees to 1e-6
relative. Above 20,000 orientations the pass uses the near field of 4 mean radii, compared
with the FP64 C oracle (pinned to the dense oracle by tests/test_oracle_pin.py). The FP32
gather walks 2.5 of the 4 mean radii first and keeps the two best chords; a point whose
choice it cannot prove (second best within the FP32 chord error, or nearest possibly beyond
the first ball) goes to the exact FP64 search.
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


def _spacing_vs_oracle(engine, ops32, group, count, seed, q_in=None):
    gid = GROUPS.index(group)
    ops = ops32[group]
    grid = engine.haar(group, count, seed) if q_in is None else engine.from_quaternions(q_in, group)
    with grid:
        grid.spacing()
        degrees = grid.point_values("separation")
        neighbours = grid.point_neighbours()
        report = grid.spacing_exact()
        q = grid.quaternions.astype(np.float64)
    rows = cref.near_rows(q, ops, 4)
    expected = qvm.nearest_degrees(rows)
    mismatched = np.flatnonzero(neighbours != rows["nearest_source"])
    assert len(mismatched) == 0, (len(mismatched), mismatched[:10], report)
    np.testing.assert_allclose(degrees, expected, rtol=1e-6)
    assert report["exact_ties"] == 0
    return report


def test_spacing_indices_exact_at_one_million(engine, ops32):
    """Config 3's group and seed at N=1M: every index equals the FP64 oracle's; the exact
    search settles the few hundred points whose two best FP32 chords are within error."""
    report = _spacing_vs_oracle(engine, ops32, "I", 1_000_000, 7)
    assert 0 < report["exact_search"] < 20_000


@pytest.mark.slow
def test_spacing_indices_exact_at_ten_million(engine, ops32):
    """Config 3's spacing workload itself: I, N=10M, seed 7."""
    report = _spacing_vs_oracle(engine, ops32, "I", 10_000_000, 7)
    assert report["exact_search"] < 200_000


def test_spacing_exact_search_beyond_first_ball(engine, ops32):
    """A point whose whole neighbourhood within 3.2 mean radii is emptied has its nearest
    beyond the first walk's 2.5 radii: the exact search over the full 4 radii finds it."""
    group, count = "I", 60_000
    gid = GROUPS.index(group)
    ops = ops32[group]
    q = qvm.fold(qvm.haar(count, 13), gid, ops, f32=True).astype(np.float64)
    radius = qvm.mean_radius(count * len(ops))
    x = qvm.normalize(q)
    chord = 2 * np.sin(3.2 * radius / 2)
    far = np.ones(count, bool)
    for k in range(len(ops)):
        y = qvm.normalize(qvm.qmul(x, ops[k]))
        d = np.minimum(np.linalg.norm(y - x[0], axis=1), np.linalg.norm(y + x[0], axis=1))
        far &= d > chord
    far[0] = True
    q_in = q[far].astype(np.float32)
    report = _spacing_vs_oracle(engine, ops32, group, int(far.sum()), 0, q_in=q_in)
    assert report["exact_search"] >= 1


def test_spacing_matches_all_pairs(engine):
    """tests/test_measures.py:122-131 of the reference: above 20,000 orientations the spacing
    pass (near field of 4 mean radii) gives the same per-point nearest angles as a measure
    over all pairs (O 60k is above O's ratio limit, so measure() is an all-pairs quick pass)."""
    with engine.haar("O", 60000, 3) as grid:
        spacing = grid.spacing()
        near = grid.point_values("separation").copy()
        near_index = grid.point_neighbours().copy()
        assert spacing["quey_energy"] is None and "energy not measured" in spacing["precision"]
        grid.measure()
        assert np.abs(near - grid.point_values("separation")).max() < 1e-5
        assert abs(spacing["separation_deg"] - grid.stats["separation_deg"]) < 1e-5
        assert np.array_equal(near_index, grid.point_neighbours())


def test_spacing_walk_fraction_changes_no_result(engine, ops32):
    """The first walk's fraction of the cutoff (zo_near_walk, picked per size by the tuner)
    moves sources between the FP32 walk and the exact FP64 search, never a result: indices
    and degrees are the same bit for bit for every fraction and tile shape, and equal the FP64
    oracle's. A shorter walk leaves more sources to the exact search."""
    group, count, seed = "I", 200_000, 7
    runs = {}
    with engine.haar(group, count, seed) as grid:
        lib, h = grid._lib, grid._handle
        for shape in ((1, 1.5), (4, 2.0)):
            grid._check(lib.zo_near_tiles(h, *shape))
            for walk in (0.3, 0.45, 0.625, 1.0):
                grid._check(lib.zo_near_walk(h, walk))
                grid.spacing()
                runs[shape, walk] = (grid.point_neighbours().copy(), grid.point_values("separation").copy(),
                                     grid.spacing_exact()["exact_search"])
        for bad in (0.1, 1.5, -1.0):
            with pytest.raises(RuntimeError, match="InvalidWalk"):
                grid._check(lib.zo_near_walk(h, bad))
        grid._check(lib.zo_near_walk(h, 0.0))
        grid._check(lib.zo_near_tiles(h, 0, 0.0))
        q = grid.quaternions.astype(np.float64)
    first = runs[(1, 1.5), 0.625]
    for key, (neighbours, degrees, _) in runs.items():
        assert np.array_equal(neighbours, first[0]), key
        assert np.array_equal(degrees, first[1]), key
    for shape in ((1, 1.5), (4, 2.0)):
        listed = [runs[shape, w][2] for w in (0.3, 0.45, 0.625, 1.0)]
        assert listed == sorted(listed, reverse=True) and listed[0] > listed[-1], (shape, listed)
    rows = cref.near_rows(q, ops32[group], 4)
    assert np.array_equal(first[0], rows["nearest_source"])
    np.testing.assert_allclose(first[1], qvm.nearest_degrees(rows), rtol=1e-6)
