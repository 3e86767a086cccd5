"""Covering radius on the GPU (zo_cover): the largest empty cap of the full orbit on S3,
against the Qhull oracle over the full orbit (oracle/covering.py, the reference's own test
oracle) and the reference's published radii; per-point largest caps and Voronoi faces
against the hull (the reference's tests/test_covering.py and tests/test_point_values.py,
mirrored). Tolerances are the reference's: 2e-4 degrees in the radius, 2e-3 per point,
faces exact (on samples in general position; lattices have co-spherical points, where any
triangulation is valid, so only their radius is compared)."""
import math

import numpy as np
import pytest

from conftest import GROUPS
from oracle import covering as cov
from test_oracle_covering import PUBLISHED, published_grid

pytestmark = pytest.mark.gpu


def hull_of(grid):
    return cov.covering(grid.quaternions.astype(np.float64), grid.operations.astype(np.float64))


def cover_mode(grid, mode):
    grid._check(grid._lib.zo_debug_cover_mode(grid._handle, mode))


@pytest.mark.parametrize("mode", [1, 2], ids=["every-image", "chart-grid"])
@pytest.mark.parametrize("group", PUBLISHED)
def test_published_radii(engine, group, mode):
    rows, radius = published_grid(group)
    with engine.from_quaternions(rows.astype(np.float32), group) as grid:
        cover_mode(grid, mode)
        stats = grid.covering()
        assert abs(stats["covering_radius_deg"] - radius) < 2e-4
        assert abs(stats["covering_radius_deg"] - hull_of(grid)["radius_deg"]) < 2e-4
        assert stats["covering_unresolved_caps"] == 0


@pytest.mark.parametrize("group", GROUPS)
def test_covering_full_orbit_and_stale_state(engine, group):
    with engine.generate(group, h=2) as grid:
        assert grid.stats["covering_radius_deg"] is None
        for stage in range(2):
            if stage:
                previous = grid.stats["covering_radius_deg"]
                grid.relax(5)
                assert grid.stats["covering_radius_deg"] == previous
                assert not grid.stats["covering_current"]
            measured = grid.covering()
            expected = hull_of(grid)["radius_deg"]
            assert abs(measured["covering_radius_deg"] - expected) < 2e-4
            count = 2 * len(grid.operations) * len(grid)
            bound = sum(c * count ** (-(2 * i + 1) / 3) for i, c in enumerate(cov.SIMPLEX_SERIES)) * 360 / math.pi
            assert abs(measured["simplex_bound_deg"] - bound) < 1e-12
            assert abs(measured["covering_excess"] - (measured["covering_radius_deg"] / measured["simplex_bound_deg"]
                                                       - 1)) < 1e-12
            if stage:
                assert abs(measured["mesh_ratio"] - measured["covering_radius_deg"] / measured["separation_deg"]) < 1e-12
            assert measured["covering_current"]
            assert measured["covering_iteration"] == grid.stats["iteration"]
            assert measured["triangulation_backend"] == "cuda"
            assert measured["covering_certificate_probes"] > 0
            assert measured["covering_domain_bound_deg"] >= measured["covering_radius_deg"]
            assert measured["covering_unresolved_caps"] == 0
            assert np.isfinite(measured["covering_witness"]).all()


@pytest.mark.parametrize("group,count", [("O", 300), ("D6", 250), ("C2", 120)])
def test_point_values_match_hull(engine, group, count):
    with engine.haar(group, count, 5) as grid:
        grid.relax(30)
        stats = grid.covering()
        hull = hull_of(grid)
        faces = grid.point_values("faces")
        covering = grid.point_values("covering")
        assert faces is not None and covering is not None
        assert np.array_equal(faces, hull["faces"])
        assert np.allclose(covering, hull["point_covering"], atol=2e-3)
        assert covering.max() == pytest.approx(stats["covering_radius_deg"], abs=1e-3)
        assert stats["point_covering_iteration"] == stats["iteration"]
        # The witness is a cap centre: every orbit point is at least the radius away from it.
        points, _ = cov.orbit(grid.quaternions.astype(np.float64), grid.operations.astype(np.float64))
        witness = np.asarray(stats["covering_witness"], np.float64)
        nearest = np.degrees(2 * np.arccos(np.clip((points @ witness).max(), -1, 1)))
        assert nearest == pytest.approx(stats["covering_radius_deg"], abs=1e-5)


def test_imported_grid_covering_and_regeneration_invalidates(engine):
    q = np.random.default_rng(197).normal(size=(65, 4))
    with engine.from_quaternions(q, "I") as grid:
        result = grid.covering()
        assert abs(result["covering_radius_deg"] - hull_of(grid)["radius_deg"]) < 2e-4
        grid.set(q, "O")
        assert grid.stats["covering_radius_deg"] is None
        assert grid.point_values("covering") is None


def test_covering_result_is_kept_for_an_unchanged_sample(engine):
    with engine.haar("O", 1000, 11) as grid:
        first = grid.covering()
        assert not first["covering_cached"] and first["covering_unresolved_caps"] == 0
        again = grid.covering()
        assert again["covering_cached"] and again["covering_radius_deg"] == first["covering_radius_deg"]
        grid.relax(1)
        moved = grid.covering()
        assert not moved["covering_cached"] and moved["covering_radius_deg"] != first["covering_radius_deg"]
        grid.set(grid.quaternions, "T")  # same orientations, another group
        assert not grid.covering()["covering_cached"]


def test_too_few_orientations(engine):
    with engine.from_quaternions(np.eye(4)[:3], "O") as grid:
        with pytest.raises(RuntimeError, match="Covering radius: TooFewOrientations"):
            grid.covering()


def _per_point(grid, mode):
    cover_mode(grid, mode)
    stats = grid.covering()
    return stats, grid.point_values("covering").copy(), grid.point_values("faces").copy()


@pytest.mark.parametrize("group,count", [("O", 20_000), ("I", 4_000), ("C2", 60_000)])
def test_chart_grid_and_every_image_agree(engine, group, count):
    """The two ways of collecting neighbours build the same stars (same points, same order)."""
    with engine.haar(group, count, 5) as grid:
        dense, dense_cov, dense_faces = _per_point(grid, 1)
        near, near_cov, near_faces = _per_point(grid, 2)
    assert dense["covering_unresolved_caps"] == 0 and near["covering_unresolved_caps"] == 0
    assert near["covering_shell_points"] > 0 and dense["covering_shell_points"] == 0
    assert np.array_equal(near_cov, dense_cov) and np.array_equal(near_faces, dense_faces)
    assert near["covering_radius_deg"] == dense["covering_radius_deg"]


def test_chart_grid_against_hull(engine):
    """The chart-grid collection at a size Qhull still finishes in seconds."""
    with engine.haar("C2", 40_000, 3) as grid:
        cover_mode(grid, 2)  # the chart grid (by size it would scan every image)
        stats = grid.covering()
        assert stats["covering_shell_points"] > 0 and stats["covering_unresolved_caps"] == 0
        hull = hull_of(grid)
        assert abs(stats["covering_radius_deg"] - hull["radius_deg"]) < 2e-4
        assert np.allclose(grid.point_values("covering"), hull["point_covering"], atol=2e-3)
        assert np.array_equal(grid.point_values("faces"), hull["faces"])


def test_covering_at_the_headline_size(engine):
    """O, N = 100,000 (seed 193): every star proven and the same as every image's; a cell has
    about 15.5 Voronoi faces on average (the mean vertex degree of a random 3-D Delaunay
    triangulation). Every source the first (narrow) pass left short ran again, all of them
    from the chart grid: a reach past the grid's is tried at the grid's full reach first."""
    with engine.haar("O", 100_000, 193) as grid:
        near, near_cov, near_faces = _per_point(grid, 0)
        dense, dense_cov, dense_faces = _per_point(grid, 1)
    assert near["covering_unresolved_caps"] == 0 and near["covering_shell_points"] > 0
    first = near["covering_first_pass_short"] + near["covering_first_pass_sparse"]
    assert 0 < first <= near["covering_rerun_grid"] and near["covering_rerun_dense"] == 0
    assert np.array_equal(near_cov, dense_cov) and np.array_equal(near_faces, dense_faces)
    assert 13 < near_faces.mean() < 17
    assert near["covering_domain_bound_deg"] >= near["covering_radius_deg"] > near["simplex_bound_deg"]


def test_actual_shell_mesh_export(engine):
    """The reference's tests/test_explorer.py:17-23, mirrored (Hopf grid instead of the FCC
    transport, which this engine does not build)."""
    with engine.generate("O", h=2) as grid:
        mesh = grid.triangulation()
        assert len(mesh["stereographic"]) >= len(grid)
        assert len(mesh["tetrahedra"]) > 0
        assert mesh["tetrahedra"].max() < len(mesh["stereographic"])
        assert grid.stats["covering_current"]


@pytest.mark.parametrize("group,count", [("O", 300), ("D6", 250)])
def test_mesh_is_the_hull_around_the_zone(engine, group, count):
    """Every tetrahedron of the exported mesh is a facet of the orbit's convex hull that
    touches an orientation's identity image, and every such facet is exported once; the
    vertices are the orbit points' stereographic coordinates, the orientations first."""
    from scipy.spatial import ConvexHull, cKDTree

    with engine.haar(group, count, 5) as grid:
        grid.relax(30)
        mesh = grid.triangulation()
        q = grid.quaternions.astype(np.float64)
        ops = grid.operations.astype(np.float64)
    points, _ = cov.orbit(q, ops)
    chart = points[:, 1:] / (1 + points[:, :1])
    tree = cKDTree(chart)
    distance, index = tree.query(mesh["stereographic"].astype(np.float64))
    assert distance.max() < 1e-5
    assert np.array_equal(index[:count], np.arange(count))
    exported = {tuple(sorted(index[t])) for t in mesh["tetrahedra"]}
    assert len(exported) == len(mesh["tetrahedra"])
    hull = ConvexHull(points)
    around = {tuple(sorted(s)) for s in hull.simplices if (s < count).any()}
    assert exported == around


@pytest.mark.parametrize("group,count", [("C2", 4), ("C2", 7), ("D2", 5), ("C4", 12), ("T", 4), ("I", 4)])
def test_covering_of_tiny_samples(engine, group, count):
    """A handful of orientations: caps of tens of degrees, reaches up to a hemisphere."""
    q = np.random.default_rng(count).normal(size=(count, 4))
    with engine.from_quaternions(q, group) as grid:
        stats = grid.covering()
        hull = hull_of(grid)
        assert stats["covering_unresolved_caps"] == 0
        assert abs(stats["covering_radius_deg"] - hull["radius_deg"]) < 2e-4
        assert np.allclose(grid.point_values("covering"), hull["point_covering"], atol=2e-3)
