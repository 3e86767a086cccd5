"""Covering optimisation (zo_cover_optimize, zo_cover_kicks; the reference's
Grid.optimize_covering): lowers the covering radius, keeps the zone and returns the best
sample it saw, holds a fixed identity and a separation floor, stops on a callback. Mirrors
the reference's tests/test_covering_optimizer.py; the radius is checked against the Qhull
oracle over the full orbit."""
import numpy as np
import pytest

from oracle import covering as cov

pytestmark = pytest.mark.gpu


def in_zone(grid):
    q = grid.quaternions.astype(np.float64)
    ops = grid.operations.astype(np.float64)
    return np.max(np.abs(q @ ops.T) - q[:, :1]) < 1e-6


@pytest.mark.parametrize("group,mode", [("O", "tet"), ("D4", "face"), ("I", "face")])
def test_optimizer_lowers_covering_and_keeps_zone(engine, group, mode):
    with engine.haar(group, 300, 11) as grid:
        grid.relax(20)
        before = grid.covering()["covering_radius_deg"]
        grid.optimize_covering(250, mode=mode)
        stats = grid.stats
        assert len(grid) == 300
        assert stats["covering_current"]
        assert stats["covering_radius_deg"] < before
        # Only the covering radius is measured: energy and separation wait for measure().
        assert stats["measures_current"] is False
        assert grid.measure()["measures_current"]
        # The engine keeps the best sample it saw, so the result is that sample.
        assert stats["covering_radius_deg"] == pytest.approx(stats["covering_optimizer_best_deg"], abs=1e-5)
        assert np.max(np.abs(np.linalg.norm(grid.quaternions, axis=1) - 1)) < 1e-5
        assert in_zone(grid)
        expected = cov.covering(grid.quaternions, grid.operations)["radius_deg"]
        assert expected == pytest.approx(stats["covering_radius_deg"], abs=2e-3)


def test_optimizer_holds_fixed_identity_and_stops_on_best(engine):
    with engine.generate("O", count=400, exact=True, fixed_identity=True) as grid:
        index = grid.stats["identity_index"]
        calls = []
        grid.optimize_covering(600, batch=50,
                               callback=lambda g, s: calls.append(s["covering_optimizer_steps"]) or len(calls) < 3)
        stats = grid.stats
        assert len(calls) == 3 and stats["covering_optimizer_steps"] == 150
        np.testing.assert_array_equal(grid.quaternions[index], [1, 0, 0, 0])
        assert stats["covering_radius_deg"] == pytest.approx(stats["covering_optimizer_best_deg"], abs=1e-5)
        with pytest.raises(ValueError):
            grid.optimize_covering(1, mode="everything")


def test_separation_floor_holds(engine):
    with engine.haar("D4", 400, 9) as grid:
        grid.relax(30)
        before = grid.covering()["covering_radius_deg"]
        floor = 0.95 * grid.measure()["separation_deg"]
        grid.optimize_covering(200, min_separation_deg=floor)
        assert grid.stats["covering_radius_deg"] < before
        assert grid.measure()["separation_deg"] >= floor * (1 - 1e-5)
        with pytest.raises(ValueError):
            grid.optimize_covering(1, min_separation_deg=200)


def test_plateau_kicks_keep_the_best(engine):
    with engine.haar("T", 300, 3) as grid:
        grid.relax(20)
        before = grid.covering()["covering_radius_deg"]
        grid.optimize_covering(120, patience=5, kick=0.05)
        stats = grid.stats
        assert stats["covering_optimizer_kicks"] > 0
        assert stats["covering_radius_deg"] == pytest.approx(stats["covering_optimizer_best_deg"], abs=1e-5)
        assert stats["covering_radius_deg"] < before and in_zone(grid)
        assert stats["covering_kick_settings"]["patience"] == 5


def test_invalid_settings_through_the_abi(engine):
    with engine.haar("O", 100, 1) as grid:
        assert grid._lib.zo_cover_kicks(grid._handle, 0, 5e-4, 0.04, 0.03) == -1
        assert grid._lib.zo_error(grid._handle).decode() == "Covering kicks: InvalidKickPatience"
        assert grid._lib.zo_cover_optimize(grid._handle, 1, 2, 1, 0.0) == -1
        assert grid._lib.zo_error(grid._handle).decode() == "Covering optimization: InvalidCoveringMode"


def test_undone_steps_bring_back_the_covering_they_set_aside(engine):
    """A step that does not lower the radius is undone, and the covering measured before it
    comes back instead of being measured again: after a batch that ends without the
    finishing pass, the engine's covering (radius, per-point caps and faces, and the mesh
    built from its stars and chart grid) equals a fresh measurement of the same sample."""
    with engine.haar("O", 4000, 4) as grid:
        grid._check(grid._lib.zo_debug_cover_mode(grid._handle, 2))  # the chart grid's path
        grid.relax(20)
        grid.covering()
        grid._check(grid._lib.zo_cover_optimize(grid._handle, 40, 1, 0, 0.0))
        stats = grid.stats
        assert stats["covering_optimizer_skipped"] > 0 and stats["covering_optimizer_improved"] > 0
        assert stats["covering_current"]
        kept = (stats["covering_radius_deg"], grid.point_values("covering").copy(),
                grid.point_values("faces").copy())
        kept_mesh = grid.triangulation()
        grid._check(grid._lib.zo_debug_cover_mode(grid._handle, 2))  # drops the covering
        fresh_mesh = grid.triangulation()
        fresh = grid.stats
        assert fresh["covering_radius_deg"] == kept[0]
        assert np.array_equal(grid.point_values("covering"), kept[1])
        assert np.array_equal(grid.point_values("faces"), kept[2])
        assert np.array_equal(fresh_mesh["tetrahedra"], kept_mesh["tetrahedra"])
        assert np.array_equal(fresh_mesh["stereographic"], kept_mesh["stereographic"])
