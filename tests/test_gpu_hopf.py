"""zo_generate: inverse-Hopf product grids folded into the zone on the GPU (src/engine.zig:
244-281), against the reference's SO3K_Grids fixture and the oracle fold.

Mirrors the reference's tests/test_hopf.py: rows in the reference's order, each an image of
the fixture row's orbit (chord < 1e-6), in the zone, with stats grid "hopf" and h = f;
frequency selection by nearest count; the count limit; and the haar() bootstrap of the
reference's Python API (`Grid(group, h=1, count=8)` before zo_random).
"""
import numpy as np
import pytest

from conftest import GROUPS
from oracle import qvm
from test_hopf import CASES, FIXTURE, expected_count, orbit_chord, qmul

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group,f", [c for c in CASES if c[1] <= 6 or c in [("O", 14), ("I", 12), ("D6", 10)]])
def test_generate_matches_fixture(engine, ops32, ops64, group, f):
    gid = GROUPS.index(group)
    with engine.generate(group, h=f) as grid:
        q = grid.quaternions.astype(np.float64)
        stats = grid.stats
    assert stats["grid"] == "hopf" and stats["h"] == f and stats["count"] == len(q) == expected_count(group, f)
    assert stats["generator"].startswith("Inverse Hopf product grid")
    # The fold of the host rows as the oracle folds float32 input: bit for bit, except rows
    # on a zone boundary (grid points often lie on symmetry planes), where the FP64
    # products' last bits decide between equivalent zone images; there both rows are in the
    # zone and images of each other.
    expected = qvm.fold(engine.hopf_points(group, f), gid, ops32[group], f32=True)
    differ = np.any(q.astype(np.float32) != expected, axis=1)
    assert differ.mean() < 0.2, differ.mean()
    if differ.any():
        assert orbit_chord(q[differ], expected[differ].astype(np.float64), ops64[group]).max() < 1e-6
    # In the zone up to rounding: no image of a row has a larger scalar part (the points on
    # a boundary satisfy the zone's strict inequalities only to within rounding).
    images = qmul(q[:, None], ops64[group][None])
    assert np.all(q[:, 0] >= np.abs(images[..., 0]).max(axis=1) - 1e-6)
    assert orbit_chord(q, FIXTURE[f"{group}_{f}"], ops64[group]).max() < 1e-6


@pytest.mark.parametrize("group", GROUPS)
def test_frequency_nearest_the_count(engine, group):
    sizes = {f: expected_count(group, f) for f in range(1, 513) if expected_count(group, f) <= 10_000_000}
    for target in (300, 900):
        with engine.generate(group, count=target) as grid:
            n = len(grid)
            assert grid.stats["grid"] == "hopf"
        assert abs(np.log(n / target)) == min(abs(np.log(m / target)) for m in sizes.values())


def test_regenerate_on_one_engine(engine):
    with engine.generate("O", h=3) as grid:
        for f in (1, 2, 5, 9):
            grid._check(grid._lib.zo_generate(grid._handle, GROUPS.index("O"), f, 2048, 0, 0))
            assert len(grid) == expected_count("O", f) and grid.stats["h"] == f


def test_frequency_beyond_the_count_limit(engine):
    with pytest.raises(RuntimeError, match="GridTooLarge"):
        engine.generate("C2", h=100)


def test_transport_is_not_built(engine):
    with pytest.raises(RuntimeError, match="TransportNotAvailable"):
        engine.generate("O", h=6, kind="transport")
    with pytest.raises(ValueError):
        engine.generate("D4", kind="transport")


def test_haar_bootstrap_of_the_reference_api(engine):
    """The reference's haar() creates Grid(group, h=1, count=8) and then calls zo_random on
    it (python/zxtalori/api.py:364-372): both calls succeed on this library."""
    grid = engine.Grid("O", h=1, count=8)
    try:
        assert len(grid) == 1 and grid.stats["grid"] == "hopf"
        grid._check(grid._lib.zo_random(grid._handle, GROUPS.index("O"), 1000, 193))
        assert len(grid) == 1000 and grid.stats["grid"] is None and grid.stats["h"] == 0
    finally:
        grid.close()


def test_relax_a_generated_grid(engine):
    """A generated grid relaxes and measures like any other sample (the reference's default
    constructor path)."""
    with engine.generate("I", h=6) as grid:
        before = grid.measure()["quey_energy"]
        grid.relax(10)
        after = grid.measure()["quey_energy"]
        assert grid.stats["iteration"] == 10 and grid.stats["grid"] == "hopf"
    assert after <= before * (1 + 1e-9)


def test_identity_keeps_grid_fields(engine):
    with engine.generate("T", h=3, identity=True) as grid:
        stats = grid.stats
        assert stats["grid"] == "hopf" and stats["h"] == 3
        assert stats["base_count"] == expected_count("T", 3)
        assert stats["identity_index"] is not None
