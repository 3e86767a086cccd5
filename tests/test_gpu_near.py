"""Near-field force pass on the GPU against the oracle (tests/test_near_field.py's checks).

FP64 mode matches the dense FP64 near-field rows to 1e-10; FP32 mode to 2e-5 in force and
curvature (relative to the largest), 1e-6 in energy, 5e-5 in the raw nearest chord (the
float32 images' rounding, ~3e-8 per coordinate, on chords near 0.01; the separation the API
reports is recomputed in FP64). The stats energy of a near-field pass matches the
reference's own dense model within its 2e-6.
"""
import numpy as np
import pytest

from conftest import GROUPS
from oracle import cref, qvm

pytestmark = pytest.mark.gpu

TOL = {"fp32": (2e-5, 2e-5, 1e-6, 5e-5), "fp64": (1e-10, 1e-10, 1e-10, 1e-10)}


def compare(rows, o, precision):
    tf, tc, te, tn = TOL[precision]
    scale = np.linalg.norm(o["force"], axis=1).max()
    assert np.linalg.norm(rows[:, :3] - o["force"], axis=1).max() / scale < tf
    assert np.max(np.abs(rows[:, 3] - o["curvature"]) / o["curvature"].max()) < tc
    assert np.max(np.abs(rows[:, 4] - o["energy"]) / np.maximum(o["energy"], 1e-300)) < te
    assert np.max(np.abs(rows[:, 5] - o["nearest"]) / o["nearest"]) < tn


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group,count", [("O", 600), ("D6", 500), ("C2", 400), ("I", 300), ("T", 400), ("D3", 400)])
def test_near_rows_match_dense_oracle(engine, ops32, ops64, group, count, precision):
    gid = GROUPS.index(group)
    ops = ops32[group] if precision == "fp32" else ops64[group]
    with engine.haar(group, count, 11, precision=precision) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64) if precision == "fp32" else qvm.fold(qvm.haar(count, 11), gid, ops,
                                                                                     f32=False)
    compare(rows, qvm.near_rows(q, ops, 20), precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_near_rows_large_against_c_oracle(engine, ops32, ops64, precision):
    group, count, gid = "O", 30000, 9
    ops = ops32[group] if precision == "fp32" else ops64[group]
    with engine.haar(group, count, 21, precision=precision) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64) if precision == "fp32" else qvm.fold(qvm.haar(count, 21), gid, ops,
                                                                                     f32=False)
    compare(rows, cref.near_rows(q, ops, 20), precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group,count", [("C2", 120000), ("D3", 60000), ("T", 40000), ("I", 20000)])
def test_chart_grid_path_across_groups(engine, ops32, ops64, group, count, precision):
    """Cutoffs below 0.5 rad take the shell and chart-grid path in both modes; the small-N
    cases above take the dense path. Each group's grid path against the C oracle."""
    gid = GROUPS.index(group)
    ops = ops32[group] if precision == "fp32" else ops64[group]
    with engine.haar(group, count, 31, precision=precision) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64) if precision == "fp32" else qvm.fold(qvm.haar(count, 31), gid, ops,
                                                                                     f32=False)
    assert qvm.near_radius(count, len(ops), 20)[0] < 0.5
    compare(rows, cref.near_rows(q, ops, 20), precision)


@pytest.mark.parametrize("group,count", [("C2", 20000), ("O", 4000), ("D6", 3300), ("I", 1800)])
def test_grid_path_wide_cutoffs(engine, ops32, group, count):
    """FP32 mode keeps the chart grid for cutoffs of 0.5 to 0.9 rad when the sample has
    more than 1e8 image pairs (its gather walks exact chart balls); these samples take it,
    checked against the C oracle."""
    gid = GROUPS.index(group)
    ops = ops32[group]
    r = qvm.near_radius(count, len(ops), 20)[0]
    assert 0.5 <= r < 0.9 and count * count * len(ops) > 1e8
    with engine.haar(group, count, 41) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64)
    compare(rows, cref.near_rows(q, ops, 20), "fp32")


@pytest.mark.parametrize("group,count", [("O", 1000), ("D6", 1000), ("C2", 800)])
def test_near_sums_match_dense_reference(engine, ops32, group, count):
    """test_near_field.py:43-54 with its tolerances."""
    with engine.haar(group, count, 11) as grid:
        grid.relax(20)
        grid.relax(1, neighbourhood=20)
        stats = grid.stats
        assert stats["energy_neighbourhood"] == 20 and stats["relax_neighbourhood"] == 20
        q = grid.quaternions.astype(np.float64)
        rows = qvm.near_rows(q, ops32[group], 20)
        n, order = len(q), len(ops32[group])
        assert stats["energy"] == pytest.approx(rows["energy"].sum() / (n * order * (n - 1)), rel=2e-6)
        assert stats["separation_deg"] == pytest.approx(qvm.separation_deg(rows["nearest"].min()), rel=1e-4)
        grid.relax(1, neighbourhood=0)
        assert grid.stats["energy_neighbourhood"] is None


def test_near_relaxation_approaches_all_pairs(engine):
    """test_near_field.py:57-65."""
    outcomes = {}
    for delta in (0, 20):
        with engine.haar("O", 1000, 7) as grid:
            grid.relax(200, neighbourhood=delta)
            grid.relax(0, neighbourhood=0)
            grid.measure()
            outcomes[delta] = grid.stats
    assert outcomes[20]["energy"] == pytest.approx(outcomes[0]["energy"], rel=1e-5)
    assert outcomes[20]["separation_deg"] > 0.95 * outcomes[0]["separation_deg"]


def test_neighbourhood_range(engine):
    with engine.haar("O", 200, 3) as grid:
        with pytest.raises(RuntimeError, match="NeighbourhoodOutside2To1000"):
            grid.relax(1, neighbourhood=1)


def _nudged(q, seed):
    up = np.random.default_rng(seed).random(q.shape) < 0.5
    return np.nextafter(q, np.where(up, np.float32(np.inf), np.float32(-np.inf))).astype(np.float32)


def test_near_relax_fp32_vs_fp64(engine, ops32):
    """The same 20 near-field steps from the same float32 start in both modes. The energy of
    the FP32-refined trajectory stays within 1e-6 of the FP64 one. The separation, a single
    pair's distance after a chaotic descent, is compared with the FP64 method's own
    sensitivity: the FP64 run started one float32 ulp away moves it by about as much (at
    this size, up to 1e-4 relative). The FP32 run must stay within three times the largest
    of three such nudges, and its reported separation must equal the FP64 oracle's of its
    own relaxed sample to 1e-6."""
    with engine.haar("O", 5000, 5) as grid:
        start = grid.quaternions

    def relaxed(q, mode):
        with engine.from_quaternions(q, "O", precision=mode) as grid:
            grid.relax(20, neighbourhood=20)
            return grid.stats, grid.quaternions.astype(np.float64)

    (s64, _), (s32, q32) = relaxed(start, "fp64"), relaxed(start, "fp32")
    assert s32["energy"] == pytest.approx(s64["energy"], rel=1e-6)
    sensitivity = max(abs(relaxed(_nudged(start, k), "fp64")[0]["separation_deg"] - s64["separation_deg"])
                      for k in range(3))
    assert abs(s32["separation_deg"] - s64["separation_deg"]) <= 3 * sensitivity + 1e-6 * s64["separation_deg"]
    own = qvm.separation_deg(qvm.near_rows(q32, ops32["O"], 20)["nearest"].min())
    assert s32["separation_deg"] == pytest.approx(own, rel=1e-6)


@pytest.mark.parametrize("sources_per_warp,sites_per_cell",
                         [(2, 1.5), (2, 3.0), (8, 1.0), (8, 3.0), (4, 1.25), (4, 2.0), (1, 1.0), (1, 3.0)])
def test_every_tile_shape_matches_the_oracle(engine, ops32, sources_per_warp, sites_per_cell):
    """Each tile shape the tuner may choose (zo_near_tiles) gives the oracle's rows (near
    field, O 30k) and the oracle's spacing indices (I 40k). Shape 1 (one source per thread)
    is the spacing pass's alone; the relaxation pass then keeps 4 sources per warp."""
    with engine.haar("O", 30000, 23) as grid:
        grid._check(grid._lib.zo_near_tiles(grid._handle, sources_per_warp, sites_per_cell))
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64)
    compare(rows, cref.near_rows(q, ops32["O"], 20), "fp32")
    with engine.haar("I", 40000, 29) as grid:
        grid._check(grid._lib.zo_near_tiles(grid._handle, sources_per_warp, sites_per_cell))
        grid.spacing()
        neighbours = grid.point_neighbours()
        q = grid.quaternions.astype(np.float64)
    assert np.array_equal(neighbours, cref.near_rows(q, ops32["I"], 4)["nearest_source"])


def test_tile_override_rejects_bad_shapes(engine):
    with engine.haar("O", 1000, 3) as grid:
        with pytest.raises(RuntimeError, match="InvalidTiles"):
            grid._check(grid._lib.zo_near_tiles(grid._handle, 3, 2.0))
        with pytest.raises(RuntimeError, match="InvalidTiles"):
            grid._check(grid._lib.zo_near_tiles(grid._handle, 4, 100.0))
        grid._check(grid._lib.zo_near_tiles(grid._handle, 0, 0.0))  # back to the table


def test_sites_at_the_cutoff_along_the_chart_axes(engine, ops32):
    """The walk trims each cell row's run to the balls' extent along chart x; sites just
    inside the cutoff (at 1 - 1e-6 of it) in the six chart-axis directions of an isolated
    source must all be found: its nearest chord and rows equal the dense oracle's."""
    group, count = "O", 30000
    ops = ops32[group]
    base = qvm.fold(qvm.haar(2 * count, 19), 9, ops, f32=True).astype(np.float64)
    r = qvm.near_radius(count, len(ops), 20)[0]  # the cutoff of the final sample of `count` points
    # Clear the source's neighbourhood (every image within 1.2 r of the identity), then put
    # the identity and six points at angle r (1 - 1e-6) from it, along +-x, +-y, +-z.
    x = qvm.normalize(base)
    keep = np.ones(len(x), bool)
    for g in ops:
        y = qvm.normalize(qvm.qmul(x, g))
        keep &= np.minimum(np.linalg.norm(y - [1, 0, 0, 0], axis=1), np.linalg.norm(y + [1, 0, 0, 0], axis=1)) > \
            2 * np.sin(0.6 * r)
    theta = r * (1 - 1e-6)  # the S3 angle from (1, 0, 0, 0) to (cos t, sin t, 0, 0) is t
    planted = [[1.0, 0, 0, 0]]
    for axis in range(3):
        for sign in (1.0, -1.0):
            v = np.zeros(4)
            v[0], v[1 + axis] = np.cos(theta), sign * np.sin(theta)
            planted.append(v)
    q = np.vstack([np.array(planted), x[keep][: count - len(planted)]]).astype(np.float32)
    assert len(q) == count
    with engine.from_quaternions(q, group) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        got = grid.quaternions.astype(np.float64)
    dense = qvm.near_rows(got, ops, 20, sources=np.arange(7))
    assert np.all(dense["nearest"] < dense["cut"])  # the planted sites are inside the cutoff
    np.testing.assert_allclose(rows[:7, 5], dense["nearest"], rtol=5e-5)
    # The isolated source's energy is a window remainder of about 1e-11 (its sites sit where
    # the window vanishes); the planted sites' own rows are ordinary.
    np.testing.assert_allclose(rows[1:7, 4], dense["energy"][1:], rtol=1e-5)


def test_pair_counts_of_the_gather(engine, ops32):
    """zo_debug_pair_counts: the in-cutoff pairs the FP32 gather counts equal a k-d tree's
    count of orbit images within the cutoff chord (own images excluded), up to FP32 rounding at
    the boundary; the candidates it evaluates include all of them. The rows of the counting
    pass are the ordinary pass's."""
    import ctypes as C
    from scipy.spatial import cKDTree

    group, count, delta = "O", 20000, 20
    ops = ops32[group]
    with engine.haar(group, count, 41) as grid:
        grid.relax(0, neighbourhood=delta)
        before = grid.debug_rows(0)
        out = (C.c_double * 2)()
        grid._check(grid._lib.zo_debug_pair_counts(grid._handle, out))
        after = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64)
    np.testing.assert_array_equal(before, after)
    candidates, inside = out[0], out[1]
    x = qvm.normalize(q)
    images = qvm.normalize(qvm.images(x, ops))  # (|K|, n, 4)
    _, cut2 = qvm.near_radius(count, len(ops), delta)
    chord = np.sqrt(cut2)
    tree = cKDTree(np.concatenate([images, -images]).reshape(-1, 4))
    every = int(tree.query_ball_point(x, chord, return_length=True).sum())
    own = sum(int(np.count_nonzero(np.linalg.norm(s * images[k] - x, axis=1) <= chord))
              for k in range(len(ops)) for s in (1.0, -1.0))  # the identity image, and any other own image
    expected = every - own
    assert abs(inside - expected) <= 1e-5 * expected + 10, (inside, expected)
    assert candidates >= inside
    assert candidates < 3 * inside  # the walk stays near the sources' balls


def test_headline_rows_against_c_oracle(engine, ops32):
    """The headline workload (O, N = 100,000, seed 193, neighbourhood 20): the first force
    pass's rows of 3,000 sources (random ones and the nearest a zone boundary) against the
    FP64 C oracle, at the FP32 tolerances above."""
    with engine.haar("O", 100_000, 193) as grid:
        grid.relax(0, neighbourhood=20)
        rows = grid.debug_rows(0)
        q = grid.quaternions.astype(np.float64)
    ops = ops32["O"]
    rng = np.random.default_rng(0)
    margin = np.max(np.abs(q @ ops[1:].T), axis=1) / q[:, 0]  # near 1: close to a zone face
    picked = np.unique(np.concatenate([rng.choice(len(q), 2000, replace=False), np.argsort(-margin)[:1000]]))
    compare(rows[picked], cref.near_rows(q, ops, 20, sources=picked), "fp32")


def test_headline_trajectory_against_fp64(engine, ops32):
    """100 steps of the headline workload in both modes from the same float32 start. Energy:
    the FP32-refined run within 1e-6 of the FP64 run (measured 1.2e-7). Separation: within
    three times the FP64 method's own sensitivity to a one-ulp change of its start (measured
    4.6e-3 against 6.3e-3), and equal to 1e-6 to the FP64 C oracle's separation of the FP32
    run's own relaxed sample."""
    with engine.haar("O", 100_000, 193) as grid:
        start = grid.quaternions

    def relaxed(q, mode):
        with engine.from_quaternions(q, "O", precision=mode) as grid:
            grid.relax(100, neighbourhood=20)
            return grid.stats, grid.quaternions.astype(np.float64)

    (s64, _), (s32, q32) = relaxed(start, "fp64"), relaxed(start, "fp32")
    assert s32["energy"] == pytest.approx(s64["energy"], rel=1e-6)
    sensitivity = max(abs(relaxed(_nudged(start, k), "fp64")[0]["separation_deg"] - s64["separation_deg"])
                      for k in range(2))
    assert abs(s32["separation_deg"] - s64["separation_deg"]) <= 3 * sensitivity + 1e-6 * s64["separation_deg"]
    own = qvm.separation_deg(cref.near_rows(q32, ops32["O"], 20)["nearest"].min())
    assert s32["separation_deg"] == pytest.approx(own, rel=1e-6)
