"""The C oracle (oracle/qvm_ref.c) against the golden-pinned NumPy oracle (oracle/qvm.py).

Every large GPU parity case is checked against the C oracle, which finds near-field
neighbours through its own shell of images near the zone and a grid over the stereographic
chart (shaders/shell.wgsl:18-39, src/near.zig:90-152). The NumPy oracle tests every image
of the sample with no shell and no grid, and tests/test_oracle_golden.py pins it to the
reference's own dense models (tests/test_near_field.py:23-40 near_reference,
tests/test_pair_kernels.py:27-69 reference). Here the two agree, on sources drawn at random
and on the sources nearest a zone boundary (where shell membership decides), at sizes
where the C oracle takes its chart-grid path: rows to 1e-12, nearest sources equal.
"""
import numpy as np
import pytest

from conftest import GROUPS
from oracle import cref, qvm


def zone_planes(ops):
    """The 2|K|-1 bisector planes of the zone (src/covering.zig:382-396), FP64."""
    planes = []
    for k, g in enumerate(ops):
        for s in (1.0, -1.0):
            if k == 0 and s > 0:
                continue
            h = np.concatenate([[1.0 - s * g[0]], -s * g[1:]])
            planes.append(h / np.linalg.norm(h))
    return np.array(planes)


def picked_sources(q, ops, random_count, rim_count, seed=1):
    """`random_count` sources at random and the `rim_count` nearest a zone boundary."""
    x = qvm.normalize(q)
    margin = (x @ zone_planes(ops).T).min(axis=1)
    rim = np.argsort(margin, kind="stable")[:rim_count]
    rest = np.setdiff1d(np.arange(len(q)), rim)
    chosen = np.random.default_rng(seed).choice(rest, random_count, replace=False)
    return np.concatenate([rim, chosen])


def compare_rows(c, d):
    scale = np.linalg.norm(d["force"], axis=1).max()
    assert np.linalg.norm(c["force"] - d["force"], axis=1).max() / scale < 1e-12
    assert np.abs(c["curvature"] - d["curvature"]).max() / d["curvature"].max() < 1e-12
    assert np.max(np.abs(c["energy"] - d["energy"]) / np.maximum(d["energy"], 1e-300)) < 1e-12
    assert np.max(np.abs(c["nearest"] - d["nearest"]) / d["nearest"]) < 1e-12
    assert np.array_equal(c["nearest_source"], d["nearest_source"])


@pytest.mark.parametrize("group,count,delta,seed,random_count", [
    ("O", 30000, 20, 21, 250),    # the headline group and cutoff (0.297 rad) at a smaller N
    ("C2", 120000, 20, 31, 250),  # the widest chart-grid cutoff of the GPU tests (0.428 rad)
    ("I", 40000, 4, 7, 120),      # the spacing pass's neighbourhood of 4 mean radii
    ("O", 4000, 20, 41, 250),     # a wide cutoff (0.581 rad) on the chart grid
    ("D3", 60000, 20, 31, 200),
])
def test_c_oracle_near_rows_match_dense(ops32, group, count, delta, seed, random_count):
    gid = GROUPS.index(group)
    ops = ops32[group]
    q = qvm.fold(qvm.haar(count, seed), gid, ops, f32=True).astype(np.float64)
    r = qvm.near_radius(count, len(ops), delta)[0]
    assert r < 0.9  # the C oracle's chart grid, not a dense fallback
    sources = picked_sources(q, ops, random_count, 60)
    compare_rows(cref.near_rows(q, ops, delta, sources=sources),
                 qvm.near_rows(q, ops, delta, sources=sources, block=64))


@pytest.mark.parametrize("group,count", [("O", 3000), ("I", 1200), ("C6", 2000)])
def test_c_oracle_pair_rows_match_dense(ops32, group, count):
    gid = GROUPS.index(group)
    ops = ops32[group]
    q = qvm.fold(qvm.haar(count, 5), gid, ops, f32=True).astype(np.float64)
    sources = picked_sources(q, ops, 150, 50)
    compare_rows(cref.pair_rows(q, ops, sources=sources), qvm.pair_rows(q, ops, sources=sources, block=32))


def test_source_subsets_are_rows_of_the_whole(ops32):
    """A source list gives the same rows as a whole pass, in the list's order."""
    ops = ops32["O"]
    q = qvm.fold(qvm.haar(2500, 3), 9, ops, f32=True).astype(np.float64)
    pick = np.array([2499, 0, 1234, 7])
    whole, part = cref.near_rows(q, ops, 20), cref.near_rows(q, ops, 20, sources=pick)
    for key in ("force", "curvature", "energy", "nearest", "nearest_source"):
        assert np.array_equal(whole[key][pick], part[key])
    small, pick = q[:600], pick % 600
    dense, dense_all = qvm.near_rows(small, ops, 20, sources=pick), qvm.near_rows(small, ops, 20)
    for key in ("curvature", "energy", "nearest", "nearest_source"):
        np.testing.assert_allclose(dense_all[key][pick], dense[key], rtol=1e-13)
