"""Inverse-Hopf product grids (src/hopf.zig) on the host, against the reference's SO3K_Grids
fixture (tests/golden/hopf.npz, copied from tests/fixtures/hopf-reference.npz by
make_hopf.py) and its count formulas (tests/test_hopf.py:24-39). No GPU."""
import numpy as np
import pytest

from conftest import GROUPS, ROOT

ROOTS = {"C2": "I", "C3": "I", "D2": "I", "D3": "I", "T": "I", "I": "I", "C4": "O", "D4": "O", "O": "O",
         "C6": "D6", "D6": "D6"}
ORDER = {"C2": 2, "C3": 3, "C4": 4, "C6": 6, "D2": 4, "D3": 6, "D4": 8, "D6": 12, "T": 12, "O": 24, "I": 60}

with np.load(ROOT / "tests" / "golden" / "hopf.npz") as _data:
    FIXTURE = {k: _data[k] for k in _data.files}
CASES = sorted((k.split("_")[0], int(k.split("_")[1])) for k in FIXTURE)


def ring(f, j):
    mult = 12 if j == f else 6
    return max(mult, mult * int(np.floor(4 * f * np.sin(np.pi * j / (2 * f)) / mult + 0.5)))


def expected_count(group, f):
    """The reference test's closed-form row count."""
    root = ROOTS[group]
    if root == "O":
        n, nodes = (4 * f if f < 6 else 4 * f - 12 * ((2 * f + 9) // 18)), 4 * f * f + 2
    elif root == "I":
        n, nodes = 5 * f, 10 * f * f + 2
    else:
        n, nodes = 6 * int(np.ceil(4 * f / 6)), 2 + ring(f, f) + 2 * sum(ring(f, j) for j in range(1, f))
    return n * nodes // ORDER[group]


def qmul(a, b):
    w1, x1, y1, z1 = np.moveaxis(a, -1, 0)
    w2, x2, y2, z2 = np.moveaxis(b, -1, 0)
    return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], -1)


def orbit_chord(actual, expected, ops):
    """Per row, the chord from the actual row to the nearest image of the expected row's
    orbit {+-e g}."""
    images = qmul(expected[None], ops[:, None])
    return np.minimum(np.linalg.norm(actual[None] - images, axis=-1),
                      np.linalg.norm(actual[None] + images, axis=-1)).min(0)


@pytest.fixture(scope="module")
def zo():
    import zxtalori_b200

    from zxtalori_b200 import build

    build.build(verbose=False)
    return zxtalori_b200


@pytest.mark.parametrize("group,f", CASES)
def test_rows_match_fixture(zo, ops64, group, f):
    actual = zo.hopf_points(group, f).astype(np.float64)
    expected = FIXTURE[f"{group}_{f}"]
    assert len(actual) == len(expected) == expected_count(group, f)
    assert np.abs(np.linalg.norm(actual, axis=1) - 1).max() < 3e-7
    # Row order is the reference's: row i is an image of the fixture's row i (to f32).
    assert orbit_chord(actual, expected, ops64[group]).max() < 1e-6


@pytest.mark.parametrize("group", GROUPS)
def test_counts(zo, group):
    lib = zo.api._library()
    gid = GROUPS.index(group)
    for f in list(range(1, 40)) + [64, 100, 281, 512]:
        n = expected_count(group, f)
        got = lib.zo_hopf_points(gid, f, None, 0)
        assert got == (n if n <= 10_000_000 else -1), (group, f)
    assert lib.zo_hopf_points(gid, 0, None, 0) == -1
    assert lib.zo_hopf_points(gid, 513, None, 0) == -1


def test_capacity_and_group_checks(zo):
    lib = zo.api._library()
    out = np.zeros((5, 4), np.float32)
    assert lib.zo_hopf_points(9, 2, out.ctypes.data, 5) == -2  # O h=2 has 6 rows
    assert lib.zo_hopf_points(11, 2, None, 0) == -1
    with pytest.raises(ValueError):
        zo.hopf_points("C2", 100)  # 25 million rows: above the count limit


def test_orbits_are_distinct(zo, ops64):
    """No orientation twice: the minimum orbit chord between rows stays well above zero."""
    for group, f in [("O", 7), ("I", 4), ("D6", 5), ("C3", 3), ("T", 4)]:
        q = zo.hopf_points(group, f).astype(np.float64)
        images = qmul(q[:, None], ops64[group][None])  # (n, |K|, 4)
        flat = images.reshape(-1, 4)
        owner = np.repeat(np.arange(len(q)), len(ops64[group]))
        d = np.minimum(np.linalg.norm(q[:, None] - flat[None], axis=-1), np.linalg.norm(q[:, None] + flat[None], axis=-1))
        d[np.arange(len(q))[:, None] == owner[None]] = np.inf
        assert d.min() > 1e-3, (group, f, d.min())
