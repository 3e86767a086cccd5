"""The covering-radius oracle (oracle/covering.py: Qhull over the full orbit, the reference's
own test oracle, tests/test_covering.py:8-15) against the reference's published covering
radii (tests/fixtures/covering-reference.json, copied with its grids by
tests/golden/make_covering.py), and the simplex bound against its series."""
import math

import numpy as np
import pytest

from conftest import ROOT
from oracle import covering as cov

COVERING = ROOT / "tests" / "golden" / "covering.npz"
HOPF = ROOT / "tests" / "golden" / "hopf.npz"
PUBLISHED = ("C2", "C3", "C4", "D2", "D3", "D4", "D6", "T", "O", "I")


def published_grid(group):
    with np.load(COVERING) as data, np.load(HOPF) as hopf:
        rows = hopf[str(data[f"{group}_grid"])] if f"{group}_grid" in data.files else data[f"{group}_rows"]
        return np.asarray(rows, np.float64), float(data[f"{group}_radius_deg"])


@pytest.mark.parametrize("group", PUBLISHED)
def test_oracle_matches_published_radii(group, ops64):
    rows, radius = published_grid(group)
    result = cov.covering(rows, ops64[group])
    assert abs(result["radius_deg"] - radius) < 1e-5
    assert result["point_covering"].max() == pytest.approx(result["radius_deg"], abs=1e-9)


def test_simplex_bound_series():
    coefficients = cov.SIMPLEX_SERIES
    for count in (8, 400, 48_000, 2_400_000):
        direct = sum(c * count ** (-(2 * i + 1) / 3) for i, c in enumerate(coefficients)) * 360 / math.pi
        assert cov.simplex_degrees(count) == pytest.approx(direct, rel=1e-13)
    assert cov.simplex_degrees(0) is None


def test_point_values_follow_their_definition(ops64):
    """Per point: the largest cap of any facet touching an image of the point, and its
    identity image's distinct hull neighbours; the witness is the largest cap's centre, as
    far from every orbit point as the radius says."""
    rng = np.random.default_rng(3)
    q = rng.normal(size=(40, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    result = cov.covering(q, ops64["D3"])
    points, _ = cov.orbit(q, ops64["D3"])
    nearest = np.degrees(2 * np.arccos(np.clip((points @ result["witness"]).max(), -1, 1)))
    assert nearest == pytest.approx(result["radius_deg"], abs=1e-7)
    assert (result["faces"] >= 4).all() and result["point_covering"].max() == result["radius_deg"]
