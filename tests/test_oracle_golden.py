"""The oracle pinned against the reference's own dense models (tests/golden/golden.npz,
made by tests/golden/make_golden.py from tests/test_pair_kernels.py:reference,
tests/test_measures.py:expected_measures and tests/test_near_field.py:near_reference)."""
import math

import numpy as np
import pytest

from conftest import GROUPS
from oracle import qvm

# Reference row columns (tests/test_pair_kernels.py:27-69).
COLUMNS = {0: "riesz1", 1: "riesz2", 2: "riesz3", 3: "log", 4: "green", 5: "energy", 6: "nearest", 11: "curvature"}


@pytest.mark.parametrize("group", GROUPS)
def test_rows_match_reference_model(group, golden, ops32):
    rows = qvm.pair_rows(golden["rows_q"], ops32[group], full=True)
    expected = golden[f"rows_{group}"]
    for col, key in COLUMNS.items():
        np.testing.assert_allclose(rows[key], expected[:, col], rtol=1e-11, atol=1e-11, err_msg=f"{group} {key}")
    np.testing.assert_allclose(rows["force"], expected[:, 8:11], rtol=1e-10, atol=1e-11)


def test_rows_antipodal_invariance(golden, ops32):
    signed = qvm.pair_rows(golden["rows_signed_q"], ops32["O"], full=True)
    expected = golden["rows_signed_O"]
    np.testing.assert_allclose(signed["energy"], expected[:, 5], rtol=1e-11)
    plain = qvm.pair_rows(golden["rows_q"], ops32["O"], full=True)
    np.testing.assert_allclose(signed["energy"], plain["energy"], rtol=1e-11)
    np.testing.assert_allclose(signed["log"], plain["log"], rtol=1e-11)


@pytest.mark.parametrize("group", GROUPS)
def test_measures_match_reference_model(group, golden, ops32):
    keys = [str(k) for k in golden["measures_keys"]]
    got = qvm.full_measures(qvm.pair_rows(golden["measures_q"], ops32[group], full=True), len(ops32[group]))
    for key, value in zip(keys, golden[f"measures_{group}"]):
        assert got[key] == pytest.approx(value, rel=1e-10, abs=1e-12), key


def test_near_pair_measures(golden, ops32):
    keys = [str(k) for k in golden["measures_keys"]]
    got = qvm.full_measures(qvm.pair_rows(golden["near_pair_q"], ops32["C2"], full=True), 2)
    for key, value in zip(keys, golden["near_pair_measures"]):
        assert got[key] == pytest.approx(value, rel=1e-9), key


def test_mean_radius(golden):
    for count, value in zip(golden["radius_counts"], golden["radius_values"]):
        assert qvm.mean_radius(int(count)) == value


@pytest.mark.parametrize("group", ["O", "D6", "C2", "I"])
def test_near_field_matches_reference_model(group, golden, ops32):
    q = golden[f"near_{group}_q"]
    energy, separation, delta = golden[f"near_{group}"]
    rows = qvm.near_rows(q, ops32[group], delta)
    n, order = len(q), len(ops32[group])
    assert rows["energy"].sum() / (n * order * (n - 1)) == pytest.approx(energy, rel=1e-12)
    assert qvm.separation_deg(rows["nearest"].min()) == pytest.approx(separation, rel=1e-12)


def test_haar_hash_known_answers():
    # Independent integer restatement of the shader's hash (shaders/haar.wgsl:3).
    def h(v):
        x = v & 0xFFFFFFFF
        x ^= x >> 16
        x = (x * 0x7FEB352D) & 0xFFFFFFFF
        x ^= x >> 15
        x = (x * 0x846CA68B) & 0xFFFFFFFF
        return x ^ (x >> 16)

    values = np.array([0, 1, 193, 0xFFFFFFFF, 123456789], dtype=np.uint64)
    assert [int(v) for v in qvm.hash32(values)] == [h(int(v)) for v in values]
    q = qvm.haar(1000, 193).astype(np.float64)
    np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1.0, atol=2e-7)
    # Uniform on S3: the mean of w^2 is 1/4.
    assert abs((q[:, 0] ** 2).mean() - 0.25) < 0.02


@pytest.mark.parametrize("group", GROUPS)
def test_fold_lands_in_zone(group, ops32):
    gid = GROUPS.index(group)
    q = qvm.haar(500, 11)
    folded = qvm.fold(q, gid, ops32[group], f32=False)
    assert qvm.in_zone(folded, gid, ops32[group]).all()
    # A fold changes only the orbit representative: some image of the input equals it.
    images = qvm.normalize(qvm.qmul(qvm.normalize(q.astype(np.float64))[None], ops32[group][:, None]))
    chord = np.minimum(np.linalg.norm(folded[None] - images, axis=-1), np.linalg.norm(folded[None] + images, axis=-1))
    assert chord.min(0).max() < 1e-12


def test_relax_descends(ops32):
    q = qvm.fold(qvm.haar(120, 5), 9, ops32["O"], f32=False)
    relax = qvm.Relax(q, 9, ops32["O"])
    start = qvm.quick_measures(qvm.pair_rows(relax.q, ops32["O"]), 24)["quey_energy"]
    relax.run(3)
    end = qvm.quick_measures(qvm.pair_rows(relax.q, ops32["O"]), 24)["quey_energy"]
    assert end <= start + 1e-12
    np.testing.assert_allclose(np.linalg.norm(relax.q, axis=1), 1.0, atol=1e-14)
    assert relax.iteration == 3


def test_exact_median():
    v = np.array([3.0, -1.0, 2.0, 5.0])
    assert qvm.exact_median(v) == 2.5  # -1 counts as 0: sorted 0, 2, 3, 5
    assert qvm.exact_median(np.array([4.0, 1.0, 7.0])) == 4.0
    assert qvm.exact_median(np.array([-2.0, -3.0])) == 1e-12
