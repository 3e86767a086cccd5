"""All-pairs rows, full measures, sampler and fold on the GPU against the oracle.

Mirrors the reference's tests/test_pair_kernels.py and tests/test_measures.py: every group,
random inputs from the same recipes, antipodal invariance, duplicates, singletons, a pair
5e-5 rad apart, import scale invariance. The oracle runs on the engine's own state (its
float32 positions in FP32 mode; the FP64 fold of the same float32 input in FP64 mode).

Tolerances (relative unless stated). FP64 mode: 1e-10 rows, 1e-8 measures. FP32 mode
(FP32 pair arithmetic, FP64 sums): rows 5e-6 force (relative to the largest), 2e-6
curvature and energy, 2e-6 nearest chord; measures 2e-6, Green and log ratios 5e-5
(they are small remainders of large sums).
"""
import math

import numpy as np
import pytest

from conftest import GROUPS
from oracle import qvm

pytestmark = pytest.mark.gpu

TOL = {
    "fp32": {"force": 5e-6, "curv": 2e-6, "energy": 2e-6, "nearest": 2e-6, "riesz": 2e-6, "green": 2e-6, "log": 1e-11},
    "fp64": {"force": 1e-10, "curv": 1e-10, "energy": 1e-10, "nearest": 1e-10, "riesz": 1e-10, "green": 1e-10,
             "log": 1e-11},
}


def engine_state(grid, q_in, group, precision, ops32, ops64):
    """The positions the engine holds and the table it uses, as FP64 arrays."""
    gid = GROUPS.index(group)
    if precision == "fp32":
        return grid.quaternions.astype(np.float64), ops32[group]
    return qvm.fold(np.asarray(q_in, np.float32), gid, ops64[group], f32=False), ops64[group]


def rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group", GROUPS)
def test_force_and_full_rows(engine, golden, ops32, ops64, group, precision):
    q_in = golden["rows_q"]
    with engine.from_quaternions(q_in, group, precision=precision) as grid:
        q, ops = engine_state(grid, q_in, group, precision, ops32, ops64)
        rows = grid.debug_rows(0)
        full = grid.debug_rows(1)
    o = qvm.pair_rows(q, ops, full=True)
    t = TOL[precision]
    scale = np.linalg.norm(o["force"], axis=1).max()
    for r in (rows, full):
        assert np.linalg.norm(r[:, :3] - o["force"], axis=1).max() / scale < t["force"]
        assert rel(r[:, 3], o["curvature"]) < t["curv"]
        assert rel(r[:, 4], o["energy"]) < t["energy"]
        assert rel(r[:, 5], o["nearest"]) < t["nearest"]
    n = len(q)
    assert np.array_equal(rows[:, 6].astype(np.int64) % n, o["nearest_source"])
    assert rel(full[:, 6] + 0.5, o["riesz1"]) < t["riesz"]
    assert rel(full[:, 7] + 0.25, o["riesz2"]) < t["riesz"]
    assert rel(full[:, 8] + 0.125, o["riesz3"]) < t["riesz"]
    green = full[:, 9] - 3 / (8 * math.pi ** 2)
    assert np.abs(green - o["green"]).max() < t["green"] * np.abs(o["green"]).max()
    assert np.abs(full[:, 10] + 0.25 - math.log(2) - o["log"]).max() < t["log"] * len(q) * len(ops)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_measures_all_groups(engine, golden, ops32, ops64, precision):
    q_in = golden["measures_q"]
    keys = ("riesz_1", "riesz_2", "riesz_3", "green_ratio", "log_ratio", "quey_energy", "separation_deg", "force_rms")
    with engine.from_quaternions(q_in, "C2", precision=precision) as grid:
        for group in GROUPS:
            grid.set(q_in, group)
            got = grid.measure()
            q, ops = engine_state(grid, q_in, group, precision, ops32, ops64)
            expected = qvm.full_measures(qvm.pair_rows(q, ops, full=True), len(ops))
            for key in keys:
                tol = 1e-8 if precision == "fp64" else (5e-5 if key in ("green_ratio", "log_ratio") else 2e-6)
                assert got[key] == pytest.approx(expected[key], rel=tol), (group, key)
            # The reference's own model on its own inputs, at its tolerance (test_measures.py:228).
            ref = dict(zip([str(k) for k in golden["measures_keys"]], golden[f"measures_{group}"]))
            for key in keys:
                assert got[key] == pytest.approx(ref[key], rel=4e-4, abs=4e-4), (group, key)
            assert got["energy_ratios_current"] is True
            # Antipodal representatives change nothing (test_measures.py:229-233).
            signed = grid.quaternions.copy()
            signed[::2] *= -1
            grid.set(signed, group)
            again = grid.measure()
            for key in keys:
                assert again[key] == pytest.approx(got[key], rel=1e-5, abs=1e-9), (group, key)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_haar_and_fold_bit_exact(engine, ops32, ops64, precision):
    for group in ("C2", "D3", "T", "O", "I"):
        gid = GROUPS.index(group)
        ops = ops32[group] if precision == "fp32" else ops64[group]
        with engine.haar(group, 4000, 17, precision=precision) as grid:
            q = grid.quaternions
        expected = qvm.fold(qvm.haar(4000, 17), gid, ops, f32=False).astype(np.float32)
        assert np.array_equal(q, expected), group
        assert qvm.in_zone(q.astype(np.float64), gid, ops).mean() > 0.999


def test_duplicates_rejected(engine):
    with engine.from_quaternions(np.array([[1, 0, 0, 0], [1, 0, 0, 0]], np.float32), "C2") as grid:
        with pytest.raises(RuntimeError, match="Measure failed: DuplicateOrientations"):
            grid.measure()
        rows = grid.debug_rows(0)
        assert (rows[:, 5] == 0).all() and np.isfinite(rows[:, :5]).all()


def test_singleton_force_zero(engine, golden):
    with engine.from_quaternions(golden["rows_q"][:1], "C2") as grid:
        rows = grid.debug_rows(0)
        assert (rows[:, :3] == 0).all()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_near_pair_resolved(engine, golden, ops32, precision):
    pair = golden["near_pair_q"]
    with engine.from_quaternions(pair, "C2", precision=precision) as grid:
        got = grid.measure()
        q = grid.quaternions.astype(np.float64)
    expected = qvm.full_measures(qvm.pair_rows(q, ops32["C2"], full=True), 2)
    assert got["separation_deg"] > 0
    assert got["separation_deg"] == pytest.approx(expected["separation_deg"], rel=1e-5)


def test_import_scale_invariance(engine):
    q = np.random.default_rng(198).normal(size=(29, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    with engine.from_quaternions(q, "I") as grid:
        expected = grid.quaternions
        grid.set(q * np.geomspace(1e-8, 3e38, len(q))[:, None])
        actual = grid.quaternions
        assert np.isfinite(actual).all()
        np.testing.assert_allclose(actual, expected, rtol=0, atol=4e-7)
        np.testing.assert_allclose(np.linalg.norm(actual, axis=1), 1, rtol=0, atol=3e-7)
        extreme = np.array([[1, 1, 1, 1], [1, .1, .3, .4]], np.float32)
        grid.set(extreme, "C2")
        expected = grid.quaternions
        grid.set(extreme * np.float32(3e38), "C2")
        np.testing.assert_allclose(grid.quaternions, expected, rtol=0, atol=4e-7)


def test_import_errors(engine):
    with engine.from_quaternions(np.eye(4, dtype=np.float32), "O") as grid:
        with pytest.raises(RuntimeError, match="Import failed: NonFiniteQuaternion"):
            grid.set(np.array([[1, np.nan, 0, 0]], np.float32))
        with pytest.raises(RuntimeError, match="Import failed: ZeroQuaternion"):
            grid.set(np.zeros((1, 4), np.float32))
        with pytest.raises(RuntimeError, match="Spacing failed: TooFewOrientations"):
            grid.set(np.eye(4, dtype=np.float32)[:1])
            grid.spacing()


@pytest.mark.parametrize("group,count", [("T", 700), ("O", 1000), ("D4", 400)])
def test_chunked_sums_match(engine, group, count):
    """Splitting the all-pairs work over more chunks changes only rounding (test_pair_chunks.py)."""
    def run(scale):
        with engine.haar(group, count, 5) as grid:
            grid._lib.zo_pair_budget(grid._handle, scale)
            m = dict(grid.measure())
            grid.relax(1)
            return m, grid.quaternions

    whole, moved_whole = run(1.0)
    chunked, moved_chunked = run(1e-5)
    for key in ("quey_energy", "riesz_1", "riesz_2", "riesz_3", "green_ratio", "log_ratio", "separation_deg"):
        assert chunked[key] == pytest.approx(whole[key], rel=2e-5, abs=2e-6), key
    assert np.max(np.abs(moved_chunked - moved_whole)) < 2e-5


def _turn(q, axis, h):
    """Left rotation by angle h about a coordinate axis (tests/test_pair_kernels.py:151-153)."""
    d = np.zeros(4)
    d[0], d[axis + 1] = math.cos(h), math.sin(h)
    return qvm.qmul(d, q)


@pytest.mark.parametrize("precision,rtol", [("fp64", 2e-6), ("fp32", 1e-5)])
def test_force_is_half_energy_gradient(engine, golden, precision, rtol):
    """Force sign, left-tangent frame and factor of two against finite differences
    (tests/test_pair_kernels.py:147-159): turning source 0 by +-h (h = 1e-6) about each axis,
    d(sum E)/d(theta) = -2 F_0. The engine's force is taken at its own positions; the energy
    sums come from the FP64 oracle at the same positions turned (a float32 import would round
    away the 1e-6 turn)."""
    base = golden["rows_q"][:9].astype(np.float64)
    base /= np.linalg.norm(base, axis=-1, keepdims=True)
    ops = golden["ops_C2"].astype(np.float64) if precision == "fp64" else \
        golden["ops_C2"].astype(np.float32).astype(np.float64)
    with engine.from_quaternions(base.astype(np.float32), "C2", precision=precision) as grid:
        q = grid.quaternions.astype(np.float64)
        force = grid.debug_rows(0)[:, :3]
    if precision == "fp64":  # the engine's FP64 state: the FP64 fold of the float32 input
        q = qvm.fold(base.astype(np.float32), GROUPS.index("C2"), ops, f32=False)
    h = 1e-6
    for axis in range(3):
        energy = []
        for sign in (1, -1):
            moved = q.copy()
            moved[0] = _turn(q[0], axis, sign * h)
            energy.append(qvm.pair_rows(moved, ops)["energy"].sum())
        derivative = (energy[0] - energy[1]) / (2 * h)
        assert abs(derivative + 2 * force[0, axis]) <= rtol * max(1.0, abs(derivative)), (axis, derivative, force[0])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("group,source", [("O", "random"), ("I", "random"), ("T", "hopf"), ("O", "hopf")])
def test_log_ratio_against_dense_fp64(engine, ops32, ops64, group, source, precision):
    """tests/test_log_scale.py of the reference: the log ratio of about a thousand points
    within 1e-5 (absolute) of the dense FP64 value, for random points and generated grids
    (the reference also uses its FCC transports, which this engine does not build)."""
    gid = GROUPS.index(group)
    if source == "random":
        q = np.random.default_rng(936).normal(size=(1000, 4))
        grid = engine.from_quaternions(q / np.linalg.norm(q, axis=1, keepdims=True), group, precision=precision)
    else:
        grid = engine.generate(group, count=1000, precision=precision)
    with grid:
        actual = grid.measure()["log_ratio"]
        q = grid.quaternions.astype(np.float64)
    ops = ops32[group] if precision == "fp32" else ops64[group]
    expected = qvm.full_measures(qvm.pair_rows(q, ops, full=True), len(ops))["log_ratio"]
    assert abs(actual - expected) < 1e-5
