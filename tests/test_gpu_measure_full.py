"""measure(full=True) (zo_measure_full, an extension): every energy ratio over all pairs at
any count. Below the ratio limit it is measure() itself; above it (where the reference's
measure gives energy and separation only, src/engine.zig:308-351) the sums are taken in FP64
in both modes, so the FP32-refined engine's ratios match the FP64 method's on the same
float32 sample to 1e-5 (the two engines' FP64 positions differ by the float32 rounding)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("riesz_1", "riesz_2", "riesz_3", "green_ratio", "log_ratio", "quey_energy", "separation_deg")


def test_full_measure_below_the_ratio_limit_is_measure(engine):
    with engine.haar("I", 2000, 3) as grid:
        m = grid.measure()
        f = grid.measure(full=True)
    for k in KEYS:
        assert f[k] == m[k]
    assert f["energy_ratios_current"]


def test_full_measure_above_the_ratio_limit(engine):
    with engine.haar("I", 30_000, 7) as grid:
        assert len(grid) > grid.stats["ratio_limit"]
        m = grid.measure()
        assert m["riesz_1"] is None and not m["energy_ratios_current"]
        f = grid.measure(full=True)
        q = grid.quaternions
    assert f["energy_ratios_current"] and f["precision"] == "All measures current"
    assert f["quey_energy"] == pytest.approx(m["quey_energy"], rel=1e-6)
    assert f["separation_deg"] == pytest.approx(m["separation_deg"], rel=1e-6)
    with engine.from_quaternions(q, "I", precision="fp64") as g64:
        f64 = g64.measure(full=True)
    errors = {k: abs(f[k] - f64[k]) / abs(f64[k]) for k in KEYS}
    print(errors)
    for k in KEYS:
        assert np.isfinite(f[k]) and errors[k] < 1e-5, (k, errors)
