"""Failure paths driven from the host, and the sample file formats.

- Shell overflow: a development hook (zo_debug_shell_capacity) makes the next near-field
  workspace too small, so a pass produces more shell sites than it holds. The engine then
  sizes the workspace again and redoes the pass, as the reference does (src/pairs.zig:
  391-394 for the closing pass of a relaxation, :311 measure, :330 spacing): the results
  equal those of a run that never overflowed, bit for bit.
- Cancel: zo_cancel from another thread stops a long relaxation at the next step
  (src/engine.zig:58, 911); the call still ends with the closing pass and reports no error.
- Save and load: the "zxtalori-1" JSON and NPZ formats (python/zxtalori/api.py:336-362)
  hold the float32 quaternions exactly; loading imports them, which renormalises each one
  (src/engine.zig:282-307), so the loaded sample equals the saved one to a float32 rounding.
No GPU fault is involved in any of them.
"""
import json
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def shrink(grid, sites):
    grid._check(grid._lib.zo_debug_shell_capacity(grid._handle, sites))


def test_shell_overflow_resize_and_redo(engine):
    with engine.haar("O", 30000, 5) as a, engine.haar("O", 30000, 5) as b:
        a.relax(3, neighbourhood=20)
        b.relax(3, neighbourhood=20)
        np.testing.assert_array_equal(a.quaternions, b.quaternions)
        # The closing pass of a relaxation (zo_relax with no steps): it overflows, is sized
        # again and redone.
        a._check(a._lib.zo_relax(a._handle, 0))
        shrink(b, 1000)
        b._check(b._lib.zo_relax(b._handle, 0))
        sa, sb = a.stats, b.stats
        assert sb["energy"] == sa["energy"] and sb["separation_deg"] == sa["separation_deg"]
        np.testing.assert_array_equal(a.point_values("separation"), b.point_values("separation"))
        # A measure (N below O's ratio limit: full measures, then the near-field pass).
        ma = a.measure()
        shrink(b, 1000)
        mb = b.measure()
        for key in ("quey_energy", "separation_deg", "riesz_2", "log_ratio"):
            assert mb[key] == ma[key], key
        # The spacing pass (neighbourhood 4 above 20,000 points).
        a.spacing()
        shrink(b, 500)
        b.spacing()
        np.testing.assert_array_equal(a.point_neighbours(), b.point_neighbours())
        np.testing.assert_array_equal(a.point_values("separation"), b.point_values("separation"))
        # Steps after the redo continue on a workspace of the right size.
        a.relax(2)
        b.relax(2)
        np.testing.assert_array_equal(a.quaternions, b.quaternions)


def test_cancel_from_another_thread(engine):
    with engine.haar("O", 100_000, 193) as grid:
        grid.relax(1, neighbourhood=20)
        start = grid.stats["iteration"]
        timer = threading.Timer(0.3, lambda: grid._lib.zo_cancel(grid._handle))
        timer.start()
        try:
            grid.relax(1000)  # about 2.7 s of steps on one B200
        finally:
            timer.join()
        stopped = grid.stats["iteration"] - start
        assert 0 < stopped < 1000
        assert np.isfinite(grid.stats["energy"])
        np.testing.assert_allclose(np.linalg.norm(grid.quaternions, axis=1), 1, atol=3e-7)
        # The flag is cleared by the next call.
        grid.relax(5)
        assert grid.stats["iteration"] == start + stopped + 5


@pytest.mark.parametrize("suffix", [".json", ".npz"])
def test_save_load_round_trip(engine, tmp_path, suffix):
    with engine.haar("D6", 3000, 17) as grid:
        grid.relax(4)
        path = grid.save(tmp_path / f"sample{suffix}")
        q, stats = grid.quaternions, grid.stats
    if suffix == ".json":
        data = json.loads(path.read_text(encoding="utf-8"))
        assert data["format"] == "zxtalori-1" and data["group"] == "D6"
        assert data["metadata"]["iteration"] == 4
        np.testing.assert_array_equal(np.asarray(data["quaternions"], np.float32), q)
    else:
        with np.load(path) as data:
            np.testing.assert_array_equal(data["quaternions"], q)
            assert json.loads(str(data["metadata"]))["group"] == "D6"
    with engine.load(path) as again:
        loaded = again.quaternions.astype(np.float64)
        chord = np.minimum(np.linalg.norm(loaded - q, axis=1), np.linalg.norm(loaded + q, axis=1))
        assert chord.max() <= 1.2e-7
        assert again.stats["group"] == "D6" and again.stats["count"] == stats["count"]
        assert again.measure()["quey_energy"] == pytest.approx(stats["quey_energy"], rel=1e-6)
