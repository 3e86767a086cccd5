"""The reference's own, unchanged Python API (python/zxtalori/api.py) driving this library.

The reference's api.py loads its engine from $ZXTALORI_LIBRARY and binds all 28 zo_* names
eagerly with getattr (api.py:18-55); a missing name would fail there. This test runs it in
a fresh process against zxtalori_b200/_lib/libzxtalori.so: every binding must succeed, and
a Grid must either come up (on a machine with a B200) or fail with the reference's error
convention, RuntimeError carrying zo_create_error() (api.py:104-106). With a GPU it also
runs haar -> relax -> measure -> spacing -> save/load through that API.

It needs a checkout of the reference project (never part of this repository): set
ZXTALORI_REFERENCE to its root. Without it the test is skipped.
"""
import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REFERENCE = os.environ.get("ZXTALORI_REFERENCE")

SCRIPT = textwrap.dedent('''
    import json, sys, tempfile, pathlib
    sys.path.insert(0, sys.argv[1])
    import zxtalori as zo
    from zxtalori import api
    api._library()  # binds every name the reference binds
    out = {"bound": True, "module": api.__file__}
    try:
        grid = zo.haar("O", 3000, 193)
    except RuntimeError as e:
        out["create_error"] = str(e)
    else:
        with grid:
            grid.relax(20, neighbourhood=20)
            m = grid.measure()
            s = grid.spacing()
            path = grid.save(pathlib.Path(tempfile.mkdtemp()) / "sample.json")
            q = grid.quaternions
        with zo.load(path) as again:
            out["round_trip_equal"] = bool((again.quaternions == q).all())
        out.update({"energy": m["quey_energy"], "separation": s["separation_deg"], "iteration": m["iteration"],
                    "riesz_2": m["riesz_2"]})
    print(json.dumps(out))
''')


@pytest.mark.skipif(not REFERENCE or not (Path(REFERENCE or ".") / "python" / "zxtalori" / "api.py").is_file(),
                    reason="needs a reference checkout in $ZXTALORI_REFERENCE")
def test_reference_api_drives_this_library():
    lib = ROOT / "zxtalori_b200" / "_lib" / "libzxtalori.so"
    if not lib.is_file():
        pytest.fail(f"engine library missing: {lib}")
    env = dict(os.environ, ZXTALORI_LIBRARY=str(lib))
    done = subprocess.run([sys.executable, "-c", SCRIPT, str(Path(REFERENCE) / "python")], env=env,
                          capture_output=True, text=True, timeout=600)
    assert done.returncode == 0, done.stderr[-2000:]
    out = json.loads(done.stdout.strip().splitlines()[-1])
    assert out["bound"] and out["module"].startswith(str(Path(REFERENCE)))
    if "create_error" in out:  # no CUDA device here: the reference's error path
        assert out["create_error"].startswith("GPU init:")
    else:
        assert out["round_trip_equal"] and out["iteration"] == 20
        assert out["energy"] > 0 and out["separation"] > 0 and out["riesz_2"] > 0
