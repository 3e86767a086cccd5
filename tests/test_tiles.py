"""The near-field tile table (no GPU): its file format, the nearest-bucket rule and the
defaults, through zo_tiles_lookup in a fresh process (the table is read once per process)."""
import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

LOOKUP = textwrap.dedent('''
    import ctypes as C, json, sys
    lib = C.CDLL(sys.argv[1])
    lib.zo_tiles_lookup.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]
    out, got = (C.c_double * 3)(), []
    for kind, group, n in json.loads(sys.argv[2]):
        rc = lib.zo_tiles_lookup(kind, group, n, out)
        got.append([rc, out[0], out[1], out[2]])
    print(json.dumps(got))
''')


def lookups(table_text, queries, tmp_path):
    table = tmp_path / "tiles.txt"
    table.write_text(table_text)
    lib = ROOT / "zxtalori_b200" / "_lib" / "libzxtalori.so"
    env = dict(os.environ, ZXTALORI_TILES=str(table))
    done = subprocess.run([sys.executable, "-c", LOOKUP, str(lib), json.dumps(queries)], env=env,
                          capture_output=True, text=True, timeout=120, check=True)
    return json.loads(done.stdout)


def test_tile_table_lookup(tmp_path):
    text = ("# kind group bucket sources_per_warp sites_per_cell [walk]\n"
            "relax O 16 4 2.0\n"
            "relax O 12 2 1.5\n"
            "relax I 14 8 3\n"
            "spacing I 20 4 1.5\n"
            "spacing I 22 1 1.5 0.5\n"
            "spacing I 23 1 1.5 0.1\n"  # walk below the accepted range: ignored
            "relax O 13 5 2.0\n"        # invalid shape: ignored
            "nonsense line\n")
    O, I, C2 = 9, 10, 0
    W = 0.625  # the default first-walk fraction
    got = lookups(text, [[0, O, 70_000], [0, O, 1 << 12], [0, O, 9000], [0, O, 3000], [0, O, 10_000_000],
                         [0, I, 5], [1, I, 1 << 20], [1, O, 1 << 20], [0, C2, 50_000], [2, O, 1000],
                         [1, I, 5_000_000], [1, I, 10_000_000]], tmp_path)
    assert got[0] == [0, 4, 2.0, W]         # bucket 16 exactly
    assert got[1] == [0, 2, 1.5, W]         # bucket 12 exactly
    assert got[2] == [0, 2, 1.5, W]         # bucket 13 (invalid line ignored): nearest 12
    assert got[3] == [0, 2, 1.5, W]         # bucket 11: nearest 12
    assert got[4] == [0, 4, 2.0, W]         # bucket 23: nearest 16
    assert got[5] == [0, 8, 3.0, W]         # the group's only entry
    assert got[6] == [0, 4, 1.5, W]         # the spacing kind has its own entries
    assert got[7] == [0, 4, 2.0, W]         # no spacing entry for O: the defaults
    assert got[8] == [0, 4, 2.0, W]         # no entry for C2: the defaults
    assert got[9][0] == -1                  # unknown kind
    assert got[10] == [0, 1, 1.5, 0.5]      # bucket 22, with its walk
    assert got[11] == [0, 1, 1.5, 0.5]      # bucket 23's line is ignored: nearest 22


def test_missing_table_gives_defaults(tmp_path):
    lib = ROOT / "zxtalori_b200" / "_lib" / "libzxtalori.so"
    env = dict(os.environ, ZXTALORI_TILES=str(tmp_path / "absent.txt"))
    done = subprocess.run([sys.executable, "-c", LOOKUP, str(lib), json.dumps([[0, 9, 100_000]])], env=env,
                          capture_output=True, text=True, timeout=120, check=True)
    assert json.loads(done.stdout) == [[0, 4, 2.0, 0.625]]
