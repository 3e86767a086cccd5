"""The C-ABI library: built for sm_100a, exports exactly what include/zxtalori.h declares
(every name the reference's python/zxtalori/api.py binds), and loads without a GPU.
No compute runs here."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import GROUPS, ROOT

HEADER = ROOT / "include" / "zxtalori.h"
# The names python/zxtalori/api.py:29-50 binds eagerly with getattr.
REFERENCE_BOUND = [
    "zo_create", "zo_create_error", "zo_destroy", "zo_generate", "zo_random", "zo_set", "zo_count", "zo_order",
    "zo_quaternions", "zo_operations", "zo_measure", "zo_spacing", "zo_relax", "zo_relax_neighbourhood",
    "zo_point_values", "zo_identity", "zo_cover", "zo_cover_optimize", "zo_cover_kicks", "zo_mesh",
    "zo_mesh_vertices", "zo_mesh_tets", "zo_mesh_vertex_count", "zo_mesh_tet_count", "zo_generate_exact",
    "zo_stats", "zo_error", "zo_cancel",
]


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zo_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def library():
    from zxtalori_b200 import build

    path = build.build(verbose=False)
    return path


def test_header_covers_reference_bindings():
    names = declared()
    missing = [n for n in REFERENCE_BOUND if n not in names]
    assert not missing, missing


def test_library_exports_every_declared_symbol(library):
    lib = ctypes.CDLL(str(library))
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(library)], capture_output=True, text=True, check=True).stdout
    exported = sorted(line.split()[-1] for line in out.splitlines() if " T " in line)
    assert exported == declared(), "only the declared ABI is exported"


def test_build_targets_sm100a():
    from zxtalori_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_create_without_gpu_fails_cleanly(library):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = ctypes.CDLL(str(library))
    lib.zo_create.restype = ctypes.c_void_p
    lib.zo_create.argtypes = [ctypes.c_char_p]
    lib.zo_create_error.restype = ctypes.c_char_p
    assert not lib.zo_create(b"")
    assert lib.zo_create_error().startswith(b"GPU init:")


def test_group_tables_match_reference_fixture(golden):
    """groups_table.inc (generated) equals the reference's published operator tables."""
    text = (ROOT / "zxtalori_b200" / "csrc" / "groups_table.inc").read_text()
    body64 = text.split("kOps64")[1].split("};")[0]
    body32 = text.split("kOps32")[1].split("};")[0]
    rows64 = [[float.fromhex(v) for v in r.split(",")] for r in re.findall(r"\{([^{}]+)\}", body64)]
    rows32 = [[float.fromhex(v.strip().rstrip("f")) for v in r.split(",")] for r in re.findall(r"\{([^{}]+)\}", body32)]
    table64 = np.array(rows64)
    table32 = np.array(rows32)
    start = 0
    for g in GROUPS:
        ops = golden[f"ops_{g}"]
        assert np.array_equal(table64[start:start + len(ops)], ops), g
        assert np.array_equal(table32[start:start + len(ops)], ops.astype(np.float32).astype(np.float64)), g
        start += len(ops)
    assert start == len(table64) == len(table32)


def test_python_api_surface():
    import zxtalori_b200 as zo

    for name in ("GROUPS", "Grid", "generate", "from_quaternions", "load", "haar"):
        assert hasattr(zo, name)
    assert zo.GROUPS == GROUPS
    for method in ("relax", "measure", "spacing", "point_values", "quaternions", "stats", "operations", "set",
                   "identity", "save", "close", "covering", "triangulation", "optimize_covering"):
        assert hasattr(zo.Grid, method), method


def test_serve_structs_match_the_header(tmp_path):
    """The ctypes request and result records of serve.NativeServer have the C layout that
    include/zxtalori.h declares for zo_serve (sizes and every field's offset, from gcc)."""
    from zxtalori_b200.serve import _NativeRequest, _NativeResult

    records = {"zo_serve_request": _NativeRequest, "zo_serve_result": _NativeResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for c_name, record in records.items():
        lines.append(f'  printf("{c_name} size %zu\\n", sizeof({c_name}));')
        for field, _ in record._fields_:
            lines.append(f'  printf("{c_name} {field} %zu\\n", offsetof({c_name}, {field}));')
    lines += ["  return 0;", "}"]
    source = tmp_path / "layout.c"
    source.write_text("\n".join(lines) + "\n")
    binary = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(binary), str(source)], check=True)
    printed = dict(line.rsplit(" ", 1) for line in subprocess.run([str(binary)], check=True, capture_output=True,
                                                                   text=True).stdout.splitlines())
    for c_name, record in records.items():
        assert int(printed[f"{c_name} size"]) == ctypes.sizeof(record)
        for field, _ in record._fields_:
            assert int(printed[f"{c_name} {field}"]) == getattr(record, field).offset, (c_name, field)
