"""ctypes wrapper of the C restatement (oracle/qvm_ref.c).  TEST INFRASTRUCTURE ONLY.

Same rows as oracle.qvm.pair_rows / near_rows, FP64, threaded with OpenMP. Built by
`make -C oracle` (also run by __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libqvmref.so"
_lib = None


def library():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "qvm_ref.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    lib = C.CDLL(str(LIB))
    d = C.POINTER(C.c_double)
    i64 = C.POINTER(C.c_int64)
    lib.oracle_pair_rows.argtypes = [d, C.c_int, d, C.c_int, d, d, d, d, i64, C.c_int, C.c_int, i64]
    lib.oracle_near_rows.argtypes = [d, C.c_int, d, C.c_int, C.c_double, C.c_double, d, d, d, d, i64, C.c_int,
                                     C.c_int, i64]
    lib.oracle_mean_radius.argtypes = [C.c_double]
    lib.oracle_mean_radius.restype = C.c_double
    _lib = lib
    return lib


def threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def _ptr(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _rows(kind, q, ops, delta=0.0, taper=0.5, nthreads=None, count=0, sources=None):
    lib = library()
    q = np.ascontiguousarray(q, np.float64)
    ops = np.ascontiguousarray(ops, np.float64)
    n = len(q)
    picked = None
    if sources is not None:
        picked = np.ascontiguousarray(sources, np.int64)
        if len(picked) == 0 or picked.min() < 0 or picked.max() >= n:
            raise ValueError("sources must be indices of the sample")
        count = len(picked)
    rows = count if (count and (count < n or picked is not None)) else n
    force = np.zeros((rows, 3))
    curv, energy, nearest = np.zeros(rows), np.zeros(rows), np.zeros(rows)
    src = np.zeros(rows, np.int64)
    nthreads = nthreads or threads()
    chosen = _ptr(picked, C.c_int64) if picked is not None else None
    if kind == "pairs":
        lib.oracle_pair_rows(_ptr(q), n, _ptr(ops), len(ops), _ptr(force), _ptr(curv), _ptr(energy), _ptr(nearest),
                             _ptr(src, C.c_int64), nthreads, int(count), chosen)
    else:
        lib.oracle_near_rows(_ptr(q), n, _ptr(ops), len(ops), float(delta), float(taper), _ptr(force), _ptr(curv),
                             _ptr(energy), _ptr(nearest), _ptr(src, C.c_int64), nthreads, int(count), chosen)
    return {"force": force, "curvature": curv, "energy": energy, "nearest": nearest, "nearest_source": src}


def pair_rows(q, ops, nthreads=None, count=0, sources=None):
    """All-pairs rows; with `count`, only the first `count` sources get rows; with
    `sources`, only those (rows in its order)."""
    return _rows("pairs", q, ops, nthreads=nthreads, count=count, sources=sources)


def near_rows(q, ops, delta, taper=0.5, nthreads=None, count=0, sources=None):
    """Near-field rows; q must hold zone representatives (the shell assumes it). `count`
    and `sources` as for pair_rows."""
    return _rows("near", q, ops, delta, taper, nthreads, count, sources)
