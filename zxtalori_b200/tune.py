"""The near-field tile tuner: picks the FP32 gather's tile shape per group and sample size.

For each group and size bucket (N from 2^b to 2^(b+1)), a Haar sample of the bucket's
middle size is relaxed with every candidate tile shape - sources per warp (2, 4, 8) times
target shell sites per chart cell (1 to 3); the spacing pass also one source per
thread - and the device time of its BB steps is
taken with CUDA events (zo_bench: L2 flushed before each step). The fastest shape is
written to the tile table, which every engine reads when it sizes a near-field workspace
(zo_tiles_lookup shows its choice). Sizes whose cutoff takes the dense path (every image
tested, no tiles) are skipped. The spacing pass (nearest neighbour only, neighbourhood 4)
is tuned the same way for the groups asked, with zo_bench_spacing, and then, with its
fastest shape, the fraction of the cutoff that its first FP32 walk covers (WALKS): a
shorter walk tests fewer sites but leaves more sources to the exact FP64 search.

    python -m zxtalori_b200.tune [--out near_tiles.txt] [--groups O I ...] [--spacing-groups I]

The reference's own tiling is fixed at compile time (src/pairs.zig:100-128,
src/near.zig:22-29); here a measured table replaces those constants.
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import time
from pathlib import Path

import numpy as np

from .api import GROUPS, haar

ORDER = {"C2": 2, "C3": 3, "C4": 4, "C6": 6, "D2": 4, "D3": 6, "D4": 8, "D6": 12, "T": 12, "O": 24, "I": 60}
CELLS = (1.0, 1.25, 1.5, 2.0, 3.0)  # target shell sites per chart cell
SHAPES = [(g, spc) for g in (2, 4, 8) for spc in CELLS]
# The spacing pass may also search one source per thread (tile shape 1).
SPACING_SHAPES = SHAPES + [(1, spc) for spc in CELLS]
WALKS = (0.45, 0.5, 0.55, 0.625, 0.75)
DEFAULT_WALK = 0.625
DEFAULT_TABLE = Path(__file__).resolve().parent / "near_tiles.txt"
FLUSH_BYTES = 256 << 20


def mean_radius(count):
    """d_r of `count` orbit points (the engine's bisection, src/pairs.zig:205-215)."""
    target = math.pi * math.pi / count
    lo, hi = 0.0, math.pi
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if math.pi * (mid - math.sin(mid)) < target:
            lo = mid
        else:
            hi = mid
    return 0.25 * (lo + hi)


def takes_grid(group, n, delta=20.0):
    """Whether an FP32 near-field pass of this size uses the chart grid (and so the tiles):
    cutoffs below 0.5 rad, or below 0.9 rad for samples of more than 1e8 image pairs."""
    r = min(1.5, delta * mean_radius(n * ORDER[group]))
    return r < 0.5 or (r < 0.9 and n * n * ORDER[group] > 1e8)


def _relax_step_ms(grid, shape, steps, warmup):
    lib, h = grid._lib, grid._handle
    grid._check(lib.zo_near_tiles(h, shape[0], shape[1]))
    out = np.zeros(4 + steps)
    grid._check(lib.zo_bench(h, steps, warmup, float(FLUSH_BYTES), out.ctypes.data_as(C.POINTER(C.c_double)),
                             len(out)))
    return float(np.median(out[4:4 + steps]))


def _spacing_ms(grid, shape, passes, warmup, walk=0.0):
    lib, h = grid._lib, grid._handle
    grid._check(lib.zo_near_tiles(h, shape[0], shape[1]))
    grid._check(lib.zo_near_walk(h, walk))
    out = np.zeros(6)
    grid._check(lib.zo_bench_spacing(h, passes, warmup, float(FLUSH_BYTES), out.ctypes.data_as(C.POINTER(C.c_double)),
                                     len(out)))
    return float(out[0])


def tune(groups=GROUPS, buckets=range(10, 19), spacing_groups=("I",), spacing_buckets=range(15, 24), steps=4,
         warmup=2, log=print):
    """Times every shape per (kind, group, bucket); returns {(kind, group, bucket): (best, {shape: ms})}."""
    found = {}
    for group in groups:
        for b in buckets:
            n = int(round(2 ** (b + 0.5)))
            if not takes_grid(group, n):
                continue
            with haar(group, n, 1000 + b) as grid:
                grid.relax(0, neighbourhood=20)
                times = {shape: _relax_step_ms(grid, shape, steps, warmup) for shape in SHAPES}
            best = min(times, key=times.get)
            found[("relax", group, b)] = (best, times)
            log(f"relax {group} {b} n={n}: best {best} {times[best]:.3f} ms (default {times[(4, 2.0)]:.3f} ms)")
    for group in spacing_groups:
        for b in spacing_buckets:
            n = int(round(2 ** (b + 0.5)))
            if n > 10_000_000 or n <= 20_000:
                continue
            with haar(group, n, 2000 + b) as grid:
                times = {shape: _spacing_ms(grid, shape, steps, warmup) for shape in SPACING_SHAPES}
                shape = min(times, key=times.get)
                walks = {w: _spacing_ms(grid, shape, steps, warmup, w) for w in WALKS}
            walk = min(walks, key=walks.get)
            best = shape + (walk,)
            times[best] = walks[walk]
            found[("spacing", group, b)] = (best, times)
            log(f"spacing {group} {b} n={n}: best {best} {times[best]:.3f} ms (default {times[(4, 2.0)]:.3f} ms, "
                f"walk {DEFAULT_WALK} {walks[DEFAULT_WALK]:.3f} ms)")
    return found


def write_table(found, path=DEFAULT_TABLE, device=""):
    lines = ["# FP32 near-field gather tile table, written by python -m zxtalori_b200.tune",
             f"# measured {time.strftime('%Y-%m-%d')} on {device or 'one GPU'}; device ms per BB step (relax) or",
             "# per spacing pass, L2 flushed; columns: kind group log2-size-bucket sources-per-warp sites-per-cell",
             "# (spacing lines: then the first walk's fraction of the cutoff), then the best time and the",
             "# default shape's (4 sources per warp, 2 sites per cell, walk 0.625)"]
    for (kind, group, b), (best, times) in sorted(found.items(), key=lambda kv: (kv[0][0], GROUPS.index(kv[0][1]),
                                                                                  kv[0][2])):
        walk = f" {best[2]:g}" if len(best) > 2 else ""
        lines.append(f"{kind} {group} {b} {best[0]} {best[1]:g}{walk}  # {times[best]:.4f} ms, default "
                     f"{times[(4, 2.0)]:.4f} ms")
    Path(path).write_text("\n".join(lines) + "\n")
    return path


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(DEFAULT_TABLE))
    p.add_argument("--groups", nargs="*", default=list(GROUPS))
    p.add_argument("--spacing-groups", nargs="*", default=["I"])
    p.add_argument("--buckets", nargs=2, type=int, default=[10, 18], help="first and last log2 size bucket")
    p.add_argument("--steps", type=int, default=4)
    args = p.parse_args(argv)
    t = time.perf_counter()
    found = tune(args.groups, range(args.buckets[0], args.buckets[1] + 1), args.spacing_groups, steps=args.steps)
    with haar("O", 64, 1) as g:
        device = g.stats["adapter"]
    write_table(found, args.out, device)
    print(f"wrote {args.out} ({len(found)} entries) in {time.perf_counter() - t:.0f} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
