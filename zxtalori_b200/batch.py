"""Many samples relaxed side by side on one GPU.

Each sample is an engine with its own CUDA stream and resident state; in FP32 mode a step
replays the sample's captured CUDA graph. `relax_batch` enqueues every sample's steps
before waiting for any, so samples of uneven sizes and different groups run concurrently,
then closes each with its force pass and readback (zo_batch_relax).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .api import Grid, haar


@dataclass
class Sample:
    group: str
    count: int
    seed: int
    neighbourhood: float = 20.0


def neighbours(count, order, neighbourhood):
    """Orbit points a source feels (the reference's count, src/engine.zig:905-907)."""
    return min(count * order, 0.94 * neighbourhood ** 3 + 64) if neighbourhood > 0 else count * order


def pair_evals(count, order, neighbourhood, steps):
    """Pair evaluations of `steps` BB steps plus the closing force pass."""
    return (steps + 1) * count * neighbours(count, order, neighbourhood)


def make_grids(samples, precision="fp32"):
    grids = []
    try:
        for s in samples:
            g = haar(s.group, s.count, s.seed, precision=precision)
            grids.append(g)
            g._check(g._lib.zo_relax_neighbourhood(g._handle, float(s.neighbourhood)))
    except BaseException:
        for g in grids:
            g.close()
        raise
    return grids


def relax_batch(grids, steps):
    """Relax every grid by `steps` BB steps side by side; raises if any failed."""
    if not grids:
        return []
    lib = grids[0]._lib
    handles = (C.c_void_p * len(grids))(*[g._handle for g in grids])
    status = (C.c_int32 * len(grids))()
    lib.zo_batch_relax(handles, len(grids), int(steps), status)
    errors = [g._lib.zo_error(g._handle).decode(errors="replace") for g, s in zip(grids, status) if s != 0]
    if errors:
        raise RuntimeError("; ".join(errors))
    for g in grids:
        g.history.append(g.stats)
    return [g.stats for g in grids]


def random_samples(count, seed=0, groups=("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I"),
                   n_min=1000, n_max=200_000, neighbourhood=20.0):
    """Batched workload: groups uniform, N log-uniform in [n_min, n_max], seeds 0..count-1."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        out.append(Sample(str(rng.choice(groups)), n, k, neighbourhood))
    return out


__all__ = ["Sample", "make_grids", "relax_batch", "random_samples", "pair_evals", "neighbours", "Grid"]
