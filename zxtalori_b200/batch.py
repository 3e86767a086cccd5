"""Many samples relaxed together on one GPU, and split over GPUs.

Each sample is an engine with its own CUDA stream and resident state. `relax_batch` runs
zo_batch_relax: every step of the batch is one CUDA graph over all its FP32 samples, whose
near-field gathers run in one persistent launch per tile variant, then each sample closes
with its force pass and readback. `shard` splits a batch over ranks (one process per GPU).
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


def shard(samples, rank, world, steps=50):
    """This rank's share of `samples` when `world` GPUs relax a batch together (one process
    per GPU, no collective: samples are independent). Samples go, largest first by pair
    evaluations, to the rank with the least work so far (ties to the lower rank), so every
    rank computes the same split and the ranks finish close together. Returns the rank's
    samples in their original order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    order = {"C2": 2, "C3": 3, "C4": 4, "C6": 6, "D2": 4, "D3": 6, "D4": 8, "D6": 12, "T": 12, "O": 24, "I": 60}
    work = [pair_evals(s.count, order[s.group], s.neighbourhood, steps) for s in samples]
    load = [0.0] * world
    owner = [0] * len(samples)
    for k in sorted(range(len(samples)), key=lambda k: (-work[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[k] = r
        load[r] += work[k]
    return [s for s, o in zip(samples, owner) if o == rank]


def random_samples(count, seed=0, groups=("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I"),
                   n_min=1000, n_max=200_000, neighbourhood=20.0):
    """Batched workload: groups uniform, N log-uniform in [n_min, n_max], seeds 0..count-1."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        out.append(Sample(str(rng.choice(groups)), n, k, neighbourhood))
    return out


__all__ = ["Sample", "make_grids", "relax_batch", "random_samples", "shard", "pair_evals", "neighbours", "Grid"]
