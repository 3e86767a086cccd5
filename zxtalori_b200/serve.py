"""Continuous-batching relax + measure service on one GPU.

Requests (group, N, steps, seed, neighbourhood) arrive over time. The loop admits waiting
requests in arrival order while their device memory fits the budget, keeps each admitted
sample resident in its own engine (own CUDA stream, FP32 steps replayed from a captured
graph), and advances every active sample a chunk of steps whenever its stream is idle, so
the kernels of all active samples overlap on the device. A request whose steps are done is
handed to a worker thread for its blocking part - closing force pass, measure() (every
energy ratio below the ratio limit), positions read back, engine closed - while the loop
keeps feeding the others; its memory then goes to the next admission. Admission counts
each resident sample at the device bytes its engine reports once its workspace is sized
(an estimate before that). Results do not depend on what else is running: every sample's
kernels read only its own buffers and sum in a fixed order.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .api import GROUPS, _library, haar
from .batch import neighbours

ORDER = {"C2": 2, "C3": 3, "C4": 4, "C6": 6, "D2": 4, "D3": 6, "D4": 8, "D6": 12, "T": 12, "O": 24, "I": 60}


@dataclass
class Request:
    id: int
    group: str
    count: int
    steps: int
    seed: int
    neighbourhood: float
    arrival: float = 0.0


@dataclass
class Result:
    id: int
    arrival: float
    admitted: float
    finished: float
    stats: dict
    quaternions: np.ndarray | None = None

    @property
    def latency(self):
        return self.finished - self.arrival


def estimate_bytes(count, group, neighbourhood):
    """Device memory a request holds while resident (generous): positions, rows and BB
    history ~450 B per source; a near field adds shell sites (~80 B each, a few per
    source), partial rows of up to 64 slices and the chart grids."""
    order = ORDER[group]
    total = 450 * count + (64 << 20)
    if neighbourhood > 0:
        slices = min(64, max(1, math.ceil(148 * 48 / max(1, count / 32))))
        total += count * 80 * min(2 * order, 10) + slices * count * 52 + (40 << 20)
    else:
        total += 32 * 52 * count
    return total


def device_free_bytes():
    import torch

    free, _ = torch.cuda.mem_get_info()
    return free


@dataclass
class _Active:
    request: Request
    grid: object
    remaining: int
    admitted: float
    bytes: int
    per_step_s: float = 0.0
    sized: bool = False  # bytes is the engine's own report (its workspace is sized)


@dataclass
class Server:
    """Continuous-batching loop. `memory_budget` bytes (default: 80% of free device memory)
    bound the resident samples; `max_active` caps concurrency; each chunk aims at
    `chunk_seconds` of estimated device work per sample; `workers` threads run the finishing
    part of completed requests; `measure` runs measure() on each result."""
    precision: str = "fp32"
    memory_budget: int | None = None
    max_active: int = 64
    chunk_seconds: float = 0.02
    keep_quaternions: bool = False
    measure: bool = True
    workers: int = 4
    pair_rate: float = 2.5e11  # pair evaluations per second, for chunk sizing only
    results: list = field(default_factory=list)

    def _admit(self, r, now):
        g = haar(r.group, r.count, r.seed, precision=self.precision)
        g._check(g._lib.zo_relax_neighbourhood(g._handle, float(r.neighbourhood)))
        evals = r.count * neighbours(r.count, ORDER[r.group], r.neighbourhood)
        return _Active(r, g, r.steps, now, estimate_bytes(r.count, r.group, r.neighbourhood),
                       per_step_s=evals / self.pair_rate)

    def _finish(self, a, t0, clock):
        """The blocking part of a request (a worker thread; the engine is no longer stepped)."""
        lib, h = a.grid._lib, a.grid._handle
        try:
            a.grid._check(lib.zo_relax_finish(h))
            if self.measure:
                a.grid._check(lib.zo_measure(h))
            stats = a.grid.stats
            q = a.grid.quaternions if self.keep_quaternions else None
            return Result(a.request.id, a.request.arrival, a.admitted, clock() - t0, stats, q)
        finally:
            a.grid.close()

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times in seconds from the start); returns the results
        in completion order."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.id))
        budget = self.memory_budget if self.memory_budget is not None else int(0.8 * device_free_bytes())
        stepping: list[_Active] = []
        finishing = {}  # future -> _Active
        t0 = clock()
        held = 0
        with ThreadPoolExecutor(max_workers=max(1, self.workers)) as pool:
            while pending or stepping or finishing:
                now = clock() - t0
                resident = len(stepping) + len(finishing)
                # One sample at a time is admitted on its estimate: the next waits until the
                # first chunk has sized its workspace and its engine has reported its bytes.
                if (pending and pending[0].arrival <= now and resident < self.max_active
                        and all(a.sized for a in stepping)
                        and (held + estimate_bytes(pending[0].count, pending[0].group, pending[0].neighbourhood)
                             <= budget or resident == 0)):
                    a = self._admit(pending.pop(0), now)
                    held += a.bytes
                    stepping.append(a)
                progressed = False
                for a in list(stepping):
                    lib, h = a.grid._lib, a.grid._handle
                    idle = lib.zo_idle(h)
                    if idle < 0:
                        a.grid._check(-1)
                    if not idle:
                        continue
                    if a.remaining > 0:
                        k = max(1, min(a.remaining, int(self.chunk_seconds / max(a.per_step_s, 1e-9))))
                        a.grid._check(lib.zo_relax_async(h, k))
                        a.remaining -= k
                        if not a.sized:  # the first chunk sized the workspace: count real bytes
                            real = int(lib.zo_device_bytes(h))
                            held += real - a.bytes
                            a.bytes, a.sized = real, True
                        progressed = True
                        continue
                    stepping.remove(a)
                    finishing[pool.submit(self._finish, a, t0, clock)] = a
                    progressed = True
                for fut in [f for f in finishing if f.done()]:
                    a = finishing.pop(fut)
                    held -= a.bytes
                    self.results.append(fut.result())  # re-raises a failed request's error
                    progressed = True
                if not progressed:
                    if not stepping and not finishing and pending:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                    else:
                        time.sleep(0.0005)
        return self.results


class _NativeRequest(C.Structure):
    _fields_ = [("id", C.c_uint32), ("group", C.c_uint32), ("count", C.c_uint32), ("steps", C.c_uint32),
                ("seed", C.c_uint32), ("neighbourhood", C.c_float), ("arrival", C.c_double)]


class _NativeResult(C.Structure):
    _fields_ = [("id", C.c_uint32), ("iteration", C.c_uint32), ("count", C.c_uint32), ("order", C.c_uint32),
                ("arrival", C.c_double), ("admitted", C.c_double), ("finished", C.c_double),
                ("neighbourhood", C.c_double), ("energy", C.c_double), ("separation_deg", C.c_double),
                ("status", C.c_int32), ("error", C.c_char * 108)]


@dataclass
class NativeServer:
    """The same continuous-batching loop run inside the library (zo_serve): admission,
    chunked stepping and the finishing workers in C++ threads, one blocking call for the
    whole request stream (arrival times from the call). Results carry the numbers the
    summary needs (count, order, iteration, neighbourhood, Quey energy, separation)."""
    precision: str = "fp32"
    memory_budget: int | None = None
    max_active: int = 64
    chunk_seconds: float = 0.02
    measure: bool = True
    workers: int = 4
    pair_rate: float = 2.5e11

    def run(self, requests):
        lib = _library()
        if not hasattr(lib, "_serve_bound"):
            lib.zo_serve.argtypes = [C.POINTER(_NativeRequest), C.c_uint32, C.POINTER(C.c_double), C.c_uint32,
                                     C.POINTER(_NativeResult), C.c_char_p, C.c_size_t]
            lib.zo_serve.restype = C.c_int
            lib._serve_bound = True
        reqs = (_NativeRequest * len(requests))()
        for k, r in enumerate(requests):
            reqs[k] = _NativeRequest(r.id, GROUPS.index(r.group), r.count, r.steps, r.seed, r.neighbourhood, r.arrival)
        settings = (C.c_double * 7)(float(self.memory_budget or 0), float(self.max_active), float(self.chunk_seconds),
                                    1.0 if self.measure else 0.0, 1.0 if self.precision == "fp64" else 0.0,
                                    float(self.workers), float(self.pair_rate))
        out = (_NativeResult * len(requests))()
        error = C.create_string_buffer(512)
        if lib.zo_serve(reqs, len(requests), settings, 7, out, error, len(error)) != 0:
            raise RuntimeError(error.value.decode(errors="replace"))
        results = []
        for r in out:
            if r.status != 0:
                raise RuntimeError(f"request {r.id}: {r.error.decode(errors='replace')}")
            stats = {"count": r.count, "order": r.order, "iteration": r.iteration,
                     "relax_neighbourhood": r.neighbourhood or None, "quey_energy": r.energy,
                     "separation_deg": r.separation_deg}
            results.append(Result(r.id, r.arrival, r.admitted, r.finished, stats))
        return results


def shard_requests(requests, rank, world):
    """This rank's share of a request stream when `world` GPUs serve it together (one process
    and one Server per GPU, no collective): request k goes to rank k mod world, so each rank
    sees a thinned Poisson stream at 1/world of the rate."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return [r for r in requests if r.id % world == rank]


def serve_one_at_a_time(requests, precision="fp64", clock=time.perf_counter, keep_quaternions=False, measure=True):
    """The plain path: requests in arrival order, one at a time, each relaxed with zo_relax
    (no graphs, no overlap) and then measured; FP64 by default."""
    pending = sorted(requests, key=lambda r: (r.arrival, r.id))
    results = []
    t0 = clock()
    for r in pending:
        now = clock() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        admitted = clock() - t0
        g = haar(r.group, r.count, r.seed, precision=precision)
        try:
            g._check(g._lib.zo_graphs(g._handle, 0))
            g.relax(r.steps, neighbourhood=r.neighbourhood)
            if measure:
                g.measure()
            results.append(Result(r.id, r.arrival, admitted, clock() - t0, g.stats,
                                  g.quaternions if keep_quaternions else None))
        finally:
            g.close()
    return results


def poisson_requests(rate, duration, seed=0, n_min=500, n_max=1_000_000, steps=(10, 200), all_pairs_below=5000):
    """Serving workload: Poisson arrivals at `rate` per second over `duration` seconds,
    group uniform over the eleven, N log-uniform in [n_min, n_max], steps uniform in
    `steps`, all pairs below `all_pairs_below` orientations else a neighbourhood of 20,
    a per-request seed."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            return out
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        out.append(Request(len(out), str(rng.choice(GROUPS)), n, int(rng.integers(steps[0], steps[1] + 1)),
                           int(rng.integers(0, 2 ** 31)), 0.0 if n < all_pairs_below else 20.0, t))


def summary(results, duration=None):
    """Throughput (pair-evals/s counted as the reference counts them) and latency percentiles."""
    if not results:
        return {}
    lat = np.array([r.latency for r in results])
    span = duration or max(r.finished for r in results)
    evals = 0.0
    for r in results:
        s = r.stats
        n, order = s["count"], s["order"]
        delta = s.get("relax_neighbourhood") or 0.0
        evals += (s["iteration"] + 1) * n * neighbours(n, order, delta)
    return {"requests": len(results), "pair_evals_per_s": evals / span, "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)), "span_s": span}
