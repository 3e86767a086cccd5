"""Benchmark of the QVM relaxation hot path on B200 (one JSON line on rank 0).

Workload (the headline configuration): group O, N = 100,000 Haar-random orientations
(seed 193, folded into the zone), near field of 20 mean orientation radii (~7,584
neighbours per source, smooth fade from half the cutoff), Barzilai-Borwein steps with FP32
pair arithmetic and FP64 BB products, sums and renormalisation. A step is one BB step over
the resident sample: near-field force pass, BB statistics, exact median, move and fold.

Metric: pair-evals/s counted as the reference counts them (src/engine.zig:905-907): per
force pass N * min(N|K|, 0.94 delta^3 + 64). `value` is device time (CUDA events on the
engine's stream, L2 flushed by a 256 MB memset before every step, outside the events);
`e2e` goes through the public API with host buffers (import from pinned memory, relax,
read the positions back). Multi-GPU: independent replicas, one per rank (weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
_T0 = time.perf_counter()  # the whole run's wall clock starts here

GROUP, COUNT, SEED, DELTA, TAPER = "O", 100_000, 193, 20.0, 0.5
ORDER = 24
STEPS_PER_REQUEST = 100  # config: 100 BB steps
FLUSH_BYTES = 256 * 1024 * 1024
# Algorithmic FP32 operations of one windowed near-field Quey pair, counted from the
# reference formulation (shaders/pairs.wgsl:250-262, 352-361, 403-409): chord tests and
# dot products 23, near/far and the half-angle t 6, angle and the four powers 14, sine 5,
# sign 2, direction 21, force/curvature/energy 14, window and its slope term 29,
# accumulation 6; each add, multiply, divide, sqrt, atan, sin, min/max/select counts 1.
FLOPS_PER_NEAR_PAIR = 120
# The same count for one all-pairs Quey pair (shaders/pairs.wgsl:250-262, 293-300): chord
# tests and dot products 22, nearest 2, near/far and t 6, angle and powers 14, sine 5, sign
# 2, direction 21, force/curvature/energy 14, accumulation 5.
FLOPS_PER_PAIR = 91


def neighbours_of(n, order, delta):
    return min(n * order, 0.94 * delta ** 3 + 64) if delta > 0 else n * order


EVALS_PER_PASS = COUNT * neighbours_of(COUNT, ORDER, DELTA)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-extras", action="store_true",
                   help="skip the all-pairs, spacing, batched and served sections")
    return p.parse_args()


# ---------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def reduce(self, value, op):
        if not self.pg:
            return value
        import torch

        t = torch.tensor([float(value)], dtype=torch.float64)
        self.pg.all_reduce(t, op={"max": self.pg.ReduceOp.MAX, "sum": self.pg.ReduceOp.SUM}[op])
        return float(t.item())

    def gather(self, obj):
        """Every rank's `obj`, in rank order, on every rank."""
        if not self.pg:
            return [obj]
        out = [None] * self.world
        self.pg.all_gather_object(out, obj)
        return out

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks during the timed region
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *_):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded or sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------- CPU baseline (the oracle port)
def cpu_relaxation(threads=None):
    """The workload's plain FP64 relaxation on the host cores: the oracle's BB step
    (oracle/qvm.py Relax, restating shaders/relax.wgsl) over near-field rows from the C/OpenMP
    restatement (oracle/qvm_ref.c: shell of images, chart grid, windowed pairs) of all
    sources. Returns the relaxation and the thread count."""
    from oracle import cref, qvm

    ops = np.load(ROOT / "tests/golden/golden.npz")["ops_O"].astype(np.float32).astype(np.float64)
    gid = qvm.GROUPS.index(GROUP)
    threads = threads or cref.threads()
    q = qvm.fold(qvm.haar(COUNT, SEED), gid, ops, f32=False)
    rows = lambda x: cref.near_rows(x, ops, DELTA, TAPER, nthreads=threads)  # noqa: E731
    return qvm.Relax(q, gid, ops, delta=DELTA, rows_fn=rows), threads


def cpu_steps(relax, count):
    """Seconds of each of `count` whole BB steps (force pass over every source + update)."""
    times = []
    for _ in range(count):
        t = time.perf_counter()
        relax.step()
        times.append(time.perf_counter() - t)
    return times


def cpu_sample(steps=3, warmup=1):
    """Our line's cpu_baseline: a few whole FP64 steps of the workload on the host cores."""
    relax, threads = cpu_relaxation()
    cpu_steps(relax, warmup)
    times = cpu_steps(relax, steps)
    per_step = statistics.mean(times)
    return EVALS_PER_PASS / per_step, threads, (
        f"{steps} whole FP64 BB steps of the workload after {warmup} untimed (near-field rows of all {COUNT} "
        f"sources by the C/OpenMP restatement, shell and chart grid rebuilt each step as on the GPU, then the "
        f"BB update), {per_step:.2f} s per step")


def run_reference(args, dist):
    """Reference arm: the reference has no CPU implementation of this path and its own
    engine (Zig + WGSL through wgpu-native) cannot run here, so the arm is the oracle port
    of the same workload on the host cores: W untimed and K timed whole FP64 steps, each a
    near-field force pass over all sources and the BB update; ms_per_step is measured."""
    if dist.rank != 0:
        return 0
    relax, threads = cpu_relaxation()
    cpu_steps(relax, args.warmup)
    times = cpu_steps(relax, args.steps)
    per_step = statistics.mean(times)
    value = EVALS_PER_PASS / per_step
    desc = (f"{args.steps} timed whole FP64 BB steps after {args.warmup} untimed, all {COUNT} sources each "
            f"(C/OpenMP near-field rows + oracle BB update), {threads} threads")
    line = {
        "impl": "reference", "metric": "pair-evals/s", "value": value, "unit": "pair-evals/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(args),
        "step_ms": {"p50": 1e3 * float(np.percentile(times, 50)), "max": 1e3 * max(times)},
        "cpu_baseline": {"value": value, "unit": "pair-evals/s", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "pair-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config(args):
    return {"workload": f"QVM near-field relaxation, group {GROUP}, N={COUNT} Haar (seed {SEED}), "
                        f"neighbourhood {DELTA:g} mean radii, taper {TAPER}",
            "group": GROUP, "n": COUNT, "neighbourhood": DELTA, "steps_per_request": STEPS_PER_REQUEST,
            "pair_evals_per_pass": EVALS_PER_PASS, "parallelism": f"replicas x{args.gpus}",
            "l2": "flushed before every timed step (256 MB memset)",
            "arithmetic": "FP32 pairs, FP64 sums/BB/renormalisation (fp32-refined)"}


# ---------------------------------------------------------------- our arm
def bench_engine(zo, precision, steps, warmup, seed):
    grid = zo.haar(GROUP, COUNT, seed, precision=precision)
    grid.relax(0, neighbourhood=DELTA)
    out = np.zeros(4 + steps, np.float64)
    grid._check(grid._lib.zo_bench(grid._handle, steps, warmup, float(FLUSH_BYTES),
                                   out.ctypes.data_as(C.POINTER(C.c_double)), len(out)))
    return grid, out


def e2e_requests(zo, seed, requests):
    """Public-API requests: import from pinned host memory, set the neighbourhood, relax
    100 steps, read the positions back. Returns (pair-evals/s, latencies s, bytes)."""
    import torch

    base = zo.haar(GROUP, COUNT, seed)
    start = base.quaternions
    base.close()
    pinned = torch.empty((COUNT, 4), dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = start
    out = torch.empty((COUNT, 4), dtype=torch.float32, pin_memory=True)
    grid = zo.Grid(GROUP, _empty=True)
    lib, h = grid._lib, grid._handle
    ptr = C.cast(pinned.data_ptr(), C.POINTER(C.c_float))

    def request():
        grid._check(lib.zo_set(h, 9, ptr, COUNT))
        grid._check(lib.zo_relax_neighbourhood(h, DELTA))
        grid._check(lib.zo_relax(h, STEPS_PER_REQUEST))
        C.memmove(out.data_ptr(), lib.zo_quaternions(h), COUNT * 16)
        return json.loads(lib.zo_stats(h))

    request()  # warm-up
    lat = []
    for _ in range(requests):
        t = time.perf_counter()
        stats = request()
        lat.append(time.perf_counter() - t)
    grid.close()
    evals = (STEPS_PER_REQUEST + 1) * EVALS_PER_PASS
    return evals * len(lat) / sum(lat), lat, stats


def batched_section(zo, samples=256, steps=50, dist=None):
    """Config 4: 256 samples (groups uniform over the eleven, N log-uniform in [1e3, 2e5],
    seeds 0..255, neighbourhood 20), 50 BB steps each, relaxed together by zo_batch_relax:
    each step is one CUDA graph over all samples, whose near-field gathers run in one
    persistent launch per tile variant (tile shapes from the tuned table); pair-evals/s over
    the whole batch (steps plus each sample's closing force pass), wall clock."""
    from zxtalori_b200 import batch, serve

    rank, world = (dist.rank, dist.world) if dist else (0, 1)
    specs = batch.shard(batch.random_samples(samples), rank, world)  # all of them on one GPU
    t = time.perf_counter()
    grids = batch.make_grids(specs)
    setup = time.perf_counter() - t
    evals = sum(batch.pair_evals(s.count, serve.ORDER[s.group], s.neighbourhood, steps) for s in specs)
    sum_n = sum(s.count for s in specs)
    try:
        if dist:
            dist.barrier()
        t = time.perf_counter()
        batch.relax_batch(grids, steps)
        dt = time.perf_counter() - t
    finally:
        for g in grids:
            g.close()
    if dist:  # every rank's share at once: the slowest rank's time, all ranks' work
        dt, setup = dist.reduce(dt, "max"), dist.reduce(setup, "max")
        evals, sum_n = dist.reduce(evals, "sum"), int(dist.reduce(sum_n, "sum"))
    lib = zo.api._library()
    out = (C.c_double * 3)()
    shapes = {}
    for sp in specs:
        lib.zo_tiles_lookup(0, zo.GROUPS.index(sp.group), sp.count, out)
        shapes[f"{int(out[0])}x{out[1]:g}"] = shapes.get(f"{int(out[0])}x{out[1]:g}", 0) + 1
    return {"samples": samples, "steps": steps, "sum_n": sum_n, "pair_evals_per_s": evals / dt,
            "seconds": dt, "setup_seconds": setup, "tile_shapes_from_table": shapes, "gpus": world,
            "split": "samples over ranks, largest first to the least-loaded rank; no collective",
            "timing": "wall clock of zo_batch_relax (all steps and closing passes), samples created beforehand"}


def served_split_section(zo, device_rate, dist, factor=1.4, per_rate=200):
    """Config 5 over several GPUs: one request stream at `factor` times the whole job's
    capacity, request k served by rank k mod N (its own zo_serve loop, no collective); the ranks'
    results are gathered for the whole-job throughput (all pair evaluations over the longest
    rank's span) and latency percentiles."""
    from zxtalori_b200 import serve

    probe = serve.poisson_requests(1.0, 20_000.0, seed=11)
    mean_evals = float(np.mean([(r.steps + 1) * r.count * serve.neighbours(r.count, serve.ORDER[r.group],
                                                                           r.neighbourhood) for r in probe]))
    rate = factor * dist.world * device_rate / mean_evals
    reqs = serve.poisson_requests(rate, 1.5 * per_rate / rate, seed=5)[:per_rate]
    mine = serve.shard_requests(reqs, dist.rank, dist.world)
    dist.barrier()
    served = serve.NativeServer().run(mine)
    everything = [r for part in dist.gather(served) for r in part]
    return {"rate_per_s": rate, "rate_over_capacity": factor, "gpus": dist.world,
            "split": "request k to rank k mod N, one zo_serve loop per GPU, no collective",
            **serve.summary(everything)}


def served_section(zo, device_rate, factors=(0.7, 1.4), per_rate=200, plain_requests=20):
    """Config 5: Poisson arrivals of relax+measure requests (group uniform, N log-uniform in
    [500, 1e6], steps uniform in [10, 200], all pairs below 5,000 orientations else
    neighbourhood 20), served by the library's continuous-batching loop (zo_serve) in
    FP32-refined mode, at
    rates below and above the GPU's capacity: capacity = the headline's device
    pair-evals/s over the mean pair evaluations of a request. `per_rate` requests per rate
    (p50 and p99 from that many latencies). The plain FP64 path serves a fixed subsample
    (every k-th request of the higher-rate stream) one at a time; both throughputs count
    pair evaluations as the reference does (relax steps and closing pass)."""
    from zxtalori_b200 import serve

    probe = serve.poisson_requests(1.0, 20_000.0, seed=11)
    mean_evals = float(np.mean([(r.steps + 1) * r.count * serve.neighbours(r.count, serve.ORDER[r.group],
                                                                           r.neighbourhood) for r in probe]))
    capacity = device_rate / mean_evals
    sweep = []
    streams = {}
    for f in factors:
        rate = f * capacity
        reqs = serve.poisson_requests(rate, 1.5 * per_rate / rate, seed=5)[:per_rate]
        streams[f] = reqs
        t = time.perf_counter()
        served = serve.NativeServer().run(reqs)
        wall = time.perf_counter() - t
        sweep.append({"rate_per_s": rate, "rate_over_capacity": f, "wall_s": wall,
                      "arrival_window_s": reqs[-1].arrival, **serve.summary(served)})
    middle = sweep[len(sweep) // 2]
    stream = streams[factors[len(factors) // 2]]
    stride = max(1, len(stream) // plain_requests)
    chosen = stream[::stride][:plain_requests]
    plain_in = [serve.Request(r.id, r.group, r.count, r.steps, r.seed, r.neighbourhood, 0.0) for r in chosen]
    t = time.perf_counter()
    plain = serve.summary(serve.serve_one_at_a_time(plain_in))
    plain["wall_s"] = time.perf_counter() - t
    # The same subsample served by the batching loop, for a like-for-like throughput ratio.
    same = serve.summary(serve.NativeServer().run([serve.Request(r.id, r.group, r.count, r.steps, r.seed,
                                                           r.neighbourhood, 0.0) for r in chosen]))
    return {**{k: middle[k] for k in ("requests", "pair_evals_per_s", "latency_p50_s", "latency_p99_s")},
            "capacity_requests_per_s": capacity, "mean_pair_evals_per_request": mean_evals,
            "sweep": sweep, "plain_fp64_one_at_a_time": plain, "served_same_subsample": same,
            "served_over_plain_same_subsample": same["pair_evals_per_s"] / plain["pair_evals_per_s"],
            "requests_measured": "every request runs measure() after its steps (every energy ratio below "
                                 "the ratio limit)"}


def _device_seconds(lib, handle, steps, warmup):
    out = np.zeros(4 + steps, np.float64)
    rc = lib.zo_bench(handle, steps, warmup, float(FLUSH_BYTES), out.ctypes.data_as(C.POINTER(C.c_double)), len(out))
    if rc != 0:
        raise RuntimeError(lib.zo_error(handle).decode())
    return out


def allpairs_section(zo, peak, count=1048, steps=30, kernel_count=16384):
    """Config 1 (group O, N=1,048 Haar seed 193, all pairs, 30 steps then every measure) as
    requests through the public API in both precision modes, and the all-pairs row kernel
    on the FP32 roofline at N=16,384 (6.4e9 pairs per pass)."""
    result = {"workload": f"O, N={count} Haar (seed {SEED}), all pairs, {steps} steps + measure"}
    evals = (steps + 1) * count * count * ORDER
    for precision in ("fp64", "fp32"):
        lat = []
        for rep in range(4):
            t = time.perf_counter()
            g = zo.haar(GROUP, count, SEED, precision=precision)
            g.relax(steps)
            m = g.measure()
            dt = time.perf_counter() - t
            g.close()
            if rep:
                lat.append(dt)
        result[precision] = {"request_s_p50": float(np.median(lat)), "pair_evals_per_s": evals / float(np.median(lat)),
                             "quey_energy": m["quey_energy"], "separation_deg": m["separation_deg"],
                             "riesz_2": m["riesz_2"], "log_ratio": m["log_ratio"]}
    g = zo.haar(GROUP, kernel_count, SEED)
    g.relax(0, neighbourhood=0)
    out = _device_seconds(g._lib, g._handle, 5, 3)
    g.close()
    avg = out[1] / max(1, out[2]) / 1e3
    pairs = kernel_count * kernel_count * ORDER
    achieved = pairs * FLOPS_PER_PAIR / avg / 1e12
    result["kernel"] = {"kernel": "k_pairs32 (all-pairs rows)", "n": kernel_count, "pairs_per_pass": pairs,
                        "kernel_ms_avg": avg * 1e3, "pair_evals_per_s": pairs / avg, "achieved_tflops": achieved,
                        "peak_tflops": peak, "frac": achieved / peak, "flops_per_pair": FLOPS_PER_PAIR,
                        "step_ms": out[0] / 5}
    return result


def spacing_section(zo, peak, count=10_000_000, seed=7, measure_count=None):
    """Config 3: the spacing pass (per-orientation nearest SO(3) angle and neighbour index;
    neighbourhood 4 above 20,000 orientations) over group I, N=10M Haar seed 7: wall clock
    through the public API (the second of two calls: the first sizes the workspace), device
    time per pass and the gather kernel's HBM roofline from zo_bench_spacing, and the
    indices and angles checked against the FP64 method on the same float32 sample. With
    `measure_count`, the default measures of I at that size (all pairs, FP32)."""
    g = zo.haar("I", count, seed)
    t = time.perf_counter()
    g.spacing()
    first = time.perf_counter() - t
    t = time.perf_counter()
    sep = g.spacing()["separation_deg"]
    dt = time.perf_counter() - t
    degrees = g.point_values("separation")
    neighbours = g.point_neighbours()
    exact = g.spacing_exact()
    q = g.quaternions
    out = np.zeros(6, np.float64)
    g._check(g._lib.zo_bench_spacing(g._handle, 5, 1, float(FLUSH_BYTES), out.ctypes.data_as(C.POINTER(C.c_double)),
                                     len(out)))
    g.close()
    n_pairs = count * neighbours_of(count, 60, 4.0)
    tiles = (C.c_double * 3)()
    zo.api._library().zo_tiles_lookup(1, zo.GROUPS.index("I"), count, tiles)
    lane = int(tiles[0]) == 1
    # Algorithmic bytes of one gather launch: every source read once (16 B), every shell
    # site read once (its 16 B position; the warp-tiled search also reads a 4 B code and a
    # 4 B chart x), the chosen site written per source (4 B; the tiled search also writes
    # the 8 B chord).
    sites = out[3]
    algorithmic = count * 16 + sites * (16 if lane else 24) + count * (4 if lane else 12)
    achieved = algorithmic / (out[1] * 1e-3) / 1e9
    result = {"workload": f"I, N={count} Haar (seed {seed}), spacing with neighbourhood 4",
              "seconds": dt, "first_call_seconds": first, "pair_evals_per_s": n_pairs / dt,
              "device_ms_per_pass": out[0], "separation_deg": sep, "median_nearest_deg": float(np.median(degrees)),
              "exact_search_points": exact["exact_search"], "exact_ties": exact["exact_ties"],
              "roofline": {"bound": "hbm",
                           "kernel": ("k_nearest_lane (one source per thread" if lane else
                                      "k_near32<nearest only> (") + f"; tile shape {int(tiles[0])}, "
                                     f"{tiles[1]:g} sites per cell, first walk {tiles[2]:g} of the cutoff)",
                           "kernel_ms_avg": out[1], "launches": int(out[2]), "shell_sites": int(sites),
                           "algorithmic_bytes": algorithmic, "achieved": achieved, "peak": peak[0],
                           "peak_source": peak[1], "unit": "GB/s", "frac": achieved / peak[0],
                           "limiter": "not HBM: each source reads every site of its first ball's cell rows (tens "
                                      "per source) from L1/L2; ncu on the 1M launch shows the ALU pipe at 71 % "
                                      "and 13 of 32 lanes active (each thread walks its own rows)"}}
    # The same float32 sample through the FP64 method: indices must agree except exact ties.
    g64 = zo.from_quaternions(q, "I", precision="fp64")
    g64.spacing()
    d64, n64 = g64.point_values("separation"), g64.point_neighbours()
    g64.close()
    mismatched = int(np.count_nonzero(neighbours != n64))
    rel = np.abs(degrees - d64) / d64
    result["vs_fp64"] = {"index_mismatches": mismatched, "index_mismatches_allowed": exact["exact_ties"],
                         "degrees_max_rel_error": float(rel.max()), "degrees_p99_rel_error": float(np.percentile(rel, 99)),
                         "note": "FP32-refined mode forms images with the float32 operator tables the reference "
                                 "uploads, the FP64 method with the FP64 tables; the tables differ by up to 6e-8 per "
                                 "component, which at the smallest separations (1e-5 rad) is 1e-4 of the angle. "
                                 "Against the FP64 oracle with the same float32 tables the angles agree to 1e-6 "
                                 "(tests/test_gpu_spacing.py)."}
    if measure_count:
        g = zo.haar("I", measure_count, seed)
        t = time.perf_counter()
        m = g.measure()
        dt = time.perf_counter() - t
        g.close()
        pairs = measure_count * measure_count * 60
        result["measure"] = {"workload": f"I, N={measure_count} Haar (seed {seed}), measure(): above I's ratio "
                                         "limit, so Quey energy and separation over all pairs (FP32)",
                             "n": measure_count, "seconds": dt, "pair_evals_per_s": pairs / dt,
                             "quey_energy": m["quey_energy"], "separation_deg": m["separation_deg"]}
    return result


def covering_section(zo):
    """The covering radius (zo_cover: every orientation's Delaunay star on the GPU), exact-count
    generation and covering optimisation: wall clock through the public API."""
    out = {}
    for group, count, seed in (("O", 100_000, SEED), ("I", 1_000_000, 7)):
        with zo.haar(group, count, seed) as g:
            t = time.perf_counter()
            s = g.covering()
            first = time.perf_counter() - t
            g.relax(1, neighbourhood=DELTA)  # a near-field step (all pairs at 1M would take minutes)
            t = time.perf_counter()
            s = g.covering()
            again = time.perf_counter() - t
        out[f"{group}_{count}"] = {"seconds_first_call": first, "seconds_after_a_step": again,
                                   **{k: s[k] for k in ("covering_radius_deg", "simplex_bound_deg",
                                                        "covering_unresolved_caps", "covering_rounds",
                                                        "covering_shell_points", "covering_tetrahedra",
                                                        "covering_certificate_probes")}}
    t = time.perf_counter()
    with zo.generate("O", count=4000, exact=True) as g:
        out["exact_O_4000"] = {"seconds": time.perf_counter() - t, "base_count": g.stats["base_count"],
                               "inserted_count": g.stats["inserted_count"]}
    with zo.haar("O", 1000, 11) as g:
        g.relax(20)
        before = g.covering()["covering_radius_deg"]
        t = time.perf_counter()
        g.optimize_covering(200, mode="face")
        s = g.stats
        out["optimize_O_1000"] = {"steps": 200, "seconds": time.perf_counter() - t, "radius_before_deg": before,
                                  "radius_after_deg": s["covering_radius_deg"],
                                  "improved_steps": s["covering_optimizer_improved"],
                                  "kicks": s["covering_optimizer_kicks"]}
    return out


def hbm_peak():
    """HBM copy bandwidth in GB/s and where it comes from: the measured figure in
    MEASURED_PEAKS.json when present, else an earlier copy measurement on B200 (6,650 GB/s)."""
    try:
        data = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        for key in ("hbm_gbs", "hbm_GBs", "hbm_copy_gbs"):
            if isinstance(data.get(key), (int, float)):
                return float(data[key]), "measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback (earlier B200 copy measurement)"


def _rel(a, b):
    return abs(a - b) / abs(b) if b else abs(a - b)


def _chord(a, b, ops):
    """Per-point distance between two samples of the same orbits: the smallest chord from a
    to any image of b (b g_k, either sign), so a point folded to another equivalent zone
    image counts by its orbit."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    ops = np.asarray(ops, np.float64)
    best = np.full(len(a), np.inf)
    for g in ops:
        w = b[:, :1] * g[0] - (b[:, 1:] * g[1:]).sum(1, keepdims=True)
        v = b[:, :1] * g[1:] + g[0] * b[:, 1:] + np.cross(b[:, 1:], g[1:])
        y = np.concatenate([w, v], axis=1)
        y /= np.linalg.norm(y, axis=1, keepdims=True)
        best = np.minimum(best, np.minimum(np.linalg.norm(a - y, axis=1), np.linalg.norm(a + y, axis=1)))
    return best


def _nudged(q):
    """Every component moved by one float32 ulp, in a seeded random direction."""
    q = np.asarray(q, np.float32)
    up = np.random.default_rng(0).random(q.shape) < 0.5
    return np.nextafter(q, np.where(up, np.float32(np.inf), np.float32(-np.inf))).astype(np.float32)


def errors_section(zo):
    """Every result's error against the FP64 method (the plain path: FP64 arithmetic,
    positions and sums throughout), for configs 1 and 2, three ways:
    - trajectory: the FP32-refined run against the FP64 run from the same start;
    - same sample: the FP32-refined engine's measures of its own relaxed sample against the
      FP64 method's measures of that same float32 sample (the arithmetic alone);
    - conditioning: the FP64 run against itself started one float32 ulp away. A relaxed
      sample's minimum separation follows the trajectory's sensitivity to its start, so
      this is the floor below which no trajectory comparison can go."""
    keys = ("quey_energy", "separation_deg", "riesz_1", "riesz_2", "riesz_3", "green_ratio", "log_ratio")
    out = {}
    # Config 1: O, N=1,048, all pairs, 30 steps, then every measure.
    ops = None

    def run1(precision, q=None):
        nonlocal ops
        g = zo.haar("O", 1048, SEED, precision=precision) if q is None else zo.from_quaternions(q, "O", precision)
        ops = g.operations
        start = g.quaternions
        g.relax(30)
        m, q_end = g.measure(), g.quaternions
        g.close()
        return m, q_end, start

    m64, q64, start = run1("fp64")
    m32, q32, _ = run1("fp32")
    g = zo.from_quaternions(q32, "O", precision="fp64")
    same = g.measure()
    g.close()
    m64n, q64n, _ = run1("fp64", _nudged(start))
    m64s, _, _ = run1("fp64", start)  # the same start imported, for the comparison above
    out["config1"] = {
        "workload": "O, N=1048 Haar (seed 193), all pairs, 30 BB steps, then measure()",
        "trajectory": {**{k: _rel(m32[k], m64[k]) for k in keys}, "positions_chord_max": float(_chord(q32, q64, ops).max())},
        "same_sample": {k: _rel(m32[k], same[k]) for k in keys},
        "conditioning": {**{k: _rel(m64n[k], m64s[k]) for k in keys},
                         "positions_chord_max": float(_chord(q64n, q64, ops).max())},
    }
    # Config 2: O, N=100,000, neighbourhood 20, 100 steps.
    def run2(precision, q=None):
        g = zo.haar(GROUP, COUNT, SEED, precision=precision) if q is None else zo.from_quaternions(q, GROUP, precision)
        start = g.quaternions
        g.relax(STEPS_PER_REQUEST, neighbourhood=DELTA)
        st, q_end = g.stats, g.quaternions
        g.close()
        return st, q_end, start

    def all_pairs(q):
        g = zo.from_quaternions(q, GROUP, precision="fp64")
        g.relax(0, neighbourhood=0)
        m = g.measure()  # above O's ratio limit: energy and separation over all pairs
        g.close()
        return m

    s64, p64, start = run2("fp64")
    s32, p32, _ = run2("fp32")
    s64n, p64n, _ = run2("fp64", _nudged(start))
    s64s, p64s, _ = run2("fp64", start)
    g = zo.from_quaternions(p32, GROUP, precision="fp64")
    g.relax(0, neighbourhood=DELTA)  # sets the neighbourhood; measure() then uses the near field
    near_same = g.measure()
    g.close()
    a32, a64, a64s, a64n = all_pairs(p32), all_pairs(p64), all_pairs(p64s), all_pairs(p64n)
    near = ("quey_energy", "separation_deg")
    chords = _chord(p32, p64, ops)
    out["config2"] = {
        "workload": f"{GROUP}, N={COUNT} Haar (seed {SEED}), neighbourhood {DELTA:g}, {STEPS_PER_REQUEST} BB steps",
        "trajectory": {**{f"near_{k}": _rel(s32[k], s64[k]) for k in near},
                       **{f"allpairs_{k}": _rel(a32[k], a64[k]) for k in near},
                       "positions_chord_max": float(chords.max()),
                       "positions_chord_p99": float(np.percentile(chords, 99))},
        "same_sample": {f"near_{k}": _rel(s32[k], near_same[k]) for k in near},
        "conditioning": {**{f"near_{k}": _rel(s64n[k], s64s[k]) for k in near},
                         **{f"allpairs_{k}": _rel(a64n[k], a64s[k]) for k in near},
                         "positions_chord_max": float(_chord(p64n, p64s, ops).max())},
        "fp64_allpairs": {k: a64[k] for k in near},
    }
    return out


def traffic_from_profile():
    """DRAM bytes per launch of the near-field row kernel from the committed ncu summary."""
    path = ROOT / "profiles" / "near_rows_kernel.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_ours(args, dist):
    os.environ["ZXTALORI_DEVICE"] = str(dist.local)
    import zxtalori_b200 as zo

    seed = SEED + dist.rank
    # FP32-refined: the product path.
    dist.barrier()
    with Clocks(dist.local) as clocks:
        grid, out = bench_engine(zo, "fp32", args.steps, args.warmup, seed)
    total_ms = out[0]
    per_step = out[4:4 + args.steps]
    kernel_ms, kernel_launches, launches_per_step = out[1], out[2], out[3]
    peak = grid._lib.zo_fp32_peak(grid._handle)
    separation = grid.measure()["separation_deg"]
    # Pairs the gather evaluates and those inside the cutoff, from one counting pass (outside
    # the timed steps), beside the metric's nominal count.
    counted = (C.c_double * 2)()
    grid._check(grid._lib.zo_debug_pair_counts(grid._handle, counted))
    grid.close()
    dist.barrier()
    t_max = dist.reduce(total_ms, "max")
    work = dist.reduce(args.steps * EVALS_PER_PASS, "sum")
    value = work / (t_max / 1e3)
    # Plain FP64 method on the same workload (fewer steps).
    k64 = max(1, min(args.steps, 3))
    g64, out64 = bench_engine(zo, "fp64", k64, 1, seed)
    g64.close()
    t64 = dist.reduce(out64[0], "max")
    fp64_value = dist.reduce(k64 * EVALS_PER_PASS, "sum") / (t64 / 1e3)
    # End to end through the public API.
    e2e_value, lat, _ = e2e_requests(zo, seed, requests=4)
    e2e_value = dist.reduce(e2e_value, "sum")
    extras = {}
    if args.gpus > 1 and not args.no_extras:
        extras["batched"] = batched_section(zo, dist=dist)  # config 4 split over the ranks
        extras["served"] = served_split_section(zo, value / args.gpus, dist)  # config 5 split over the ranks
    if dist.rank != 0:
        return 0
    # All pairs, spacing, batched and served workloads (configs 1, 3, 4, 5) on one GPU.
    if args.gpus == 1 and not args.no_extras:
        sections = (("allpairs", lambda: allpairs_section(zo, peak)),
                    ("spacing", lambda: spacing_section(zo, hbm_peak(), measure_count=1_000_000)),
                    ("errors_vs_fp64", lambda: errors_section(zo)),
                    ("covering", lambda: covering_section(zo)),
                    ("batched", lambda: batched_section(zo)),
                    ("served", lambda: served_section(zo, value)))
        wall = {}
        for name, run in sections:
            t = time.perf_counter()
            extras[name] = run()
            wall[name] = time.perf_counter() - t
        extras["section_seconds"] = wall
    kernel_avg_s = kernel_ms / max(1, kernel_launches) / 1e3
    achieved = EVALS_PER_PASS * FLOPS_PER_NEAR_PAIR / kernel_avg_s / 1e12
    traffic = traffic_from_profile()
    cpu_value, cpu_threads, cpu_desc = cpu_sample() if args.gpus == 1 else (None, None, "rank 0 only at N=1")
    line = {
        "metric": "pair-evals/s", "value": value, "unit": "pair-evals/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config(args),
        "latency_ms": {"step_p50": float(np.percentile(per_step, 50)), "step_p99": float(np.percentile(per_step, 99)),
                       "request_p50": 1e3 * float(np.percentile(lat, 50)),
                       "request_p99": 1e3 * float(np.percentile(lat, 99))},
        "fp64_plain": {"value": fp64_value, "ms_per_step": t64 / k64, "steps": k64,
                       "ratio_fp32_refined_over_fp64": value / fp64_value},
        "separation_deg": separation,
        "pairs_per_pass": {"nominal": EVALS_PER_PASS, "in_cutoff": counted[1], "candidates": counted[0],
                           "note": "nominal: the reference's metric count, N min(N|K|, 0.94 delta^3 + 64); "
                                   "in_cutoff: orbit pairs within the cutoff that exert a force; candidates: "
                                   "sites the gather evaluates (the union of its warp's four sources' balls, "
                                   "cell row by cell row); the metric and the roofline use nominal"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_near32 (near-field rows)",
                     "peak_source": "FP32 FMA probe on this GPU (zo_fp32_peak); MEASURED_PEAKS.json has no FP32 figure",
                     "flops_per_pair": FLOPS_PER_NEAR_PAIR, "kernel_ms_avg": kernel_avg_s * 1e3},
        "cpu_baseline": {"value": cpu_value, "unit": "pair-evals/s", "cores": cpu_threads, "kind": "port",
                         "sample": cpu_desc},
        "e2e": {"value": e2e_value, "unit": "pair-evals/s", "h2d_bytes_per_step": COUNT * 16,
                "d2h_bytes_per_step": COUNT * 16,
                "step": f"one request: import N quaternions from pinned host memory, relax {STEPS_PER_REQUEST} "
                        f"steps (+1 closing force pass), read N quaternions back"},
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "clocks": clocks.summary(),
        **extras,
        "bench_wall_seconds": time.perf_counter() - _T0,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            return run_reference(args, dist)
        return run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    sys.exit(main())
