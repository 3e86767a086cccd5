"""Batched and served relaxation: every sample's result is the same alone and in the mix.

Each sample's kernels read only its own buffers and sum in a fixed order, and a captured
step graph replays exactly the launches it captured, so the comparisons are exact
(tolerance 0); the energies are also checked against the oracle's measure of the result.
"""
import numpy as np
import pytest

from oracle import qvm

pytestmark = pytest.mark.gpu

SAMPLES = [("O", 3000, 1, 20.0), ("I", 1500, 2, 20.0), ("C4", 900, 3, 0.0), ("D6", 6000, 4, 20.0), ("T", 700, 5, 0.0)]


def test_graph_replay_equals_direct_launches(engine):
    out = []
    for graphs in (1, 0):
        with engine.haar("O", 4000, 8) as grid:
            grid._check(grid._lib.zo_graphs(grid._handle, graphs))
            grid.relax(12, neighbourhood=20)
            out.append((grid.quaternions, grid.stats))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1]["energy"] == out[1][1]["energy"]


def test_batch_matches_alone(engine, ops32):
    from zxtalori_b200 import batch

    specs = [batch.Sample(g, n, s, d) for g, n, s, d in SAMPLES]
    grids = batch.make_grids(specs)
    try:
        stats = batch.relax_batch(grids, 10)
        mixed = [g.quaternions for g in grids]
    finally:
        for g in grids:
            g.close()
    for spec, q_mix, s_mix in zip(specs, mixed, stats):
        with engine.haar(spec.group, spec.count, spec.seed) as grid:
            grid.relax(10, neighbourhood=spec.neighbourhood)
            assert np.array_equal(grid.quaternions, q_mix), spec
            assert grid.stats["energy"] == s_mix["energy"]
        assert s_mix["iteration"] == 10


# (group, N, seed, neighbourhood, tile shape forced or None, precision): the shared gather's
# chord form (O 40k, cutoff 0.27 rad) and arctangent form (O 3000, I 1500: 0.59-0.64 rad),
# a forced tile shape (8 sources per warp, 3 sites per cell), a dense cutoff (C2 2000: every
# image tested), all pairs, and an FP64 engine, which steps alongside the shared launches.
MIX = [("O", 40000, 11, 20.0, None, "fp32"), ("O", 3000, 12, 20.0, None, "fp32"),
       ("I", 1500, 13, 20.0, (8, 3.0), "fp32"), ("D6", 6000, 14, 20.0, (2, 1.5), "fp32"),
       ("C2", 2000, 15, 20.0, None, "fp32"), ("C4", 900, 16, 0.0, None, "fp32"), ("T", 1200, 17, 20.0, None, "fp64")]


def _mix_grid(engine, group, n, seed, delta, tiles, precision):
    g = engine.haar(group, n, seed, precision=precision)
    if tiles:
        g._check(g._lib.zo_near_tiles(g._handle, tiles[0], tiles[1]))
    g._check(g._lib.zo_relax_neighbourhood(g._handle, delta))
    return g


def test_shared_gather_batch_matches_alone(engine):
    """zo_batch_relax with every kind of sample: each result equals its own zo_relax, bit for
    bit, over 12 steps (the first direct, then one graph for the whole batch, replayed), and
    again over a second call (the step after a closing pass)."""
    from zxtalori_b200 import batch

    grids = [_mix_grid(engine, *m) for m in MIX]
    try:
        first = batch.relax_batch(grids, 12)
        q_first = [g.quaternions for g in grids]
        second = batch.relax_batch(grids, 5)
        q_second = [g.quaternions for g in grids]
    finally:
        for g in grids:
            g.close()
    for m, s1, q1, s2, q2 in zip(MIX, first, q_first, second, q_second):
        with _mix_grid(engine, *m) as alone:
            alone.relax(12)
            assert np.array_equal(alone.quaternions, q1), m
            assert alone.stats["energy"] == s1["energy"] and s1["iteration"] == 12
            alone.relax(5)
            assert np.array_equal(alone.quaternions, q2), m
            assert alone.stats["energy"] == s2["energy"] and s2["iteration"] == 17


def test_server_results_same_alone_and_in_mix(engine):
    from zxtalori_b200 import serve

    requests = [serve.Request(k, g, n, 8 + 3 * k, 100 + k, d, arrival=0.01 * k) for k, (g, n, _, d) in enumerate(SAMPLES)]
    mixed = serve.Server(keep_quaternions=True, chunk_seconds=0.001).run(requests)
    assert sorted(r.id for r in mixed) == list(range(len(requests)))
    by_id = {r.id: r for r in mixed}
    for req in requests:
        alone = serve.Server(keep_quaternions=True).run([serve.Request(req.id, req.group, req.count, req.steps, req.seed,
                                                                       req.neighbourhood, 0.0)])[0]
        assert np.array_equal(alone.quaternions, by_id[req.id].quaternions), req
        assert alone.stats["energy"] == by_id[req.id].stats["energy"]
        assert by_id[req.id].stats["iteration"] == req.steps
    info = serve.summary(mixed)
    assert info["requests"] == len(requests) and info["latency_p99_s"] >= info["latency_p50_s"] > 0


def test_served_energy_matches_oracle(engine, ops32):
    from zxtalori_b200 import serve

    req = serve.Request(0, "C4", 900, 6, 77, 0.0)
    res = serve.Server(keep_quaternions=True).run([req])[0]
    q = res.quaternions.astype(np.float64)
    expected = qvm.quick_measures(qvm.pair_rows(q, ops32["C4"]), 4)
    assert res.stats["energy"] == pytest.approx(expected["quey_energy"], rel=1e-6)


def test_plain_one_at_a_time(engine):
    from zxtalori_b200 import serve

    reqs = [serve.Request(0, "O", 1048, 5, 193, 0.0), serve.Request(1, "D3", 800, 4, 5, 0.0, 0.001)]
    res = serve.serve_one_at_a_time(reqs)
    assert [r.id for r in res] == [0, 1]
    assert all(r.stats["arithmetic"] == "fp64" for r in res)


def test_native_server_same_alone_in_mix_and_as_the_python_loop(engine):
    """zo_serve (the loop inside the library): every request completes once with exactly its
    steps; each result's energy and separation are the same served alone, in the mix, and by
    the Python loop (results do not depend on what else runs)."""
    from zxtalori_b200 import serve

    requests = [serve.Request(k, g, n, 8 + 3 * k, 100 + k, d, arrival=0.01 * k) for k, (g, n, _, d) in enumerate(SAMPLES)]
    mixed = serve.NativeServer(chunk_seconds=0.001).run(requests)
    assert sorted(r.id for r in mixed) == list(range(len(requests)))
    by_id = {r.id: r for r in mixed}
    python = {r.id: r for r in serve.Server(chunk_seconds=0.001).run(requests)}
    for req in requests:
        alone = serve.NativeServer().run([serve.Request(req.id, req.group, req.count, req.steps, req.seed,
                                                        req.neighbourhood, 0.0)])[0]
        got = by_id[req.id]
        assert got.stats["iteration"] == req.steps
        assert alone.stats["quey_energy"] == got.stats["quey_energy"] == python[req.id].stats["quey_energy"]
        assert alone.stats["separation_deg"] == got.stats["separation_deg"] == python[req.id].stats["separation_deg"]
        assert got.finished >= got.admitted >= got.arrival - 1e-9
    info = serve.summary(mixed)
    assert info["requests"] == len(requests) and info["pair_evals_per_s"] > 0


def test_native_server_tight_budget_runs_one_at_a_time(engine):
    from zxtalori_b200 import serve

    requests = [serve.Request(k, "O", 2000, 5, k, 0.0) for k in range(4)]
    results = serve.NativeServer(memory_budget=1).run(requests)
    assert sorted(r.id for r in results) == [0, 1, 2, 3]
    spans = sorted((r.admitted, r.finished) for r in results)
    assert all(spans[k + 1][0] >= spans[k][1] - 1e-3 for k in range(3))  # admitted after the last finished
