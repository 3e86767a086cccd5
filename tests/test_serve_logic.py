"""Host logic of the continuous-batching server, with a fake engine in place of the GPU:
admission in arrival order within the memory budget and the concurrency cap, a request
larger than the budget still served when nothing else is resident, every request relaxed
for exactly its steps, and the Poisson workload generator's shape."""
import numpy as np
import pytest

from zxtalori_b200 import serve


class FakeLib:
    def __init__(self, log):
        self.log = log

    def zo_idle(self, h):
        return 1

    def zo_relax_async(self, h, k):
        h.done += k
        self.log.append(("steps", h.request_id, k))
        return 0

    def zo_relax_finish(self, h):
        self.log.append(("finish", h.request_id))
        return 0

    def zo_measure(self, h):
        self.log.append(("measure", h.request_id))
        return 0

    def zo_device_bytes(self, h):
        return serve.estimate_bytes(h.count, h.group, h.neighbourhood)


class FakeGrid:
    live = 0
    most_live = 0

    def __init__(self, request_id, count, group, log):
        self._handle = self
        self._lib = FakeLib(log)
        self.request_id = request_id
        self.count = count
        self.group = group
        self.done = 0
        self.neighbourhood = 0.0
        FakeGrid.live += 1
        FakeGrid.most_live = max(FakeGrid.most_live, FakeGrid.live)

    def _check(self, rc):
        assert rc == 0

    @property
    def stats(self):
        return {"count": self.count, "order": serve.ORDER[self.group], "iteration": self.done,
                "relax_neighbourhood": self.neighbourhood or None}

    @property
    def quaternions(self):
        return np.zeros((self.count, 4), np.float32)

    def close(self):
        FakeGrid.live -= 1


class Clock:
    """Advances 1 ms on every reading, so the loop's waits end."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


@pytest.fixture
def fake(monkeypatch):
    log = []
    FakeGrid.live = 0
    FakeGrid.most_live = 0
    ids = {}

    def haar(group, count, seed, precision="fp32"):
        return FakeGrid(ids[seed], count, group, log)

    def neighbourhood(h, delta):
        h.neighbourhood = delta
        return 0

    monkeypatch.setattr(serve, "haar", haar)
    monkeypatch.setattr(FakeLib, "zo_relax_neighbourhood", lambda self, h, d: neighbourhood(h, d), raising=False)
    return log, ids


def _requests(ids, specs):
    out = []
    for k, (group, count, steps, delta, arrival) in enumerate(specs):
        seed = 1000 + k
        ids[seed] = k
        out.append(serve.Request(k, group, count, steps, seed, delta, arrival))
    return out


def test_every_request_runs_exactly_its_steps(fake):
    log, ids = fake
    reqs = _requests(ids, [("O", 2000, 37, 0.0, 0.0), ("I", 800, 5, 0.0, 0.002), ("C2", 9000, 120, 20.0, 0.004)])
    results = serve.Server(memory_budget=1 << 40, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert sorted(r.id for r in results) == [0, 1, 2]
    for r in results:
        assert r.stats["iteration"] == reqs[r.id].steps
        assert r.finished >= r.admitted >= r.arrival
    # Each sample is finished and measured once, after all its steps.
    for k in range(3):
        events = [e for e in log if e[1] == k]
        assert events[-2:] == [("finish", k), ("measure", k)]
        assert sum(e[2] for e in events if e[0] == "steps") == reqs[k].steps
    assert FakeGrid.live == 0


def test_admission_respects_budget_and_cap(fake):
    log, ids = fake
    specs = [("O", 3000, 10, 0.0, 0.0) for _ in range(6)]
    reqs = _requests(ids, specs)
    one = serve.estimate_bytes(3000, "O", 0.0)
    serve.Server(memory_budget=2 * one + one // 2, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert FakeGrid.most_live == 2
    FakeGrid.most_live = 0
    log.clear()
    ids.clear()
    reqs = _requests(ids, specs)
    serve.Server(memory_budget=1 << 40, max_active=3, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert FakeGrid.most_live == 3


def test_admission_uses_the_engines_reported_bytes(fake, monkeypatch):
    """Once a sample's workspace is sized, admission counts the bytes its engine reports:
    engines that hold twice their estimate leave room for fewer samples."""
    log, ids = fake
    specs = [("O", 3000, 200, 0.0, 0.01 * k) for k in range(6)]
    one = serve.estimate_bytes(3000, "O", 0.0)
    reqs = _requests(ids, specs)
    serve.Server(memory_budget=3 * one, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert FakeGrid.most_live == 3
    monkeypatch.setattr(FakeLib, "zo_device_bytes", lambda self, h: 2 * one)
    FakeGrid.most_live = 0
    ids.clear()
    reqs = _requests(ids, specs)
    results = serve.Server(memory_budget=3 * one, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert FakeGrid.most_live == 2 and len(results) == 6


def test_oversize_request_runs_alone(fake):
    log, ids = fake
    reqs = _requests(ids, [("O", 50_000, 4, 20.0, 0.0), ("T", 1000, 4, 0.0, 0.0)])
    results = serve.Server(memory_budget=1, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert sorted(r.id for r in results) == [0, 1]
    assert FakeGrid.most_live == 1


def test_admission_follows_arrival_order(fake):
    log, ids = fake
    reqs = _requests(ids, [("O", 1000, 3, 0.0, 0.05), ("O", 1000, 3, 0.0, 0.01), ("O", 1000, 3, 0.0, 0.03)])
    results = serve.Server(memory_budget=1, chunk_seconds=1e-6).run(reqs, clock=Clock())
    assert [r.id for r in results] == [1, 2, 0]
    assert all(r.admitted >= r.arrival for r in results)


def test_poisson_workload_shape():
    reqs = serve.poisson_requests(2.0, 200.0, seed=3)
    again = serve.poisson_requests(2.0, 200.0, seed=3)
    assert [(r.group, r.count, r.steps, r.seed, r.arrival) for r in reqs] == \
        [(r.group, r.count, r.steps, r.seed, r.arrival) for r in again]
    assert 300 < len(reqs) < 500  # 400 expected
    arrivals = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arrivals) > 0) and arrivals[-1] <= 200.0
    assert {r.group for r in reqs} <= set(serve.ORDER)
    assert all(500 <= r.count <= 1_000_000 and 10 <= r.steps <= 200 for r in reqs)
    assert all((r.neighbourhood == 0.0) == (r.count < 5000) for r in reqs)
    logs = np.log([r.count for r in reqs])
    assert abs(np.median(logs) - 0.5 * (np.log(500) + np.log(1e6))) < 0.6  # log-uniform


def test_summary_counts_pairs_as_the_reference():
    res = [serve.Result(0, 0.0, 0.0, 2.0, {"count": 1000, "order": 24, "iteration": 10, "relax_neighbourhood": None}),
           serve.Result(1, 1.0, 1.0, 4.0, {"count": 100_000, "order": 24, "iteration": 5, "relax_neighbourhood": 20.0})]
    info = serve.summary(res)
    evals = 11 * 1000 * 1000 * 24 + 6 * 100_000 * min(100_000 * 24, 0.94 * 20 ** 3 + 64)
    assert info["pair_evals_per_s"] == pytest.approx(evals / 4.0)
    assert info["requests"] == 2
    assert info["latency_p50_s"] == pytest.approx(2.5)


def test_batch_shards_cover_every_sample_once_and_balance():
    from zxtalori_b200 import batch

    specs = batch.random_samples(256)
    work_of = {s.seed: batch.pair_evals(s.count, serve.ORDER[s.group], s.neighbourhood, 50) for s in specs}
    for world in (1, 2, 3, 8):
        shares = [batch.shard(specs, r, world) for r in range(world)]
        assert sorted(s.seed for share in shares for s in share) == list(range(256))
        work = [sum(work_of[s.seed] for s in share) for share in shares]
        assert max(work) <= sum(work) / world + max(work_of.values())  # greedy balance bound
        assert shares == [batch.shard(specs, r, world) for r in range(world)]  # the same split on every rank
    with pytest.raises(ValueError):
        batch.shard(specs, 2, 2)


class FakeServeLib:
    """Stands in for the library's zo_serve: checks what NativeServer passes and answers
    with one result per request, in reverse order (completion order is not arrival order)."""

    _serve_bound = True  # the argument types are the real library's business

    def __init__(self, fail_id=None):
        self.fail_id = fail_id
        self.seen = None

    def zo_serve(self, requests, n, settings, n_settings, results, error, error_len):
        self.seen = ([(requests[k].id, requests[k].group, requests[k].count, requests[k].steps, requests[k].seed,
                       requests[k].neighbourhood, requests[k].arrival) for k in range(n)],
                     [settings[k] for k in range(n_settings)])
        for slot, k in enumerate(reversed(range(n))):
            r = results[slot]
            r.id, r.count, r.order, r.iteration = requests[k].id, requests[k].count, 24, requests[k].steps
            r.arrival, r.admitted, r.finished = requests[k].arrival, requests[k].arrival + 0.5, requests[k].arrival + 1.0
            r.neighbourhood, r.energy, r.separation_deg = requests[k].neighbourhood, 1.5, 2.0
            r.status = -1 if requests[k].id == self.fail_id else 0
            if r.status:
                r.error = b"Measure: Cancelled"
        return 0


def test_native_server_marshals_requests_settings_and_results(monkeypatch):
    """NativeServer (the Python face of zo_serve) passes each request and its settings as the
    header lays them out and turns the records back into results; a failed request raises."""
    fake = FakeServeLib()
    monkeypatch.setattr(serve, "_library", lambda: fake)
    reqs = [serve.Request(7, "O", 2000, 30, 5, 20.0, 0.25), serve.Request(9, "I", 600, 10, 6, 0.0, 1.5)]
    out = serve.NativeServer(memory_budget=1 << 30, max_active=8, workers=2).run(reqs)
    passed, settings = fake.seen
    assert passed == [(7, serve.GROUPS.index("O"), 2000, 30, 5, 20.0, 0.25), (9, serve.GROUPS.index("I"), 600, 10, 6,
                                                                             0.0, 1.5)]
    assert settings == [float(1 << 30), 8.0, 0.02, 1.0, 0.0, 2.0, 2.5e11]
    assert [r.id for r in out] == [9, 7]
    assert out[1].stats == {"count": 2000, "order": 24, "iteration": 30, "relax_neighbourhood": 20.0,
                            "quey_energy": 1.5, "separation_deg": 2.0}
    assert out[0].stats["relax_neighbourhood"] is None  # all pairs
    assert (out[1].arrival, out[1].admitted, out[1].finished) == (0.25, 0.75, 1.25)
    monkeypatch.setattr(serve, "_library", lambda: FakeServeLib(fail_id=9))
    with pytest.raises(RuntimeError, match="request 9: Measure: Cancelled"):
        serve.NativeServer().run(reqs)
