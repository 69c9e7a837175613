"""CPU tests of the serving scheduler (fastvid_b200.serve.Server) with a
stand-in backend: admission under the memory budget, batching of requests
that arrive while others run, batches of one kind, per-request errors, and
the release of idle workspaces.  The CUDA backend is covered on the GPU by
test_serve_gpu.py."""

import threading
import time

import pytest

from fastvid_b200.serve import Request, Server, percentile


class FakeBackend:
    """Requests carry their sizes; a batch 'runs' for `delay` seconds and
    answers payload * 2 (payload 'bad' fails its batch)."""

    def __init__(self, delay=0.01):
        self.delay = delay
        self.lock = threading.Lock()
        self.peak = 0          # largest accounted device bytes seen at a batch start
        self.server = None
        self.runs = []

    def encode_request(self, payload, ws=10, out=5, pixels=1):
        return Request("encode", payload, {}, pixels, ws, out)

    def decode_request(self, payload, header=None, predictor="wavefront"):
        return Request("decode", payload, {"predictor": predictor}, 1, 10, 5)

    def make_worker_codec(self):
        return {"resident": 0}

    def resident_bytes(self, codec):
        return codec["resident"]

    def release(self, codec):
        codec["resident"] = 0

    def stream(self):
        return None

    def bind(self, stream):
        pass

    def run(self, codec, kind, reqs):
        with self.lock:
            s = self.server
            with s._cv:
                self.peak = max(self.peak, sum(s._resident) + s._inflight)
            self.runs.append((kind, len(reqs)))
        codec["resident"] = max(codec["resident"], sum(r.ws_bytes for r in reqs))
        time.sleep(self.delay)
        if any(r.payload == "bad" for r in reqs):
            raise RuntimeError("frame 0: bad frame")
        return [r.payload * 2 for r in reqs]


def _server(backend, **kw):
    s = Server(backend=backend, **kw)
    backend.server = s
    return s


def test_results_and_batching_of_arrivals_during_a_run():
    b = FakeBackend(delay=0.02)
    with _server(b, memory_budget=10_000, workers=2, max_batch_frames=16) as s:
        first = s.submit_encode(1)
        time.sleep(0.005)  # the first batch is running
        futs = [s.submit_encode(i) for i in range(2, 40)]
        assert first.result(timeout=10) == 2
        assert [f.result(timeout=10) for f in futs] == [2 * i for i in range(2, 40)]
    sizes = [n for _, n in s.batches]
    assert sum(sizes) == 39
    assert max(sizes) > 1            # arrivals were batched
    assert max(sizes) <= 16
    assert s.max_concurrent == 2     # two batches on the device at once


def test_batches_hold_one_kind():
    b = FakeBackend(delay=0.005)
    with _server(b, workers=1) as s:
        futs = [s.submit_encode(i) if i % 2 else s.submit_decode(i) for i in range(30)]
        assert [f.result(timeout=10) for f in futs] == [2 * i for i in range(30)]
    assert len(b.runs) >= 2
    assert all(kind in ("encode", "decode") for kind, _ in b.runs)


def test_budget_bounds_what_is_on_the_device():
    b = FakeBackend(delay=0.005)
    # each request: 10 workspace + 5 output; 40 bytes admit two at a time
    # beside one other worker's workspace
    with _server(b, memory_budget=40, workers=3, max_batch_frames=64) as s:
        futs = [s.submit_encode(i) for i in range(60)]
        assert [f.result(timeout=20) for f in futs] == [2 * i for i in range(60)]
    assert b.peak <= 40
    assert max(n for _, n in s.batches) <= 2


def test_request_above_the_budget_is_rejected():
    b = FakeBackend()
    with _server(b, memory_budget=100, workers=1) as s:
        big = s.submit_encode(1, ws=90, out=20)
        with pytest.raises(MemoryError, match="above the server budget"):
            big.result(timeout=5)
        assert s.submit_encode(3).result(timeout=5) == 6


def test_failing_request_fails_alone():
    b = FakeBackend(delay=0.01)
    with _server(b, workers=1, max_batch_frames=8) as s:
        s.submit_encode(0)  # keep the worker busy so the next ones batch
        futs = [s.submit_encode(i) for i in (1, 2)] + [s.submit_encode("bad")] + [s.submit_encode(i) for i in (3, 4)]
        with pytest.raises(RuntimeError, match="bad frame"):
            futs[2].result(timeout=10)
        assert [futs[i].result(timeout=10) for i in (0, 1, 3, 4)] == [2, 4, 6, 8]


def test_idle_workspaces_are_released_for_a_large_request():
    b = FakeBackend(delay=0.002)
    with _server(b, memory_budget=100, workers=3, max_batch_frames=1) as s:
        # grow every worker's resident workspace to 30
        futs = [s.submit_encode(i, ws=30, out=1) for i in range(9)]
        for f in futs:
            f.result(timeout=10)
        # 80 + 10 fits an empty server but not beside two idle 30s
        assert s.submit_encode(5, ws=80, out=10).result(timeout=10) == 10


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert percentile(v, 50) == 50
    assert percentile(v, 99) == 99
    assert percentile([7.0], 99) == 7.0


def test_open_loop_driver_reports_every_request():
    from fastvid_b200.serve import report, run_open_loop

    b = FakeBackend(delay=0.002)
    with _server(b, workers=2) as s:
        items = [("encode", i, {}) for i in range(50)] + [("decode", 7, {})]
        recs, t0, kept = run_open_loop(s, items, rate=5000, seed=3, keep=(0, 50))
    assert len(recs) == 51 and all(r.ok for r in recs)
    assert kept == {0: 0, 50: 14}
    rep = report(recs, t0)
    assert rep["requests"] == 51 and rep["failed"] == 0
    assert 0 < rep["p50_ms"] <= rep["p99_ms"] <= rep["max_ms"]


class BrokenBackend(FakeBackend):
    def make_worker_codec(self):
        raise RuntimeError("no device")


def test_worker_failure_fails_requests_instead_of_hanging():
    b = BrokenBackend()
    s = Server(backend=b, workers=1)
    b.server = s
    for t in s._threads:
        t.join(timeout=5)
    with pytest.raises(RuntimeError, match="serving worker failed"):
        s.submit_encode(1)
    s.close()
