"""The fit server: admission (slots, HBM budget, arrival order) with a stand-in for the GPU work
on the CPU, and on the GPU that every request's result is the same alone and in a mix of
concurrent requests of different models and sizes."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from larmor_b200.serve import FitServer


class _FakeJob:
    def __init__(self, name, need, seconds):
        self.name, self.need, self.seconds = name, need, seconds


class _FakeServer(FitServer):
    """Runs each request as a sleep, recording what ran at once."""

    def __init__(self, *a, **k):
        self.lock = threading.Lock()
        self.live = set()
        self.live_bytes = 0
        self.max_live = 0
        self.max_bytes = 0
        self.order = []
        super().__init__(*a, **k)

    def request_bytes(self, job):
        return job.need

    def _run(self, slot, job):
        with self.lock:
            assert slot not in self.live
            self.live.add(slot)
            self.live_bytes += job.need
            self.max_live = max(self.max_live, len(self.live))
            self.max_bytes = max(self.max_bytes, self.live_bytes)
            self.order.append(job.name)
        time.sleep(job.seconds)
        with self.lock:
            self.live.discard(slot)
            self.live_bytes -= job.need
        return {"name": job.name}


def test_admission_respects_slots_budget_and_arrival_order():
    server = _FakeServer(budget_bytes=100, slots=3)
    jobs = [_FakeJob(f"j{i}", need, 0.02) for i, need in enumerate([40, 30, 20, 50, 10, 60, 5, 5])]
    futures = [server.submit(j) for j in jobs]
    results = [f.result(timeout=30) for f in futures]
    server.close()
    assert [r["name"] for r in results] == [j.name for j in jobs]
    assert server.max_live <= 3
    assert server.max_bytes <= 100
    # Arrival order: a request never starts before one that arrived earlier.
    assert server.order == [j.name for j in jobs]
    assert len(server.latencies_ms()) == len(jobs)


def test_requests_overlap_when_they_fit():
    server = _FakeServer(budget_bytes=1000, slots=4)
    futures = [server.submit(_FakeJob(f"j{i}", 10, 0.1)) for i in range(4)]
    for f in futures:
        f.result(timeout=30)
    server.close()
    assert server.max_live == 4


def test_a_request_above_the_budget_is_refused():
    server = _FakeServer(budget_bytes=100, slots=2)
    with pytest.raises(ValueError):
        server.submit(_FakeJob("big", 101, 0.0))
    server.close()


def test_a_failing_request_reaches_its_future_and_frees_its_slot():
    class Failing(_FakeServer):
        def _run(self, slot, job):
            if job.name == "bad":
                raise RuntimeError("fit failed")
            return super()._run(slot, job)

    server = Failing(budget_bytes=100, slots=1)
    bad = server.submit(_FakeJob("bad", 10, 0.0))
    good = server.submit(_FakeJob("good", 10, 0.0))
    with pytest.raises(RuntimeError):
        bad.result(timeout=30)
    assert good.result(timeout=30) == {"name": "good"}
    server.close()


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_a_mix(cuda):
    from larmor_b200.batch import generate_jobs

    jobs = generate_jobs(seed=6, n_volumes=9, min_voxels=500, max_voxels=5000, mix=(1, 1, 1))
    assert {j.kind for j in jobs} == {"dti", "dki", "mfod"}
    alone = []
    server = FitServer(budget_bytes=40 << 30, slots=1)
    for j in jobs:
        alone.append(server.submit(j).result(timeout=600))
    server.close()
    mixed_server = FitServer(budget_bytes=40 << 30, slots=6)
    futures = [mixed_server.submit(j) for j in reversed(jobs)]
    mixed = [f.result(timeout=600) for f in reversed(futures)]
    mixed_server.close()
    assert mixed_server.peak_running > 1
    for j, a, m in zip(jobs, alone, mixed):
        assert a.keys() == m.keys()
        for k in a:
            np.testing.assert_array_equal(a[k], m[k], err_msg=f"{j.kind} {k}")
