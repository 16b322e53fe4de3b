"""Host logic of the request loop (ktcountermemorygreedy_b200.serving), with a
fake counter in place of the GPU handle: requests are submitted at their
arrival times, results are collected in arrival order, latency is the
scheduled arrival to the job's end, and a failing request is reported
without stopping the others."""
import threading
import time
from types import SimpleNamespace

import numpy as np

from ktcountermemorygreedy_b200 import serving


class FakeCounter:
    """Runs each job on a thread for `service_ms`, one worker at a time."""

    def __init__(self, service_ms=5.0, fail_k=None):
        self.service_ms = service_ms
        self.fail_k = fail_k
        self.jobs = {}
        self.next = 1
        self.lock = threading.Lock()
        self.worker = threading.Lock()
        self.submit_times = []

    def submit(self, files, k, **kw):
        if k == self.fail_k:
            raise RuntimeError("KC_ERR_INVALID: k must be in 1..32")
        with self.lock:
            jid = self.next
            self.next += 1
        t_sub = time.perf_counter()
        self.submit_times.append(t_sub)
        done = threading.Event()
        rec = {"t_sub": t_sub, "done": done, "k": k, "n": sum(len(f) for f in files)}
        self.jobs[jid] = rec

        def run():
            with self.worker:
                rec["t_start"] = time.perf_counter()
                if not rec.get("cancel"):
                    time.sleep(self.service_ms / 1000.0)
                rec["t_end"] = time.perf_counter()
            done.set()

        threading.Thread(target=run, daemon=True).start()
        return jid

    def wait(self, jid):
        self.jobs[jid]["done"].wait()
        if self.jobs[jid].get("cancel"):
            raise RuntimeError("KC_ERR_CANCELLED: cancelled")

    def cancel(self, jid):
        r = self.jobs[jid]
        if r["done"].is_set():
            return False
        r["cancel"] = True   # a job not yet on the worker is dropped when its turn comes
        return True

    def result(self, jid, k, copy=True):
        r = self.jobs[jid]
        return SimpleNamespace(queue_ms=1000 * (r["t_start"] - r["t_sub"]), run_ms=1000 * (r["t_end"] - r["t_start"]),
                               device_ms=self.service_ms,
                               occurrences=r["n"], distinct=r["n"] // 2, le2_keys=np.zeros(3, np.uint64),
                               hist=np.array([1, 2, 3]))


def test_requests_submitted_at_arrival_times_and_latency_accounted():
    fc = FakeCounter(service_ms=20.0)
    reqs = [serving.Request(0.01 * i, [b"x" * (100 + i)], 31) for i in range(8)]
    t0 = time.perf_counter()
    stats, wall = serving.serve(fc, reqs)
    assert len(stats) == 8 and all(not s.error for s in stats)
    # submissions follow the schedule (never early)
    for i, ts in enumerate(fc.submit_times):
        assert ts - t0 >= 0.01 * i - 1e-3
    # one 20 ms worker for jobs 10 ms apart: queueing grows, latency >= service time
    assert all(s.latency_ms >= 19.0 for s in stats)
    assert stats[-1].queue_ms > stats[0].queue_ms
    assert wall >= 8 * 0.020 - 0.005
    summ = serving.summarize(stats, wall)
    assert summ["jobs"] == 8 and summ["failed"] == 0
    assert summ["p50_ms"] <= summ["p99_ms"]
    assert summ["occurrences"] == sum(100 + i for i in range(8))


def test_failed_request_is_reported_and_others_complete():
    fc = FakeCounter(service_ms=1.0, fail_k=33)
    reqs = [serving.Request(0.0, [b"ab"], 31), serving.Request(0.001, [b"abc"], 33),
            serving.Request(0.002, [b"abcd"], 21)]
    stats, wall = serving.serve(fc, reqs)
    assert not stats[0].error and not stats[2].error
    assert "k must be" in stats[1].error
    summ = serving.summarize(stats, wall)
    assert summ["failed"] == 1 and summ["occurrences"] == 2 + 4


def test_results_collected_in_arrival_order_when_listed_out_of_order():
    fc = FakeCounter(service_ms=1.0)
    reqs = [serving.Request(0.004, [b"late"], 31), serving.Request(0.0, [b"e"], 31)]
    stats, _ = serving.serve(fc, reqs)
    assert stats[0].occurrences == 4 and stats[1].occurrences == 1
    assert fc.submit_times[0] <= fc.submit_times[1]


def test_request_past_its_deadline_is_cancelled_and_others_complete():
    """One 30 ms worker, five jobs arriving together: the fourth has a 40 ms
    deadline and is still queued then, so it is cancelled (and reported as
    such); the others complete with their results."""
    fc = FakeCounter(service_ms=30.0)
    reqs = [serving.Request(0.0, [b"x" * (10 + i)], 31, deadline_ms=(40.0 if i == 3 else None)) for i in range(5)]
    stats, wall = serving.serve(fc, reqs)
    assert "cancelled at its deadline" in stats[3].error
    assert all(not stats[i].error for i in (0, 1, 2, 4))
    assert [stats[i].occurrences for i in (0, 1, 2, 4)] == [10, 11, 12, 14]
    summ = serving.summarize(stats, wall)
    assert summ["failed"] == 1
