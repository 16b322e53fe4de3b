"""Request loop for served counting jobs.

Requests arrive at their own times (a Poisson process in the benchmark) and
are submitted to a KmerCounter handle as they arrive.  The handle's workers
admit queued jobs in FIFO order as soon as a worker stream and enough of the
device-memory budget are free, so a request that arrives while others are on
the GPU starts without waiting for them to finish and its kernels overlap with
theirs.  Each job's partitions and table stay on the device for the length of
the job; its histogram and queries (and, when asked for, its sorted records)
come back to pinned host memory.

serve() returns one RequestStats per request (latency from the scheduled
arrival to the end of the job, host clock) and the wall time of the stream.
A request with a deadline that has not finished by then is cancelled
(``kc_cancel``: taken off the queue, or stopped at its next stage boundary
with its device memory given back) and reported with an error; the other
jobs are not affected.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np


@dataclass
class Request:
    arrival_s: float                 # seconds after the stream starts
    files: Sequence                  # FASTQ buffers (bytes or uint8 arrays), kept alive by the caller
    k: int
    job: dict = field(default_factory=dict)   # further KmerCounter.submit keywords
    deadline_ms: float | None = None          # cancelled when not done this long after its arrival


@dataclass
class RequestStats:
    latency_ms: float                # scheduled arrival -> job end
    queue_ms: float                  # submission -> start on a worker
    run_ms: float                    # start -> end
    submit_late_ms: float            # actual submission - scheduled arrival
    device_ms: float                 # device time of the job's pipeline
    passes: int                      # counting passes (more than one when the device was short of memory)
    occurrences: int
    distinct: int
    n_le2: int
    hist_sum: int
    error: str = ""


def serve(counter, requests: Sequence[Request]):
    """Submits every request at its arrival time, waits for all, returns
    (stats in request order, wall seconds from the first arrival to the last
    job end)."""
    order = sorted(range(len(requests)), key=lambda i: requests[i].arrival_s)
    ids: List[int] = [0] * len(requests)
    late = [0.0] * len(requests)
    submitted = [threading.Event() for _ in requests]
    errors: List[str] = [""] * len(requests)
    t0 = time.perf_counter()

    def submitter():
        for i in order:
            r = requests[i]
            delay = t0 + r.arrival_s - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            late[i] = 1000.0 * (time.perf_counter() - t0 - r.arrival_s)
            try:
                ids[i] = counter.submit(r.files, k=r.k, **r.job)
            except Exception as e:   # reported per request
                errors[i] = str(e)
            submitted[i].set()

    th = threading.Thread(target=submitter, daemon=True)
    th.start()

    # deadlines: a watchdog cancels every job still unfinished at its deadline
    collected = set()
    lock = threading.Lock()
    cancelled = set()
    timed = sorted((requests[i].arrival_s * 1000.0 + requests[i].deadline_ms, i) for i in range(len(requests))
                   if requests[i].deadline_ms is not None)
    stop = threading.Event()

    def watchdog():
        for when, i in timed:
            delay = t0 + when / 1000.0 - time.perf_counter()
            if delay > 0 and stop.wait(delay):
                return
            submitted[i].wait()
            with lock:
                if i in collected or errors[i]:
                    continue
                try:
                    if counter.cancel(ids[i]):
                        cancelled.add(i)
                except Exception:   # finished and released meanwhile
                    pass

    wd = threading.Thread(target=watchdog, daemon=True)
    wd.start()
    stats: List[RequestStats] = [None] * len(requests)
    end_max = 0.0
    for i in order:
        submitted[i].wait()
        r = requests[i]
        if errors[i]:
            stats[i] = RequestStats(math.nan, 0, 0, late[i], 0, 0, 0, 0, 0, 0, errors[i])
            continue
        try:
            counter.wait(ids[i])
            with lock:
                collected.add(i)
            res = counter.result(ids[i], r.k, copy=False)
        except Exception as e:
            with lock:
                collected.add(i)
            msg = str(e)
            if i in cancelled:
                msg = f"cancelled at its deadline ({r.deadline_ms} ms): {msg}"
            stats[i] = RequestStats(math.nan, 0, 0, late[i], 0, 0, 0, 0, 0, 0, msg)
            continue
        lat = late[i] + res.queue_ms + res.run_ms
        end_max = max(end_max, r.arrival_s * 1000.0 + lat)
        stats[i] = RequestStats(lat, res.queue_ms, res.run_ms, late[i], res.device_ms, int(getattr(res, "passes", 1)),
                                int(res.occurrences),
                                int(res.distinct),
                                int(len(res.le2_keys)), int(np.asarray(res.hist).sum()))
        del res
    th.join()
    stop.set()
    wd.join()
    first = min((r.arrival_s for r in requests), default=0.0)
    return stats, max(end_max / 1000.0 - first, 1e-9)


def summarize(stats: Sequence[RequestStats], wall_s: float) -> dict:
    ok = [s for s in stats if not s.error]
    lat = np.array([s.latency_ms for s in ok]) if ok else np.zeros(1)
    occ = sum(s.occurrences for s in ok)
    return {"jobs": len(stats), "failed": len(stats) - len(ok),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "kmers_per_s": occ / wall_s, "wall_s": wall_s, "occurrences": occ,
            "mean_queue_ms": float(np.mean([s.queue_ms for s in ok])) if ok else 0.0,
            "mean_run_ms": float(np.mean([s.run_ms for s in ok])) if ok else 0.0,
            "mean_device_ms": float(np.mean([s.device_ms for s in ok])) if ok else 0.0,
            "multi_pass_jobs": sum(1 for s in ok if s.passes > 1)}
