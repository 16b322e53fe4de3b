"""Failure detection on the GPU, in forms that fault, trap or hang nothing.

Each failure is forced through kc_job.fault_inject and takes the path a real
failure of its kind takes: a device wait that runs out (a bounded poll of a
flag nothing sets, about a millisecond) sets the wait-timeout flag and the
job ends KC_ERR_DEVICE; a table that reports itself full is regrown or split
and counted again (exact results) or, every time, ends the job after its
retries; a device allocation that fails ends the job KC_ERR_NOMEM.  After
every failure the same handle counts a job exactly, so the context and the
handle stay usable.  Cancellation (kc_cancel) of queued, running and served
jobs leaves the other jobs' results unchanged.  Integer work: exact
comparisons against the oracle."""
import time

import numpy as np
import pytest

import fixtures
import oracle_lib as O

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


@pytest.fixture(scope="module")
def kc():
    import ktcountermemorygreedy_b200 as kc
    return kc


@pytest.fixture(scope="module")
def data():
    return fixtures.plain_small()


@pytest.fixture(scope="module")
def want(data):
    return O.exact_records([data], 31)


def _exact(r, want):
    return np.array_equal(r.keys, want[0]) and np.array_equal(r.counts, want[1])


def test_device_wait_that_runs_out_ends_the_job_with_a_status(kc, data, want):
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        with pytest.raises(kc.KcError) as e:
            c.count([data], k=31, count_max=U32, fault_inject=kc.INJECT_WAIT_TIMEOUT)
        assert e.value.code == 6 and "bounded wait expired" in str(e.value)
        assert _exact(c.count([data], k=31, count_max=U32), want)   # the context is usable


def test_table_full_once_is_regrown_with_exact_results(kc, data, want):
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        r = c.count([data], k=31, count_max=U32, fault_inject=kc.INJECT_TABLE_FULL_ONCE)
        assert _exact(r, want)
        # Bloom job, shared-memory sub-buckets: the first bucket is split and counted again
        m = want[1] >= 2
        rb = c.count([data], k=31, count_max=U32, bloom=True, memory_gb=1, min_count=2,
                     fault_inject=kc.INJECT_TABLE_FULL_ONCE)
        assert np.array_equal(rb.keys, want[0][m]) and np.array_equal(rb.counts, want[1][m])
        assert rb.smem_passes == 1


def test_table_full_every_time_fails_after_retries(kc, data, want):
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        with pytest.raises(kc.KcError) as e:
            c.count([data], k=31, count_max=U32, fault_inject=kc.INJECT_TABLE_FULL)
        assert e.value.code == 6 and "counting table overflow" in str(e.value)
        assert _exact(c.count([data], k=31, count_max=U32), want)


def test_failed_device_allocation_ends_the_job_with_nomem(kc, data, want):
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        with pytest.raises(kc.KcError) as e:
            c.count([data], k=31, count_max=U32, fault_inject=kc.INJECT_NOMEM)
        assert e.value.code == 3
        assert _exact(c.count([data], k=31, count_max=U32), want)


def test_cancelled_queued_job_leaves_the_others_exact(kc, data, want):
    big = fixtures.random_fastq(7, 60000, (150, 150), genome_len=2_000_000, sub=0.01, n_rate=0.0)
    big_want = O.exact_records([big], 25)
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        a = c.submit([big], k=25, count_max=U32)
        b = c.submit([data], k=31, count_max=U32)
        cj = c.submit([data], k=31, count_max=U32)
        took = c.cancel(cj)
        if took:
            with pytest.raises(kc.KcError) as e:
                c.wait(cj)
            assert e.value.code == kc.KC_ERR_CANCELLED
        else:   # it had finished already: its results stand
            c.wait(cj)
            assert _exact(c.result(cj, 31), want)
        c.wait(a)
        ra = c.result(a, 25)
        assert np.array_equal(ra.keys, big_want[0]) and np.array_equal(ra.counts, big_want[1])
        c.wait(b)
        assert not c.cancel(b)   # finished: nothing to cancel
        assert _exact(c.result(b, 31), want)


def test_cancelled_running_job_gives_back_its_memory(kc, data, want):
    big = fixtures.random_fastq(8, 60000, (150, 150), genome_len=2_000_000, sub=0.01, n_rate=0.0)
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        for _ in range(3):
            j = c.submit([big], k=31, count_max=U32, bloom=True, memory_gb=2, min_count=2)
            time.sleep(0.002)
            if c.cancel(j):
                with pytest.raises(kc.KcError) as e:
                    c.wait(j)
                assert e.value.code == kc.KC_ERR_CANCELLED
            else:
                c.wait(j)
                c.release(j)
        assert _exact(c.count([data], k=31, count_max=U32), want)


def test_served_jobs_past_their_deadline_are_cancelled_others_same_as_alone(kc):
    from ktcountermemorygreedy_b200 import serving
    files = [fixtures.random_fastq(20 + i, 3000 + 500 * i, (150, 150), genome_len=200_000, sub=0.01, n_rate=0.0)
             for i in range(6)]
    job = dict(count_max=U32, min_count=1, hist_min=1, hist_max=1000)
    with kc.KmerCounter(max_inflight_jobs=2) as c:
        alone = [c.count([f], k=21, **job) for f in files]
        # request 4 has a deadline it cannot meet (0 ms): it is cancelled, queued or running
        reqs = [serving.Request(0.001 * i, [f], 21, dict(job, keep_records=True),
                                deadline_ms=(0.0 if i == 4 else None)) for i, f in enumerate(files)]
        stats, _ = serving.serve(c, reqs)
    for i, s in enumerate(stats):
        if i == 4 and s.error:
            assert "cancelled at its deadline" in s.error
            continue
        assert not s.error, s.error
        assert s.occurrences == alone[i].occurrences and s.distinct == alone[i].distinct
        assert s.hist_sum == int(alone[i].hist.sum())
