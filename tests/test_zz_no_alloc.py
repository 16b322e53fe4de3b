"""kc_sort_records_noalloc: the record sort for callers that cannot allocate
device memory (a fixed device-memory budget owned by another allocator, or a
path that must not stall on an allocation).  It sorts the caller's device
arrays in place with working memory compiled into libkc.so.

The test calls it through the C ABI on device buffers the test owns (the test
may allocate; the entry point must not) and compares with kc_sort_records, the
existing entry point, on two calls in a row -- the second call reuses the same
shared scratch array, so stale contents from the first would show.  Integer
keys: the comparison is exact."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sorted_by_existing_entry_point(kc, keys, counts, bits):
    return kc.sort_records(keys, counts, bits)


# 62 bits: 8 passes of 8 bits; 42: 6; 40: 5 (an odd pass count leaves the
# result in the scratch array, from where it is copied back to the caller's)
@pytest.mark.parametrize("n,bits", [(1 << 20, 62), (300_001, 42), (300_001, 40), (1 << 20, 33)])
def test_noalloc_sort_matches_existing_sort_twice(n, bits):
    import torch
    import ktcountermemorygreedy_b200 as kc

    assert torch.cuda.is_available()
    lib = kc.lib()
    stream = torch.cuda.current_stream()
    # n = 0: the one-time set-up only (array lookup, kernels loaded)
    assert lib.kc_sort_records_noalloc(None, None, 0, bits, C.c_void_p(stream.cuda_stream)) == 0
    for call in range(2):
        rng = np.random.default_rng(1000 * call + bits)
        keys = rng.integers(0, 2**62, size=n, dtype=np.uint64) & np.uint64((1 << bits) - 1)
        keys[: n // 10] = keys[n // 2: n // 2 + n // 10]          # duplicate keys: stability matters
        counts = rng.integers(1, 1 << 30, size=n, dtype=np.uint32)
        want_k, want_c = _sorted_by_existing_entry_point(kc, keys, counts, bits)
        # and independently of the library: numpy's stable sort
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(want_k, keys[order]) and np.array_equal(want_c, counts[order])

        d_keys = torch.from_numpy(keys.view(np.int64)).to("cuda")
        d_counts = torch.from_numpy(counts.view(np.int32)).to("cuda")
        torch.cuda.synchronize()
        rc = lib.kc_sort_records_noalloc(C.c_void_p(d_keys.data_ptr()), C.c_void_p(d_counts.data_ptr()), n, bits,
                                         C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.kc_last_error()
        got_k = d_keys.cpu().numpy().view(np.uint64)
        got_c = d_counts.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_k, want_k), f"call {call}: keys differ"
        assert np.array_equal(got_c, want_c), f"call {call}: counts differ"


def test_noalloc_sort_rejects_too_many_records():
    import ktcountermemorygreedy_b200 as kc
    lib = kc.lib()
    n = (1 << 20) + 1
    rc = lib.kc_sort_records_noalloc(C.c_void_p(16), C.c_void_p(16), n, 62, None)
    assert rc == 1
    assert b"at most" in lib.kc_last_error()
