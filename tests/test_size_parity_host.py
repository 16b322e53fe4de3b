"""The at-size parity checks of tests/size_parity.py, on the CPU: the oracle's
exact records pass them, and records with a planted mistake (two records
swapped, one count changed) fail them.  The mistakes are planted in copies of
the oracle's output."""
import numpy as np
import pytest

import fixtures
import oracle_lib as O
import size_parity as SP


@pytest.fixture(scope="module")
def fq():
    return fixtures.random_fastq(3, 20000, (150, 150), genome_len=300000, sub=0.01, n_rate=0.0)


def _hist(counts, lo, hi):
    return np.bincount(counts, minlength=hi + 1)[lo: hi + 1].astype(np.int64)


def test_spot_check_kmer1(fq):
    buf = np.frombuffer(fq, np.uint8)
    uk, uc = O.count(O.extract(fq, 31))
    keys, counts = O.sort_string_order(uk[uc >= 2], uc[uc >= 2], 31)
    hist = _hist(uc, 2, 1000)
    r = SP.full_spot_check(buf, 31, keys, counts, hist, 2, 2, threads=4, sample_bits=4)
    assert r["identical"] and r["sampled_kmers"] > 1000
    k2 = keys.copy()
    k2[[10, 11]] = k2[[11, 10]]
    assert not SP.full_spot_check(buf, 31, k2, counts, hist, 2, 2, threads=4, sample_bits=4)["records_sorted"]
    c2 = counts.copy()
    c2[O.sampled_mask(keys, 4).nonzero()[0][0]] += 1
    r = SP.full_spot_check(buf, 31, keys, c2, hist, 2, 2, threads=4, sample_bits=4)
    assert not r["sampled_records_identical"] and not r["hist_equals_records_hist"]


@pytest.mark.parametrize("k", [45, 100])
def test_spot_check_wide(fq, k):
    buf = np.frombuffer(fq, np.uint8)
    keys, counts = O.exact_records_wide([fq], k, min_count=2)
    _, uc = O.count_wide(O.extract_wide(fq, k))
    hist = _hist(uc, 2, 1000)
    r = SP.full_spot_check_wide(buf, k, keys, counts, hist, 2, 2, threads=4, sample_bits=4)
    assert r["identical"] and r["sampled_kmers"] > 1000
    k2 = keys.copy()
    k2[[10, 11]] = k2[[11, 10]]
    assert not SP.full_spot_check_wide(buf, k, k2, counts, hist, 2, 2, threads=4, sample_bits=4)["records_sorted"]
    c2 = counts.copy()
    c2[((O.sample_hash_wide_np(keys) & np.uint64(15)) == 0).nonzero()[0][0]] += 1
    r = SP.full_spot_check_wide(buf, k, keys, c2, hist, 2, 2, threads=4, sample_bits=4)
    assert not r["sampled_records_identical"] and not r["hist_equals_records_hist"]
    # the folded sample hash of the oracle's C code and of numpy agree
    one = np.ascontiguousarray(keys[:50])
    for i in range(len(one)):
        assert O.lib().kco_sample_hash_wide(O.P(np.ascontiguousarray(one[i])), one.shape[1]) == \
            int(O.sample_hash_wide_np(one[i:i + 1])[0])
