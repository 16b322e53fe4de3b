"""Properties of the reference's Bloom singleton split, checked on the oracle
(oracle/kc_oracle.c kco_bloom_classify, which restates
src/BloomFilter.h:233-273) on the CPU.

* Order: which occurrence of a k-mer the filter calls FIRST depends on the
  order in which occurrences meet the filter (the reference's threads, the
  GPU's blocks), so the singletons kept as FIRST vary between orders. The
  counts rebuilt from the split are exact in every order: the non-FIRST
  occurrences go to the table and the FIRST ones to their own list
  (src/FastqClassifier.h:533-548), and the precise tools merge that list into
  the table's records, +1 on a hit and a count-1 record on a miss
  (tool/histogram_tool.cpp:735-791).
* Filter block ranges: a k-mer touches only the one block of its prefix's
  filter that its hash selects, so the filter can be cut into ranges of
  consecutive blocks and each range's k-mers classified on their own. Keeping
  the relative order inside every range gives each occurrence the same class
  as the undivided filter. The shared-memory count relies on this: each
  thread block holds one range of blocks and sees only the k-mers that land
  in it."""
import numpy as np
import pytest

import fixtures
import oracle_lib as O

FIRST, ONCE, TWICE = 0, 1, 2   # kco_bloom_classify: first sight, seen once before, seen twice before


def _keys(seed=11, n_reads=400, k=21):
    data = fixtures.random_fastq(seed, n_reads, read_len=(100, 150), genome_len=6000, sub=0.01)
    return O.extract(data, k)


def _blocks(keys, caps):
    return np.array([O.bloom_probe(int(w), int(caps[int(w) >> 56]))[0] for w in keys], np.uint64)


def _rebuild(keys, cls):
    """Counts the reference derives from one classified stream: a table over
    the non-FIRST occurrences, then the FIRST list merged into it."""
    tk, tc = O.count(keys[cls != FIRST])
    fk = keys[cls == FIRST]
    hit = np.isin(fk, tk)
    counts = dict(zip(tk.tolist(), tc.tolist()))
    for w in fk[hit].tolist():
        counts[w] += 1
    low_only = fk[~hit]
    for w in low_only.tolist():
        assert w not in counts
        counts[w] = 1
    return counts, len(low_only)


@pytest.mark.parametrize("cap", [8, 64, 4096])
def test_split_counts_are_exact_in_every_occurrence_order(cap):
    keys = _keys()
    uk, uc = O.count(keys)
    exact = dict(zip(uk.tolist(), uc.tolist()))
    singletons = int(np.count_nonzero(uc == 1))
    caps = np.full(256, cap, np.uint64)
    rng = np.random.default_rng(5)
    low_counts = set()
    for t in range(5):
        ks = keys if t == 0 else keys[rng.permutation(len(keys))]
        cls = O.bloom_classify(ks, caps)
        first = cls == FIRST
        # at most one FIRST per k-mer, and only at its first occurrence in this order
        _, first_pos = np.unique(ks, return_index=True)
        first_occ = np.zeros(len(ks), bool)
        first_occ[first_pos] = True
        assert not np.any(first & ~first_occ)
        counts, low_only = _rebuild(ks, cls)
        assert counts == exact
        # singletons are kept as FIRST or, after a false positive, counted once in the table
        assert low_only <= singletons
        low_counts.add(low_only)
    if cap == 8:
        # a filter this small answers "seen" for many new k-mers, and which ones depends on the order
        assert len(low_counts) > 1


@pytest.mark.parametrize("shift", [0, 2, 4, 6])
def test_classes_are_the_same_when_the_filter_is_cut_into_block_ranges(shift):
    keys = _keys(seed=12)
    rng = np.random.default_rng(shift)
    caps = rng.choice(np.array([64, 128, 256], np.uint64), size=256)
    cls = O.bloom_classify(keys, caps)
    blocks = _blocks(keys, caps)
    prefix = (keys >> np.uint64(56)).astype(np.uint64)
    # range of consecutive blocks: 2^shift blocks each, numbered within the prefix's filter
    sub = prefix * np.uint64(1 << 16) + (blocks >> np.uint64(shift))
    order = np.argsort(sub, kind="stable")
    assert np.array_equal(O.bloom_classify(keys[order], caps), cls[order])
    # the ranges in the opposite order, each still in stream order inside
    order_rev = np.lexsort((np.arange(len(keys)), -sub.astype(np.int64)))
    assert np.array_equal(O.bloom_classify(keys[order_rev], caps), cls[order_rev])


def test_reordering_inside_a_block_range_keeps_counts_exact():
    """Within one range the order matters: a shuffled range gives other
    occurrences the FIRST class, but each k-mer still has at most one FIRST
    occurrence and the counts rebuilt from it stay exact."""
    keys = _keys(seed=13)
    caps = np.full(256, 32, np.uint64)
    blocks = _blocks(keys, caps)
    sub = (keys >> np.uint64(56)) * np.uint64(1 << 16) + (blocks >> np.uint64(3))
    rng = np.random.default_rng(1)
    order = np.lexsort((rng.random(len(keys)), sub))      # ranges in order, shuffled inside each
    ks = keys[order]
    cls = O.bloom_classify(ks, caps)
    counts, _ = _rebuild(ks, cls)
    uk, uc = O.count(keys)
    assert counts == dict(zip(uk.tolist(), uc.tolist()))
    base = O.bloom_classify(keys, caps)[order]
    assert not np.array_equal(cls, base)
    _, first_pos = np.unique(ks, return_index=True)
    first_occ = np.zeros(len(ks), bool)
    first_occ[first_pos] = True
    assert not np.any((cls == FIRST) & ~first_occ)
