"""Parity of the CUDA path (libkc.so, called through the C ABI) with the oracle
and with the golden outputs of the reference's own programs.  Integer work:
every comparison is exact."""
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fixtures
import oracle_lib as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))
U32 = 0xFFFFFFFF


@pytest.fixture(scope="module")
def kc():
    import ktcountermemorygreedy_b200 as kc
    return kc


@pytest.fixture(scope="module")
def counter(kc):
    c = kc.KmerCounter(max_inflight_jobs=4)
    yield c
    c.close()


def _case_files(name):
    for n, files, _ in fixtures.E2E_CASES:
        if n == name:
            return files
    raise KeyError(name)


def test_hashes_bit_exact(kc):
    keys = np.array([int(r[0], 16) for r in GOLDEN["hashes"]], np.uint64)
    h = kc.hash_kmers(keys)
    for row, got in zip(GOLDEN["hashes"], h):
        assert [int(x) for x in got] == [int(row[1], 16), int(row[2], 16), int(row[3], 16), int(row[4], 16),
                                         int(row[5], 16)]


def test_extract_matches_getkmer_golden(kc):
    for case in GOLDEN["getkmer"]:
        bases = case["bases"]
        fq = f"@x\n{bases}\n+\n{'I' * len(bases)}\n".encode()
        got = np.sort(kc.extract_kmers(fq, case["k"]))
        want = np.sort(np.array([int(x, 16) for x in case["canonical"]], np.uint64))
        assert got.tolist() == want.tolist(), case["k"]


@pytest.mark.parametrize("name", [c[0] for c in fixtures.E2E_CASES])
@pytest.mark.parametrize("k", [1, 5, 11, 16, 21, 25, 31, 32])
def test_extract_matches_oracle(kc, name, k):
    for f in _case_files(name):
        got = np.sort(kc.extract_kmers(f, k))
        want = np.sort(O.extract(f, k))
        assert len(got) == len(want)
        assert np.array_equal(got, want)


def test_extract_empty_and_tiny(kc):
    assert len(kc.extract_kmers(b"", 21)) == 0
    assert len(kc.extract_kmers(b"@a\n", 21)) == 0
    assert kc.extract_kmers(b"@a\nACGTA", 5).tolist() == O.extract(b"@a\nACGTA", 5).tolist()
    # exactly one tile, and one byte more
    for n in (8192 - 7, 8192, 8193, 3 * 8192 + 5):
        seq = ("ACGT" * (n // 4 + 1))[: max(0, n - 12)]
        fq = f"@a\n{seq}\n+\n".encode()[:n]
        assert np.array_equal(np.sort(kc.extract_kmers(fq, 31)), np.sort(O.extract(fq, 31)))


@pytest.mark.parametrize("bits", [1, 8, 13, 42, 62, 64])
def test_radix_sort_is_stable_and_ordered(kc, bits):
    rng = np.random.default_rng(bits)
    n = 300_001
    keys = rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    if bits < 64:
        keys &= np.uint64((1 << bits) - 1)
    vals = np.arange(n, dtype=np.uint32)
    sk, sv = kc.sort_records(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(sk, keys[order])
    assert np.array_equal(sv, vals[order])


@pytest.mark.parametrize("case", GOLDEN["e2e"], ids=lambda c: f"{c['name']}-k{c['k']}-cm{c['count_max']}")
def test_job_matches_reference_tools(counter, kc, case):
    files = _case_files(case["name"])
    r = counter.count(files, k=case["k"], count_max=case["count_max"], hist_min=1, hist_max=10000)
    sparse = {str(i + 1): int(v) for i, v in enumerate(r.hist) if v}
    assert sparse == case["hist"]
    text = kc.dump_text(r.keys, r.counts, case["k"]).encode()
    assert text.count(b"\n") == case["dump_lines"]
    assert hashlib.sha256(text).hexdigest() == case["dump_sha256"]
    assert r.occurrences == sum(len(O.extract(f, case["k"])) for f in files)


@pytest.mark.parametrize("name,k", [("plain_small", 31), ("repeat", 21), ("mixed", 21), ("edge", 25), ("edge", 5),
                                    ("mixed", 11), ("plain_small", 32)])
@pytest.mark.parametrize("min_count", [1, 2])
def test_bloom_job_exact(counter, name, k, min_count):
    files = _case_files(name)
    want_k, want_c = O.exact_records(files, k, U32, min_count=min_count)
    r = counter.count(files, k=k, count_max=U32, bloom=True, memory_gb=1, min_count=min_count, hist_min=1,
                      hist_max=5000)
    assert np.array_equal(r.keys, want_k)
    assert np.array_equal(r.counts, want_c)
    all_k, all_c = O.exact_records(files, k, U32)
    assert r.hist.tolist() == O.histogram(all_c, 1, 5000).tolist()
    assert r.distinct == len(all_k)


@pytest.mark.parametrize("rec", GOLDEN["prepass"], ids=lambda r: r["name"])
def test_bloom_plan_matches_reference(kc, rec):
    import test_oracle_golden as T
    files = T._prepass_files(rec["name"])
    pc, avg, caps, mx = kc.bloom_plan(files, rec["k"], rec["memory_gb"])
    assert pc.tolist() == rec["raw_prefix_counts"]
    assert avg == rec["avg_quality"]
    assert mx == rec["max_bloom_capacity"]
    assert caps.tolist() == rec["bloom_capacities"]


def test_plain_job_full_size(counter):
    """The plain job at its full size (1 Mbp genome, 200k x 150 bp)."""
    import ktcountermemorygreedy_b200.synth as S
    fq, k = S.plain_job()
    fq = fq.tobytes()
    want_k, want_c = O.exact_records([fq], k, U32)
    r = counter.count([fq], k=k, count_max=U32, hist_max=10000)
    # about 4.3M distinct k-mers: too many for one L2-resident table, so the
    # job is counted through the root-prefix buckets
    assert r.high_len == r.occurrences
    assert r.occurrences == int(want_c.sum(dtype=np.uint64))
    assert np.array_equal(r.keys, want_k)
    assert np.array_equal(r.counts, want_c)
    assert r.hist.tolist() == O.histogram(want_c, 1, 10000).tolist()


def test_plain_partitioned_job_queries_and_filters(counter, kc):
    """A plain job on the partitioned path, k = 25, with count filters,
    saturation and both queries, against the oracle."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(31, 3_000_000)
    fq = S.reads(g, 31, 60_000, (150, 150), 0.01, 0.0).tobytes()
    k = 25
    small = counter.count([fq[: 4000 * 316]], k=k, count_max=U32)
    assert small.high_len == 0                      # a small job keeps one table
    all_k, all_c = O.exact_records([fq], k, 7)
    r = counter.count([fq], k=k, count_max=7, min_count=2, max_count=6, top_n=500, want_le2=True, hist_max=20)
    assert r.high_len == r.occurrences
    m = (all_c >= 2) & (all_c <= 6)
    assert np.array_equal(r.keys, all_k[m]) and np.array_equal(r.counts, all_c[m])
    assert r.hist.tolist() == O.histogram(all_c, 1, 20).tolist()
    keep_k, keep_c = all_k[m], all_c[m]
    strs = [kc.string_key(int(w), k) for w in keep_k]
    order = sorted(range(len(keep_k)), key=lambda i: (-int(keep_c[i]), strs[i]))[:500]
    assert r.top_keys.tolist() == [int(keep_k[i]) for i in order]
    le = keep_c <= 2
    assert r.le2_keys.tolist() == keep_k[le].tolist()


def test_bloom_job_sampled_census(counter):
    """Inputs of 512+ tiles size the root-prefix buckets from a 1-in-8 tile
    sample of the census; the result stays exact."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(21, 2_000_000)
    fq = S.reads(g, 21, 30_000, (150, 150), 0.01, 0.0).tobytes()
    assert len(fq) > 512 * 8192
    for mc in (1, 2):
        want_k, want_c = O.exact_records([fq], 31, U32, min_count=mc)
        r = counter.count([fq], k=31, count_max=U32, bloom=True, memory_gb=2, min_count=mc)
        assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)


def test_gzip_inputs_count_like_plain_ones(counter):
    """gzip FASTQ (one member, several concatenated members, mixed with an
    uncompressed file) is inflated on the host and counts exactly like the
    uncompressed input, in single, Bloom and batched jobs; corrupt or
    truncated gzip data is reported as an error."""
    import gzip
    a = fixtures.random_fastq(501, 400, (100, 150), genome_len=5000)
    b = fixtures.random_fastq(502, 300, (90, 150), genome_len=4000)
    half = len(a) // 2
    cut = a.index(b"\n@", half) + 1   # a record boundary
    multi = gzip.compress(a[:cut]) + gzip.compress(a[cut:])
    for kw in (dict(), dict(bloom=True, memory_gb=1, min_count=1)):
        want = counter.count([a, b], k=25, count_max=U32, **kw)
        for files in ([gzip.compress(a), b], [multi, gzip.compress(b)]):
            got = counter.count(files, k=25, count_max=U32, **kw)
            assert np.array_equal(got.keys, want.keys) and np.array_equal(got.counts, want.counts)
            assert got.input_bytes == len(a) + len(b)
    res = counter.count_batch([[gzip.compress(a)], [b], [multi]], [21, 31, 21], count_max=U32)
    for files, k, r in zip([[a], [b], [a]], [21, 31, 21], res):
        one = counter.count(files, k=k, count_max=U32)
        assert np.array_equal(r.keys, one.keys) and np.array_equal(r.counts, one.counts)
    bad = bytearray(gzip.compress(a))
    bad[len(bad) // 2] ^= 0xFF
    import ktcountermemorygreedy_b200 as kcm
    for data in (bytes(bad), gzip.compress(a)[:-40]):
        with pytest.raises(kcm.KcError):
            counter.count([data], k=25)


def test_tuning_changes_speed_not_results(kc):
    """The handle's settings (table load factors, sort group size) and the
    autotuner that picks them change no record: plain, partitioned and
    batched jobs give the same results under every setting."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(61, 2_000_000)
    big = S.reads(g, 61, 45_000, (150, 150), 0.01, 0.0).tobytes()
    small = fixtures.random_fastq(62, 300, (100, 150), genome_len=3000)
    with kc.KmerCounter(max_inflight_jobs=2) as c:
        ref = [c.count([f], k=31, count_max=U32) for f in (big, small)]
        refb = c.count_batch([[small], [big]], [21, 31], count_max=U32)
        for t in (dict(bucket_table_factor=1.2, table_factor=1.1, sort_group_records=1000),
                  dict(bucket_table_factor=5.0, table_factor=2.5, sort_group_records=1 << 24)):
            c.set_tuning(**t)
            assert c.tuning["table_factor"] == t["table_factor"]
            for f, want in zip((big, small), ref):
                got = c.count([f], k=31, count_max=U32)
                assert np.array_equal(got.keys, want.keys) and np.array_equal(got.counts, want.counts)
            for want, got in zip(refb, c.count_batch([[small], [big]], [21, 31], count_max=U32)):
                assert np.array_equal(got.keys, want.keys) and np.array_equal(got.counts, want.counts)
        # the search starts from the current settings (the last ones set
        # above) and moves only for a clear gain
        best = c.autotune([[big]], [31], count_max=U32)
        assert best["bucket_table_factor"] in (2.0, 3.0, 4.0, 5.0) and best["table_factor"] in (1.3, 1.6, 2.2, 2.5)
        got = c.count([big], k=31, count_max=U32)
        assert np.array_equal(got.keys, ref[0].keys) and np.array_equal(got.counts, ref[0].counts)
        import ktcountermemorygreedy_b200 as kcm
        with pytest.raises(kcm.KcError):
            c.set_tuning(table_factor=1.0)


def test_dump_text_on_device_matches_oracle(kc):
    """kc_dump_text formats records on the device exactly as the tool's text
    (k from 1 to 32, counts from 0 to 2^32 - 1, more records than one block,
    no records)."""
    rng = np.random.default_rng(77)
    for k, n in ((1, 3), (21, 1000), (31, 4099), (32, 257)):
        keys = rng.integers(0, 2**63, size=n, dtype=np.uint64)
        if k < 32:
            keys &= np.uint64(((1 << (2 * k)) - 1) << (64 - 2 * k))
        counts = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        counts[: min(n, 5)] = [0, 1, 9, 10, 0xFFFFFFFF][: min(n, 5)]
        assert kc.dump_bytes(keys, counts, k) == O.dump_text(keys, counts, k), k
    assert kc.dump_bytes(np.zeros(0, np.uint64), np.zeros(0, np.uint32), 31) == b""


def test_multi_pass_jobs_match_single_pass(counter):
    """A job whose pass budget is smaller than its k-mer arrays, filters and
    tables runs in several passes over ranges of root prefixes, each pass's
    records kept in pinned host memory until the final sort.  Bloom and plain
    jobs, with count filters and queries, against the oracle and against the
    same job in one pass."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(41, 2_000_000)
    fq = S.reads(g, 41, 45_000, (150, 150), 0.01, 0.0).tobytes()   # ~3.5M distinct: partitioned
    kw = dict(count_max=U32, top_n=300, want_le2=True, hist_max=100)
    for bloom, mc in ((True, 2), (False, 1)):
        want_k, want_c = O.exact_records([fq], 31, U32, min_count=mc)
        one = counter.count([fq], k=31, bloom=bloom, memory_gb=2, min_count=mc, **kw)
        many = counter.count([fq], k=31, bloom=bloom, memory_gb=2, min_count=mc, pass_bytes=24 << 20, **kw)
        assert one.passes == 1 and many.passes >= 4, (one.passes, many.passes)
        if bloom:   # min count 2: every pass counts its sub-buckets in shared memory
            assert many.smem_passes == many.passes and one.smem_passes == 1
        assert np.array_equal(many.keys, want_k) and np.array_equal(many.counts, want_c)
        for f in ("keys", "counts", "hist", "top_keys", "top_counts", "le2_keys", "le2_counts"):
            assert np.array_equal(getattr(many, f), getattr(one, f)), (bloom, f)
        assert many.occurrences == one.occurrences and many.distinct == one.distinct


def test_bloom_job_census_overflow_falls_back_to_exact(counter):
    """Every 8th tile random, the others one homopolymer: the sampled census
    underestimates the homopolymer's bucket, its region overflows and the job
    is redone with an exact census -- same exact result."""
    import random
    rnd = random.Random(5)
    recs = []
    for i in range(600):
        seq = "".join(rnd.choice("ACGT") for _ in range(4000)) if i % 8 == 0 else "A" * 4000
        header = "@" + "h" * 186 + "\n"
        recs.append(header + seq + "\n+\n" + "I" * 4000 + "\n")
    fq = "".join(recs).encode()
    assert all(len(r) == 8192 for r in recs)
    want_k, want_c = O.exact_records([fq], 21, U32)
    r = counter.count([fq], k=21, count_max=U32, bloom=True, memory_gb=1)
    assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)


def test_queries(counter, kc):
    files = _case_files("repeat")
    k = 21
    want_k, want_c = O.exact_records(files, k, U32)
    r = counter.count(files, k=k, count_max=U32, top_n=1000, want_le2=True)
    strs = [kc.string_key(int(w), k) for w in want_k]
    order = sorted(range(len(want_k)), key=lambda i: (-int(want_c[i]), strs[i]))[:1000]
    assert r.top_keys.tolist() == [int(want_k[i]) for i in order]
    assert r.top_counts.tolist() == [int(want_c[i]) for i in order]
    m = want_c <= 2
    assert r.le2_keys.tolist() == want_k[m].tolist()
    assert r.le2_counts.tolist() == want_c[m].tolist()


def test_count_filters_and_saturation(counter):
    files = _case_files("repeat")
    for cm, lo, hi in [(255, 1, U32), (100, 50, 100), (U32, 3, 7)]:
        want_k, want_c = O.exact_records(files, 31, cm, min_count=lo, max_count=hi)
        r = counter.count(files, k=31, count_max=cm, min_count=lo, max_count=hi)
        assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)


def test_batch_matches_oracle(counter):
    samples, ks = [], []
    for i, (name, files, kl) in enumerate(fixtures.E2E_CASES):
        samples.append(files)
        ks.append(kl[-1])
    samples.append([fixtures.random_fastq(40, 50, (120, 120), genome_len=1000)])
    ks.append(21)
    res = counter.count_batch(samples, ks, count_max=U32)
    for files, k, r in zip(samples, ks, res):
        want_k, want_c = O.exact_records(files, k, U32)
        assert np.array_equal(r.keys, want_k), k
        assert np.array_equal(r.counts, want_c)
        assert r.hist.tolist() == O.histogram(want_c, 1, 10000).tolist()


def test_batch_spanning_several_sort_groups_matches_single_jobs(counter):
    """A batch of more than 4M records is sorted in several groups of
    samples; each sample (k = 21, 25 and 31 mixed, so the samples take 6, 7
    and 8 radix passes) must equal the same sample counted alone, and the
    per-sample totals must add up."""
    import ktcountermemorygreedy_b200.synth as S
    samples, ks = [], []
    for i in range(7):
        g = S.genome(7000 + i, 3_000_000)
        samples.append([S.reads(g, 7000 + i, 12_000 + 1000 * i, (150, 150), 0.02, 0.0)])
        ks.append([21, 25, 31][i % 3])
    res = counter.count_batch(samples, ks, count_max=U32, hist_max=4095)
    assert sum(len(r.keys) for r in res) > (4 << 20)
    for files, k, r in zip(samples, ks, res):
        one = counter.count(files, k=k, count_max=U32, hist_max=4095)
        assert np.array_equal(r.keys, one.keys), k
        assert np.array_equal(r.counts, one.counts), k
        assert np.array_equal(r.hist, one.hist), k
        assert r.occurrences == one.occurrences


def test_pinned_arena_results_match(kc):
    """Results carved from a pinned arena set aside at kc_open (records and
    count <= 2 sets of several sizes, released and reused across rounds) are
    the same as results in blocks pinned on demand."""
    jobs = []
    for i in range(6):
        f = fixtures.random_fastq(300 + i, 200 + 150 * i, (100, 150), genome_len=3000 + 700 * i)
        jobs.append(([f], [21, 25, 31][i % 3]))
    with kc.KmerCounter(max_inflight_jobs=2) as c0:
        want = [c0.count(f, k=k, count_max=U32, want_le2=True) for f, k in jobs]
    with kc.KmerCounter(max_inflight_jobs=3, pinned_bytes=64 << 20) as c1:
        for rnd in range(3):
            ids = [c1.submit(f, k=k, count_max=U32, want_le2=True) for f, k in jobs]
            for jid, (f, k), w in zip(ids, jobs, want):
                c1.wait(jid)
                r = c1.result(jid, k, copy=(rnd != 1))
                assert np.array_equal(r.keys, w.keys) and np.array_equal(r.counts, w.counts)
                assert np.array_equal(r.le2_keys, w.le2_keys) and np.array_equal(r.le2_counts, w.le2_counts)
                del r


def test_jobs_same_alone_and_in_the_mix(kc):
    jobs = []
    for i in range(12):
        f = fixtures.random_fastq(100 + i, 300 + 97 * i, (100, 150), genome_len=2000 + 500 * i)
        jobs.append(([f], [21, 25, 31][i % 3]))
    alone = []
    with kc.KmerCounter(max_inflight_jobs=1) as c1:
        for files, k in jobs:
            alone.append(c1.count(files, k=k, count_max=U32, top_n=50, want_le2=True))
    with kc.KmerCounter(max_inflight_jobs=6) as c6:
        ids = [c6.submit(files, k=k, count_max=U32, top_n=50, want_le2=True) for files, k in jobs]
        mixed = []
        for jid, (files, k) in zip(ids, jobs):
            c6.wait(jid)
            mixed.append(c6.result(jid, k))
    for (files, k), a, m in zip(jobs, alone, mixed):
        want_k, want_c = O.exact_records(files, k, U32)
        for r in (a, m):
            assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
        assert np.array_equal(a.top_keys, m.top_keys) and np.array_equal(a.le2_keys, m.le2_keys)
        assert np.array_equal(a.hist, m.hist)


def test_resident_input(counter):
    files = _case_files("mixed")
    inp = counter.upload(files)
    try:
        r = counter.count(input=inp, k=21, count_max=U32)
        want_k, want_c = O.exact_records(files, 21, U32)
        assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
    finally:
        counter.free_input(inp)


def test_merge_records_matches_tool_merge(kc):
    """A high/low split like the reference counter writes (each k-mer in
    high.bin, low.bin or both, at most one low occurrence) merges to the
    exact counts, as histogram_tool/dump_tool precise compute them."""
    rng = np.random.default_rng(7)
    files = _case_files("plain_small")
    k = 31
    uk, uc = O.count(O.extract_files(files, k))
    in_low = rng.random(len(uk)) < 0.6
    high_part = uc.astype(np.int64) - in_low
    hm = high_part > 0
    for cm in (U32, 255, 3):
        ok, oc, hist = kc.merge_records(uk[hm], high_part[hm].clip(0, cm).astype(np.uint32), uk[in_low], k, cm,
                                        hist_min=1, hist_max=300)
        want_k, want_c = O.sort_string_order(uk, np.minimum(uc, cm).astype(np.uint32), k)
        assert np.array_equal(ok, want_k) and np.array_equal(oc, want_c)
        assert hist.tolist() == O.histogram(want_c, 1, 300).tolist()


def test_cli_round_trip():
    """kmer_counter -> tmp_dir -> histogram_tool / dump_tool, byte-identical to
    the reference tools' outputs recorded in the golden vectors."""
    bin_dir = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin")
    case = [c for c in GOLDEN["e2e"] if c["name"] == "multi" and c["k"] == 31][0]
    with tempfile.TemporaryDirectory() as tmp:
        paths = []
        for i, data in enumerate(_case_files("multi")):
            p = os.path.join(tmp, f"m{i}.fq")
            open(p, "wb").write(data)
            paths.append(p)
        d = os.path.join(tmp, "t")
        os.makedirs(d)
        subprocess.run([os.path.join(bin_dir, "kmer_counter"), ",".join(paths), "31", "8", "1", d, "1024", "2",
                        str(U32), str(U32)], check=True, capture_output=True)
        assert os.path.getsize(os.path.join(d, "low.bin")) == 0
        h = os.path.join(tmp, "h.tsv")
        subprocess.run([os.path.join(bin_dir, "histogram_tool"), "precise", d, "8", "1", h, "1", "10000"], check=True,
                       capture_output=True)
        sparse = {}
        for line in open(h):
            a, b = line.split("\t")
            if int(b):
                sparse[a] = int(b)
        assert sparse == case["hist"]
        o = os.path.join(tmp, "d.txt")
        subprocess.run([os.path.join(bin_dir, "dump_tool"), "precise", d, "8", "1", o, "1", str(U32), "--sort"],
                       check=True, capture_output=True)
        assert hashlib.sha256(open(o, "rb").read()).hexdigest() == case["dump_sha256"]


def _segment_budget_gb(k, dump, with_low, n_high, n_low, hist_bins, parts):
    """A max_memory_gb that makes the tools merge in about `parts` segments:
    their host bytes per high.bin record, per low.bin k-mer and fixed
    (seg_cost in ktcountermemorygreedy_b200/cli/cli_common.h)."""
    out = 24 + k if dump else 0
    per_high, per_low = 12 + out, (8 + out) if with_low else 0
    fixed = (4 << 20) + (1 << 20) + 2 * 4 ** min(k, 8) * 8 + hist_bins * 16
    return (fixed + (n_high * per_high + n_low * per_low) // parts) / 2 ** 30


def test_tools_segmented_mode_matches_whole_and_exact_counts():
    """histogram_tool and dump_tool given a max_memory_gb too small for all
    records merge them in segments of the k-mers' first bases: the outputs
    are byte-identical to the whole-file path's and equal the exact counts
    (precise) or the high.bin counts (approximate).  The tmp_dir is split like
    the reference counter's: each k-mer in high.bin, low.bin or both."""
    import re
    from test_tool_segments_host import write_tmpdir
    bin_dir = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin")
    rng = np.random.default_rng(11)
    k = 31
    uk, uc = O.count(O.extract_files(_case_files("plain_small"), k))
    in_low = rng.random(len(uk)) < 0.6
    high_part = uc.astype(np.int64) - in_low
    hm = high_part > 0
    with tempfile.TemporaryDirectory() as tmp:
        for cm in (U32, 255):
            d = os.path.join(tmp, f"t{cm}")
            hk, hc = uk[hm], high_part[hm].clip(0, cm).astype(np.uint32)
            write_tmpdir(d, k, cm, hk, hc, uk[in_low])
            for tool, mode in (("histogram_tool", "precise"), ("histogram_tool", "approximate"),
                               ("dump_tool", "precise"), ("dump_tool", "approximate")):
                dump, with_low = tool == "dump_tool", mode == "precise"
                tail = ["2", str(U32), "--sort"] if dump else ["1", "10000"]
                small = _segment_budget_gb(k, dump, with_low, len(hk), int(in_low.sum()), 0 if dump else 10000, 4)
                outs = []
                for mem in ("64", repr(small)):
                    o = os.path.join(tmp, f"{tool}_{mode}_{cm}_{len(outs)}")
                    p = subprocess.run([os.path.join(bin_dir, tool), mode, d, "8", mem, o] + tail,
                                       capture_output=True, text=True)
                    assert p.returncode == 0, p.stderr
                    seg = re.search(r"Segmented mode: \d+ high records in (\d+) segment", p.stdout)
                    if outs:
                        assert seg and int(seg.group(1)) >= 2, p.stdout
                    else:
                        assert seg is None
                    outs.append(open(o, "rb").read())
                assert outs[0] == outs[1]
                if with_low:
                    want_k, want_c = O.sort_string_order(uk, np.minimum(uc, cm).astype(np.uint32), k)
                else:
                    want_k, want_c = O.sort_string_order(hk, hc, k)
                if dump:
                    m = want_c >= 2
                    assert outs[0] == O.dump_text(want_k[m], want_c[m], k)
                else:
                    got = [int(line.split(b"\t")[1]) for line in outs[0].splitlines()]
                    assert got == O.histogram(want_c, 1, 10000).tolist()
        # below the fixed need of a segment: the reference tools' "insufficient memory" exit code
        for tool in ("histogram_tool", "dump_tool"):
            p = subprocess.run([os.path.join(bin_dir, tool), "precise", os.path.join(tmp, f"t{U32}"), "8", "0.001",
                                os.path.join(tmp, "x")], capture_output=True, text=True)
            assert p.returncode == 2 and "insufficient memory" in p.stderr


def test_bloom_shared_memory_path_matches_global_path(kc):
    """Bloom jobs with min count >= 2 count each filter sub-bucket in shared
    memory; the global-memory path (bloom_smem=2) and the oracle give the same
    records, histogram, queries and totals, with saturated counts too."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(81, 1_500_000)
    fq = S.reads(g, 81, 40_000, (100, 150), 0.01, 0.0).tobytes()
    files = [fq, fixtures.random_fastq(82, 500, (80, 150), genome_len=3000)]
    with kc.KmerCounter(max_inflight_jobs=2) as c:
        for k, cm, mc in ((31, U32, 2), (21, 255, 3), (25, 9, 2)):
            kw = dict(k=k, count_max=cm, bloom=True, memory_gb=1, min_count=mc, hist_min=1, hist_max=3000,
                      top_n=100, want_le2=1)
            c.set_tuning(bloom_smem=1)
            a = c.count(files, **kw)
            c.set_tuning(bloom_smem=2)
            b = c.count(files, **kw)
            assert a.smem_passes == a.passes == 1 and a.smem_fallbacks == 0
            assert b.smem_passes == 0
            for f in ("keys", "counts", "hist", "top_keys", "top_counts", "le2_keys", "le2_counts"):
                assert np.array_equal(getattr(a, f), getattr(b, f)), (k, f)
            # low_only (singletons the filter let through as FIRST) depends on
            # the order the occurrences meet the filter, as in the reference;
            # the count-1 histogram bin, which adds both kinds, is exact
            assert (a.occurrences, a.distinct) == (b.occurrences, b.distinct)
            assert a.low_len + a.high_len == a.occurrences
            want_k, want_c = O.exact_records(files, k, cm, min_count=mc)
            assert np.array_equal(a.keys, want_k) and np.array_equal(a.counts, want_c)
        c.set_tuning(bloom_smem=1)


@pytest.mark.parametrize("shape", [1, 2, 3, 4])
def test_count_shapes_give_exact_results(kc, shape):
    """Every block shape of the shared-memory count (kc_tuning.count_shape:
    512- or 256-thread blocks, 4096- or 2048-slot tables, two table hashes):
    exact records, histogram and queries, including a job whose tables
    overflow and are split."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(84, 2_000_000)
    fq = S.reads(g, 84, 50_000, (100, 150), 0.01, 0.0).tobytes()
    once = S.reads(S.genome(85, 3_000_000), 85, 15_000, (150, 150), 0.0, 0.0).tobytes()
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        c.set_tuning(bloom_smem=1, count_shape=shape)
        assert c.tuning["count_shape"] == shape
        for files, k, cm in (([fq], 31, U32), ([fq], 21, 255), ([once, once], 31, U32)):
            want_k, want_c = O.exact_records(files, k, cm)
            m = want_c >= 2
            r = c.count(files, k=k, count_max=cm, bloom=True, memory_gb=1, min_count=2, hist_min=1, hist_max=400,
                        top_n=64, want_le2=1)
            assert r.smem_passes == 1 and r.smem_fallbacks == 0
            assert np.array_equal(r.keys, want_k[m]) and np.array_equal(r.counts, want_c[m]), (shape, k)
            assert np.array_equal(r.hist, O.histogram(want_c, 1, 400))
            rk, rc = want_k[m], want_c[m]
            order = np.argsort(-rc.astype(np.int64), kind="stable")[:64]   # count desc, then printed order
            assert np.array_equal(r.top_keys, rk[order]) and np.array_equal(r.top_counts, rc[order])
            le = want_c[m] <= 2
            assert np.array_equal(r.le2_keys, want_k[m][le])
            assert r.distinct == len(want_k)


@pytest.mark.parametrize("part_shape", [1, 2])
def test_partition_round_sizes_give_exact_results(kc, part_shape):
    """The partition's two round sizes (kc_tuning.part_shape: 4096 or 2048
    k-mers staged per round) and the sub-bucket scatter's two variants
    (scatter_shape) on Bloom and large plain jobs: exact records."""
    import ktcountermemorygreedy_b200.synth as S
    fq = S.reads(S.genome(86, 2_000_000), 86, 60_000, (100, 150), 0.01, 0.0).tobytes()
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        c.set_tuning(part_shape=part_shape, scatter_shape=part_shape)
        assert c.tuning["part_shape"] == part_shape and c.tuning["scatter_shape"] == part_shape
        for kw in (dict(k=31, bloom=True, memory_gb=1, min_count=2), dict(k=25, bloom=True, memory_gb=1,
                                                                          min_count=2, pass_bytes=64 << 20),
                   dict(k=21)):
            want_k, want_c = O.exact_records([fq], kw["k"], U32, min_count=kw.get("min_count", 1))
            r = c.count([fq], count_max=U32, **kw)
            assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c), (part_shape, kw)


def test_bloom_shared_memory_tables_overflow_and_split(counter):
    """Every read twice: half the k-mers of a bucket are distinct repeated
    ones, more than one sub-bucket table holds, so the overflowing buckets are
    cut into more sub-buckets and counted again -- still exact."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(83, 4_000_000)
    once = S.reads(g, 83, 20_000, (150, 150), 0.0, 0.0).tobytes()
    files = [once, once]
    want_k, want_c = O.exact_records(files, 31, U32, min_count=2)
    r = counter.count(files, k=31, count_max=U32, bloom=True, memory_gb=1, min_count=2)
    assert r.smem_passes == 1 and r.smem_fallbacks == 0
    assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
    assert r.distinct == len(O.exact_records(files, 31, U32)[0])


def test_streamed_upload_counts_like_resident_input(kc):
    """A Bloom job's single host file of 512 MiB or more goes up in 128 MiB
    chunks that the census, the SCAN and the partition follow (bucket regions
    from the first chunks' census); the results equal those of the same input
    uploaded first and counted from device memory."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(91, 20_000_000)
    fq = S.reads(g, 91, 1_900_000, (150, 150), 0.01, 0.0).tobytes()
    assert len(fq) >= 512 << 20
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        inp = c.upload([fq])
        try:
            for mc in (2, 1):
                kw = dict(k=31, count_max=U32, bloom=True, memory_gb=8, min_count=mc, hist_max=2000)
                host = c.count([fq], **kw)
                dev = c.count(input=inp, **kw)
                for f in ("keys", "counts", "hist"):
                    assert np.array_equal(getattr(host, f), getattr(dev, f)), (mc, f)
                assert (host.occurrences, host.distinct) == (dev.occurrences, dev.distinct)
        finally:
            c.free_input(inp)


REF_BIN = os.environ.get("KC_REF_BIN") or os.path.join(ROOT, "oracle", "_ref")
GEN = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin", "fastq_gen")


def _ref_programs():
    progs = [os.path.join(REF_BIN, p) for p in ("kmer_counter", "histogram_tool", "dump_tool")]
    if not all(os.access(p, os.X_OK) for p in progs):
        pytest.skip("the reference programs (oracle/_ref) are not built here")
    return progs


def test_large_job_sample_matches_reference_programs(counter, kc):
    """The benchmarked job's settings (k = 31, the reference's Bloom split and
    sizing, min count 2, u32 counts) on the first 60k reads of its read stream:
    the histogram text and the count >= 2 part of the sorted dump equal the
    reference programs' own outputs on the same file."""
    import size_parity as SP
    kcnt, htool, dtool = _ref_programs()
    with tempfile.TemporaryDirectory() as tmp:
        fq = os.path.join(tmp, "s.fq")
        subprocess.run([GEN, "large", "100000000", "0", "60000", fq], check=True)
        d = os.path.join(tmp, "t")
        os.makedirs(d)
        subprocess.run([kcnt, fq, "31", "6", "2", d, "1024", "2", str(U32), str(U32)], check=True,
                       capture_output=True)
        subprocess.run([htool, "precise", d, "6", "2", os.path.join(tmp, "h.tsv"), "2", "10000"], check=True,
                       capture_output=True)
        subprocess.run([dtool, "precise", d, "6", "2", os.path.join(tmp, "d.txt"), "1", str(U32), "--sort"],
                       check=True, capture_output=True)
        data = np.fromfile(fq, np.uint8)
        r = counter.count([data], k=31, count_max=U32, bloom=True, memory_gb=64, min_count=2, hist_min=2,
                          hist_max=10000)
        chk = SP.reference_outputs_match(kc.histogram_text(r.hist, 2), kc.dump_bytes(r.keys, r.counts, 31),
                                         os.path.join(tmp, "h.tsv"), os.path.join(tmp, "d.txt"), 31, 2)
        assert chk["histogram_identical"]
        assert chk["dump_identical"], chk
        assert chk["dump_lines"] == len(r.keys) > 0
        # and the size-independent checks the benchmark applies to the full job
        full = SP.full_spot_check(data, 31, r.keys, r.counts, r.hist, 2, 2, threads=4, sample_bits=3)
        assert full["identical"], full


def test_reference_tools_read_our_tmpdir():
    """The unmodified reference tools (compiled from the reference's sources)
    run on the tmp_dir our kmer_counter writes (infos.bin, exact counts in
    high.bin, empty low.bin): their precise histogram and sorted dump equal
    the golden outputs the reference produced from its own tmp_dir."""
    _, htool, dtool = _ref_programs()
    bin_dir = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin")
    for name, k, cm in (("multi", 31, U32), ("repeat", 21, 255), ("repeat", 31, 1000), ("edge", 25, U32)):
        cases = [c for c in GOLDEN["e2e"] if c["name"] == name and c["k"] == k and c["count_max"] == cm]
        assert cases, (name, k, cm)
        case = cases[0]
        with tempfile.TemporaryDirectory() as tmp:
            paths = []
            for i, data in enumerate(_case_files(name)):
                p = os.path.join(tmp, f"m{i}.fq")
                open(p, "wb").write(data)
                paths.append(p)
            d = os.path.join(tmp, "t")
            os.makedirs(d)
            subprocess.run([os.path.join(bin_dir, "kmer_counter"), ",".join(paths), str(k), "8", "1", d, "1024",
                            "2", str(U32), str(cm)], check=True, capture_output=True)
            h = os.path.join(tmp, "h.tsv")
            subprocess.run([htool, "precise", d, "6", "1", h, "1", "10000"], check=True, capture_output=True)
            sparse = {}
            for line in open(h):
                a, b = line.split("\t")
                if int(b):
                    sparse[a] = int(b)
            assert sparse == case["hist"], name
            o = os.path.join(tmp, "d.txt")
            subprocess.run([dtool, "precise", d, "6", "1", o, "1", str(U32), "--sort"], check=True,
                           capture_output=True)
            assert hashlib.sha256(open(o, "rb").read()).hexdigest() == case["dump_sha256"], name


def _distinct_keys(rng, n, bits):
    k = np.unique(rng.integers(0, 1 << bits, size=int(n * 1.05) + 16, dtype=np.uint64))
    rng.shuffle(k)
    assert len(k) >= n
    return k[:n]


@pytest.mark.parametrize("n,bits,skew", [(1 << 20, 62, False), (3_000_001, 62, False), (2_000_000, 42, False),
                                         (1_200_000, 24, False), (1_500_000, 62, True), (900_000, 50, False)])
def test_distinct_record_sort_matches_numpy(kc, n, bits, skew):
    """kc_sort_distinct_records (the most-significant-bits-first sort of the
    job records) against numpy, with a skewed case whose largest bucket (40%
    of the keys share their top 16 bits) goes to the per-bucket fallback."""
    rng = np.random.default_rng(n + bits)
    keys = _distinct_keys(rng, n, bits)
    if skew:
        m = int(0.4 * n)
        low = _distinct_keys(rng, m, bits - 16)
        keys = np.unique(np.concatenate([(np.uint64(0xBEEF) << np.uint64(bits - 16)) | low, keys[: n - m]]))
        rng.shuffle(keys)
    counts = rng.integers(1, 1 << 32, size=len(keys), dtype=np.uint64).astype(np.uint32)
    got_k, got_c = kc.sort_distinct_records(keys, counts, bits)
    order = np.argsort(keys)
    assert np.array_equal(got_k, keys[order])
    assert np.array_equal(got_c, counts[order])


def test_sampled_subbucket_regions_give_exact_results(kc):
    """The shared-memory Bloom path with sub-bucket regions estimated from a
    1-in-8 sample (forced on small jobs here): exact records and histogram,
    both when the estimates hold and when a sub-bucket outgrows its region
    and the pass is counted again with exact regions."""
    big = fixtures.random_fastq(31, 40000, (150, 150), genome_len=1_500_000, sub=0.01, n_rate=0.0)
    small = fixtures.plain_small()
    redos = 0
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        c.set_tuning(bloom_smem=1, sampled_region_keys=1)
        for data, k in ((big, 31), (small, 25), (big, 21)):
            want_k, want_c = O.exact_records([data], k)
            m = want_c >= 2
            r = c.count([data], k=k, count_max=U32, bloom=True, memory_gb=2, min_count=2, hist_min=1, hist_max=500)
            assert np.array_equal(r.keys, want_k[m]) and np.array_equal(r.counts, want_c[m]), k
            assert r.hist.tolist() == O.histogram(want_c, 1, 500).tolist()
            assert r.smem_passes == 1
            redos += r.region_redos
    # the small job's buckets are a few work items each: its estimates miss
    assert redos >= 1


def test_batch_larger_than_the_budget_runs_as_sub_batches(kc):
    """A batch whose samples exceed a worker's share of the device-memory
    budget is cut into consecutive sub-batches; every sample's results equal
    the sample counted alone."""
    samples = [fixtures.random_fastq(40 + i, 1500 + 300 * i, (100, 150), genome_len=60_000, sub=0.01, n_rate=0.0)
               for i in range(6)]
    ks = [21 if i % 2 == 0 else 31 for i in range(6)]
    job = dict(count_max=U32, min_count=1, hist_min=1, hist_max=300)
    with kc.KmerCounter(max_inflight_jobs=2, hbm_budget_bytes=300 << 20) as c:
        res = c.count_batch([[s] for s in samples], ks, **job)
        alone = [c.count([s], k=k, **job) for s, k in zip(samples, ks)]
    assert len({r.batch_part for r in res}) > 1
    for r, a in zip(res, alone):
        assert np.array_equal(r.keys, a.keys) and np.array_equal(r.counts, a.counts)
        assert r.hist.tolist() == a.hist.tolist()


@pytest.mark.parametrize("record_sort", [1, 2])
def test_record_sort_variants_same_results(kc, record_sort):
    """The two record sorts (most significant bits first, LSD) give the same
    records and histogram: Bloom jobs (one pass and several), a plain job on
    the partitioned path."""
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(71, 3_000_000)
    big = S.reads(g, 71, 60_000, (150, 150), 0.01, 0.0)
    jobs = [dict(k=31, count_max=U32, bloom=True, memory_gb=4, min_count=2, hist_min=1, hist_max=1000),
            dict(k=25, count_max=U32, bloom=True, memory_gb=4, min_count=2, hist_min=1, hist_max=1000,
                 pass_bytes=96 << 20),
            dict(k=31, count_max=U32, min_count=1, hist_min=1, hist_max=1000)]
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        c.set_tuning(record_sort=record_sort)
        assert c.tuning["record_sort"] == record_sort
        got = [c.count([big], **j) for j in jobs]
    for j, r in zip(jobs, got):
        wk, wc = O.exact_records([big.tobytes()], j["k"])
        m = (wc >= j["min_count"])
        assert np.array_equal(r.keys, wk[m]) and np.array_equal(r.counts, wc[m]), j
        assert r.hist.tolist() == O.histogram(wc, 1, 1000).tolist()


def test_large_jobs_run_alone_among_small_ones(kc):
    """A job whose reservation exceeds one worker's share of the budget runs
    alone (the idle workers give their kept workspaces back first; nothing
    else starts until it ends); small jobs around it still run concurrently.
    Every job's results equal the job counted alone."""
    big = fixtures.random_fastq(91, 120_000, (150, 150), genome_len=3_000_000, sub=0.01, n_rate=0.0)
    smalls = [fixtures.random_fastq(92 + i, 2000, (100, 150), genome_len=50_000, sub=0.01, n_rate=0.0)
              for i in range(6)]
    plan = [(smalls[0], 21), (smalls[1], 31), (big, 31), (smalls[2], 25), (smalls[3], 21), (big, 25),
            (smalls[4], 31), (smalls[5], 21)]
    job = dict(count_max=U32, hist_min=1, hist_max=500)
    # a 1.2 GB budget over three workers: the 38 MB file reserves about 1 GB
    with kc.KmerCounter(max_inflight_jobs=3, hbm_budget_bytes=1_200_000_000) as c:
        ids = [c.submit([f], k=k, **job) for f, k in plan]
        for jid, (f, k) in zip(ids, plan):
            c.wait(jid)
            r = c.result(jid, k)
            want_k, want_c = O.exact_records([f], k)
            assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c), k
            assert np.array_equal(r.hist, O.histogram(want_c, 1, 500))
