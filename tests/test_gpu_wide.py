"""k-mers of 33..128 bases (the reference's kmer<2> and kmer<4> paths,
src/main.cpp:617-633) on the GPU, through the C ABI, against the oracle
(pinned to GetKmer<N> golden vectors and the reference programs' outputs) and
against the reference programs themselves.  Integer work: exact comparisons."""
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
BIN = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
U32 = 0xFFFFFFFF
WIDE_KS = [33, 40, 47, 63, 64, 65, 80, 95, 96, 97, 127, 128]


@pytest.fixture(scope="module")
def kc():
    import ktcountermemorygreedy_b200 as kc
    return kc


@pytest.fixture(scope="module")
def counter(kc):
    c = kc.KmerCounter(max_inflight_jobs=2)
    yield c
    c.close()


def _case_files(name):
    for n, files, _ in fixtures.E2E_CASES:
        if n == name:
            return files
    raise KeyError(name)


def _sorted_rows(a):
    a = np.ascontiguousarray(a)
    return a[np.lexsort(a.T[::-1])] if len(a) else a


def _sparse(hist, lo=1):
    return {str(lo + i): int(v) for i, v in enumerate(hist) if v}


@pytest.mark.parametrize("k", WIDE_KS)
def test_wide_extraction_matches_oracle(kc, k):
    for name in ("edge", "crlf", "mixed", "plain_small", "multi"):
        for f in _case_files(name):
            got = kc.extract_kmers(f, k)
            want = O.extract_wide(f, k)
            assert got.shape == want.shape, (name, k)
            assert np.array_equal(_sorted_rows(got), _sorted_rows(want)), (name, k)


@pytest.mark.parametrize("k", WIDE_KS)
def test_wide_job_records_match_oracle(counter, k):
    files = _case_files("plain_small") + _case_files("edge")
    want_k, want_c = O.exact_records_wide(files, k)
    r = counter.count(files, k=k, count_max=U32, hist_min=1, hist_max=10000)
    assert r.keys.shape == want_k.shape
    assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
    assert r.distinct == len(want_k)
    assert r.occurrences == int(want_c.astype(np.int64).sum())
    assert np.array_equal(r.hist, O.histogram(want_c, 1, 10000))


@pytest.mark.parametrize("case", GOLDEN["e2e_wide"], ids=lambda c: f"{c['name']}-k{c['k']}")
def test_wide_jobs_match_reference_programs(counter, kc, case):
    """The reference's precise histogram (every k but 96) and sorted dump (up
    to k = 64), recorded from its own programs."""
    k = case["k"]
    r = counter.count(_case_files(case["name"]), k=k, count_max=U32, hist_min=1, hist_max=10000)
    if k == 96:
        # the reference splits some 96-mers' counts (stale bases in
        # GetKmer<4>'s data[3]); the occurrences agree
        ref_occ = sum(int(c) * int(v) for c, v in case["hist"].items())
        assert r.occurrences == ref_occ and sum(case["hist"].values()) > r.distinct
    else:
        assert _sparse(r.hist) == case["hist"]
    if k <= 64:
        text = kc.dump_bytes(r.keys, r.counts, k)
        assert text.count(b"\n") == case["dump_lines"]
        assert hashlib.sha256(text).hexdigest() == case["dump_sha256"]
    else:
        assert kc.dump_bytes(r.keys, r.counts, k) == O.dump_text_wide(r.keys, r.counts, k)


@pytest.mark.parametrize("k", [33, 63, 96, 127])
def test_wide_bloom_min_count_saturation_and_queries(counter, k):
    files = [fixtures.repeat_fastq()]
    want_k, want_c = O.exact_records_wide(files, k)
    # Bloom flag, min count 2, counts saturated at 255
    r = counter.count(files, k=k, count_max=255, bloom=True, memory_gb=1, min_count=2, hist_min=1, hist_max=300,
                      top_n=50, want_le2=True)
    sat = np.minimum(want_c, 255).astype(np.uint32)
    m = sat >= 2
    assert np.array_equal(r.keys, want_k[m]) and np.array_equal(r.counts, sat[m])
    assert np.array_equal(r.hist, O.histogram(sat, 1, 300))
    # top 50 by count desc then printed string asc; records with count <= 2
    order = np.argsort(-sat[m].astype(np.int64), kind="stable")[:50]   # count desc, then printed order
    assert np.array_equal(r.top_keys, want_k[m][order]) and np.array_equal(r.top_counts, sat[m][order])
    le = sat[m] <= 2
    assert np.array_equal(r.le2_keys, want_k[m][le]) and np.array_equal(r.le2_counts, sat[m][le])


def test_wide_job_in_passes_matches_one_pass(counter):
    f = fixtures.random_fastq(31, 20000, (150, 150), genome_len=400_000, sub=0.01, n_rate=0.0)
    for k in (45, 100):
        one = counter.count([f], k=k, count_max=U32)
        many = counter.count([f], k=k, count_max=U32, pass_bytes=8 << 20)
        assert many.passes > 1 and one.passes == 1
        assert np.array_equal(one.keys, many.keys) and np.array_equal(one.counts, many.counts)
        assert np.array_equal(one.hist, many.hist)
        want_k, want_c = O.exact_records_wide([f], k)
        assert np.array_equal(one.keys, want_k) and np.array_equal(one.counts, want_c)


def test_wide_table_full_is_regrown_or_fails_after_retries(kc):
    f = fixtures.plain_small()
    want_k, want_c = O.exact_records_wide([f], 63)
    with kc.KmerCounter(max_inflight_jobs=1) as c:
        r = c.count([f], k=63, count_max=U32, fault_inject=kc.INJECT_TABLE_FULL_ONCE)
        assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
        with pytest.raises(kc.KcError) as e:
            c.count([f], k=63, count_max=U32, fault_inject=kc.INJECT_TABLE_FULL)
        assert e.value.code == 6 and "counting table overflow" in str(e.value)
        with pytest.raises(kc.KcError) as e:
            c.count([f], k=63, count_max=U32, fault_inject=kc.INJECT_WAIT_TIMEOUT)
        assert e.value.code == 6 and "bounded wait expired" in str(e.value)
        r = c.count([f], k=63, count_max=U32)
        assert np.array_equal(r.keys, want_k)


@pytest.mark.parametrize("k", [40, 64, 65, 128])
def test_wide_merge_matches_reference_tool_merge(kc, k):
    """kc_merge_records on N-word keys against the oracle's restatement of the
    tools' precise merge (tool/histogram_tool.cpp, LowFrequencyQueryThreadPool)."""
    files = _case_files("plain_small")
    keys, counts = O.exact_records_wide(files, k)
    rng = np.random.default_rng(k)
    low = rng.random(len(keys)) < 0.25          # split like the reference: some k-mers also in low.bin
    only_low = rng.random(len(keys)) < 0.1      # some only in low.bin
    hk = keys[~only_low]
    hc = np.where(low[~only_low], np.maximum(counts[~only_low], 2) - 1, counts[~only_low]).astype(np.uint32)
    lk = np.concatenate([keys[~only_low][low[~only_low]], keys[only_low]])
    mk, mc, hist = kc.merge_records(hk, hc, lk, k, U32, hist_min=1, hist_max=5000)
    nw = O.key_words(k)
    want = np.zeros(5000, np.int64)
    O.lib().kco_tool_precise_histogram(O.P(np.ascontiguousarray(hk)), O.P(hc), len(hc),
                                        O.P(np.ascontiguousarray(lk)), len(lk), nw, U32, 1, 5000, O.P(want))
    assert np.array_equal(hist, want)
    exp = np.where(low[~only_low], np.maximum(counts[~only_low], 2), counts[~only_low])
    ek, ec = O.sort_string_order_wide(np.concatenate([hk, keys[only_low]]),
                                      np.concatenate([exp, np.ones(only_low.sum())]).astype(np.uint32), k)
    assert np.array_equal(mk, ek) and np.array_equal(mc, ec)


def test_wide_cli_round_trip_and_reference_tools():
    """kmer_counter at k = 63, 70 and 97 -> tmp_dir -> our tools, and the
    unmodified reference tools on the same tmp_dir: the histogram equals the
    reference's, the dump equals it at k = 63 (and the oracle's text at 97)."""
    ref_tools = [os.path.join(REF_BIN, p) for p in ("histogram_tool", "dump_tool")]
    have_ref = all(os.access(p, os.X_OK) for p in ref_tools)
    for name, k in (("multi", 70), ("plain_small", 63), ("plain_small", 97)):
        cases = [c for c in GOLDEN["e2e_wide"] if c["name"] == name and c["k"] == k]
        case = cases[0] if cases else None
        files = _case_files(name)
        with tempfile.TemporaryDirectory() as tmp:
            paths = []
            for i, data in enumerate(files):
                p = os.path.join(tmp, f"m{i}.fq")
                open(p, "wb").write(data)
                paths.append(p)
            d = os.path.join(tmp, "t")
            os.makedirs(d)
            subprocess.run([os.path.join(BIN, "kmer_counter"), ",".join(paths), str(k), "8", "1", d, "1024", "2",
                            str(U32), str(U32)], check=True, capture_output=True)
            want_k, want_c = O.exact_records_wide(files, k)
            tools = [(os.path.join(BIN, "histogram_tool"), os.path.join(BIN, "dump_tool"), "ours")]
            if have_ref:
                tools.append((ref_tools[0], ref_tools[1], "reference"))
            for ht, dt, who in tools:
                h = os.path.join(tmp, f"h_{who}.tsv")
                subprocess.run([ht, "precise", d, "6", "1", h, "1", "10000"], check=True, capture_output=True)
                sparse = {}
                for line in open(h):
                    a, b = line.split("\t")
                    if int(b):
                        sparse[a] = int(b)
                assert sparse == _sparse(O.histogram(want_c, 1, 10000)), (who, k)
                if case:
                    assert sparse == case["hist"], (who, k)
                o = os.path.join(tmp, f"d_{who}.txt")
                subprocess.run([dt, "precise", d, "6", "1", o, "1", str(U32), "--sort"], check=True,
                               capture_output=True)
                text = open(o, "rb").read()
                if who == "ours" or k <= 64:
                    assert text == O.dump_text_wide(want_k, want_c, k), (who, k)
                if case and k <= 64:
                    assert hashlib.sha256(text).hexdigest() == case["dump_sha256"], (who, k)


def test_wide_larger_job_matches_oracle(counter):
    f = fixtures.random_fastq(32, 60_000, (100, 250), genome_len=2_000_000, sub=0.01, n_rate=0.001)
    for k in (55, 111):
        want_k, want_c = O.exact_records_wide([f], k)
        r = counter.count([f], k=k, count_max=U32, top_n=100)
        assert np.array_equal(r.keys, want_k) and np.array_equal(r.counts, want_c)
        order = np.argsort(-want_c.astype(np.int64), kind="stable")[:100]
        assert np.array_equal(r.top_counts, want_c[order]) and np.array_equal(r.top_keys, want_k[order])


@pytest.mark.parametrize("k,count_max,fmin,fmax", [(21, 255, 2, U32), (31, U32, 2, U32), (33, 0xFFFF, 3, 40),
                                                   (64, 0xFFFFFF, 2, U32), (100, U32, 1, 7), (17, 1000, 5, 60)])
def test_high_bin_packed_on_the_device_equals_the_host_packing(counter, k, count_max, fmin, fmax):
    """kc_job.pack_high: high.bin made on the device byte-identical to the
    host packing of the records and to the oracle's restatement of the
    reference's record layout (src/FinalDrainWriter.h:71-101)."""
    files = _case_files("plain_small") + _case_files("repeat")
    job = dict(k=k, count_max=count_max, filter_min=fmin, filter_max=fmax)
    with tempfile.TemporaryDirectory() as tmp:
        a, b = os.path.join(tmp, "dev"), os.path.join(tmp, "host")
        os.makedirs(a)
        os.makedirs(b)
        j = counter.submit(files, pack_high=True, keep_records=False, **job)
        counter.wait(j)
        counter.write_tmpdir(j, a)
        counter.release(j)
        j = counter.submit(files, keep_records=True, **job)
        counter.wait(j)
        counter.write_tmpdir(j, b)
        r = counter.result(j, k)
        dev = open(os.path.join(a, "high.bin"), "rb").read()
        assert dev == open(os.path.join(b, "high.bin"), "rb").read()
        assert os.path.getsize(os.path.join(a, "low.bin")) == 0
        assert open(os.path.join(a, "infos.bin"), "rb").read() == open(os.path.join(b, "infos.bin"), "rb").read()
    # the oracle's packing of the exact records
    nw = O.key_words(k)
    keys, counts = O.exact_records_wide(files, k, count_max=count_max)
    keep = (counts.astype(np.int64) + 1 >= fmin) & (counts <= fmax)
    cb = O.lib().kco_count_bytes(count_max)
    kb = O.lib().kco_packed_kmer_bytes(k)
    want = bytearray()
    one = np.zeros(kb, np.uint8)
    for w, c in zip(keys[keep], counts[keep]):
        O.lib().kco_pack_kmer(O.P(np.ascontiguousarray(w, np.uint64)), k, O.P(one))
        want += one.tobytes() + int(c).to_bytes(4, "little")[:cb]
    assert dev == bytes(want)
    assert r.keys.reshape(len(r.counts), -1).shape[1] == nw
