"""The oracle (oracle/kc_oracle.c) pinned against the reference: golden
vectors produced by the reference's own programs and headers
(tests/golden/make_golden.py), and the known-answer fixtures of the
reference's own tests."""
import hashlib
import json
import os

import numpy as np
import pytest

import fixtures
import oracle_lib as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
U32 = 0xFFFFFFFF


def test_hashes_match_reference_headers():
    for row in GOLDEN["hashes"]:
        w, lo, hi, x64, rap, komi, mix, block, mask = row
        w = int(w, 16)
        assert O.xxh3_128(w) == (int(lo, 16), int(hi, 16))
        assert O.lib().kco_xxh3_64_8(w) == int(x64, 16)
        assert O.lib().kco_rapidhash_8(w) == int(rap, 16)
        assert O.lib().kco_komihash_8(w) == int(komi, 16)
        assert O.lib().kco_mix_hash(int(komi, 16), int(rap, 16)) == int(mix, 16)
        assert O.lib().kco_concurrent_map_hash(w) == int(mix, 16)
        assert O.bloom_probe(w, 1 << 20) == (int(block), int(mask, 16))


def _wrap(bases: str) -> bytes:
    return f"@x\n{bases}\n+\n{'I' * len(bases)}\n".encode()


def test_rolling_extraction_matches_getkmer():
    for case in GOLDEN["getkmer"]:
        got = O.extract(_wrap(case["bases"]), case["k"])
        assert [f"{int(v):016x}" for v in got] == case["canonical"], case["k"]


@pytest.mark.parametrize("rec", GOLDEN["prepass"], ids=lambda r: r["name"])
def test_prepass_and_bloom_sizing_match_reference(rec):
    files = _prepass_files(rec["name"])
    limit = (256 << 20) if len(files) == 1 else (128 << 20)
    pc = np.zeros(256, np.uint32)
    qs = qn = 0
    for f in files:
        p, s, n = O.prepass(f, rec["k"], limit)
        pc += p
        qs += s
        qn += n
    assert pc.tolist() == rec["raw_prefix_counts"]
    avg = (qs // qn) & 0xFF if qn else 0
    assert avg == rec["avg_quality"]
    est = sum(len(f) for f in files)
    assert est == rec["estimated_file_size"]
    caps, mx = O.bloom_capacities(pc, avg, est, rec["memory_gb"], rec["k"])
    assert mx == rec["max_bloom_capacity"]
    assert caps.tolist() == rec["bloom_capacities"]


def _prepass_files(name):
    if name == "plain_small":
        return [fixtures.plain_small()]
    if name == "repeat":
        return [fixtures.repeat_fastq()]
    if name == "multi":
        return [c for c in fixtures.E2E_CASES if c[0] == "multi"][0][1]
    if name == "prepass_big":
        return [fixtures.random_fastq(16, 9000, (150, 150), genome_len=50000)]
    if name == "edge":
        return [fixtures.edge_fastq()]
    raise KeyError(name)


def _case_files(name):
    for n, files, _ in fixtures.E2E_CASES:
        if n == name:
            return files
    raise KeyError(name)


@pytest.mark.parametrize("case", GOLDEN["e2e"], ids=lambda c: f"{c['name']}-k{c['k']}-cm{c['count_max']}")
def test_exact_counts_match_reference_tools(case):
    files = _case_files(case["name"])
    keys, counts = O.exact_records(files, case["k"], case["count_max"])
    hist = O.histogram(counts, 1, 10000)
    sparse = {str(i + 1): int(v) for i, v in enumerate(hist) if v}
    assert sparse == case["hist"]
    text = O.dump_text(keys, counts, case["k"])
    assert text[:2000].decode() == case["dump_head"]
    assert text.count(b"\n") == case["dump_lines"]
    assert hashlib.sha256(text).hexdigest() == case["dump_sha256"]


# ---- k-mers of 33..128 bases (kmer<2>, kmer<4>) ------------------------------

@pytest.mark.parametrize("case", GOLDEN["getkmer_wide"], ids=lambda c: f"k{c['k']}-n{c['n']}")
def test_wide_rolling_extraction_matches_getkmer(case):
    k = case["k"]
    got = O.extract_wide(_wrap(case["bases"]), k)
    last = (k - 1) // 32
    assert len(got) == case["n"]
    text = "".join(" ".join(f"{int(v):016x}" for v in row[: last + 1]) + "\n" for row in got)
    assert hashlib.sha256(text.encode()).hexdigest() == case["sha256"]
    for row, want in zip(got, case["head"]):
        assert [f"{int(v):016x}" for v in row[: last + 1]] == want[: last + 1]
    # words above the k-mer's last word are zero here; GetKmer<4> leaves stale
    # bases there at k = 96 only (its data[2] is not masked when k % 32 == 0)
    assert not got[:, last + 1:].any()
    assert (case["beyond_nonzero"] > 0) == (k == 96)


def test_wide_string_keys_agree():
    r = np.random.default_rng(3)
    for k in (33, 47, 63, 64, 65, 96, 127, 128):
        nw = O.key_words(k)
        occ = O.extract_wide(fixtures.random_fastq(40 + k, 30, (150, 200), genome_len=5000), k)
        sk = O.string_keys_wide(occ, k)
        one = np.zeros(nw, np.uint64)
        for i in r.choice(len(occ), 50):
            O.lib().kco_string_key_wide(O.P(np.ascontiguousarray(occ[i])), k, O.P(one))
            assert one.tolist() == sk[i].tolist()
            # the key's bases read back give the printed string
            s = "".join("ACGT"[(int(sk[i][nw - 1 - (k - 1 - j) // 32]) >> (2 * ((k - 1 - j) % 32))) & 3]
                        for j in range(k))
            assert s == O.kmer_string_wide(occ[i], k)


@pytest.mark.parametrize("case", GOLDEN["e2e_wide"], ids=lambda c: f"{c['name']}-k{c['k']}")
def test_wide_exact_counts_match_reference_tools(case):
    k = case["k"]
    files = _case_files(case["name"])
    keys, counts = O.exact_records_wide(files, k)
    hist = O.histogram(counts, 1, 10000)
    sparse = {str(i + 1): int(v) for i, v in enumerate(hist) if v}
    if k == 96:
        # GetKmer<4>'s stale data[3] at k = 96 gives one 96-mer several keys:
        # the reference reports more distinct k-mers, the same occurrences
        ref_occ = sum(int(c) * int(v) for c, v in case["hist"].items())
        assert sum(case["hist"].values()) > len(keys)
        assert ref_occ == int(counts.astype(np.int64).sum())
        return
    assert sparse == case["hist"]
    if k <= 64:
        # the reference's sorted dump is an oracle up to k = 64
        text = O.dump_text_wide(keys, counts, k)
        assert text[:2000].decode() == case["dump_head"]
        assert text.count(b"\n") == case["dump_lines"]
        assert hashlib.sha256(text).hexdigest() == case["dump_sha256"]


# ---- the reference's own test fixtures ------------------------------------

def _words(*w):
    return np.array(w, np.uint64)


def test_low_frequency_query_deltas():
    # tests/test_low_frequency_query_thread_pool.cpp:384-436 (k = 33, two words)
    two = [0x0123456789ABCDEF, 0xC000000000000000]
    four = [0x1111222233334444, 0x8000000000000000]
    missing = [0x9999AAAABBBBCCCC, 0x4000000000000000]
    high = _words(*two, *four)
    hc = np.array([2, 4], np.uint32)
    low = _words(*two, *four, *missing)
    hist = np.zeros(4, np.int64)
    O.lib().kco_tool_low_query_deltas(O.P(high), O.P(hc), 2, O.P(low), 3, 2, U32, 1, 4, O.P(hist))
    assert hist.tolist() == [1, -1, 1, -1]


def _tool_hist(high, counts, low, n_words, lo, hi, count_max=U32):
    hist = np.zeros(hi - lo + 1, np.int64)
    hw = np.array(high, np.uint64)
    hc = np.array(counts, np.uint32)
    lw = np.array(low, np.uint64) if low else np.zeros(1, np.uint64)
    rc = O.lib().kco_tool_precise_histogram(O.P(hw), O.P(hc), len(counts), O.P(lw), len(low) // n_words,
                                            n_words, count_max, lo, hi, O.P(hist))
    return rc, hist.tolist()


def test_histogram_tool_expectations():
    # tests/test_histogram_tool.cpp:211-296 (expected vectors)
    a = [0x0123456789ABCDEF, 0xC000000000000000]
    b = [0x1111111111111111, 0x8000000000000000]
    c = [0x2222222222222222, 0x4000000000000000]
    e = [0x3333333333333333, 0x0000000000000000]
    assert _tool_hist(a + c + e, [2, 1, 4], a + b + c + e, 2, 1, 4) == (0, [1, 1, 1, 0])
    g = [0x4444444444444444, 0xC000000000000000]
    h = [0x5555555555555555, 0x8000000000000000]
    i = [0x6666666666666666, 0x4000000000000000]
    j = [0x7777777777777777, 0x0000000000000000]
    assert _tool_hist(g + h + i, [1, 2, 5], g + h + i + j, 2, 3, 5) == (0, [1, 0, 0])
    key1 = [0xAAAAAAAA55555555]
    assert _tool_hist(key1, [1], key1, 1, 1, 3) == (0, [0, 1, 0])
    key4 = [0xAAAAAAAA55555555, 0x0123456789ABCDEF, 0xC000000000000000, 0]
    assert _tool_hist(key4, [1], key4, 4, 1, 3) == (0, [0, 1, 0])
    # an empty high.bin makes the tool fail (tool/histogram_tool.cpp:296-300)
    assert _tool_hist([], [], [0], 1, 1, 3)[0] == -1


@pytest.mark.parametrize("k,n_words", [(33, 2), (64, 2), (31, 1), (21, 1), (65, 4)])
def test_export_record_packing_round_trip(k, n_words):
    # tests/test_export_reader.cpp:175-390: pack -> unpack keeps the k bases
    rng = np.random.default_rng(k)
    nb = O.lib().kco_packed_kmer_bytes(k)
    assert nb == (k // 32) * 8 + (2 * (k % 32) + 7) // 8
    for _ in range(200):
        w = rng.integers(0, 2**63, size=n_words, dtype=np.uint64) * 2 + rng.integers(0, 2, size=n_words, dtype=np.uint64)
        tail = k % 32
        if tail:
            w[k // 32] &= np.uint64(((1 << (2 * tail)) - 1) << (64 - 2 * tail))
        for t in range(k // 32 + (1 if tail else 0), n_words):
            w[t] = 0
        buf = np.zeros(nb, np.uint8)
        O.lib().kco_pack_kmer(O.P(w), k, O.P(buf))
        back = np.zeros(n_words, np.uint64)
        O.lib().kco_unpack_kmer(O.P(buf), k, n_words, O.P(back))
        assert back.tolist() == w.tolist()


def test_count_bytes_follow_count_max():
    # src/main.cpp:599-615
    for cm, cb in [(1, 1), (255, 1), (256, 2), (65535, 2), (65536, 3), (0xFFFFFF, 3), (0x1000000, 4), (U32, 4)]:
        assert O.lib().kco_count_bytes(cm) == cb


def test_oracle_radix_sort_matches_numpy():
    # the property of tests/test_and_benckmark_export_record_radix_sort.cpp:101-190
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 2**62, size=50000, dtype=np.uint64) & np.uint64((1 << 44) - 1)
    uk, uc = O.count(keys)
    ref_u, ref_c = np.unique(keys, return_counts=True)
    assert uk.tolist() == ref_u.tolist() and uc.tolist() == ref_c.tolist()


def test_string_order_is_lexicographic():
    rng = np.random.default_rng(4)
    for k in (5, 21, 31, 32):
        shift = 64 - 2 * k
        keys = (rng.integers(0, 2**63, size=300, dtype=np.uint64) >> np.uint64(max(shift - 1, 0))) << np.uint64(shift) \
            if shift else rng.integers(0, 2**63, size=300, dtype=np.uint64)
        counts = np.arange(300, dtype=np.uint32)
        sk, sc = O.sort_string_order(keys, counts, k)
        strs = [O.kmer_string(int(w), k) for w in sk]
        assert strs == sorted(strs)
