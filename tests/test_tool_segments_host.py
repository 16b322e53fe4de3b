"""The tools' segmented mode on the CPU: high.bin/low.bin decoding, the
counting pass, the segment plan and the per-segment reads of
ktcountermemorygreedy_b200/cli/cli_common.h, driven by
tests/cli_segments_check.cpp (no library call, no GPU). The merge of each
segment on the GPU is covered by the -m gpu tests."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
U32 = 0xFFFFFFFF


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("seg") / "cli_segments_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "ktcountermemorygreedy_b200", "cli"),
                    os.path.join(ROOT, "tests", "cli_segments_check.cpp"), "-o", exe], check=True)
    return exe


def count_bytes(count_max):
    return 1 if count_max <= 0xFF else 2 if count_max <= 0xFFFF else 3 if count_max <= 0xFFFFFF else 4


def key_bytes(k):
    return 8 * (k // 32) + (2 * (k % 32) + 7) // 8


def key_words(k):
    return 1 if k <= 32 else (2 if k <= 64 else 4)


def pack_keys(words, k):
    """The reference's k-mer packing (src/FinalDrainWriter.h:71-88): the full
    words, then the top tail bytes of the next word, little-endian."""
    words = words.reshape(len(words), key_words(k))
    b = words.astype("<u8").view(np.uint8).reshape(len(words), 8 * key_words(k))
    full, kb = k // 32, key_bytes(k)
    tail = kb - 8 * full
    parts = [b[:, : 8 * full]]
    if tail:
        parts.append(b[:, 8 * full + 8 - tail: 8 * full + 8])
    return np.concatenate(parts, axis=1)


def write_tmpdir(d, k, count_max, hk, hc, lk):
    os.makedirs(d, exist_ok=True)
    np.array([k, count_max], "<u4").tofile(os.path.join(d, "infos.bin"))
    cb = count_bytes(count_max)
    cnt = hc.astype("<u4").view(np.uint8).reshape(-1, 4)[:, :cb]
    np.concatenate([pack_keys(hk, k), cnt], axis=1).tofile(os.path.join(d, "high.bin"))
    pack_keys(lk, k).tofile(os.path.join(d, "low.bin"))


def base_pos(k, i):
    """(word, bit) of base i of the printed k-mer (kmer_to_buf, tool/dump_tool.cpp:103-124)."""
    if k <= 32:
        return 0, 64 - 2 * k + 2 * i
    full, tail = k // 32, k % 32
    if i < tail:
        return full, 64 - 2 * tail + 2 * i
    off = i - tail
    return full - 1 - off // 32, 2 * (off % 32)


def random_words(rng, n, k, lead_zero=0):
    """kmer<N> word arrays, shape (n, N) (N = 1 for k <= 32): every base
    random, every other bit zero; lead_zero > 0 makes the first bases A, so
    many k-mers share one lead prefix."""
    w = np.zeros((n, key_words(k)), np.uint64)
    for i in range(k):
        if i < lead_zero:
            continue
        wi, sh = base_pos(k, i)
        w[:, wi] |= rng.integers(0, 4, size=n, dtype=np.uint64) << np.uint64(sh)
    return w


def string_value(w, k):
    """The printed k-mer as a base-4 number (base 0 most significant)."""
    w = w.reshape(len(w), -1)
    v = np.zeros(len(w), dtype=object)
    for i in range(k):
        wi, sh = base_pos(k, i)
        v = v * 4 + ((w[:, wi] >> np.uint64(sh)) & np.uint64(3)).astype(object)
    return v


def lead(w, k):
    m = min(k, 8)
    return np.array([int(x) >> (2 * (k - m)) for x in string_value(w, k)], dtype=np.int64), m


def rows(a):
    return [tuple(r) for r in a.reshape(len(a), -1).tolist()]


def make_case(k, count_max, seed):
    rng = np.random.default_rng(seed)
    n = 30000
    hk = np.concatenate([random_words(rng, n, k), random_words(rng, n // 4, k, lead_zero=min(k, 3))])
    hc = rng.integers(1, min(count_max, 5000) + 1, size=len(hk)).astype(np.uint32)
    lk = np.concatenate([hk[rng.random(len(hk)) < 0.3], random_words(rng, n // 2, k)])
    return hk, hc, lk


def run_checker(exe, d, out, budget, dump, with_low):
    os.makedirs(out, exist_ok=True)
    subprocess.run([exe, d, str(budget), "1" if dump else "0", "1" if with_low else "0", out], check=True)
    return open(os.path.join(out, "plan.txt")).read().split("\n")


CASES = [(31, U32, True, True), (21, 255, False, True), (5, 0xFFFF, True, False), (32, 0xFFFFFF, False, False),
         (13, U32, True, True), (33, U32, True, True), (64, 255, False, True), (70, U32, True, False),
         (128, 0xFFFF, True, True)]


@pytest.mark.parametrize("k,count_max,dump,with_low", CASES)
def test_segments_cover_every_record_in_printed_string_order(checker, tmp_path, k, count_max, dump, with_low):
    hk, hc, lk = make_case(k, count_max, k)
    d = str(tmp_path / "t")
    write_tmpdir(d, k, count_max, hk, hc, lk)
    # first a plan with one segment, to read the cost model back
    lines = run_checker(checker, d, str(tmp_path / "o0"), 1 << 40, dump, with_low)
    ok, nseg, fixed, per_high, per_low = lines[0].split()
    assert ok == "ok" and int(nseg) == 1
    fixed, per_high, per_low = int(fixed), int(per_high), int(per_low)
    total = len(hk) * per_high + (len(lk) * per_low if with_low else 0)
    budget = fixed + total // 5
    out = str(tmp_path / "o")
    lines = run_checker(checker, d, out, budget, dump, with_low)

    # high.bin / low.bin decoded as packed
    nw = key_words(k)
    ah = np.fromfile(os.path.join(out, "all_high.bin"), np.dtype([("k", "<u8", (nw,)), ("c", "<u4")]))
    assert np.array_equal(ah["k"].reshape(-1, nw), hk) and np.array_equal(ah["c"], hc)
    assert np.array_equal(np.fromfile(os.path.join(out, "all_low.bin"), "<u8").reshape(-1, nw), lk)

    head = lines[0].split()
    assert head[0] == "ok"
    segs = [tuple(int(x) for x in l.split()) for l in lines[1:] if l.strip()]
    assert len(segs) == int(head[1]) >= 5
    hl, m = lead(hk, k)
    ll, _ = lead(lk, k)
    # contiguous ranges over every lead prefix
    assert segs[0][0] == 0 and segs[-1][1] == 4 ** m
    assert all(a[1] == b[0] for a, b in zip(segs, segs[1:]))
    sh = np.fromfile(os.path.join(out, "seg_high.bin"), np.dtype([("k", "<u8", (nw,)), ("c", "<u4"), ("s", "<u4")]))
    sl = np.fromfile(os.path.join(out, "seg_low.bin"), np.dtype([("k", "<u8", (nw,)), ("s", "<u4")]))
    # every record exactly once, in the segment of its lead prefix
    assert sorted(zip(rows(sh["k"]), sh["c"].tolist())) == sorted(zip(rows(hk), hc.tolist()))
    if with_low:
        assert sorted(rows(sl["k"])) == sorted(rows(lk))
    else:
        assert len(sl) == 0
    p0 = np.array([s[0] for s in segs])
    p1 = np.array([s[1] for s in segs])
    shl, _ = lead(sh["k"], k)
    assert np.all((shl >= p0[sh["s"]]) & (shl < p1[sh["s"]]))
    if with_low:
        sll, _ = lead(sl["k"], k)
        assert np.all((sll >= p0[sl["s"]]) & (sll < p1[sl["s"]]))
    # each segment fits, and the next prefix would not have (ranges as long as fit)
    room = budget - fixed
    pb = np.bincount(hl, minlength=4 ** m) * per_high + (np.bincount(ll, minlength=4 ** m) * per_low if with_low else 0)
    for i, (a, b, nh, nl) in enumerate(segs):
        assert nh == int(np.count_nonzero((hl >= a) & (hl < b)))
        assert nl == (int(np.count_nonzero((ll >= a) & (ll < b))) if with_low else 0)
        used = int(pb[a:b].sum())
        assert used <= room
        if i + 1 < len(segs):
            assert used + int(pb[b]) > room
    # a segment's k-mers all print before the next segment's
    sv = string_value(sh["k"], k)
    for i in range(len(segs) - 1):
        here, there = sv[sh["s"] == i], sv[sh["s"] == i + 1]
        if len(here) and len(there):
            assert max(here) < min(there)


def test_no_plan_below_the_fixed_need_or_for_a_crowded_prefix(checker, tmp_path):
    k = 21
    hk, hc, lk = make_case(k, U32, 3)
    rng = np.random.default_rng(4)
    crowd = random_words(rng, 3000, k, lead_zero=8)      # k-mers starting with AAAAAAAA
    hk = np.concatenate([hk, crowd])
    hc = np.concatenate([hc, np.full(len(crowd), 7, np.uint32)])
    d = str(tmp_path / "t")
    write_tmpdir(d, k, U32, hk, hc, lk)
    lines = run_checker(checker, d, str(tmp_path / "o0"), 1 << 40, True, True)
    _, _, fixed, per_high, per_low = lines[0].split()
    fixed, per_high, per_low = int(fixed), int(per_high), int(per_low)
    lines = run_checker(checker, d, str(tmp_path / "o1"), fixed, True, True)
    assert lines[0] == f"nofit {0xFFFFFFFF}" and "below the" in lines[1]
    # room for every prefix but the crowded one
    hl, m = lead(hk, k)
    ll, _ = lead(lk, k)
    pb = np.bincount(hl, minlength=4 ** m) * per_high + np.bincount(ll, minlength=4 ** m) * per_low
    big = int(np.argmax(pb))
    assert pb[big] > 2 * np.sort(pb)[-2]
    lines = run_checker(checker, d, str(tmp_path / "o2"), fixed + int(pb[big]) - 1, True, True)
    assert lines[0] == f"nofit {big}"
    assert big == 0 and "start with AAAAAAAA" in lines[1] and f"need {fixed + int(pb[big])} bytes" in lines[1]


def test_errors_match_read_tmpdir(checker, tmp_path):
    d = str(tmp_path / "t")
    write_tmpdir(d, 31, U32, np.zeros((0, 1), np.uint64), np.zeros(0, np.uint32), np.zeros((0, 1), np.uint64))
    p = subprocess.run([checker, d, "1000000", "1", "1", str(tmp_path)], capture_output=True, text=True)
    assert p.returncode == 2 and "empty high.bin file" in p.stderr
