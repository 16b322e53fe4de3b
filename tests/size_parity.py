"""Parity checks of a counting job at any size (checker side only).

Used by the GPU tests and by bench.py's CPU-baseline leg, outside every timed
region, to check the job that is timed:

* ``full_spot_check`` -- the records of a job of any size against the oracle
  on a hash sample of the k-mers: the oracle extracts the whole FASTQ on many
  threads but keeps only k-mers whose sample hash (splitmix64, unrelated to
  every hash on the counting path) has its low bits zero -- all occurrences of
  those k-mers, so their exact counts are the job's counts of them.  The
  job's records with the same hash property must equal them key for key; in
  addition the records must be strictly increasing in printed-string order
  and the job's histogram must equal the histogram of its records.
* ``reference_outputs_match`` -- a job against the reference programs' own
  outputs on the same file: ``histogram_tool precise`` text, and the
  ``dump_tool precise ... 1 <max> --sort`` text filtered to count >= min
  (the reference's dump with min > 1 is wrong, tool/dump_tool.cpp:717).
"""
from __future__ import annotations

import hashlib
import time

import numpy as np

import oracle_lib as O


def record_splits(fq: np.ndarray, pieces: int):
    """Byte offsets of record starts close to `pieces` equal cuts of a FASTQ
    written by the project's generator: a header line "@r<id>" follows a
    newline, and 'r' never starts a sequence or quality line of its reads."""
    n = len(fq)
    out = []
    for i in range(1, max(1, pieces)):
        p = n * i // pieces
        w = np.asarray(fq[p:p + 8192])
        if len(w) < 3:
            continue
        hit = np.flatnonzero((w[:-2] == 10) & (w[1:-1] == 64) & (w[2:] == 114))
        if len(hit):
            out.append(p + int(hit[0]) + 1)
    return sorted(set(out))


def string_keys(words: np.ndarray) -> np.ndarray:
    """Printed-string order key of kmer<1> words (k <= 32): the 2-bit groups
    in reverse order (first base most significant), right-aligned."""
    x = np.ascontiguousarray(words, np.uint64).copy()
    m1 = np.uint64(0x3333333333333333)
    m2 = np.uint64(0x0F0F0F0F0F0F0F0F)
    x = ((x >> np.uint64(2)) & m1) | ((x & m1) << np.uint64(2))
    x = ((x >> np.uint64(4)) & m2) | ((x & m2) << np.uint64(4))
    return x.byteswap()


CHUNK = 1 << 26   # records per step of the checks below (a few GB of temporaries at most)


def full_spot_check(fq: np.ndarray, k: int, keys: np.ndarray, counts: np.ndarray, hist: np.ndarray,
                    hist_min: int, min_count: int, threads: int = 8, sample_bits: int = 6) -> dict:
    """Checks a job's records (kmer<1> words in printed-string order, exact
    counts >= min_count) and histogram (bins hist_min..) against the oracle
    on the 2^-sample_bits hash sample of the k-mers of the FASTQ `fq`.  The
    records are read in chunks, so that a job of billions of records is
    checked in bounded host memory."""
    t0 = time.perf_counter()
    occ = O.extract_sampled(fq, k, sample_bits, record_splits(fq, 4 * threads), threads)
    uk, uc = O.count(occ)
    n_occ = len(occ)
    del occ
    m = uc >= min_count
    want_k, want_c = O.sort_string_order(uk[m], uc[m], k)
    keys = np.asarray(keys)
    counts = np.asarray(counts)
    n = len(keys)
    got_k, got_c = [], []
    ordered = True
    prev = None
    hmax = hist_min + len(hist) - 1
    rec_hist = np.zeros(len(hist), np.int64)
    for a in range(0, n, CHUNK):
        kc_, cc = keys[a:a + CHUNK], counts[a:a + CHUNK]
        sel = O.sampled_mask(kc_, sample_bits)
        got_k.append(kc_[sel])
        got_c.append(cc[sel])
        sk = string_keys(kc_)
        ordered = ordered and bool(np.all(sk[1:] > sk[:-1])) and bool(prev is None or len(sk) == 0 or sk[0] > prev)
        if len(sk):
            prev = sk[-1]
        del sk
        c = cc[(cc >= hist_min) & (cc <= hmax)]
        rec_hist += np.bincount(c - np.uint32(hist_min), minlength=len(hist))[: len(hist)]
    got_k = np.concatenate(got_k) if got_k else np.zeros(0, np.uint64)
    got_c = np.concatenate(got_c) if got_c else np.zeros(0, np.uint32)
    same = bool(np.array_equal(got_k, want_k) and np.array_equal(got_c, want_c))
    hist_ok = bool(np.array_equal(rec_hist, np.asarray(hist)))
    return {
        "identical": same and ordered and hist_ok,
        "sampled_records_identical": same, "records_sorted": ordered, "hist_equals_records_hist": hist_ok,
        "sampled_kmers": int(len(want_k)), "sampled_occurrences": int(n_occ), "records": int(n),
        "how": f"oracle (C restatement) on the whole FASTQ, {threads} threads, keeping the k-mers whose "
               f"splitmix64 hash is 0 mod {1 << sample_bits} (all their occurrences): their exact counts "
               f">= {min_count} equal the job's records of those k-mers; every record in strictly "
               f"increasing printed-string order; the job's histogram equals its records' histogram",
        "check_s": round(time.perf_counter() - t0, 2),
    }


def full_spot_check_wide(fq: np.ndarray, k: int, keys: np.ndarray, counts: np.ndarray, hist: np.ndarray,
                         hist_min: int, min_count: int, threads: int = 8, sample_bits: int = 6) -> dict:
    """full_spot_check for k-mers of 33..128 bases: records are (n, N) kmer<N>
    word arrays in printed-string order."""
    t0 = time.perf_counter()
    occ = O.extract_wide_sampled(fq, k, sample_bits, record_splits(fq, 4 * threads), threads)
    uk, uc = O.count_wide(occ)
    n_occ = len(occ)
    del occ
    m = uc >= min_count
    want_k, want_c = O.sort_string_order_wide(uk[m], uc[m], k)
    keys = np.asarray(keys)
    counts = np.asarray(counts)
    n = len(counts)
    smask = np.uint64((1 << sample_bits) - 1)
    got_k, got_c = [], []
    ordered, prev = True, None
    hmax = hist_min + len(hist) - 1
    rec_hist = np.zeros(len(hist), np.int64)
    for a in range(0, n, CHUNK // 4):
        kc_, cc = keys[a:a + CHUNK // 4], counts[a:a + CHUNK // 4]
        sel = (O.sample_hash_wide_np(kc_) & smask) == 0
        got_k.append(kc_[sel])
        got_c.append(cc[sel])
        sk = O.string_keys_wide(kc_, k)
        if len(sk):
            # strictly increasing rows: the first differing word decides
            cmp = np.zeros(len(sk) - 1, np.int8)
            for w in range(sk.shape[1]):
                und = cmp == 0
                cmp[und & (sk[1:, w] > sk[:-1, w])] = 1
                cmp[und & (sk[1:, w] < sk[:-1, w])] = -1
            ordered = ordered and bool(np.all(cmp == 1))
            if prev is not None:
                ordered = ordered and bool(tuple(sk[0].tolist()) > prev)
            prev = tuple(sk[-1].tolist())
        c = cc[(cc >= hist_min) & (cc <= hmax)]
        rec_hist += np.bincount(c - np.uint32(hist_min), minlength=len(hist))[: len(hist)]
    got_k = np.concatenate(got_k) if got_k else np.zeros((0, keys.shape[1]), np.uint64)
    got_c = np.concatenate(got_c) if got_c else np.zeros(0, np.uint32)
    same = bool(np.array_equal(got_k, want_k) and np.array_equal(got_c, want_c))
    hist_ok = bool(np.array_equal(rec_hist, np.asarray(hist)))
    return {
        "identical": same and ordered and hist_ok,
        "sampled_records_identical": same, "records_sorted": ordered, "hist_equals_records_hist": hist_ok,
        "sampled_kmers": int(len(want_k)), "sampled_occurrences": int(n_occ), "records": int(n),
        "how": f"oracle (C restatement of GetKmer<N>) on the whole FASTQ, {threads} threads, keeping the k-mers "
               f"whose word-folded splitmix64 hash is 0 mod {1 << sample_bits}: their exact counts >= "
               f"{min_count} equal the job's records of those k-mers; records in strictly increasing "
               f"printed-string order; the job's histogram equals its records' histogram",
        "check_s": round(time.perf_counter() - t0, 2),
    }


def filtered_dump(path: str, k: int, min_count: int) -> bytes:
    """The reference's `dump_tool precise ... 1 <max> --sort` text with the
    lines whose count is below min_count removed."""
    buf = np.fromfile(path, np.uint8)
    if len(buf) == 0:
        return b""
    nl = np.flatnonzero(buf == 10)
    starts = np.concatenate([[0], nl[:-1] + 1]).astype(np.int64)
    first = starts + k + 1                      # first digit of the count
    ndig = nl - first
    val = np.zeros(len(nl), np.int64)
    for d in range(int(ndig.max()) if len(ndig) else 0):
        live = d < ndig
        pos = np.where(live, first + d, 0)
        val = np.where(live, val * 10 + (buf[pos].astype(np.int64) - 48), val)
    keep = val >= min_count
    mask = np.repeat(keep, nl - starts + 1)
    return buf[: len(mask)][mask].tobytes()


def reference_outputs_match(hist_text: str, dump_bytes: bytes, hist_path: str, dump_path: str, k: int,
                            min_count: int) -> dict:
    """A job's histogram text and sorted dump text against the reference
    programs' files on the same input."""
    ref_hist = open(hist_path).read()
    ref_dump = filtered_dump(dump_path, k, min_count)
    h_ok = hist_text == ref_hist
    d_ok = dump_bytes == ref_dump
    return {
        "identical": h_ok and d_ok, "histogram_identical": h_ok, "dump_identical": d_ok,
        "dump_sha256": hashlib.sha256(dump_bytes).hexdigest(),
        "reference_dump_sha256": hashlib.sha256(ref_dump).hexdigest(),
        "dump_lines": dump_bytes.count(b"\n"),
        "how": f"histogram_tool precise ... {min_count} <max> text equal byte for byte; dump_tool precise "
               f"... 1 <max> --sort text filtered to count >= {min_count} equal byte for byte "
               f"(SHA-256 given)",
    }
