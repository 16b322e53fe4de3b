"""ctypes binding of the oracle (oracle/liboracle.so), the CPU restatement of
the reference path.  Test infrastructure only: the tests compare the CUDA
path against it."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "oracle", "liboracle.so")
_L = None
U64P = C.POINTER(C.c_uint64)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(PATH):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)
        L = C.CDLL(PATH)
        vp, u32, u64, u8 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint8
        sig = {
            "kco_extract": (u64, [vp, u64, u32, vp, u64]),
            "kco_key_words": (u32, [u32]),
            "kco_extract_wide": (u64, [vp, u64, u32, vp, u64]),
            "kco_string_key_wide": (None, [vp, u32, vp]),
            "kco_sample_hash_wide": (u64, [vp, u32]),
            "kco_extract_wide_sampled": (u64, [vp, u64, u32, u32, vp, u64]),
            "kco_sample_hash": (u64, [u64]),
            "kco_extract_sampled": (u64, [vp, u64, u32, u32, vp, u64]),
            "kco_prepass": (None, [vp, u64, u32, u64, vp, U64P, U64P]),
            "kco_count_sorted": (u64, [vp, u64, vp, vp]),
            "kco_sort_records_string_order": (None, [vp, vp, u64, u32]),
            "kco_string_key": (u64, [u64, u32]),
            "kco_kmer_to_string": (None, [vp, u32, C.c_char_p]),
            "kco_histogram": (None, [vp, u64, u32, u32, vp]),
            "kco_xxh3_128_8": (None, [u64, U64P, U64P]),
            "kco_xxh3_64_8": (u64, [u64]),
            "kco_rapidhash_8": (u64, [u64]),
            "kco_komihash_8": (u64, [u64]),
            "kco_mix_hash": (u64, [u64, u64]),
            "kco_concurrent_map_hash": (u64, [u64]),
            "kco_bloom_probe": (None, [u64, u64, U64P, U64P]),
            "kco_bloom_classify": (None, [vp, u64, vp, vp]),
            "kco_bloom_capacities": (None, [vp, u8, u64, u64, u32, vp, U64P]),
            "kco_packed_kmer_bytes": (u32, [u32]),
            "kco_count_bytes": (u32, [u32]),
            "kco_pack_kmer": (None, [vp, u32, vp]),
            "kco_unpack_kmer": (None, [vp, u32, u32, vp]),
            "kco_tool_precise_histogram": (C.c_int, [vp, vp, u64, vp, u64, u32, u32, u32, u32, vp]),
            "kco_tool_low_query_deltas": (None, [vp, vp, u64, vp, u64, u32, u32, u32, u32, vp]),
            "kco_tool_precise_dump": (u64, [vp, vp, u64, vp, u64, u32, u32, u32, u32, vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def P(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def extract(data: bytes, k: int) -> np.ndarray:
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    cap = max(len(data), 1)
    out = np.zeros(cap, np.uint64)
    n = lib().kco_extract(P(buf), len(data), k, P(out), cap)
    return out[:n].copy()


def key_words(k: int) -> int:
    """Words of the reference's kmer<N> for k: 1 (k <= 32), 2 (<= 64), 4."""
    return 1 if k <= 32 else (2 if k <= 64 else 4)


def extract_wide(data: bytes, k: int) -> np.ndarray:
    """Canonical k-mer occurrences as kmer<N> word arrays, shape (n, N)."""
    nw = key_words(k)
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    cap = max(len(data), 1)
    out = np.zeros(cap * nw, np.uint64)
    n = lib().kco_extract_wide(P(buf), len(data), k, P(out), cap)
    return out[: n * nw].reshape(n, nw).copy()


def string_keys_wide(words: np.ndarray, k: int) -> np.ndarray:
    """Printed-string order keys of kmer<N> word arrays, shape (n, N), most
    significant word first: the 2-bit groups of the whole array reversed."""
    w = np.ascontiguousarray(words, np.uint64)
    m1 = np.uint64(0x3333333333333333)
    m2 = np.uint64(0x0F0F0F0F0F0F0F0F)
    x = w.copy()
    x = ((x >> np.uint64(2)) & m1) | ((x & m1) << np.uint64(2))
    x = ((x >> np.uint64(4)) & m2) | ((x & m2) << np.uint64(4))
    return np.ascontiguousarray(x.byteswap()[:, ::-1])


def count_wide(keys: np.ndarray):
    """Distinct rows and their counts."""
    keys = np.ascontiguousarray(keys, np.uint64)
    if len(keys) == 0:
        return keys.reshape(0, keys.shape[1] if keys.ndim == 2 else 1), np.zeros(0, np.uint32)
    uk, uc = np.unique(keys, axis=0, return_counts=True)
    return uk, uc.astype(np.uint32)


def sort_string_order_wide(keys, counts, k):
    sk = string_keys_wide(keys, k)
    order = np.lexsort(sk.T[::-1])   # the last key passed to lexsort is the primary one
    return np.ascontiguousarray(keys[order]), np.ascontiguousarray(counts[order])


def exact_records_wide(files, k, count_max=0xFFFFFFFF, min_count=1, max_count=0xFFFFFFFF):
    """exact_records for any k: (keys (n, N), counts) in printed-string order."""
    nw = key_words(k)
    occ = np.concatenate([extract_wide(f, k) for f in files]) if files else np.zeros((0, nw), np.uint64)
    uk, uc = count_wide(occ)
    uc = np.minimum(uc, np.uint32(count_max)).astype(np.uint32)
    m = (uc >= min_count) & (uc <= max_count)
    return sort_string_order_wide(uk[m], uc[m], k)


def kmer_string_wide(words, k: int) -> str:
    w = np.ascontiguousarray(words, np.uint64)
    buf = C.create_string_buffer(k + 1)
    lib().kco_kmer_to_string(P(w), k, buf)
    return buf.value.decode()


def dump_text_wide(keys, counts, k) -> bytes:
    return "".join(f"{kmer_string_wide(w, k)}\t{int(c)}\n" for w, c in zip(keys, counts)).encode()


def sample_hash_np(keys: np.ndarray) -> np.ndarray:
    """kco_sample_hash of every word (the splitmix64 finaliser), vectorised."""
    w = np.ascontiguousarray(keys, np.uint64).copy()
    with np.errstate(over="ignore"):
        w ^= w >> np.uint64(30)
        w *= np.uint64(0xbf58476d1ce4e5b9)
        w ^= w >> np.uint64(27)
        w *= np.uint64(0x94d049bb133111eb)
        w ^= w >> np.uint64(31)
    return w


def sampled_mask(keys: np.ndarray, sample_bits: int) -> np.ndarray:
    return (sample_hash_np(keys) & np.uint64((1 << sample_bits) - 1)) == 0


def extract_sampled(buf: np.ndarray, k: int, sample_bits: int, splits=None, threads: int = 1) -> np.ndarray:
    """Occurrences of the sampled k-mers (kco_extract_sampled) of one FASTQ
    held in the uint8 array `buf`.  `splits` are byte offsets of record starts
    (ascending, inside buf); the pieces between them are extracted on
    `threads` threads (ctypes releases the GIL) and concatenated."""
    import concurrent.futures as cf
    buf = np.ascontiguousarray(buf, np.uint8)
    bounds = [0] + [int(x) for x in (splits or []) if 0 < int(x) < len(buf)] + [len(buf)]
    L = lib()
    base = buf.ctypes.data

    def one(i):
        a, b = bounds[i], bounds[i + 1]
        # occurrences <= bytes of the piece; the sample keeps about 2^-bits of them
        cap = max(1024, ((b - a) >> max(0, sample_bits - 2)) + 4096)
        while True:
            out = np.zeros(cap, np.uint64)
            n = L.kco_extract_sampled(C.c_void_p(base + a), b - a, k, sample_bits, P(out), cap)
            if n <= cap:
                return out[:n]
            cap = int(n)

    with cf.ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        parts = list(ex.map(one, range(len(bounds) - 1)))
    return np.concatenate(parts) if parts else np.zeros(0, np.uint64)


def sample_hash_wide_np(keys: np.ndarray) -> np.ndarray:
    """kco_sample_hash_wide of every row of (n, N) word arrays."""
    keys = np.ascontiguousarray(keys, np.uint64)
    h = sample_hash_np(keys[:, 0])
    for i in range(1, keys.shape[1]):
        h = sample_hash_np(h ^ keys[:, i])
    return h


def extract_wide_sampled(buf: np.ndarray, k: int, sample_bits: int, splits=None, threads: int = 1) -> np.ndarray:
    """extract_sampled for N-word k-mers: rows of the sampled occurrences."""
    import concurrent.futures as cf
    nw = key_words(k)
    buf = np.ascontiguousarray(buf, np.uint8)
    bounds = [0] + [int(x) for x in (splits or []) if 0 < int(x) < len(buf)] + [len(buf)]
    L = lib()
    base = buf.ctypes.data

    def one(i):
        a, b = bounds[i], bounds[i + 1]
        cap = max(1024, ((b - a) >> max(0, sample_bits - 2)) + 4096)
        while True:
            out = np.zeros(cap * nw, np.uint64)
            n = L.kco_extract_wide_sampled(C.c_void_p(base + a), b - a, k, sample_bits, P(out), cap)
            if n <= cap:
                return out[: n * nw].reshape(n, nw)
            cap = int(n)

    with cf.ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        parts = list(ex.map(one, range(len(bounds) - 1)))
    return np.concatenate(parts) if parts else np.zeros((0, nw), np.uint64)


def extract_files(files, k):
    return np.concatenate([extract(f, k) for f in files]) if files else np.zeros(0, np.uint64)


def count(keys: np.ndarray):
    keys = keys.astype(np.uint64).copy()
    uk = np.zeros(max(len(keys), 1), np.uint64)
    uc = np.zeros(max(len(keys), 1), np.uint32)
    n = lib().kco_count_sorted(P(keys), len(keys), P(uk), P(uc))
    return uk[:n].copy(), uc[:n].copy()


def sort_string_order(keys, counts, k):
    keys = np.ascontiguousarray(keys, np.uint64).copy()
    counts = np.ascontiguousarray(counts, np.uint32).copy()
    lib().kco_sort_records_string_order(P(keys), P(counts), len(keys), k)
    return keys, counts


def exact_records(files, k, count_max=0xFFFFFFFF, min_count=1, max_count=0xFFFFFFFF):
    """Exact canonical counts of the files, saturated at count_max, filtered,
    sorted in printed-string order (what the precise tools emit)."""
    uk, uc = count(extract_files(files, k))
    uc = np.minimum(uc, np.uint32(count_max)).astype(np.uint32)
    m = (uc >= min_count) & (uc <= max_count)
    return sort_string_order(uk[m], uc[m], k)


def histogram(counts, lo, hi):
    h = np.zeros(hi - lo + 1, np.int64)
    c = np.ascontiguousarray(counts, np.uint32)
    lib().kco_histogram(P(c), len(c), lo, hi, P(h))
    return h


def kmer_string(w: int, k: int) -> str:
    words = np.array([w], np.uint64)
    buf = C.create_string_buffer(k + 1)
    lib().kco_kmer_to_string(P(words), k, buf)
    return buf.value.decode()


def dump_text(keys, counts, k) -> bytes:
    return "".join(f"{kmer_string(int(w), k)}\t{int(c)}\n" for w, c in zip(keys, counts)).encode()


def xxh3_128(w):
    lo, hi = C.c_uint64(), C.c_uint64()
    lib().kco_xxh3_128_8(w, C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def bloom_probe(w, cap):
    b, m = C.c_uint64(), C.c_uint64()
    lib().kco_bloom_probe(w, cap, C.byref(b), C.byref(m))
    return b.value, m.value


def bloom_classify(keys, caps):
    keys = np.ascontiguousarray(keys, np.uint64)
    caps = np.ascontiguousarray(caps, np.uint64)
    out = np.zeros(max(len(keys), 1), np.uint8)
    lib().kco_bloom_classify(P(keys), len(keys), P(caps), P(out))
    return out[: len(keys)]


def prepass(data: bytes, k: int, limit: int):
    buf = np.frombuffer(data, np.uint8)
    pc = np.zeros(256, np.uint32)
    qs, qn = C.c_uint64(0), C.c_uint64(0)
    lib().kco_prepass(P(buf), len(data), k, limit, P(pc), C.byref(qs), C.byref(qn))
    return pc, qs.value, qn.value


def bloom_capacities(prefix_counts, avg_quality, est_size, memory_gb, k):
    pc = np.ascontiguousarray(prefix_counts, np.uint32)
    caps = np.zeros(256, np.uint64)
    mx = C.c_uint64()
    lib().kco_bloom_capacities(P(pc), avg_quality, est_size, memory_gb, k, P(caps), C.byref(mx))
    return caps, mx.value
