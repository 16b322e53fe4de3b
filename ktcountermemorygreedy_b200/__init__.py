"""B200 k-mer counter: Python binding of libkc.so (include/kc.h).

The reference (ScorchShana/KTCounterMemoryGreedy) is driven through three
programs: ``kmer_counter`` (src/main.cpp:481) writes ``tmp_dir/{infos,high,
low}.bin``; ``histogram_tool precise`` (tool/histogram_tool.cpp:905) and
``dump_tool precise --sort`` (tool/dump_tool.cpp:1447) turn those files into
the exact count histogram and the sorted ``KMER\\tcount`` dump.  This module
mirrors that surface on top of the C ABI:

* :class:`KmerCounter` -- a handle (``kc_open``); ``count()`` runs one job
  (FASTQ bytes in, exact sorted records + histogram + queries out),
  ``submit()``/``wait()`` run jobs concurrently, ``count_batch()`` counts many
  samples in one set of device passes.
* :func:`histogram_text` / :func:`dump_text` -- the text outputs of the two
  reference tools for a result.
* :func:`kmer_string` -- ``kmer_to_buf`` (tool/dump_tool.cpp:103).

k-mer words follow the reference's ``kmer<1>`` layout (src/kmer.h:15): base i
of the printed canonical string at bit ``64 - 2k + 2i``.

There is no CPU path: every call runs on the GPU through libkc.so and raises
:class:`KcError` when the library or a device is unavailable.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Iterable, List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkc.so")

KC_OK = 0
ERRORS = {
    1: "KC_ERR_INVALID", 2: "KC_ERR_CUDA", 3: "KC_ERR_NOMEM", 4: "KC_ERR_TIMEOUT",
    5: "KC_ERR_NOT_FOUND", 6: "KC_ERR_DEVICE", 7: "KC_ERR_IO", 8: "KC_ERR_NO_DEVICE",
    9: "KC_ERR_FAILED", 10: "KC_ERR_CANCELLED",
}
KC_ERR_TIMEOUT, KC_ERR_CANCELLED = 4, 10
# kc_job.fault_inject bits (testing aid)
INJECT_WAIT_TIMEOUT, INJECT_TABLE_FULL_ONCE, INJECT_TABLE_FULL, INJECT_NOMEM = 1, 2, 4, 8
U32_MAX = 0xFFFFFFFF


class KcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class kc_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight_jobs", C.c_uint32),
                ("hbm_budget_bytes", C.c_uint64), ("workspace_bytes", C.c_uint64), ("pinned_bytes", C.c_uint64),
                ("reserved", C.c_uint64 * 4)]


class kc_tuning(C.Structure):
    _fields_ = [("bucket_table_factor", C.c_double), ("table_factor", C.c_double),
                ("sort_group_records", C.c_uint64), ("bloom_smem", C.c_uint64), ("record_sort", C.c_uint64),
                ("sampled_region_keys", C.c_uint64), ("count_shape", C.c_uint64), ("part_shape", C.c_uint64),
                ("scatter_shape", C.c_uint64), ("reserved", C.c_uint64 * 3)]


class kc_buffer(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_uint64)]


class kc_job(C.Structure):
    _fields_ = [("files", C.POINTER(kc_buffer)), ("n_files", C.c_uint32), ("k", C.c_uint32),
                ("input", C.c_void_p), ("count_max", C.c_uint32), ("bloom", C.c_uint32),
                ("memory_gb", C.c_uint64), ("filter_min", C.c_uint32), ("filter_max", C.c_uint32),
                ("min_count", C.c_uint32), ("max_count", C.c_uint32), ("hist_min", C.c_uint32),
                ("hist_max", C.c_uint32), ("top_n", C.c_uint32), ("want_le2", C.c_uint32),
                ("keep_records", C.c_uint32), ("fault_inject", C.c_uint32), ("pass_bytes", C.c_uint64),
                ("pack_high", C.c_uint32), ("reserved_u32", C.c_uint32), ("reserved", C.c_uint64 * 4)]


class kc_result_t(C.Structure):
    _fields_ = [("n_records", C.c_uint64), ("keys", C.POINTER(C.c_uint64)), ("counts", C.POINTER(C.c_uint32)),
                ("hist_len", C.c_uint64), ("hist", C.POINTER(C.c_int64)),
                ("n_top", C.c_uint64), ("top_keys", C.POINTER(C.c_uint64)), ("top_counts", C.POINTER(C.c_uint32)),
                ("n_le2", C.c_uint64), ("le2_keys", C.POINTER(C.c_uint64)), ("le2_counts", C.POINTER(C.c_uint32)),
                ("occurrences", C.c_uint64), ("distinct", C.c_uint64), ("low_only", C.c_uint64),
                ("table_capacity", C.c_uint64), ("device_ms", C.c_double), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("phase_ms", C.c_double * 12), ("phase_launches", C.c_uint64 * 12),
                ("low_len", C.c_uint64), ("high_len", C.c_uint64), ("input_bytes", C.c_uint64),
                ("n_records_total", C.c_uint64), ("passes", C.c_uint32), ("smem_passes", C.c_uint16),
                ("smem_fallbacks", C.c_uint16), ("region_redos", C.c_uint32), ("batch_part", C.c_uint32),
                ("key_words", C.c_uint32), ("reserved_u32", C.c_uint32)]

# stage names of kc_result_t.phase_ms
PHASES = ["census", "scan", "count_pass", "insert_high", "merge_low", "compact", "sort", "queries", "bloom",
          "sub_partition", "smem_count", "pack_high"]


# (name, restype, argtypes) of every symbol include/kc.h declares
SIGNATURES = [
    ("kc_open", C.c_int, [C.POINTER(kc_config), C.POINTER(C.c_void_p)]),
    ("kc_close", None, [C.c_void_p]),
    ("kc_last_error", C.c_char_p, []),
    ("kc_job_defaults", None, [C.POINTER(kc_job)]),
    ("kc_input_upload", C.c_int, [C.c_void_p, C.POINTER(kc_buffer), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("kc_input_free", None, [C.c_void_p, C.c_void_p]),
    ("kc_submit", C.c_int, [C.c_void_p, C.POINTER(kc_job), C.POINTER(C.c_uint64)]),
    ("kc_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_int32]),
    ("kc_result", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(kc_result_t)]),
    ("kc_write_tmpdir", C.c_int, [C.c_void_p, C.c_uint64, C.c_char_p]),
    ("kc_release", C.c_int, [C.c_void_p, C.c_uint64]),
    ("kc_cancel", C.c_int, [C.c_void_p, C.c_uint64]),
    ("kc_submit_batch", C.c_int, [C.c_void_p, C.POINTER(kc_job), C.c_uint32, C.POINTER(C.c_uint64)]),
    ("kc_host_alloc", C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
    ("kc_host_free", C.c_int, [C.c_void_p]),
    ("kc_extract_kmers", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p, C.c_uint64,
                                   C.POINTER(C.c_uint64)]),
    ("kc_hash_kmers", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("kc_sort_records", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32]),
    ("kc_bloom_plan", C.c_int, [C.POINTER(kc_buffer), C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p,
                                C.POINTER(C.c_uint32), C.c_void_p, C.POINTER(C.c_uint64)]),
    ("kc_kernel_launches", C.c_uint64, []),
    ("kc_key_words", C.c_uint32, [C.c_uint32]),
    ("kc_sort_distinct_records", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32]),
    ("kc_sort_records_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]),
    ("kc_atomic_peak", C.c_int, [C.c_uint64, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("kc_atomic_peak_shared", C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("kc_get_tuning", C.c_int, [C.c_void_p, C.POINTER(kc_tuning)]),
    ("kc_set_tuning", C.c_int, [C.c_void_p, C.POINTER(kc_tuning)]),
    ("kc_autotune", C.c_int, [C.c_void_p, C.POINTER(kc_job), C.c_uint32, C.c_uint32, C.POINTER(kc_tuning)]),
    ("kc_dump_text", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p, C.c_uint64,
                               C.POINTER(C.c_uint64)]),
    ("kc_plan_bloom", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p,
                                C.POINTER(C.c_uint64)]),
    ("kc_merge_records", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_uint32,
                                   C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p]),
]

_lib = None


def lib() -> C.CDLL:
    """Loads libkc.so (built in-tree by ``make -C ktcountermemorygreedy_b200``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise KcError(8, f"{LIB_PATH} is missing; build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != KC_OK:
        msg = lib().kc_last_error()
        raise KcError(rc, msg.decode() if msg else "")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _buffers(files: Sequence[bytes]):
    arr = (kc_buffer * max(len(files), 1))()
    keep = []
    for i, f in enumerate(files):
        if isinstance(f, np.ndarray):
            mv = f
            arr[i].data = f.ctypes.data
            arr[i].size = f.nbytes
        else:
            mv = np.frombuffer(f, dtype=np.uint8) if len(f) else np.zeros(1, np.uint8)
            arr[i].data = mv.ctypes.data
            arr[i].size = len(f)
        keep.append(mv)
    return arr, keep


def kmer_string(key: int, k: int) -> str:
    """Printed form of a kmer<1> word (tool/dump_tool.cpp:103-124)."""
    return "".join("ACGT"[(key >> (64 - 2 * k + 2 * i)) & 3] for i in range(k))


def string_key(key: int, k: int) -> int:
    """Printed-string order key: the k bases packed first-base-high
    (tool/dump_tool.cpp:346-354)."""
    s = 0
    for i in range(k):
        s = (s << 2) | ((key >> (64 - 2 * k + 2 * i)) & 3)
    return s


@dataclass
class Result:
    """Outputs of one job: the precise histogram/dump of the reference tools."""
    k: int
    keys: np.ndarray               # uint64 kmer<N> words, printed-string order: shape (n,) for k <= 32,
                                   # (n, N) for k > 32 (N = 2 up to k = 64, else 4; data[0] first)
    counts: np.ndarray             # uint32 exact counts (saturated at count_max)
    hist: np.ndarray               # int64, bins hist_min..hist_max
    hist_min: int
    top_keys: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint64))
    top_counts: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    le2_keys: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint64))
    le2_counts: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    occurrences: int = 0
    distinct: int = 0
    low_only: int = 0
    table_capacity: int = 0
    device_ms: float = 0.0
    queue_ms: float = 0.0
    run_ms: float = 0.0
    phase_ms: tuple = ()
    phase_launches: tuple = ()
    low_len: int = 0
    high_len: int = 0
    input_bytes: int = 0
    n_records_total: int = 0
    passes: int = 1
    smem_passes: int = 0      # passes counted per sub-bucket in shared memory (Bloom mode)
    smem_fallbacks: int = 0   # passes recounted on global-memory tables after a sub-bucket table overflowed
    region_redos: int = 0     # shared-memory passes counted again after a sub-bucket outgrew its estimated region
    batch_part: int = 0       # batched jobs: the sub-batch the sample was counted in


def _copy(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def key_words(k: int) -> int:
    """64-bit words of one k-mer (the reference's kmer<N>): 1, 2 or 4."""
    return 1 if k <= 32 else (2 if k <= 64 else 4)


def _keys(flat: np.ndarray, words: int) -> np.ndarray:
    """k-mer key arrays: 1-D for one word per k-mer, (n, words) otherwise."""
    return flat if words <= 1 else flat.reshape(-1, words)


class _JobLease:
    """Keeps a finished job (and the pinned result memory it owns) alive
    while numpy views of its results exist; releases it afterwards."""

    def __init__(self, counter, jid):
        self.counter, self.jid = counter, jid

    def __del__(self):
        try:
            if self.counter._h:
                self.counter.release(self.jid)
        except Exception:
            pass


def _view(ptr, n, dtype, lease):
    if n == 0 or not ptr:
        return np.zeros(0, dtype)
    ctype = C.c_uint64 if dtype == np.uint64 else C.c_uint32
    raw = (ctype * n).from_address(C.addressof(ptr.contents))
    raw._lease = lease   # the array's base keeps the job alive
    return np.frombuffer(raw, dtype=dtype)


class KmerCounter:
    """Handle on one GPU (``kc_open``).  ``max_inflight_jobs`` jobs run on the
    device at once; further jobs are admitted in submission order as device
    memory frees up."""

    def __init__(self, device: int = 0, max_inflight_jobs: int = 4, hbm_budget_bytes: int = 0,
                 workspace_bytes: int = 0, pinned_bytes: int = 0):
        cfg = kc_config()
        cfg.device = device
        cfg.max_inflight_jobs = max_inflight_jobs
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.workspace_bytes = workspace_bytes
        cfg.pinned_bytes = pinned_bytes
        h = C.c_void_p()
        _check(lib().kc_open(C.byref(cfg), C.byref(h)))
        self._h = h
        self._inputs = {}

    def close(self):
        if self._h:
            lib().kc_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- jobs -------------------------------------------------------------
    @staticmethod
    def make_job(k: int = 31, count_max: int = 255, bloom: bool = False, memory_gb: int = 4,
                 filter_min: int = 2, filter_max: int = U32_MAX, min_count: int = 1,
                 max_count: int = U32_MAX, hist_min: int = 1, hist_max: int = 10000, top_n: int = 0,
                 want_le2: bool = False, keep_records: bool = True, pass_bytes: int = 0,
                 fault_inject: int = 0, pack_high: bool = False) -> kc_job:
        j = kc_job()
        lib().kc_job_defaults(C.byref(j))
        j.k, j.count_max, j.bloom, j.memory_gb = k, count_max, int(bloom), memory_gb
        j.filter_min, j.filter_max, j.min_count, j.max_count = filter_min, filter_max, min_count, max_count
        j.hist_min, j.hist_max, j.top_n, j.want_le2 = hist_min, hist_max, top_n, int(want_le2)
        j.keep_records = int(keep_records)
        j.pass_bytes = pass_bytes
        j.fault_inject = fault_inject
        j.pack_high = int(pack_high)
        return j

    def upload(self, files: Sequence[bytes]):
        """Device-resident copy of the inputs (``kc_input_upload``)."""
        arr, keep = _buffers(files)
        p = C.c_void_p()
        _check(lib().kc_input_upload(self._h, arr, len(files), C.byref(p)))
        return p

    def free_input(self, p):
        lib().kc_input_free(self._h, p)

    def submit(self, files: Sequence[bytes] = (), input=None, **kw) -> int:
        j = self.make_job(**kw)
        arr, keep = _buffers(files)
        j.files = C.cast(arr, C.POINTER(kc_buffer))
        j.n_files = len(files)
        if input is not None:
            j.input = input
        jid = C.c_uint64()
        _check(lib().kc_submit(self._h, C.byref(j), C.byref(jid)))
        self._inputs[jid.value] = (arr, keep)   # host buffers stay alive until wait()
        return jid.value

    def submit_batch(self, samples: Sequence[Sequence[bytes]], ks: Sequence[int], **kw) -> List[int]:
        n = len(samples)
        jobs = (kc_job * n)()
        keep = []
        for i, (files, k) in enumerate(zip(samples, ks)):
            j = self.make_job(k=k, **kw)
            arr, kk = _buffers(files)
            keep.append((arr, kk))
            j.files = C.cast(arr, C.POINTER(kc_buffer))
            j.n_files = len(files)
            jobs[i] = j
        ids = (C.c_uint64 * n)()
        _check(lib().kc_submit_batch(self._h, jobs, n, ids))
        for i in range(n):
            self._inputs[ids[i]] = keep[i]
        return list(ids)

    def wait(self, jid: int, timeout_ms: int = -1):
        try:
            _check(lib().kc_wait(self._h, jid, timeout_ms))
        finally:
            pass

    def result(self, jid: int, k: int, release: bool = True, copy: bool = True) -> Result:
        """Results of a finished job.  copy=False returns the sorted records
        and the count <= 2 set as views of the job's pinned host memory; the
        job is released when the last view is gone."""
        r = kc_result_t()
        _check(lib().kc_result(self._h, jid, C.byref(r)))
        w = max(1, r.key_words)
        if copy:
            keys, counts = _copy(r.keys, r.n_records * w, np.uint64), _copy(r.counts, r.n_records, np.uint32)
            le2_keys, le2_counts = _copy(r.le2_keys, r.n_le2 * w, np.uint64), _copy(r.le2_counts, r.n_le2, np.uint32)
        else:
            # records and the count <= 2 set (often most of the k-mers) stay in
            # the job's pinned memory until the last view is gone
            lease = _JobLease(self, jid)
            keys = _view(r.keys, r.n_records * w, np.uint64, lease)
            counts = _view(r.counts, r.n_records, np.uint32, lease)
            le2_keys = _view(r.le2_keys, r.n_le2 * w, np.uint64, lease)
            le2_counts = _view(r.le2_counts, r.n_le2, np.uint32, lease)
            release = False
        out = Result(
            k=k,
            keys=_keys(keys, w), counts=counts,
            hist=_copy(r.hist, r.hist_len, np.int64), hist_min=0,
            top_keys=_keys(_copy(r.top_keys, r.n_top * w, np.uint64), w),
            top_counts=_copy(r.top_counts, r.n_top, np.uint32),
            le2_keys=_keys(le2_keys, w), le2_counts=le2_counts,
            occurrences=r.occurrences, distinct=r.distinct, low_only=r.low_only,
            table_capacity=r.table_capacity, device_ms=r.device_ms, queue_ms=r.queue_ms, run_ms=r.run_ms,
            phase_ms=tuple(r.phase_ms), phase_launches=tuple(r.phase_launches), low_len=r.low_len,
            high_len=r.high_len, input_bytes=r.input_bytes, n_records_total=r.n_records_total, passes=r.passes,
            smem_passes=r.smem_passes, smem_fallbacks=r.smem_fallbacks, region_redos=r.region_redos,
            batch_part=r.batch_part)
        if release:
            self.release(jid)
        return out

    def cancel(self, jid: int) -> bool:
        """Cancels a queued or running job (``kc_cancel``); its wait() then
        raises KC_ERR_CANCELLED.  False when the job had already finished."""
        rc = lib().kc_cancel(self._h, jid)
        if rc == KC_OK:
            return True
        if rc == 1:   # KC_ERR_INVALID: finished already, its results stand
            return False
        _check(rc)
        return False

    def release(self, jid: int):
        self._inputs.pop(jid, None)
        _check(lib().kc_release(self._h, jid))

    def write_tmpdir(self, jid: int, path: str):
        _check(lib().kc_write_tmpdir(self._h, jid, path.encode()))

    def count(self, files: Sequence[bytes] = (), input=None, copy: bool = True, **kw) -> Result:
        """One job: FASTQ files -> exact canonical counts (blocking)."""
        jid = self.submit(files, input=input, **kw)
        self.wait(jid)
        res = self.result(jid, kw.get("k", 31), copy=copy)
        res.hist_min = kw.get("hist_min", 1)
        return res

    @property
    def tuning(self) -> dict:
        """The handle's speed/memory settings (``kc_get_tuning``)."""
        t = kc_tuning()
        _check(lib().kc_get_tuning(self._h, C.byref(t)))
        return {"bucket_table_factor": t.bucket_table_factor, "table_factor": t.table_factor,
                "sort_group_records": t.sort_group_records, "bloom_smem": t.bloom_smem, "record_sort": t.record_sort,
                "sampled_region_keys": t.sampled_region_keys, "count_shape": t.count_shape,
                "part_shape": t.part_shape, "scatter_shape": t.scatter_shape}

    def set_tuning(self, bucket_table_factor: float = 0.0, table_factor: float = 0.0, sort_group_records: int = 0,
                   bloom_smem: int = 0, record_sort: int = 0, sampled_region_keys: int = 0, count_shape: int = 0,
                   part_shape: int = 0, scatter_shape: int = 0):
        """0 (or less) keeps a setting.  bloom_smem: 1 counts Bloom jobs (min
        count >= 2) per sub-bucket in shared memory, 2 on global-memory tables.
        record_sort: 1 sorts large jobs' records most significant bits first,
        2 with the LSD radix sort.  count_shape: the shared-memory count's
        block shape, 1..4; part_shape: the partition's round size, 1 or 2;
        scatter_shape: the sub-bucket scatter's variant, 1 or 2 (kc_tuning in
        include/kc.h)."""
        t = kc_tuning()
        t.bucket_table_factor, t.table_factor, t.sort_group_records = bucket_table_factor, table_factor, \
            sort_group_records
        t.bloom_smem = bloom_smem
        t.record_sort = record_sort
        t.sampled_region_keys = sampled_region_keys
        t.count_shape = count_shape
        t.part_shape = part_shape
        t.scatter_shape = scatter_shape
        _check(lib().kc_set_tuning(self._h, C.byref(t)))

    def autotune(self, samples: Sequence[Sequence[bytes]] = (), ks: Sequence[int] = (), batch: bool = False,
                 inputs: Sequence = (), **kw) -> dict:
        """Runs the given jobs (FASTQ files per job, or resident inputs) once
        per candidate setting and keeps the fastest settings (``kc_autotune``)."""
        n = len(inputs) if inputs else len(samples)
        jobs = (kc_job * n)()
        keep = []
        for i in range(n):
            j = self.make_job(k=ks[i] if ks else kw.get("k", 31), **{x: y for x, y in kw.items() if x != "k"})
            if inputs:
                j.input = inputs[i]
            else:
                arr, kk = _buffers(samples[i])
                j.files = C.cast(arr, C.POINTER(kc_buffer))
                j.n_files = len(samples[i])
                keep.append((arr, kk))
            jobs[i] = j
        best = kc_tuning()
        _check(lib().kc_autotune(self._h, jobs, n, int(batch), C.byref(best)))
        return self.tuning

    def count_batch(self, samples: Sequence[Sequence[bytes]], ks: Sequence[int], copy: bool = True,
                    **kw) -> List[Result]:
        """Many samples as one batched job (``kc_submit_batch``); copy=False
        returns each sample's records as views of pinned host memory."""
        ids = self.submit_batch(samples, ks, **kw)
        out = []
        for jid, k in zip(ids, ks):
            self.wait(jid)
            r = self.result(jid, k, copy=copy)
            r.hist_min = kw.get("hist_min", 1)
            out.append(r)
        return out


# ---- single steps ----------------------------------------------------------

def kernel_launches() -> int:
    """Kernel launches issued by libkc.so in this process."""
    return int(lib().kc_kernel_launches())


def atomic_peak(buffer_bytes: int, repeats: int = 5):
    """(atomics/s, ms per launch) of random 32-bit atomicAdd over a device
    buffer of buffer_bytes (power of two)."""
    rate, ms = C.c_double(), C.c_double()
    _check(lib().kc_atomic_peak(buffer_bytes, repeats, C.byref(rate), C.byref(ms)))
    return rate.value, ms.value


def atomic_peak_shared(table_bytes: int = 16384, repeats: int = 5):
    """(atomics/s, ms per launch) of random 32-bit atomicAdd on a
    shared-memory table of table_bytes per block."""
    rate, ms = C.c_double(), C.c_double()
    _check(lib().kc_atomic_peak_shared(table_bytes, repeats, C.byref(rate), C.byref(ms)))
    return rate.value, ms.value


def extract_kmers(fastq: bytes, k: int) -> np.ndarray:
    """Canonical k-mer occurrences of one FASTQ file (unordered): shape (n,)
    for k <= 32, (n, N) kmer<N> word arrays for k > 32."""
    data = np.frombuffer(fastq, dtype=np.uint8) if len(fastq) else np.zeros(1, np.uint8)
    w = key_words(k)
    cap = max(len(fastq), 1)
    out = np.zeros(cap * w, np.uint64)
    n = C.c_uint64()
    _check(lib().kc_extract_kmers(_ptr(data), len(fastq), k, _ptr(out), cap, C.byref(n)))
    return _keys(out[: n.value * w].copy(), w)


def hash_kmers(keys: np.ndarray) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.zeros(5 * max(len(keys), 1), np.uint64)
    _check(lib().kc_hash_kmers(_ptr(keys), len(keys), _ptr(out)))
    return out[: 5 * len(keys)].reshape(-1, 5)


def sort_records(keys: np.ndarray, counts: np.ndarray, bits: int):
    keys = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    counts = np.ascontiguousarray(counts, dtype=np.uint32).copy()
    _check(lib().kc_sort_records(_ptr(keys), _ptr(counts), len(keys), bits))
    return keys, counts


def sort_distinct_records(keys: np.ndarray, counts: np.ndarray, bits: int):
    """Records with distinct keys sorted on their low `bits` bits
    (``kc_sort_distinct_records``)."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    counts = np.ascontiguousarray(counts, dtype=np.uint32).copy()
    _check(lib().kc_sort_distinct_records(_ptr(keys), _ptr(counts), len(keys), bits))
    return keys, counts


def bloom_plan(files: Sequence[bytes], k: int, memory_gb: int):
    arr, keep = _buffers(files)
    pc = np.zeros(256, np.uint32)
    caps = np.zeros(256, np.uint64)
    avg = C.c_uint32()
    mx = C.c_uint64()
    _check(lib().kc_bloom_plan(arr, len(files), k, memory_gb, _ptr(pc), C.byref(avg), _ptr(caps), C.byref(mx)))
    return pc, avg.value, caps, mx.value


def plan_bloom(raw_prefix_counts, avg_quality: int, est_file_size: int, memory_gb: int, k: int):
    """The reference's Bloom filter sizing (host arithmetic only)."""
    pc = np.ascontiguousarray(raw_prefix_counts, dtype=np.uint32)
    caps = np.zeros(256, np.uint64)
    mx = C.c_uint64()
    _check(lib().kc_plan_bloom(_ptr(pc), avg_quality, est_file_size, memory_gb, k, _ptr(caps), C.byref(mx)))
    return caps, mx.value


def merge_records(high_keys, high_counts, low_keys, k: int, count_max: int, min_count: int = 1,
                  max_count: int = U32_MAX, hist_min: int = 1, hist_max: int = 10000):
    w = key_words(k)
    hk = np.ascontiguousarray(high_keys, dtype=np.uint64).reshape(-1)
    hc = np.ascontiguousarray(high_counts, dtype=np.uint32)
    lk = np.ascontiguousarray(low_keys, dtype=np.uint64).reshape(-1)
    nh, nl = len(hc), len(lk) // w
    cap = max(nh + nl, 1)
    ok = np.zeros(cap * w, np.uint64)
    oc = np.zeros(cap, np.uint32)
    hist = np.zeros(hist_max - hist_min + 1, np.int64)
    n = C.c_uint64()
    _check(lib().kc_merge_records(_ptr(hk), _ptr(hc), nh, _ptr(lk), nl, k, count_max, min_count,
                                  max_count, hist_min, hist_max, _ptr(ok), _ptr(oc), cap, C.byref(n), _ptr(hist)))
    return _keys(ok[: n.value * w], w), oc[: n.value], hist


# ---- text outputs of the reference tools -------------------------------------

def histogram_text(hist: np.ndarray, hist_min: int) -> str:
    """histogram_tool output: ``f\\tcount\\n`` for every f (tool/histogram_tool.cpp:462-478)."""
    return "".join(f"{hist_min + i}\t{int(v)}\n" for i, v in enumerate(hist))


def dump_text(keys: np.ndarray, counts: np.ndarray, k: int) -> str:
    """dump_tool output: ``KMER\\tcount\\n`` lines (tool/dump_tool.cpp:1172-1193),
    formatted on the device (``kc_dump_text``)."""
    return dump_bytes(keys, counts, k).decode("ascii")


def dump_bytes(keys: np.ndarray, counts: np.ndarray, k: int) -> bytes:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    n = len(counts)   # k > 32: keys has shape (n, N)
    need = C.c_uint64()
    _check(lib().kc_dump_text(_ptr(keys), _ptr(counts), n, k, None, 0, C.byref(need)))
    out = np.empty(max(need.value, 1), np.uint8)
    got = C.c_uint64()
    _check(lib().kc_dump_text(_ptr(keys), _ptr(counts), n, k, _ptr(out), out.nbytes, C.byref(got)))
    return out[: got.value].tobytes()
