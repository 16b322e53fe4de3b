#!/usr/bin/env python
"""Benchmark of the counting path: k-mers counted per second, bit-exact.

Default workload (N=1): the single large job -- a seeded 100 Mbp genome with
5% from 200 repeat families, 30x coverage of 150 bp reads (~20M reads, ~6.3 GB
FASTQ), 1% substitutions, k = 31, the reference's Bloom singleton split with
its filter sizing, min count 2, outputs sorted records + histogram.  Synthetic
input of that shape stands in for sequencing data (the reference measures no
public dataset).

A step is one counting job over the whole FASTQ:
  value -- input resident in HBM (kc_input_upload once), device time of the
           job from CUDA events on its stream (sum over the timed steps);
  e2e   -- the same job through the C ABI from pinned host buffers (after two
           untimed warm-up jobs that bring the worker to steady state): upload,
           counting, and the sorted records + histogram copied back, timed by
           the host clock.
--impl reference times the reference's own CPU programs (compiled from its
sources into oracle/_ref, or the directory KC_REF_BIN names) on a bounded
sample of the same workload (the first --ref-reads reads): kmer_counter and
histogram_tool precise, i.e. the records seen at least twice (high.bin) and
the histogram, the same outputs as a job here less the sort; where they are
absent it times the oracle's C restatement of the path instead ("kind":
"port").  Both arms print the same "config".

Multi-GPU: the path is run as independent replicas (one job per GPU); value is
all replicas' k-mers over the slowest replica's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

U32 = 0xFFFFFFFF
METRIC = "k-mers counted/s (bit-exact)"
MEMORY_GB = 64          # reference <memory_limit_gb>: sizes the Bloom filters
READ_LEN = 150
WORKLOAD = ("single large job (100 Mbp genome, 5% repeats from 200 families, 30x 150 bp, 1% errors, k=31, "
            "Bloom singleton filter, min count 2)")


def large_job_fastq_bytes(n_reads: int) -> int:
    """Bytes of the generator's FASTQ of n_reads reads of READ_LEN bases:
    "@r<i>\n", the bases, "\n+\n", the qualities, "\n" for i = 0 .. n - 1."""
    digits, lo, width = 0, 0, 1
    while lo < n_reads:
        hi = min(n_reads, 10 ** width)
        digits += (hi - lo) * width
        lo, width = hi, width + 1
    return n_reads * (2 * READ_LEN + 7) + digits


def workload_config(scale: float, world: int) -> dict:
    """The "config" object of both arms' lines: the large job at this scale
    (genome, reads, FASTQ bytes, occurrences; the reads carry no N, so every
    read holds READ_LEN - 31 + 1 windows)."""
    genome_len = max(1_000_000, int(100_000_000 * scale))
    n_reads = int(math.ceil(30.0 * genome_len / READ_LEN))
    return {"workload": WORKLOAD, "genome_bp": genome_len, "reads": n_reads,
            "fastq_bytes": large_job_fastq_bytes(n_reads), "occurrences_per_step": n_reads * (READ_LEN - 31 + 1),
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (FASTQ > 126 MB)",
            "memory_gb": MEMORY_GB, "scale": scale}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def make_input(scale: float, kc):
    """The large-job FASTQ, written straight into pinned host memory."""
    import ctypes as C
    import numpy as np
    import ktcountermemorygreedy_b200.synth as S
    genome_len = max(1_000_000, int(100_000_000 * scale))
    n_reads = S.large_job_reads(30.0, genome_len)
    size = S.reads_size(2, n_reads, (150, 150))
    p = C.c_void_p()
    kc._check(kc.lib().kc_host_alloc(size, C.byref(p)))
    buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(size,))
    g = S.large_job_genome(genome_len)
    fq = S.reads(g, 2, n_reads, (150, 150), 0.01, 0.0, out=buf)
    return fq, p, genome_len, n_reads


JOB = dict(k=31, count_max=U32, bloom=True, memory_gb=MEMORY_GB, min_count=2, hist_min=2, hist_max=10000)


def algorithmic_bytes(phase: str, r):
    """Bytes a stage must move at minimum (per launch), from the unit costs:
    S FASTQ bytes, O occurrences, h/l the non-FIRST/FIRST list lengths,
    cap table slots, U distinct k-mers."""
    S, O = r.input_bytes, r.occurrences
    if phase == "count_pass":          # Bloom mode: FASTQ + bucketed k-mer write; plain: FASTQ + table update
        return S + 8 * O if r.low_len + r.high_len else S + 16 * O
    if phase == "bloom":               # bucketed k-mers read + list write (16 B) + two filter words (16 B)
        return 32 * O
    if phase == "sub_partition":       # bucketed k-mers read + written in sub-bucket order, plus the
        # count that sizes the sub-buckets: 1 in 8 keys sampled on a large pass, every key otherwise
        return 16 * O + (O if O >= (64 << 20) else 8 * O)
    if phase == "smem_count":          # sub-bucket k-mers read, FIRST ones written back and read again, records
        return 8 * O + 16 * r.low_len + 12 * r.n_records_total
    if phase == "insert_high":         # list read (8 B) + slot key read and count update (16 B)
        return 24 * r.high_len
    if phase == "merge_low":
        return 24 * r.low_len
    if phase == "compact":
        return 16 * r.table_capacity + 12 * r.n_records_total
    if phase == "sort":
        # the sort row's unit: P 8-bit passes over 62 bits, each reading and
        # writing a 12 B record (P * 24 * R).  The most-significant-bits-first
        # sort of 1M-201M records moves less for the same result (a bucket
        # histogram, two scatter passes and the bucket sort: 8R + 3 * 24R)
        R = r.n_records_total
        return math.ceil(2 * 31 / 8) * 24 * R
    if phase == "census":
        return S
    if phase == "scan":
        # Bloom jobs read the 1-in-8 census tiles and the pre-pass sample
        # (the first 256 MiB); plain jobs every tile
        return S // 8 + min(S, 256 << 20) if r.low_len + r.high_len else S
    return 0


def traffic_for(phase: str, r):
    """DRAM bytes per launch of the stage's kernel from a committed ncu summary
    (profiles/dram_traffic.json), scaled by the occurrences it processed."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(phase)
    if not d:
        return None
    per_occ = d["dram_bytes"] / max(1, d["occurrences"])
    return int(per_occ * r.occurrences)


# ---------------------------------------------------------------------------
# the reference's CPU programs
# ---------------------------------------------------------------------------

def reference_dir() -> str:
    return os.environ.get("KC_REF_BIN") or os.path.join(ROOT, "oracle", "_ref")


def reference_programs_present() -> bool:
    return all(os.access(os.path.join(reference_dir(), p), os.X_OK)
               for p in ("kmer_counter", "histogram_tool", "dump_tool"))


def reference_run(fastq_path: str, threads: int, mem_gb: int, tmp: str, dump: bool = False):
    """kmer_counter + histogram_tool precise (min 2), timed: the records seen
    at least twice (high.bin) and the histogram.  dump: then, untimed,
    dump_tool precise --sort (min 1: the tool's output above min 1 is not
    deterministic), for a byte comparison.  Returns (wall seconds of the
    timed programs, occurrences); the histogram is left in tmp/h.tsv and the
    dump in tmp/d.txt."""
    ref = reference_dir()
    d = os.path.join(tmp, "t")
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(d)
    t0 = time.perf_counter()
    p = subprocess.run([os.path.join(ref, "kmer_counter"), fastq_path, "31", str(threads), str(mem_gb), d, "1024",
                        "2", str(U32), str(U32)], capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"reference kmer_counter failed: {p.stderr[-500:]}")
    subprocess.run([os.path.join(ref, "histogram_tool"), "precise", d, str(threads), str(mem_gb),
                    os.path.join(tmp, "h.tsv"), "2", "10000"], check=True, capture_output=True)
    wall = time.perf_counter() - t0
    if dump:
        subprocess.run([os.path.join(ref, "dump_tool"), "precise", d, str(threads), str(mem_gb),
                        os.path.join(tmp, "d.txt"), "1", str(U32), "--sort"], check=True, capture_output=True)
    occ = 0
    for line in p.stdout.splitlines():
        if line.startswith("Total read k-mer count:"):
            occ = int(line.split(":")[1])
    return wall, occ


def port_run(fastq_path: str):
    """The oracle's C restatement of the same path on one thread, where the
    reference programs are absent: extraction, exact counts, records in
    printed-string order and the histogram (no text).  Returns (wall seconds,
    occurrences)."""
    for p in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "tests", "golden")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import oracle_lib as O
    data = open(fastq_path, "rb").read()
    t0 = time.perf_counter()
    keys = O.extract(data, 31)
    uk, uc = O.count(keys)
    sk, sc = O.sort_string_order(uk, uc, 31)
    O.histogram(sc, 2, 10000)
    return time.perf_counter() - t0, len(keys)


def cpu_sample_run(path: str, threads: int, mem_gb: int, tmp: str, dump: bool = False):
    """(wall seconds, occurrences, kind, cores, what ran) for one sample."""
    if reference_programs_present():
        w, occ = reference_run(path, threads, mem_gb, tmp, dump=dump)
        return w, occ, "reference", threads, ("kmer_counter + histogram_tool precise: the records seen at least "
                                                "twice (high.bin) and the histogram")
    w, occ = port_run(path)
    return w, occ, "port", 1, "oracle port (extraction, exact counts, sort, histogram), one thread"


GEN = os.path.join(ROOT, "ktcountermemorygreedy_b200", "bin", "fastq_gen")


def write_workload(path: str, n_reads: int, first_read: int = 0, genome_bp: int = 100_000_000) -> int:
    """Reads first_read .. first_read + n_reads - 1 of the large job's stream
    written to `path` by the generator program (a separate process: the
    caller maps no library of this project).  Returns the file's size."""
    if not os.access(GEN, os.X_OK):
        raise RuntimeError(f"{GEN} is missing; build it with __graft_entry__.build()")
    subprocess.run([GEN, "large", str(genome_bp), str(first_read), str(n_reads), path], check=True)
    return os.path.getsize(path)


def reference_sample(sample_reads: int, tmp: str):
    """First `sample_reads` reads of the large job's stream (same genome and
    read generator) written to a file."""
    path = os.path.join(tmp, "sample.fq")
    return path, write_workload(path, sample_reads)


def cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return os.cpu_count() or 1, model


REF_ARM_BUDGET_S = 240.0   # seconds for the whole --impl reference run (warm-up and timed steps)
REF_ARM_MIN_READS = 100_000


def run_reference_arm(args):
    """The reference's programs on the first --ref-reads reads, W warm-up and
    K timed steps.  When the first warm-up step shows that W + K steps of
    that sample would take longer than REF_ARM_BUDGET_S (KC_REF_BUDGET_S),
    the sample shrinks to fit (not below REF_ARM_MIN_READS reads); the line
    names the sample that was timed."""
    threads, model = cpu_info()
    threads = max(6, threads)
    mem = int(os.environ.get("KC_REF_MEM_GB", "32"))
    budget = float(os.environ.get("KC_REF_BUDGET_S", REF_ARM_BUDGET_S))
    reads = args.ref_reads
    with tempfile.TemporaryDirectory() as tmp:
        path, nbytes = reference_sample(reads, tmp)
        w0 = cpu_sample_run(path, threads, mem, tmp)[0]
        per_step = budget / max(1, args.steps + args.warmup)
        if w0 > per_step and reads > REF_ARM_MIN_READS:
            reads = max(REF_ARM_MIN_READS, int(reads * per_step / w0))
            path, nbytes = reference_sample(reads, tmp)
            cpu_sample_run(path, threads, mem, tmp)
        for _ in range(args.warmup - 1):
            cpu_sample_run(path, threads, mem, tmp)
        walls, occ = [], 0
        for _ in range(args.steps):
            w, occ, kind, cores, what = cpu_sample_run(path, threads, mem, tmp)
            walls.append(w)
    t = sum(walls)
    value = occ * args.steps / t
    sample = f"first {reads} reads of the large job ({nbytes} B FASTQ, {occ} k-mers), {what}"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "k-mers/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": workload_config(args.scale, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": "k-mers/s", "cores": cores, "kind": kind,
                         "sample": sample, "cpu": model},
        "e2e": {"value": value, "unit": "k-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line, default=_json_default), flush=True)


# ---------------------------------------------------------------------------
# CPU leg of our arm: the reference's programs timed on a sample of the
# workload, and the parity checks of what the GPU counted (the oracle and the
# reference programs are the checkers here; nothing of this is timed as ours
# except the GPU's own runs on the sample)
# ---------------------------------------------------------------------------

def _checker():
    for p in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "tests", "golden")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import size_parity
    return size_parity


def sample_on_gpu(counter, kc, path: str, reps: int = 3):
    """The GPU on the same sample file as the CPU baseline: device-resident
    k-mers/s (CUDA events) and end to end from pinned host memory (host
    clock), and the records + histogram of one run."""
    import ctypes as C
    import numpy as np
    size = os.path.getsize(path)
    p = C.c_void_p()
    kc._check(kc.lib().kc_host_alloc(size, C.byref(p)))
    buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(size,))
    buf[:] = np.fromfile(path, np.uint8)
    inp = counter.upload([buf])
    dev, occ = [], 0
    for i in range(reps + 2):
        r = counter.count(input=inp, keep_records=False, **JOB)
        if i >= 2:
            dev.append(r.device_ms)
            occ = r.occurrences
    counter.free_input(inp)
    walls = []
    res = None
    for i in range(reps + 2):
        res = None
        t0 = time.perf_counter()
        res = counter.count([buf], keep_records=True, **JOB)
        if i >= 2:
            walls.append(time.perf_counter() - t0)
    kc.lib().kc_host_free(p)
    value = {"device": occ / (statistics.median(dev) / 1000.0), "e2e": occ / statistics.median(walls),
             "unit": "k-mers/s", "occurrences": occ,
             "note": "the GPU on the cpu_baseline sample file (same bytes), median of "
                     f"{reps}: device-resident (CUDA events) and from pinned host memory (host clock)"}
    return value, res


def full_reference_check(args, counter, fq, full):
    """The reference programs once on the whole workload (its FASTQ written
    to a file by the generator program): counter + histogram_tool precise
    (min 2), wall time, and the histogram text against the GPU job's."""
    import ktcountermemorygreedy_b200 as kc
    threads, model = cpu_info()
    mem = int(os.environ.get("KC_REF_MEM_GB", "64"))
    ram_gb = None
    try:
        ram_gb = round(os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2**30)
    except (ValueError, OSError):
        pass
    if not reference_programs_present():
        return {"status": "not run: the reference programs are absent"}
    with tempfile.TemporaryDirectory(dir=os.environ.get("KC_REF_TMP")) as tmp:
        path = os.path.join(tmp, "full.fq")
        n_reads = int(math.ceil(30.0 * 100_000_000 / 150))
        nbytes = write_workload(path, n_reads)
        if nbytes != len(fq):
            return {"status": f"not run: the generator wrote {nbytes} B, the job has {len(fq)} B"}
        w, occ = reference_run(path, max(6, threads), mem, tmp, dump=False)
        if full is None:
            full = counter.count([fq], keep_records=False, **JOB)
        same = open(os.path.join(tmp, "h.tsv")).read() == kc.histogram_text(full.hist, JOB["hist_min"])
    return {"histogram_identical": same, "wall_s": round(w, 2), "occurrences": occ,
            "kmers_per_s": occ / w, "cores": max(6, threads), "cpu": model, "ram_gb": ram_gb, "memory_gb_arg": mem,
            "how": "kmer_counter <fq> 31 <cores> <mem> <tmp> 1024 2 u32max u32max + histogram_tool precise "
                   "<tmp> <cores> <mem> h.tsv 2 10000 on the whole 20M-read FASTQ; h.tsv against the GPU job's "
                   "histogram text"}


def cpu_leg(args, counter, fq, full):
    """cpu_baseline: the reference programs (or the oracle port) timed on the
    first --ref-reads reads, and the GPU on the same file (sample_value);
    parity: the GPU's histogram text and sorted dump against the reference
    programs' on the first --parity-reads reads (their dump lists every
    k-mer, singletons included, so its sample is the smaller one), and the
    whole job against the oracle's hash sample."""
    import ktcountermemorygreedy_b200 as kc
    SP = _checker()
    threads, model = cpu_info()
    mem = int(os.environ.get("KC_REF_MEM_GB", "32"))
    cpu = sample_value = None
    parity = {}
    try:
        with tempfile.TemporaryDirectory() as tmp:
            path, nbytes = reference_sample(args.ref_reads, tmp)
            w, o, kind, cores, what = cpu_sample_run(path, max(6, threads), mem, tmp)
            cpu = {"value": o / w, "unit": "k-mers/s", "cores": cores, "kind": kind,
                   "sample": f"first {args.ref_reads} reads of the workload ({nbytes} B, {o} k-mers), "
                             f"{what}, {model}"}
            sample_value, _ = sample_on_gpu(counter, kc, path)
            os.unlink(path)
            if kind == "reference":
                ppath = os.path.join(tmp, "parity.fq")
                write_workload(ppath, args.parity_reads)
                reference_run(ppath, max(6, threads), mem, tmp, dump=True)
                res = counter.count([open(ppath, "rb").read()], keep_records=True, **JOB)
                chk = SP.reference_outputs_match(kc.histogram_text(res.hist, JOB["hist_min"]),
                                                 kc.dump_bytes(res.keys, res.counts, JOB["k"]),
                                                 os.path.join(tmp, "h.tsv"), os.path.join(tmp, "d.txt"),
                                                 JOB["k"], JOB["min_count"])
                chk["reads"] = args.parity_reads
                parity["sample"] = "identical" if chk["identical"] else "DIFFERENT"
                parity["sample_detail"] = chk
            else:
                parity["sample"] = "not checked (the reference programs are absent)"
    except Exception as e:   # the baseline is reported, never required
        cpu = cpu or {"value": None, "unit": "k-mers/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}
        parity.setdefault("sample", f"failed: {e}")
    if args.full_reference:
        parity["full_reference"] = full_reference_check(args, counter, fq, full)
    try:
        if full is None:
            full = counter.count([fq], keep_records=True, copy=False, **JOB)
        chk = SP.full_spot_check(fq, JOB["k"], full.keys, full.counts, full.hist, JOB["hist_min"],
                                 JOB["min_count"], threads=max(1, threads))
        parity["full"] = "identical" if chk["identical"] else "DIFFERENT"
        parity["full_detail"] = chk
    except Exception as e:
        parity["full"] = f"failed: {e}"
    return cpu, parity, sample_value


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


SERVED_JOB = dict(count_max=U32, min_count=1, hist_min=1, hist_max=10000, top_n=1000, want_le2=True,
                  keep_records=False)


def served_bench(kc, args, local):
    """Served request stream: Poisson arrivals, log-normal job sizes (median
    200k reads, sigma 1.5), 150 bp reads at 1% from one shared 50 Mbp genome,
    k from {21, 25, 31}; every job returns its histogram, top-1000 and
    count <= 2 queries.  Jobs are contiguous runs of a pool of reads drawn from
    the genome (the pool bounds the largest job).  Each rate is measured on
    its own stream of jobs; 'plain' is the same jobs one at a time through a
    handle with one worker."""
    import ctypes as C
    import numpy as np
    import ktcountermemorygreedy_b200.synth as S
    from ktcountermemorygreedy_b200 import serving
    pool_reads = args.served_pool_reads
    g = S.genome(4, 50_000_000)
    size = S.reads_size(4, pool_reads, (150, 150))
    p = C.c_void_p()
    kc._check(kc.lib().kc_host_alloc(size, C.byref(p)))
    buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(size,))
    fq = S.reads(g, 4, pool_reads, (150, 150), 0.01, 0.0, out=buf)
    nl = np.flatnonzero(fq == 10)
    starts = np.concatenate([[0], nl[3::4] + 1]).astype(np.int64)   # byte offset of read i (and the end)

    def make_requests(rate, n_jobs, seed):
        rng = np.random.default_rng(seed)
        t, reqs = 0.0, []
        for _ in range(n_jobs):
            t += float(rng.exponential(1.0 / rate))
            n = int(min(pool_reads, max(1.0, math.exp(rng.normal(math.log(200_000), 1.5)))))
            k = int(rng.choice([21, 25, 31]))
            i0 = int(rng.integers(0, pool_reads - n + 1))
            reqs.append(serving.Request(t, [fq[starts[i0]:starts[i0 + n]]], k, dict(SERVED_JOB)))
        return reqs

    # every worker's device workspace is grown to the largest job shape (the
    # whole pool, k=21: the most k-mers) before the timed streams, as a server
    # sized for its largest request would be
    def warm(h, workers):
        big = [serving.Request(0.0, [fq], 21, dict(SERVED_JOB)) for _ in range(workers)]
        serving.serve(h, big)

    out = {"workload": f"served stream: Poisson arrivals, log-normal sizes (median 200k reads, sigma 1.5, "
                       f"capped at the {pool_reads}-read pool), 150 bp at 1% from a 50 Mbp genome, "
                       f"k in {{21,25,31}}, histogram + top-1000 + count<=2 per job",
           "max_inflight_jobs": args.served_inflight, "pinned_arena_gb": args.served_pinned_gb, "rates": {}}
    pinned = args.served_pinned_gb << 30
    with kc.KmerCounter(device=local, max_inflight_jobs=1, pinned_bytes=pinned) as plain:
        warm(plain, 1)
        reqs = make_requests(1e9, args.served_jobs, 4000)   # all at once, one worker: back to back
        stats, wall = serving.serve(plain, reqs)
        out["plain"] = serving.summarize(stats, wall)
    with kc.KmerCounter(device=local, max_inflight_jobs=args.served_inflight) as srv:   # shares the arena
        warm(srv, args.served_inflight)
        for rate in args.served_rates:
            reqs = make_requests(rate, args.served_jobs, 4000 + int(rate))
            stats, wall = serving.serve(srv, reqs)
            out["rates"][str(rate)] = serving.summarize(stats, wall)
    kc.lib().kc_host_free(p)
    return out


def _json_default(o):
    """numpy scalars (and anything else with .item()) as plain JSON values."""
    if hasattr(o, "item"):
        return o.item()
    raise TypeError(f"not JSON serializable: {type(o).__name__}")


def records_digest(r):
    """Position-dependent digest of a job's records and histogram (in chunks,
    so that billions of records need no large temporaries)."""
    import numpy as np
    keys, counts = np.asarray(r.keys).reshape(-1), np.asarray(r.counts)
    mix = np.uint64(0x9E3779B97F4A7C15)
    acc = [len(counts), int(np.asarray(r.hist).astype(np.int64).sum()),
           hash(np.asarray(r.hist).tobytes())]
    s1 = s2 = np.uint64(0)
    step = 1 << 24
    with np.errstate(over="ignore"):
        for a in range(0, len(keys), step):
            kk = keys[a:a + step]
            idx = np.arange(a, a + len(kk), dtype=np.uint64)
            s1 += np.bitwise_xor(kk, idx * mix).sum(dtype=np.uint64)
            s2 += ((kk >> np.uint64(17)) * (idx | np.uint64(1))).sum(dtype=np.uint64)
        for a in range(0, len(counts), step):
            cc = counts[a:a + step].astype(np.uint64)
            idx = np.arange(a, a + len(cc), dtype=np.uint64)
            s2 += (cc * (idx * mix | np.uint64(1))).sum(dtype=np.uint64)
    return tuple(acc) + (int(s1), int(s2))


def batched_bench(kc, args, local):
    """Batched samples: each sample has its own seeded 5-50 Mbp genome,
    log-uniform read count in [1e4, 2e6] (times --batch-scale), read lengths
    U[100, 250], substitutions U[0.5%, 2%], k = 21 / 31 alternating.  All
    samples go to the device as one batched job (per-sample tables in one
    arena, one extraction launch over all samples, segmented sort) and, for
    comparison, as one job per sample through a one-worker handle.  Both
    include the host->device upload and the records + histograms coming back
    to pinned host memory."""
    import ctypes as C
    import numpy as np
    import ktcountermemorygreedy_b200.synth as S
    samples = S.batch_samples(args.batch_samples, scale=args.batch_scale)
    # the samples sit in pinned host memory, as a server's receive buffers would
    total = sum(len(fq) for fq, _ in samples)
    p = C.c_void_p()
    kc._check(kc.lib().kc_host_alloc(max(total, 1), C.byref(p)))
    buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(max(total, 1),))
    files, off = [], 0
    for fq, _ in samples:
        buf[off:off + len(fq)] = fq
        files.append([buf[off:off + len(fq)]])
        off += len(fq)
    ks = [k for _, k in samples]
    del samples
    job = dict(count_max=U32, min_count=1, hist_min=1, hist_max=4095)
    # pinned host memory for the results set aside up front, as a server sized
    # for its batches would (about 2 bytes of records per FASTQ byte at these
    # error rates): pinning tens of GB on demand costs more than the batch
    host_bytes = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    pinned = min(2 * total, int(host_bytes * 0.4))
    with kc.KmerCounter(device=local, max_inflight_jobs=1, pinned_bytes=pinned) as h:
        # settings chosen by the autotuner on the first 32 samples (untimed)
        tuning = h.autotune(files[:32], ks[:32], batch=True, **job)
        for _ in range(2):                                   # warm-up: steady state of the worker
            h.count_batch(files, ks, copy=False, **job)
        t0 = time.perf_counter()
        res_b = h.count_batch(files, ks, copy=False, **job)
        t_b = time.perf_counter() - t0
        occ = sum(r.occurrences for r in res_b)
        # a batch larger than the device runs as sub-batches, each with its device time
        parts = {}
        for r in res_b:
            parts[r.batch_part] = r.device_ms
        dev_b = sum(parts.values())
        first_of = {}
        for r in res_b:
            first_of.setdefault(r.batch_part, r)
        stages_b = {kc.PHASES[i]: sum(r.phase_ms[i] for r in first_of.values()) for i in range(len(kc.PHASES))
                    if any(r.phase_ms[i] > 0 for r in first_of.values())}
        # digests of the batch's results, which then go back to the pinned
        # pool (two arms of full-size results would not fit in host memory)
        dig_b = [records_digest(r) for r in res_b]
        del res_b, first_of
        for f, k in zip(files, ks):                          # warm-up
            h.count(f, k=k, copy=False, **job)
        # one job per sample; each job's results are digested and released
        # between the timed calls
        t_p, dev_p, same = 0.0, 0.0, True
        for i, (f, k) in enumerate(zip(files, ks)):
            t0 = time.perf_counter()
            r = h.count(f, k=k, copy=False, **job)
            t_p += time.perf_counter() - t0
            dev_p += r.device_ms
            same = same and records_digest(r) == dig_b[i]
            del r
    fastq_bytes = int(sum(len(f[0]) for f in files))
    del files
    kc.lib().kc_host_free(p)
    return {"workload": f"{len(ks)} samples, own 5-50 Mbp genomes, log-uniform 1e4-2e6 reads x "
                        f"{args.batch_scale}, 100-250 bp, 0.5-2% errors, k=21/31",
            "samples": len(ks), "fastq_bytes": fastq_bytes, "occurrences": int(occ), "inputs": "pinned host memory",
            "batched_kmers_per_s": occ / t_b, "batched_s": t_b, "batched_device_ms": dev_b,
            "sub_batches": len(parts),
            "batched_stages_ms": stages_b,
            "plain_kmers_per_s": occ / t_p, "plain_s": t_p, "plain_device_ms": dev_p,
            "speedup_vs_plain": t_p / t_b, "identical_to_plain": bool(same), "tuning": tuning,
            "pinned_arena_gb": round(pinned / 2 ** 30, 1)}


def wide_bench(kc, args, counter, inp, fq):
    """k-mers of more than 32 bases (the reference's kmer<2>/kmer<4> paths)
    on the same resident workload and job settings (Bloom flag, min count 2):
    device k-mers/s over 3 timed jobs after one warm-up, then one job with
    records whose hash sample is checked against the oracle (CPU leg)."""
    out = {}
    for k in args.wide:
        try:
            out[str(k)] = wide_one(kc, args, counter, inp, fq, k)
        except Exception as e:   # reported in the line, never fatal to the headline
            out[str(k)] = {"k": k, "failed": str(e)}
    return out


def wide_one(kc, args, counter, inp, fq, k):
    """One k of wide_bench."""
    job = dict(JOB, k=k)
    counter.count(input=inp, keep_records=False, **job)
    rs = [counter.count(input=inp, keep_records=False, **job) for _ in range(3)]
    dev = sum(r.device_ms for r in rs) / len(rs)
    r0 = rs[-1]
    o = {"k": k, "key_words": kc.key_words(k), "occurrences": r0.occurrences, "device_ms": dev,
         "kmers_per_s": r0.occurrences / (dev / 1000.0), "records": r0.n_records_total, "passes": r0.passes,
         "stages_ms": {kc.PHASES[i]: r0.phase_ms[i] for i in range(len(kc.PHASES)) if r0.phase_ms[i] > 0}}
    if args.cpu_baseline:
        try:
            r = counter.count(input=inp, keep_records=True, copy=False, **job)
            threads, _ = cpu_info()
            chk = _checker().full_spot_check_wide(fq, k, r.keys, r.counts, r.hist, JOB["hist_min"],
                                                  JOB["min_count"], threads=max(1, threads), sample_bits=8)
            o["parity"] = "identical" if chk["identical"] else "DIFFERENT"
            o["parity_detail"] = chk
            del r
        except Exception as e:
            o["parity"] = f"failed: {e}"
    return o


def out_of_core_bench(kc, args, local):
    """Out-of-core single job: a seeded 3.1 Gbp genome with 45% repeats
    (2000 families of 0.3-6 kbp, 1-10^5 copies, 1-15% divergence), 10x of
    150 bp reads (about 207M reads, 65 GB FASTQ) with 1% substitutions, k=31,
    the reference's Bloom split, min count 2.  The job counts in passes over
    ranges of root prefixes within the device memory, each pass's records
    parked in pinned host memory until the final sort.  One job from pinned
    host buffers (upload included), host clock, and its device time; then the
    oracle checks a hash sample of its records (CPU leg)."""
    import ctypes as C
    import numpy as np
    import ktcountermemorygreedy_b200.synth as S
    glen = max(10_000_000, int(S.OUT_OF_CORE_GENOME_BP * args.ooc_scale))
    n_reads = S.out_of_core_reads(10.0, glen)
    size = S.reads_size(5, n_reads, (150, 150))
    t0 = time.perf_counter()
    p = C.c_void_p()
    kc._check(kc.lib().kc_host_alloc(size, C.byref(p)))
    buf = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(size,))
    g = S.out_of_core_genome(glen)
    fq = S.reads(g, 5, n_reads, (150, 150), 0.01, 0.0, out=buf)
    del g
    gen_s = time.perf_counter() - t0
    job = dict(JOB)
    out = {"workload": f"out-of-core job: {glen} bp genome, 45% repeats (2000 families 0.3-6 kbp, 1-1e5 copies, "
                       f"1-15% divergence), 10x 150 bp, 1% errors, k=31, Bloom, min count 2",
           "genome_bp": glen, "reads": n_reads, "fastq_bytes": int(size), "generate_s": round(gen_s, 1)}
    with kc.KmerCounter(device=local, max_inflight_jobs=1) as h:
        t0 = time.perf_counter()
        r = h.count([fq], keep_records=True, copy=False, **job)
        wall = time.perf_counter() - t0
        out.update({"passes": r.passes, "occurrences": r.occurrences, "records": int(len(r.keys)),
                    "distinct": r.distinct, "e2e_s": wall, "e2e_kmers_per_s": r.occurrences / wall,
                    "device_ms": r.device_ms, "device_kmers_per_s": r.occurrences / (r.device_ms / 1000.0),
                    "spill_bytes": int(12 * len(r.keys)) if r.passes > 1 else 0,
                    "stages_ms": {kc.PHASES[i]: r.phase_ms[i] for i in range(len(kc.PHASES)) if r.phase_ms[i] > 0},
                    "smem_passes": r.smem_passes})
        if args.cpu_baseline:
            try:
                threads, _ = cpu_info()
                chk = _checker().full_spot_check(fq, 31, r.keys, r.counts, r.hist, JOB["hist_min"],
                                                 JOB["min_count"], threads=max(1, threads), sample_bits=8)
                out["parity"] = "identical" if chk["identical"] else "DIFFERENT"
                out["parity_detail"] = chk
            except Exception as e:
                out["parity"] = f"failed: {e}"
        del r
    kc.lib().kc_host_free(p)
    return out


def run_ours(args):
    world, rank, local = dist_setup(args)
    import numpy as np
    import ktcountermemorygreedy_b200 as kc

    fq, pinned, genome_len, n_reads = make_input(args.scale, kc)
    counter = kc.KmerCounter(device=local, max_inflight_jobs=1)
    inp = counter.upload([fq])
    if args.tuning:
        # settings given on the command line (name=value), no autotuner run
        counter.set_tuning(**{k: (float(v) if "factor" in k else int(v))
                              for k, v in (t.split("=", 1) for t in args.tuning)})
        tuning = counter.tuning
    else:
        # settings chosen by the project's autotuner on this workload (untimed)
        tuning = counter.autotune(inputs=[inp], keep_records=False, **JOB)
    for _ in range(args.warmup):
        counter.count(input=inp, keep_records=False, **JOB)
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    l0 = kc.kernel_launches()
    results = []
    for _ in range(args.steps):
        results.append(counter.count(input=inp, keep_records=False, **JOB))
    launches = kc.kernel_launches() - l0
    clocks = sampler.stop()
    barrier(world)
    dev_ms = sum(r.device_ms for r in results)
    occ = sum(r.occurrences for r in results)
    t_max = max_over_ranks(dev_ms, world)
    occ_all = sum_over_ranks(occ, world)
    value = occ_all / (t_max / 1000.0)

    # end to end through the C ABI from pinned host buffers
    e2e_val, h2d, d2h = None, 0, 0
    last_full = None
    if args.e2e_steps > 0:
        walls, occ_e = [], 0
        r = None
        # untimed host-buffer jobs: the first one's device memory beyond the
        # worker's workspace comes from the stream-ordered pool, the next job
        # grows the workspace to fit it all (and the pinned result blocks are
        # in the pool); from the third job on the worker is in steady state
        for _ in range(2):
            r = counter.count([fq], keep_records=True, copy=False, **JOB)
            del r
        d2h = 0
        for i in range(args.e2e_steps):
            last_full = None   # its pinned block goes back to the pool before the next job
            t0 = time.perf_counter()
            r = counter.count([fq], keep_records=True, copy=False, **JOB)
            walls.append(time.perf_counter() - t0)
            occ_e += r.occurrences
            d2h = len(r.keys) * 12 + r.hist.nbytes
            last_full = r   # the last job's records are checked below, outside the timed steps
            del r
        h2d = len(fq)
        w = max_over_ranks(sum(walls), world)
        e2e_val = sum_over_ranks(occ_e, world) / w

    # roofline of the dominant single-kernel stage
    phases = kc.PHASES
    ns = len(phases)
    mean_ms = [statistics.mean(r.phase_ms[i] for r in results) for i in range(ns)]
    single = [i for i in range(ns) if results[0].phase_launches[i] == 1 and mean_ms[i] > 0]
    dom = max(single, key=lambda i: mean_ms[i]) if single else max(range(ns), key=lambda i: mean_ms[i])
    r0 = results[-1]
    alg = algorithmic_bytes(phases[dom], r0)
    achieved = alg / (mean_ms[dom] / max(1, r0.phase_launches[dom]) / 1000.0) / 1e9
    peak, peak_kind = peaks()
    roof = {"bound": "hbm", "kernel": phases[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic_for(phases[dom], r0),
            "algorithmic_bytes": alg}
    stages = {phases[i]: {"ms": mean_ms[i], "launches": int(r0.phase_launches[i]),
                          "alg_GBps": (algorithmic_bytes(phases[i], r0) / (mean_ms[i] / 1000.0) / 1e9)
                          if mean_ms[i] > 0 else None} for i in range(ns) if mean_ms[i] > 0}

    # atomic throughput of the table inserts against random-atomicAdd peaks
    # measured here.  The job's own path (shared-memory sub-bucket tables):
    # one count atomicAdd per non-FIRST occurrence and one per FIRST
    # occurrence of a k-mer in the table, against random adds on a 16 KiB
    # shared-memory table per block (the sub-bucket table's count array).
    # The global-memory tables (kc_tuning.bloom_smem = 2), timed on one more
    # untimed job: one count atomicAdd per non-FIRST occurrence, against a
    # 4 GiB buffer (DRAM sector RMW) and a 32 MiB one (L2-resident, like one
    # bucket's table).
    atomics = None
    sc = phases.index("smem_count")
    if mean_ms[sc] > 0:
        pk_smem, _ = kc.atomic_peak_shared(16384)
        adds = r0.high_len + (r0.low_len - r0.low_only)
        rate = adds / (mean_ms[sc] / 1000.0)
        atomics = {"kernel": "smem_count", "table_adds_per_s": rate, "unit": "atomics/s",
                   "table_adds_per_job": int(adds), "peak_smem_random": pk_smem, "frac_of_smem_peak": rate / pk_smem,
                   "note": "count atomicAdds on the shared-memory sub-bucket tables (non-FIRST occurrences and "
                           "FIRST occurrences found in the table); the kernel also reads and hashes every key "
                           "and updates the filter slice, so the fraction is a floor on the insert's share"}
        prev = counter.tuning["bloom_smem"]
        counter.set_tuning(bloom_smem=2)
        rg = counter.count(input=inp, keep_records=False, **JOB)
        counter.set_tuning(bloom_smem=prev)
        ih = phases.index("insert_high")
        if rg.phase_ms[ih] > 0:
            pk_dram, _ = kc.atomic_peak(4 << 30)
            pk_l2, _ = kc.atomic_peak(32 << 20)
            g = rg.high_len / (rg.phase_ms[ih] / 1000.0)
            atomics["global_tables"] = {"kernel": "insert_high", "inserts_per_s": g, "inserts_per_job": int(rg.high_len),
                                        "ms": rg.phase_ms[ih], "peak_dram_random": pk_dram, "peak_l2_random": pk_l2,
                                        "frac_of_dram_peak": g / pk_dram, "frac_of_l2_peak": g / pk_l2,
                                        "same_counts": bool(rg.occurrences == r0.occurrences and
                                                            rg.distinct == r0.distinct and
                                                            np.array_equal(rg.hist, r0.hist))}
    else:
        ih = phases.index("insert_high")
        if mean_ms[ih] > 0:
            pk_dram, _ = kc.atomic_peak(4 << 30)
            pk_l2, _ = kc.atomic_peak(32 << 20)
            rate = r0.high_len / (mean_ms[ih] / 1000.0)
            atomics = {"kernel": "insert_high", "inserts_per_s": rate, "unit": "atomics/s",
                       "peak_dram_random": pk_dram, "peak_l2_random": pk_l2,
                       "frac_of_dram_peak": rate / pk_dram, "frac_of_l2_peak": rate / pk_l2,
                       "note": "one slot-key read and one count atomicAdd per non-FIRST occurrence"}

    cpu = parity = sample_value = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        cpu, parity, sample_value = cpu_leg(args, counter, fq, last_full)
    last_full = None
    wide = wide_bench(kc, args, counter, inp, fq) if (rank == 0 and world == 1 and args.wide) else None
    counter.free_input(inp)
    counter.close()
    kc.lib().kc_host_free(pinned)
    served = batched = ooc = None
    if rank == 0 and world == 1 and args.out_of_core:
        ooc = out_of_core_bench(kc, args, local)
    if rank == 0 and world == 1 and args.served:
        served = served_bench(kc, args, local)
    if rank == 0 and world == 1 and args.batched:
        batched = batched_bench(kc, args, local)
    if rank == 0:
        config = workload_config(args.scale, world)
        # the measured job, should the generator ever differ from the formula
        config.update(genome_bp=genome_len, reads=n_reads, fastq_bytes=len(fq),
                      occurrences_per_step=results[0].occurrences)
        line = {
            "metric": METRIC, "value": value, "unit": "k-mers/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": config, "records": results[0].n_records_total, "tuning": tuning,
            "e2e": {"value": e2e_val, "unit": "k-mers/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof, "cpu_baseline": cpu, "sample_value": sample_value, "parity": parity,
            "clocks": clocks, "gpu_launches": int(launches),
            "stages": stages, "atomics": atomics, "served": served, "batched": batched, "out_of_core": ooc,
            "wide": wide,
        }
        print(json.dumps(line, default=_json_default), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="genome size factor (1.0 = the 100 Mbp workload)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    # the CPU baseline's sample: 4M reads (1.25 GB, 480M k-mers), large enough that the reference's
    # fixed start-up (its memory map, the pre-pass) is a small share of a step
    ap.add_argument("--ref-reads", type=int, default=4_000_000)
    ap.add_argument("--parity-reads", type=int, default=1_000_000,
                    help="reads of the sample whose histogram and sorted dump are compared with the reference's")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-served", dest="served", action="store_false")
    ap.add_argument("--served-jobs", type=int, default=200)
    ap.add_argument("--served-rates", type=float, nargs="+", default=[10.0, 50.0, 200.0])
    # one job on the device at a time: each served job already fills the GPU, and concurrent jobs
    # slowed each other (a 2000-job stream at 100-500 jobs/s: 3.7-4.0 G k-mers/s with one worker,
    # 0.8-1.1 G with four)
    ap.add_argument("--served-inflight", type=int, default=1)
    ap.add_argument("--served-pool-reads", type=int, default=4_000_000)
    ap.add_argument("--served-pinned-gb", type=int, default=24)
    ap.add_argument("--no-batched", dest="batched", action="store_false")
    ap.add_argument("--batch-samples", type=int, default=256)
    ap.add_argument("--batch-scale", type=float, default=0.125)
    ap.add_argument("--tuning", nargs="*", default=[],
                    help="handle settings name=value (kc_tuning fields) instead of the autotuner's")
    ap.add_argument("--wide", type=int, nargs="*", default=[63, 127],
                    help="also time k-mers of more than 32 bases on the same workload (none: --wide)")
    ap.add_argument("--out-of-core", action="store_true",
                    help="also run the out-of-core job (3.1 Gbp, 10x, 65 GB FASTQ; minutes, host memory ~100 GB)")
    ap.add_argument("--ooc-scale", type=float, default=1.0, help="genome size factor of the out-of-core job")
    ap.add_argument("--full-reference", action="store_true",
                    help="also run the reference programs once on the whole workload (minutes; ~20 GB of disk "
                         "under $KC_REF_TMP) and compare their histogram with the GPU's")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference_arm(args)
        return
    run_ours(args)


if __name__ == "__main__":
    main()
