"""Seeded synthetic FASTQ for the workloads the reference is measured on
(libkcgen.so).  The reference measures no public dataset; these inputs have
its workloads' shapes: uniform-ACGT genomes (optionally with repeat families),
reads from uniform positions on either strand, uniform substitution errors,
optional N bases, Phred+33 qualities uniform in [20, 40].
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_gen = None


def gen() -> C.CDLL:
    global _gen
    if _gen is None:
        L = C.CDLL(os.path.join(_HERE, "libkcgen.so"))
        L.kcgen_genome.restype = C.c_uint64
        L.kcgen_genome.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_uint32, C.c_double, C.c_void_p, C.c_int]
        L.kcgen_genome_div.restype = C.c_uint64
        L.kcgen_genome_div.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_void_p, C.c_int]
        L.kcgen_reads_size.restype = C.c_uint64
        L.kcgen_reads_size.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32]
        L.kcgen_reads.restype = C.c_uint64
        L.kcgen_reads.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32,
                                  C.c_uint32, C.c_double, C.c_double, C.c_void_p, C.c_uint64, C.c_int]
        _gen = L
    return _gen


def threads() -> int:
    return max(1, min(64, os.cpu_count() or 1))


def genome(seed: int, length: int, repeat_frac: float = 0.0, n_families: int = 0, fam_len=(1000, 5000),
           copies=(10, 500), divergence: float = 0.0) -> np.ndarray:
    g = np.zeros(length, np.uint8)
    gen().kcgen_genome(seed, length, repeat_frac, n_families, fam_len[0], fam_len[1], copies[0], copies[1],
                       divergence, g.ctypes.data, threads())
    return g


def genome_div(seed: int, length: int, repeat_frac: float, n_families: int, fam_len, copies, divergence) -> np.ndarray:
    """Genome whose repeat families each draw a divergence from U[divergence]."""
    g = np.zeros(length, np.uint8)
    gen().kcgen_genome_div(seed, length, repeat_frac, n_families, fam_len[0], fam_len[1], copies[0], copies[1],
                           divergence[0], divergence[1], g.ctypes.data, threads())
    return g


def reads(g: np.ndarray, seed: int, n_reads: int, length=(150, 150), sub_rate: float = 0.0, n_rate: float = 0.0,
          first_id: int = 0, out: np.ndarray | None = None) -> np.ndarray:
    """FASTQ bytes as a uint8 array (``out`` may be a preallocated, e.g.
    pinned, buffer of at least ``reads_size`` bytes)."""
    size = gen().kcgen_reads_size(seed, first_id, n_reads, length[0], length[1])
    if out is None:
        out = np.zeros(max(size, 1), np.uint8)
    assert out.nbytes >= size
    n = gen().kcgen_reads(g.ctypes.data, len(g), seed, first_id, n_reads, length[0], length[1], sub_rate, n_rate,
                          out.ctypes.data, out.nbytes, threads())
    assert n == size
    return out[:size]


def reads_size(seed: int, n_reads: int, length=(150, 150), first_id: int = 0) -> int:
    return gen().kcgen_reads_size(seed, first_id, n_reads, length[0], length[1])


# ---- the workload configurations ---------------------------------------------

def plain_job(scale: float = 1.0):
    """Plain single job: 1 Mbp uniform genome (seed 1), 200k x 150 bp reads,
    0.5% substitutions, 0.1% N, k = 31, min count 1."""
    g = genome(1, 1_000_000)
    n = max(1, int(200_000 * scale))
    return reads(g, 1, n, (150, 150), 0.005, 0.001), 31


def large_job_genome(genome_len: int = 100_000_000):
    """100 Mbp genome (seed 2) with 5% from 200 repeat families of 1-5 kbp,
    10-500 copies each (scaled to the 5% total), 2% divergence."""
    return genome(2, genome_len, 0.05, 200, (1000, 5000), (10, 500), 0.02)


def large_job(coverage: float = 30.0, genome_len: int = 100_000_000, out: np.ndarray | None = None):
    """Single large job: 30x of 150 bp reads (about 20M reads) with 1%
    substitutions, k = 31, Bloom singleton filtering, min count 2."""
    g = large_job_genome(genome_len)
    n = int(math.ceil(coverage * genome_len / 150))
    return reads(g, 2, n, (150, 150), 0.01, 0.0, out=out), 31


def large_job_reads(coverage: float = 30.0, genome_len: int = 100_000_000) -> int:
    return int(math.ceil(coverage * genome_len / 150))


OUT_OF_CORE_GENOME_BP = 3_100_000_000


def out_of_core_genome(genome_len: int = OUT_OF_CORE_GENOME_BP):
    """Out-of-core job genome (seed 5): 45% from 2000 repeat families of
    0.3-6 kbp with 1-10^5 copies (scaled to the 45% total), each family at a
    divergence drawn from U[1%, 15%]."""
    return genome_div(5, genome_len, 0.45, 2000, (300, 6000), (1, 100_000), (0.01, 0.15))


def out_of_core_reads(coverage: float = 10.0, genome_len: int = OUT_OF_CORE_GENOME_BP) -> int:
    """10x of 150 bp reads (about 207M for 3.1 Gbp); 1% substitutions, seed 5."""
    return int(math.ceil(coverage * genome_len / 150))


def batch_samples(n_samples: int = 256, scale: float = 1.0, seed_base: int = 3000):
    """Batched samples: sample s has its own uniform genome of 5-50 Mbp,
    log-uniform read count in [1e4, 2e6] (times `scale`), lengths U[100, 250],
    substitutions U[0.5%, 2%]; k = 21 for even s, 31 for odd s."""
    out = []
    for s in range(n_samples):
        rng = np.random.default_rng(seed_base + s)
        glen = int(rng.integers(5_000_000, 50_000_001))
        nreads = max(1, int(math.exp(rng.uniform(math.log(1e4), math.log(2e6))) * scale))
        sub = float(rng.uniform(0.005, 0.02))
        g = genome(seed_base + s, glen)
        fq = reads(g, seed_base + s, nreads, (100, 250), sub, 0.0)
        out.append((fq, 21 if s % 2 == 0 else 31))
    return out


def served_jobs(n_jobs: int = 2000, rate: float = 100.0, seed: int = 4, genome_len: int = 50_000_000,
                size_scale: float = 1.0, cap_reads: int = 20_000_000):
    """Served request stream: Poisson arrivals at `rate` jobs/s, log-normal job
    sizes (median 200k reads, sigma 1.5, capped at 20M; times `size_scale`),
    150 bp reads at 1% from one shared genome, k drawn from {21, 25, 31}.
    Returns (genome, [(arrival_s, n_reads, k, read_seed)])."""
    rng = np.random.default_rng(seed)
    g = genome(seed, genome_len)
    t = 0.0
    jobs = []
    for i in range(n_jobs):
        t += float(rng.exponential(1.0 / rate))
        n = int(min(cap_reads, math.exp(rng.normal(math.log(200_000), 1.5))) * size_scale)
        k = int(rng.choice([21, 25, 31]))
        jobs.append((t, max(1, n), k, seed * 1_000_003 + i))
    return g, jobs
