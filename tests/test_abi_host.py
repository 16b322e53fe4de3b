"""CPU-side checks of the product: libkc.so loads and exports every entry
point include/kc.h declares; host-only logic (Bloom sizing, argument
validation of the CLIs, the synthetic generator) matches the oracle and the
reference.  No kernel is launched here."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ktcountermemorygreedy_b200")
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))


def _build():
    if not os.path.exists(os.path.join(PKG, "libkc.so")) or not os.path.exists(os.path.join(PKG, "bin", "kmer_counter")):
        subprocess.run(["make", "-s", "-C", PKG], check=True)


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "kc.h")).read()
    return sorted(set(re.findall(r"\b(kc_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    _build()
    lib = ctypes.CDLL(os.path.join(PKG, "libkc.so"))
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_binding_covers_the_header():
    import ktcountermemorygreedy_b200 as kc
    bound = {s[0] for s in kc.SIGNATURES}
    assert bound == set(declared_symbols())
    kc.lib()   # binds every signature


def test_binding_structs_have_the_header_layout(tmp_path):
    """Every struct the binding passes through the C ABI has the size and the
    field offsets that the C compiler gives include/kc.h."""
    import ktcountermemorygreedy_b200 as kc
    structs = [kc.kc_config, kc.kc_tuning, kc.kc_buffer, kc.kc_job, kc.kc_result_t]
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "kc.h"', "int main(void) {"]
    for S in structs:
        n = S.__name__
        src.append(f'printf("{n} sizeof %zu\\n", sizeof({n}));')
        for f in S._fields_:
            src.append(f'printf("{n} {f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    src.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = str(tmp_path / "layout")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(c), "-o", exe], check=True)
    got = {}
    for line in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        n, field, v = line.split()
        got[(n, field)] = int(v)
    for S in structs:
        n = S.__name__
        assert got[(n, "sizeof")] == ctypes.sizeof(S), n
        for f in S._fields_:
            assert got[(n, f[0])] == getattr(S, f[0]).offset, (n, f[0])


@pytest.mark.parametrize("rec", GOLDEN["prepass"], ids=lambda r: r["name"])
def test_host_bloom_sizing_matches_reference(rec):
    import ktcountermemorygreedy_b200 as kc
    caps, mx = kc.plan_bloom(rec["raw_prefix_counts"], rec["avg_quality"], rec["estimated_file_size"],
                             rec["memory_gb"], rec["k"])
    assert mx == rec["max_bloom_capacity"]
    assert caps.tolist() == rec["bloom_capacities"]


def test_host_bloom_sizing_matches_oracle_on_random_inputs():
    import ktcountermemorygreedy_b200 as kc
    rng = np.random.default_rng(0)
    for _ in range(200):
        pc = rng.integers(0, 5_000_000, size=256).astype(np.uint32)
        pc[rng.integers(0, 256, size=20)] = rng.integers(0, 1500, size=20)
        q = int(rng.integers(50, 80))
        est = int(rng.integers(1, 10**11))
        mem = int(rng.integers(1, 512))
        k = int(rng.integers(11, 33))
        a = kc.plan_bloom(pc, q, est, mem, k)
        b = O.bloom_capacities(pc, q, est, mem, k)
        assert a[1] == b[1] and a[0].tolist() == b[0].tolist()


def test_no_device_is_reported_not_faked():
    """Without a GPU the product refuses loudly; it has no CPU fallback."""
    import ktcountermemorygreedy_b200 as kc
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(kc.KcError) as e:
        kc.KmerCounter()
    assert e.value.code == 8
    with pytest.raises(kc.KcError):
        kc.extract_kmers(b"@a\nACGT\n+\nIIII\n", 3)


def _run(args):
    return subprocess.run(args, capture_output=True, text=True)


def test_cli_argument_validation():
    _build()
    kmc = os.path.join(PKG, "bin", "kmer_counter")
    assert _run([kmc]).returncode == 1
    r = _run([kmc, "x.fq", "31", "4", "1", "/tmp"])
    assert r.returncode == 255 and "n_thread must be >= 6" in r.stderr
    assert _run([kmc, "x.fq", "31", "8", "1", "/tmp", "1024", "5", "3"]).returncode == 1   # filter_max < filter_min
    assert _run([kmc, "x.fq", "31", "8", "1", "/tmp", "1024", "2", "9", "0"]).returncode == 1   # count_max 0
    # map_capacity is rounded up to a power of two before the 16M limit (src/main.cpp:541, :581)
    assert _run([kmc, "x.fq", "31", "8", "1", "/tmp", "9000000"]).returncode == 1
    r = _run([kmc, "x.fq", "129", "8", "1", "/tmp"])
    assert r.returncode == 1 and "k_len must be <= 128" in r.stderr   # src/main.cpp:629-632
    # infos.bin is written before any input is read (src/main.cpp:588-595)
    r = _run([kmc, "x.fq", "31", "8", "1", "/nonexistent_dir"])
    assert r.returncode == 1 and "Open infos.bin failed" in r.stderr
    ht = os.path.join(PKG, "bin", "histogram_tool")
    r = _run([ht, "fuzzy", "/tmp", "4", "1", "o.tsv"])
    assert r.returncode == 255 and "invalid mode" in r.stderr
    r = _run([ht, "precise", "/nonexistent_dir", "4", "1", "o.tsv"])
    assert r.returncode == 255 and "infos.bin" in r.stderr
    dt = os.path.join(PKG, "bin", "dump_tool")
    r = _run([dt, "precise", "/tmp", "4", "1", "o.txt", "5", "3"])
    assert r.returncode == 255 and "max_freq < min_freq" in r.stderr
    # max_memory_gb: the whole argument a positive number of GiB
    for tool in (ht, dt):
        for bad in ("1abc", "0", "-2", "", "x"):
            r = _run([tool, "precise", "/tmp", "4", bad, "o.txt"])
            assert r.returncode == 255 and f"invalid max_memory_gb: {bad}" in r.stderr
        r = _run([tool, "precise", "/tmp", "4", "1e30", "o.txt"])
        assert r.returncode == 255 and "too large" in r.stderr
        r = _run([tool, "precise", "/nonexistent_dir", "4", "0.5", "o.txt"])
        assert r.returncode == 255 and "infos.bin" in r.stderr


def test_generator_is_deterministic_across_thread_counts():
    import ktcountermemorygreedy_b200.synth as S
    g = S.genome(9, 50000)
    a = S.reads(g, 9, 3000, (100, 250), 0.01, 0.001)
    old = S.threads
    try:
        S.threads = lambda: 1
        b = S.reads(g, 9, 3000, (100, 250), 0.01, 0.001)
    finally:
        S.threads = old
    assert a.tobytes() == b.tobytes()
    text = a.tobytes().decode()
    lines = text.split("\n")
    assert lines[0] == "@r0" and lines[2] == "+" and len(lines[1]) == len(lines[3])
    assert set(lines[1]) <= set("ACGTN")
    assert all(53 <= ord(c) <= 73 for c in lines[3])


def test_generator_repeat_fraction():
    import ktcountermemorygreedy_b200.synth as S
    buf = np.zeros(1_000_000, np.uint8)
    placed = S.gen().kcgen_genome(2, 1_000_000, 0.05, 20, 1000, 5000, 10, 500, 0.02, buf.ctypes.data, 4)
    assert abs(placed - 50_000) < 6_000
