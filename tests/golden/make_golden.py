"""Regenerates tests/golden/golden.json from the reference's own programs.

Run in a checkout where the reference sources are available:

    make -C oracle ref REF=/path/to/KTCounterMemoryGreedy
    python tests/golden/make_golden.py

It runs oracle/_ref/{kmer_counter,histogram_tool,dump_tool,ref_golden} (the
reference compiled from its sources by oracle/Makefile) on the fixtures of
fixtures.py and records their outputs.  The tests never run this script; they
read the JSON it wrote.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, HERE)
import fixtures  # noqa: E402


def run(args, cwd=None):
    p = subprocess.run(args, cwd=cwd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"{args} failed ({p.returncode}): {p.stderr[-2000:]}")
    return p.stdout


def sparse_hist(path):
    out = {}
    with open(path) as f:
        for line in f:
            a, b = line.split("\t")
            if int(b):
                out[a] = int(b)
    return out


def e2e(name, files, k, count_max, tmp):
    paths = []
    for i, data in enumerate(files):
        p = os.path.join(tmp, f"{name}_{i}.fq")
        with open(p, "wb") as f:
            f.write(data)
        paths.append(p)
    d = os.path.join(tmp, f"t_{name}_{k}_{count_max}")
    os.makedirs(d, exist_ok=True)
    run([os.path.join(REF, "kmer_counter"), ",".join(paths), str(k), "8", "1", d, "1024", "2", "4294967295",
         str(count_max)])
    hist = os.path.join(tmp, "hist.tsv")
    dump = os.path.join(tmp, "dump.txt")
    run([os.path.join(REF, "histogram_tool"), "precise", d, "8", "1", hist, "1", "10000"])
    run([os.path.join(REF, "dump_tool"), "precise", d, "8", "1", dump, "1", "4294967295", "--sort"])
    with open(dump, "rb") as f:
        text = f.read()
    return {
        "name": name, "k": k, "count_max": count_max,
        "hist": sparse_hist(hist),
        "dump_sha256": hashlib.sha256(text).hexdigest(),
        "dump_lines": text.count(b"\n"),
        "dump_head": text[:2000].decode(),
    }


def main():
    g = {"source": "oracle/_ref programs built from the reference sources by oracle/Makefile"}
    # hashes
    lines = run([os.path.join(REF, "ref_golden"), "hashes", "3000", "7"]).split("\n")
    g["hashes"] = [l.split() for l in lines if l.strip()]
    # rolling canonical extraction
    gk = []
    for k, s in fixtures.getkmer_cases():
        out = run([os.path.join(REF, "ref_golden"), "getkmer", str(k), s])
        gk.append({"k": k, "bases": s, "canonical": [l.split()[1] for l in out.split("\n") if l.strip()]})
    g["getkmer"] = gk
    gw = []
    for k, s in fixtures.getkmer_wide_cases():
        out = run([os.path.join(REF, "ref_golden"), "getkmer", str(k), s])
        rows = [l.split() for l in out.split("\n") if l.strip()]
        last = (k - 1) // 32
        # the words of the k-mer (data[0..last]); words above it are counted
        # where nonzero (stale bases of GetKmer<4> at k = 96)
        text = "".join(" ".join(r[1: 2 + last]) + "\n" for r in rows)
        gw.append({"k": k, "bases": s, "n": len(rows), "sha256": hashlib.sha256(text.encode()).hexdigest(),
                   "beyond_nonzero": sum(1 for r in rows if any(int(w, 16) for w in r[2 + last:])),
                   "head": [r[1:] for r in rows[:8]]})
    g["getkmer_wide"] = gw
    with tempfile.TemporaryDirectory() as tmp:
        # pre-pass statistics and Bloom sizing
        pre = []
        big = fixtures.random_fastq(16, 9000, (150, 150), genome_len=50000)
        for name, files, k, mem in [("plain_small", [fixtures.plain_small()], 31, 4),
                                    ("repeat", [fixtures.repeat_fastq()], 21, 1),
                                    ("multi", [c for c in fixtures.E2E_CASES if c[0] == "multi"][0][1], 31, 2),
                                    ("prepass_big", [big], 31, 8),
                                    ("edge", [fixtures.edge_fastq()], 25, 1)]:
            paths = []
            for i, data in enumerate(files):
                p = os.path.join(tmp, f"pre_{name}_{i}.fq")
                with open(p, "wb") as f:
                    f.write(data)
                paths.append(p)
            out = run([os.path.join(REF, "ref_golden"), "prepass", str(k), str(mem)] + paths)
            rec = {"name": name, "k": k, "memory_gb": mem}
            for line in out.split("\n"):
                parts = line.split()
                if not parts:
                    continue
                if parts[0] in ("raw_prefix_counts", "bloom_capacities"):
                    rec[parts[0]] = [int(x) for x in parts[1:]]
                elif parts[0] in ("avg_quality", "estimated_file_size", "max_bloom_capacity"):
                    rec[parts[0]] = int(parts[1])
            pre.append(rec)
        g["prepass"] = pre
        # end to end: counter + precise tools
        cases = []
        for name, files, ks in fixtures.E2E_CASES:
            for k in ks:
                cases.append(e2e(name, files, k, 4294967295, tmp))
        cases.append(e2e("repeat", [fixtures.repeat_fastq()], 21, 255, tmp))
        cases.append(e2e("repeat", [fixtures.repeat_fastq()], 31, 1000, tmp))
        g["e2e"] = cases
        wide = []
        for name, files, ks in fixtures.E2E_WIDE_CASES:
            for k in ks:
                wide.append(e2e(name, files, k, 4294967295, tmp))
        g["e2e_wide"] = wide
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=0, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
