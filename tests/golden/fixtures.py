"""Seeded FASTQ fixtures shared by the golden-vector generator
(make_golden.py) and the tests.  Pure Python (random.Random), so the bytes are
identical wherever they are regenerated; the golden outputs committed next to
this file were produced by the reference's own programs on exactly these
bytes."""
from __future__ import annotations

import random

BASES = "ACGT"


def _comp(c: str) -> str:
    return {"A": "T", "C": "G", "G": "C", "T": "A"}.get(c, "N")


def random_fastq(seed: int, n_reads: int, read_len=(150, 150), genome_len: int = 20000, sub: float = 0.005,
                 n_rate: float = 0.001, lower: float = 0.0, u_rate: float = 0.0, crlf: bool = False,
                 final_newline: bool = True) -> bytes:
    r = random.Random(seed)
    g = "".join(r.choice(BASES) for _ in range(genome_len))
    eol = "\r\n" if crlf else "\n"
    out = []
    for i in range(n_reads):
        L = r.randint(read_len[0], read_len[1])
        p = r.randint(0, genome_len - L)
        s = list(g[p:p + L])
        if r.random() < 0.5:
            s = [_comp(c) for c in reversed(s)]
        for j in range(L):
            if r.random() < sub:
                s[j] = r.choice([b for b in BASES if b != s[j]])
            if r.random() < n_rate:
                s[j] = "N"
            if s[j] == "T" and r.random() < u_rate:
                s[j] = "U"
            if r.random() < lower:
                s[j] = s[j].lower()
        q = "".join(chr(33 + r.randint(20, 40)) for _ in range(L))
        out.append(f"@r{i}{eol}{''.join(s)}{eol}+{eol}{q}{eol}")
    text = "".join(out)
    if not final_newline:
        text = text.rstrip("\r\n")
    return text.encode()


def edge_fastq() -> bytes:
    """Hand-made records covering the reference's line semantics: bases in
    header and '+' lines (ignored), N and other invalid bytes, lowercase, U,
    CR before LF, an empty sequence line, a sequence line longer than the
    reference reader's 32 KB blocks, and a missing final newline."""
    r = random.Random(99)
    long_seq = "".join(r.choice(BASES) for _ in range(70000))
    recs = [
        ("@ACGTACGTACGTACGTACGTACGTACGTACGTACGT", "ACGTTGCAACGTTGCAACGTTGCAACGTTGCAACGTTGCA"),
        ("@r1", "acgtNNacgtacgtacgtacgtacgtacgtacgtacgtXacgtacgtacgtacgtacgtacgtacgtac"),
        ("@r2", "UUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUUU" + "AAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAA"),
        ("@r3", ""),
        ("@r4", "GATTACAGATTACAGATTACAGATTACAGATTACA\rGATTACAGATTACAGATTACAGATTACAGATTACA"),
        ("@r5", long_seq),
        ("@r6", "ACGTACGTACGTACGTACGTACGTACGTACGTAC.ACGTACGTACGTACGTACGTACGTACGTACGTAC"),
    ]
    out = []
    for h, s in recs:
        q = "I" * len(s)
        plus = "+ACGTACGTACGTACGTACGTACGTACGTACGTACGT" if h == "@r2" else "+"
        out.append(f"{h}\n{s}\n{plus}\n{q}\n")
    tail = "@r7\nTTTTGGGGCCCCAAAATTTTGGGGCCCCAAAATTTTGGGG\n+\nIIII"   # no final newline, cut quality
    return ("".join(out) + tail).encode()


def crlf_fastq() -> bytes:
    return random_fastq(11, 300, (60, 140), genome_len=3000, sub=0.01, n_rate=0.002, crlf=True)


def mixed_fastq() -> bytes:
    return random_fastq(12, 400, (40, 200), genome_len=4000, sub=0.01, n_rate=0.005, lower=0.05, u_rate=0.05)


def repeat_fastq() -> bytes:
    """Small genome and many reads: high counts, homopolymer-free repeats."""
    return random_fastq(13, 3000, (100, 150), genome_len=600, sub=0.002, n_rate=0.0)


def plain_small() -> bytes:
    """The plain-job shape at a tenth of its read count."""
    return random_fastq(1, 2000, (150, 150), genome_len=100000, sub=0.005, n_rate=0.001)


# (name, files, k values) checked end to end against the reference programs
# (k <= 32)
E2E_CASES = [
    ("edge", [edge_fastq()], [5, 21, 25, 31]),
    ("crlf", [crlf_fastq()], [21, 31]),
    ("mixed", [mixed_fastq()], [1, 11, 21, 31]),
    ("repeat", [repeat_fastq()], [21, 31]),
    ("plain_small", [plain_small()], [21, 25, 31]),
    ("multi", [random_fastq(14, 200, (80, 120), genome_len=2000, final_newline=False),
               random_fastq(15, 200, (80, 120), genome_len=2000)], [21, 31]),
]

# The same for k-mers of 33..128 bases.  The reference's histogram is an
# oracle at every k except 96, its sorted dump only up to k = 64 (above 64
# its sort key is 128 bits wide and the text is printed from that key,
# tool/dump_tool.cpp:320-324, :1181-1185).
E2E_WIDE_CASES = [
    ("edge", [edge_fastq()], [33, 63]),
    ("repeat", [repeat_fastq()], [33, 64, 65, 128]),
    ("plain_small", [plain_small()], [33, 47, 63, 64, 65, 95, 96, 97, 127, 128]),
    ("multi", [random_fastq(14, 200, (80, 120), genome_len=2000, final_newline=False),
               random_fastq(15, 200, (80, 120), genome_len=2000)], [40, 70]),
]


def getkmer_cases():
    r = random.Random(5)
    s1 = "".join(r.choice("ACGTacgtUuNn") for _ in range(400))
    s2 = "".join(r.choice(BASES) for _ in range(300))
    return [(k, s) for k in (1, 2, 5, 15, 16, 17, 21, 25, 31, 32) for s in (s1, s2)]


# k values of the reference's kmer<2> (33..64) and kmer<4> (65..128) paths
WIDE_KS = (33, 34, 47, 63, 64, 65, 80, 95, 96, 97, 127, 128)


def _revcomp(s: str) -> str:
    return s.translate(str.maketrans("ACGT", "TGCA"))[::-1]


def getkmer_wide_cases():
    """Base strings for the multi-word extraction: long valid runs with rare
    invalid bytes and mixed case, and reverse-complement palindromes of 32,
    48 and 64 bases (k-mers equal to their reverse complement, and windows
    whose forward and reverse words tie on their first words)."""
    r = random.Random(6)
    s3 = "".join(r.choice("ACGTacgtU") if r.random() > 0.004 else "N" for _ in range(900))
    parts = []
    for n in (16, 24, 32):
        h = "".join(r.choice(BASES) for _ in range(n))
        parts.append(h + _revcomp(h))
    parts.append("A" * 32 + "T" * 32)
    s4 = "".join(parts + ["".join(r.choice(BASES) for _ in range(40)) for _ in range(3)]) * 2
    return [(k, s) for k in WIDE_KS for s in (s3, s4)]
