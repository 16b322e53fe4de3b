"""bench.py's "config" object, which both arms print: the large job's FASTQ
size and occurrence count follow from its read count alone, so the reference
arm states the same workload as the GPU arm without generating or counting
it. Checked against the generator library's own size function."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


@pytest.mark.parametrize("n", [0, 1, 9, 10, 11, 99, 100, 101, 12_345, 1_000_000, 4_000_000, 20_000_000])
def test_fastq_bytes_formula_equals_the_generator(n):
    S = pytest.importorskip("ktcountermemorygreedy_b200.synth")
    try:
        want = S.reads_size(2, n, (150, 150))
    except OSError as e:   # libkcgen.so not built
        pytest.skip(str(e))
    assert bench.large_job_fastq_bytes(n) == want


def test_workload_config_of_the_default_job():
    c = bench.workload_config(1.0, 1)
    assert c["genome_bp"] == 100_000_000 and c["reads"] == 20_000_000
    assert c["fastq_bytes"] == 6_288_888_890
    assert c["occurrences_per_step"] == 2_400_000_000
    assert c["parallelism"] == "replicas x1" and c["scale"] == 1.0
    assert bench.workload_config(0.05, 2)["reads"] == 1_000_000


def test_the_generated_sample_has_the_formula_size(tmp_path):
    if not os.access(bench.GEN, os.X_OK):
        pytest.skip("the generator program is not built")
    p = str(tmp_path / "s.fq")
    assert bench.write_workload(p, 1234) == bench.large_job_fastq_bytes(1234)
    with open(p, "rb") as f:
        head = f.read(400).split(b"\n")
    assert head[0] == b"@r0" and len(head[1]) == 150 and head[2] == b"+" and len(head[3]) == 150
