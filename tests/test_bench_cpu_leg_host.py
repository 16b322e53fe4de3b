"""bench.py's CPU leg and k > 32 leg on the CPU: the reference programs
timed on one sample (counter + histogram, no text), their histogram and
sorted dump compared with a job's on a second, smaller sample, the whole-job
hash-sample check, and the k > 32 entries with their hash-sample checks.
The GPU job is stood in for by the oracle (exact counts, records in printed
order, histogram) and the device-side steps (the GPU's own timing of the
sample, the dump formatted on the device) by host equivalents, so that the
plumbing of the leg is what is tested here; the GPU tests cover the jobs."""
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import bench  # noqa: E402
import oracle_lib as O  # noqa: E402


class _Job:
    pass


class OracleCounter:
    """count() with the binding's arguments, answered by the oracle."""

    def count(self, files=(), input=None, keep_records=True, copy=True, **kw):
        data = b"".join(bytes(f) for f in files)
        uk, uc = O.count(O.extract(data, kw["k"]))
        uc = np.minimum(uc, np.uint32(kw["count_max"])).astype(np.uint32)
        m = uc >= kw["min_count"]
        r = _Job()
        r.keys, r.counts = O.sort_string_order(uk[m], uc[m], kw["k"])
        r.hist = O.histogram(uc, kw["hist_min"], kw["hist_max"])
        r.occurrences = int(uc.sum())
        return r


@pytest.fixture
def leg(monkeypatch, tmp_path):
    if not os.access(bench.GEN, os.X_OK):
        pytest.skip("the generator program is not built")
    import ktcountermemorygreedy_b200 as kc
    monkeypatch.setattr(kc, "dump_bytes", lambda keys, counts, k: O.dump_text(keys, counts, k))
    monkeypatch.setattr(bench, "sample_on_gpu",
                        lambda counter, kc_, path: ({"device": None, "e2e": None, "bytes": os.path.getsize(path)},
                                                    None))
    monkeypatch.setenv("KC_REF_MEM_GB", "4")
    p = str(tmp_path / "job.fq")
    bench.write_workload(p, 20_000)
    return np.fromfile(p, np.uint8)


def test_cpu_leg_with_the_reference_programs(leg):
    if not bench.reference_programs_present():
        pytest.skip("the reference programs are not built")
    args = types.SimpleNamespace(ref_reads=40_000, parity_reads=20_000, full_reference=False)
    cpu, parity, sample_value = bench.cpu_leg(args, OracleCounter(), leg, None)
    assert cpu["kind"] == "reference" and cpu["value"] > 0 and cpu["cores"] >= 6
    assert "first 40000 reads" in cpu["sample"] and "histogram_tool precise" in cpu["sample"]
    assert sample_value["bytes"] == bench.large_job_fastq_bytes(40_000)
    assert parity["sample"] == "identical", parity
    assert parity["sample_detail"]["reads"] == 20_000 and parity["sample_detail"]["dump_lines"] > 0
    assert parity["full"] == "identical", parity.get("full_detail")


def test_cpu_leg_with_the_port(leg, monkeypatch):
    monkeypatch.setenv("KC_REF_BIN", "/nonexistent_dir")
    args = types.SimpleNamespace(ref_reads=5_000, parity_reads=5_000, full_reference=False)
    cpu, parity, _ = bench.cpu_leg(args, OracleCounter(), leg, None)
    assert cpu["kind"] == "port" and cpu["cores"] == 1 and cpu["value"] > 0
    assert parity["sample"].startswith("not checked")
    assert parity["full"] == "identical", parity.get("full_detail")


def test_reference_run_times_counter_and_histogram_only(tmp_path):
    if not bench.reference_programs_present() or not os.access(bench.GEN, os.X_OK):
        pytest.skip("the reference programs or the generator are not built")
    p = str(tmp_path / "s.fq")
    bench.write_workload(p, 10_000)
    w, occ = bench.reference_run(p, 6, 4, str(tmp_path))
    assert w > 0 and occ == 10_000 * (150 - 31 + 1)
    assert (tmp_path / "h.tsv").exists() and not (tmp_path / "d.txt").exists()
    bench.reference_run(p, 6, 4, str(tmp_path), dump=True)
    assert (tmp_path / "d.txt").stat().st_size > 0


class OracleWideCounter:
    """count(input=...) of the resident workload for any k, answered by the
    oracle; device_ms and the stage times are placeholders."""

    def __init__(self, fq: np.ndarray):
        self.fq = fq.tobytes()

    def count(self, files=(), input=None, keep_records=True, copy=True, **kw):
        import ktcountermemorygreedy_b200 as kc
        k = kw["k"]
        occ = O.extract_wide(self.fq, k)
        uk, uc = O.count_wide(occ)
        uc = np.minimum(uc, np.uint32(kw["count_max"])).astype(np.uint32)
        m = uc >= kw["min_count"]
        r = _Job()
        r.keys, r.counts = O.sort_string_order_wide(uk[m], uc[m], k)
        r.hist = O.histogram(uc, kw["hist_min"], kw["hist_max"])
        r.occurrences = len(occ)
        r.n_records_total = int(m.sum())
        r.device_ms, r.passes = 1.0, 1
        r.phase_ms = [0.0] * len(kc.PHASES)
        return r


def test_wide_leg_reports_each_k_and_checks_its_hash_sample(leg):
    args = types.SimpleNamespace(wide=[63, 127], cpu_baseline=True)
    import ktcountermemorygreedy_b200 as kc
    out = bench.wide_bench(kc, args, OracleWideCounter(leg), None, leg)
    assert set(out) == {"63", "127"}
    for k, o in out.items():
        assert o["k"] == int(k) and o["key_words"] == (2 if k == "63" else 4)
        assert o["occurrences"] == 20_000 * (150 - int(k) + 1)
        assert o["parity"] == "identical", o.get("parity_detail")


def test_a_failing_wide_k_is_reported_not_raised(leg):
    class Failing:
        def count(self, **kw):
            raise RuntimeError("no device")

    import ktcountermemorygreedy_b200 as kc
    out = bench.wide_bench(kc, types.SimpleNamespace(wide=[63], cpu_baseline=True), Failing(), None, leg)
    assert out == {"63": {"k": 63, "failed": "no device"}}


def test_reference_arm_shrinks_its_sample_to_its_time_budget():
    import json
    import subprocess
    if not bench.reference_programs_present() or not os.access(bench.GEN, os.X_OK):
        pytest.skip("the reference programs or the generator are not built")
    env = dict(os.environ, KC_REF_BUDGET_S="1", KC_REF_MEM_GB="4", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--ref-reads", "400000"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["cpu_baseline"]["sample"].startswith(f"first {bench.REF_ARM_MIN_READS} reads")
    assert line["config"] == bench.workload_config(1.0, 1)
