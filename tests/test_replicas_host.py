"""The N>1 path of bench.py on the CPU: one process per rank under
torch.distributed.run with the gloo backend, world size 2. Each rank counts
its own replica of the workload (no collective on the data path); the only
collectives are the barrier around the timed region and the reductions that
turn per-rank device times and k-mer counts into the whole-job figure (the
slowest rank's time, the sum of the ranks' k-mers). The reference arm runs
on rank 0 alone, and times the oracle's port where the reference programs
are absent."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, {root!r})
    import bench
    world, rank, local = bench.dist_setup(None)
    assert world == 2 and local == rank
    t_max = bench.max_over_ranks(100.0 + 7.5 * rank, world)
    occ = bench.sum_over_ranks(1000.0 * (rank + 1), world)
    bench.barrier(world)
    with open(os.path.join({out!r}, f"rank{{rank}}.json"), "w") as f:
        json.dump({{"rank": rank, "t_max": t_max, "occ": occ, "value": occ / (t_max / 1000.0)}}, f)
    import torch.distributed as dist
    dist.destroy_process_group()
""")


FAILING_WORKER = textwrap.dedent("""
    import os, sys, time
    sys.path.insert(0, {root!r})
    import bench
    world, rank, local = bench.dist_setup(None)
    if rank == 1:
        raise RuntimeError("replica 1 failed before the timed region")
    bench.barrier(world)          # rank 0 waits here for a rank that is gone
    time.sleep(600)
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(script, nproc):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), script]
    return subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)


def test_two_gloo_ranks_reduce_to_slowest_time_and_total_kmers(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT, out=str(tmp_path)))
    p = _torchrun(str(script), 2)
    assert p.returncode == 0, p.stderr[-2000:]
    rows = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for row in rows:
        assert row["t_max"] == pytest.approx(107.5)
        assert row["occ"] == pytest.approx(3000.0)
        assert row["value"] == pytest.approx(3000.0 / 0.1075)


def test_a_failing_replica_ends_the_job_instead_of_leaving_the_others_waiting(tmp_path):
    import time
    script = tmp_path / "failing.py"
    script.write_text(FAILING_WORKER.format(root=ROOT))
    t0 = time.monotonic()
    p = _torchrun(str(script), 2)
    assert p.returncode != 0
    assert "replica 1 failed" in p.stderr + p.stdout
    assert time.monotonic() - t0 < 120


def test_reference_arm_times_the_oracle_port_without_the_reference_programs():
    env = dict(os.environ, KC_REF_BIN="/nonexistent_dir", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--ref-reads", "2000"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "k-mers/s"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "k-mers/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""

