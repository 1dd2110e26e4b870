"""The multi-process path of the benchmark on CPU: one process per rank over gloo, as torchrun
launches the GPU ranks (the device path runs independent replicas; its only collectives are the
timing reductions and barriers tested here)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ranks(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slowest = bench.rank_max(1.5 + rank, dist, device="cpu")
    total = bench.rank_sum(10.0 * (rank + 1), dist, device="cpu")
    dist.barrier()
    out.put((rank, slowest, total))
    dist.destroy_process_group()


def test_timing_reductions_take_the_slowest_rank_and_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_ranks, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2.5, 30.0), (1, 2.5, 30.0)]


def test_a_single_rank_reduces_to_its_own_value():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.rank_max(3.25) == 3.25 and bench.rank_sum(7.0) == 7.0


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--workload", "config1", "--steps", "3", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
