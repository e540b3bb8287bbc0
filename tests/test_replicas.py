"""The multi-GPU plumbing of bench.py on CPU: world-size-2 `gloo` process
groups stand in for NCCL ranks. The path shards as independent replicas (no
data-path collective): each rank transforms its own channels, the job's time
is the slowest rank's (max over ranks) and its throughput the units of all
ranks over that time. The reference arm runs and prints on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        units = 1000.0  # bytes per rank per step
        rate = bench.job_rate(units, world, ms * 1e-3)
        dist.barrier()
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    # every rank sees the slowest rank's time; throughput = 2 x 1000 units / 15 ms
    assert [r[1] for r in res] == [15.0, 15.0]
    assert all(abs(r[2] - 2000.0 / 0.015) < 1e-6 for r in res)


def test_reference_arm_prints_on_rank_zero_only():
    """`bench.py --impl reference` under torchrun: ranks other than 0 exit 0
    without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_weak_scaling_value_is_the_whole_job(world):
    import bench

    # the same per-rank work and slowest time: the value grows with the ranks
    assert bench.job_rate(536870912.0, world, 1e-4) == pytest.approx(world * 536870912.0 / 1e-4)


def test_reference_arm_line_is_well_formed_on_rank_zero():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["unit"] == "GB/s" and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
