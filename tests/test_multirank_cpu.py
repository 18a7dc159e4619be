"""The bench's multi-GPU path is N independent replicas (weak scaling, no data
exchange); its only cross-rank steps are the barriers and the max-over-ranks
time. Those run here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench._dist()[:2] == (world, rank)
        dist.barrier()
        my_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.max_over_ranks(my_ms, dist, "cpu")
        out[rank] = (ms, bench.job_mpx_s(world, 4 * 2048 * 2048, 10, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    ms, mpx = out[0]
    assert ms == 15.0
    assert mpx == pytest.approx(2 * 4 * 2048 * 2048 * 10 / 0.015 / 1e6)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.job_mpx_s(1, 1_000_000, 2, 1000.0) == pytest.approx(2.0)


def test_bench_starts_its_own_replicas():
    """`bench.py --gpus 2` without a launcher's environment starts two rank
    processes itself (as it does for N GPUs); the replica plumbing alone
    (rendezvous, barrier, max-over-ranks) runs here on gloo."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--workload", "ranks", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    assert lines[0]["world"] == 2 and lines[0]["max_ms"] == 15.0
    assert lines[0]["mpx_s"] == pytest.approx(2 * 4 * 2048 * 2048 * 10 / 0.015 / 1e6)
