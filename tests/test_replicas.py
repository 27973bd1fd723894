"""Replica runs over several ranks (bench.py --gpus N under torchrun), checked with two gloo
ranks on the CPU: each rank shards its own replica (its own seed), the whole-job time is the
slowest rank's and the hops are summed; the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        jobs = bench.workload_jobs("scale", rank)
        t, hops = bench.reduce_over_ranks(dist, 10.0 * (rank + 1), 100 * (rank + 1), "cpu")
        q.put((rank, jobs[0]["seed"], jobs[0]["box"], t, hops))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_replicas_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [42, 43]  # one replica per rank, its own seed
    assert got[0][2] == got[1][2] == (256, 256, 256)  # the same workload shape: weak scaling
    for g in got:
        assert g[3] == 20.0 and g[4] == 300.0  # slowest rank's time, all ranks' hops


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_runs_on_rank_zero_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
