"""N > 1 host logic of bench.py on CPU: two gloo ranks, barrier, max over
ranks, whole-job replica throughput (the GPU run uses the same helpers with
NCCL, one replica of the workload per GPU, no data-path collective)."""
import os
import socket

import pytest


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench.barrier(dist)
    ms = 10.0 + 5.0 * rank                    # rank 1 is the slow one
    mx = bench.max_over_ranks(dist, ms, "cpu")
    thr = bench.replica_throughput(world, 1_000_000, mx)
    out.put((rank, mx, thr))
    bench.barrier(dist)
    dist.destroy_process_group()


def test_two_rank_max_and_weak_scaling_throughput():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, thr in res:
        assert mx == 15.0                        # max over ranks, on every rank
        assert abs(thr - 2 * 1e6 / 15e-3 / 1e6) < 1e-9   # 2 replicas / slowest rank


def test_single_process_helpers_are_identity():
    import bench
    assert bench.max_over_ranks(None, 3.5, "cpu") == 3.5
    assert bench.replica_throughput(1, 12_582_912, 22.5) == pytest.approx(559.24, rel=1e-3)
