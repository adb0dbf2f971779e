"""The multi-GPU form of the benchmark is N independent replicas (the FMM of one point set is
not sharded); its only collective is the max over ranks of the step time. Covered here with
two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 10.0 + 5.0 * rank                     # rank 1 is the slower replica
    m = bench.max_over_ranks(ms, dist, "cpu")
    q.put((rank, m, bench.replica_throughput(1_000_000, m, world)))
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [15.0, 15.0]
    assert out[0][2] == pytest.approx(2 * 1_000_000 / 0.015)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(1000, 1.0, 1) == pytest.approx(1e6)
