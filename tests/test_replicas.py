"""Multi-GPU form of the bench: independent replicas, one process per GPU; the
only collectives are the timing reduction (max over ranks). Exercised with two
gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    local_ms = [120.0, 150.0][rank]       # the second replica is the slow one
    m = bench.max_over_ranks(local_ms, world, "cpu")
    q.put((rank, m, bench.replica_throughput(5, world, m)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, m, thr in out:
        assert m == 150.0
        assert thr == pytest.approx(2 * 5 / 0.150)
