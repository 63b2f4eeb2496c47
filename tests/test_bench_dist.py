"""Multi-rank plumbing of bench.py on CPU: two gloo ranks, each with its own
independent specimen (no data-path collective). The reported value is all
ranks' bond updates over the slowest rank's time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    bench.barrier(dist, "cpu")
    ms_local = [10.0, 25.0][rank]
    bonds_local = [1000, 3000][rank]
    value, ms, total = bench.aggregate(dist, "cpu", ms_local, bonds_local, steps=4)
    q.put((rank, value, ms, total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, value, ms, total in res:
        assert ms == 25.0
        assert total == 4000.0
        assert value == pytest.approx(4000.0 * 4 / 0.025)
