"""The N > 1 path of bench.py (independent replicas, max-over-ranks timing)
with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    v = bench.max_over_ranks(10.0 + 5 * rank, dist)
    w = bench.max_over_ranks(3.0 - rank, dist)
    out.put((rank, v, w))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, v, w in res:
        assert v == 15.0 and w == 3.0


def test_single_rank_identity():
    import bench
    assert bench.max_over_ranks(7.5, None) == 7.5
