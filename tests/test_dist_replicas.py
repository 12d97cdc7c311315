"""The multi-GPU mode of bench.py runs independent replicas (the single-box step does not shard)
and reports the max over ranks of each rank's device time.  The reduction is checked with two
gloo ranks on CPU: every rank must get the element-wise maximum, and a barrier must pass."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [1.0 + rank, 10.0 - rank, 0.5 * rank]
        got = bench.max_over_ranks(mine, dist, "cpu")
        dist.barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [float(world), 10.0, 0.5 * (world - 1)]
    assert all(res[r] == expect for r in range(world)), res
