"""Host logic of the multi-GPU bench paths, run as two gloo ranks on the CPU: how
independent systems are dealt to ranks, and the max / sum reductions of per-rank
timings that the bench reports (one process per GPU on a B200 node, NCCL there)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nsys, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    mine = bench.shard_indices(nsys, rank, world)
    t_max = bench.reduce_over_ranks(10.0 + rank, "max", world, "cpu")
    n_sum = bench.reduce_over_ranks(len(mine), "sum", world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, t_max, n_sum))


@pytest.mark.parametrize("nsys", [512, 7])
def test_two_ranks_shard_and_reduce(nsys):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nsys, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [set(o[1]) for o in out]
    assert shards[0].isdisjoint(shards[1])
    assert shards[0] | shards[1] == set(range(nsys))
    assert abs(len(shards[0]) - len(shards[1])) <= 1
    assert all(o[2] == 11.0 for o in out)          # max over ranks
    assert all(o[3] == nsys for o in out)          # every system counted once


def test_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_indices(5, 0, 1) == [0, 1, 2, 3, 4]
    assert bench.reduce_over_ranks(3.5, "max", 1, "cpu") == 3.5
