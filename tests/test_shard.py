"""Subtree sharding of one HODLR system (hmat_shard.py), run as 2 and 4 gloo ranks on
the CPU: the library's partition and collective plan, with each rank's subtree factored
and solved by the oracle's level-synchronous restatement (oracle/hmat_oracle.py
level_factor) as the local solver.  The assembled solution must match the single-rank
solve of the whole operator (the same factors) to 1e-12, and every rank must issue the
same number of collectives."""
import copy
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _operator(N, leaf):
    import hmat_b200 as H
    import hmat_oracle as O
    p = np.random.default_rng(3).random((N, 2))
    p = p[H.morton_order(p)]
    A = O.coulomb_matrix(p, 1e-3, 4.0)
    o = O.HodlrOracle(1e-9, 32, oversample=10)
    o.build_from_dense(A, leaf, O.SketchSource(7, "normal"))
    return o


class _SubtreeSolver:
    """A_g^{-1} for a rank's subtree: the oracle's factorization of a re-indexed copy."""

    def __init__(self, sub_nodes, start):
        import hmat_oracle as O
        nodes = copy.deepcopy(sub_nodes)
        ids = {id(n): i for i, n in enumerate(sub_nodes)}
        for i, n in enumerate(nodes):
            n.index = i
            n.start -= start
            n.end -= start
        for src, n in zip(sub_nodes, nodes):   # rewire children to the copies
            n.left = nodes[ids[id(src.left)]] if src.left is not None else None
            n.right = nodes[ids[id(src.right)]] if src.right is not None else None
        self.F = O.level_factor(nodes, *O._hodlr_generic(nodes))

    def solve(self, Y):
        return self.F.solve(Y)


def _worker(rank, world, port, N, leaf, q):
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200"), os.path.join(ROOT, "oracle")]
    import torch.distributed as dist

    import hmat_shard as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    try:
        o = _operator(N, leaf)
        plan = S.partition(N, leaf, world)
        sub, top, table = S.rank_share(plan, rank, o.nodes)
        s, e = plan.owner_range(rank)
        local = _SubtreeSolver(sub, s)
        sh = S.ShardedHODLR(plan, rank, local, top, table, S.NumpyOps(), S.numpy_allreduce_gloo)
        b = np.random.default_rng(11).standard_normal((N, 3))
        x = sh.solve(b[s:e])
        x2 = sh.solve(b[s:e] * 2.0)                      # factor once, solve twice
        dist.barrier()
        q.put((rank, s, e, x, x2, sh.collectives))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_solve_matches_single_rank(world):
    import torch.multiprocessing as mp
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200"), os.path.join(ROOT, "oracle")]
    import hmat_oracle as O
    N, leaf = 2048, 64
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, N, leaf, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    x = np.zeros((N, 3))
    x2 = np.zeros((N, 3))
    for rank, s, e, xr, x2r, nc in out:
        x[s:e], x2[s:e] = xr, x2r
    assert len({o[5] for o in out}) == 1          # same collectives on every rank
    b = np.random.default_rng(11).standard_normal((N, 3))
    ref = _operator(N, leaf).factor().solve(b)
    assert O.rel_err(ref, x) < 1e-12, O.rel_err(ref, x)
    assert O.rel_err(2.0 * ref, x2) < 1e-12


def test_partition_plan():
    sys.path.insert(0, os.path.join(ROOT, "hmat-omp_b200"))
    import hmat_shard as S
    plan = S.partition(1000, 64, 4)
    assert plan.p == 2 and plan.bounds == [(0, 250), (250, 500), (500, 750), (750, 1000)]
    assert [(n.start, n.mid, n.end) for n in plan.levels[1]] == [(0, 250, 500), (500, 750, 1000)]
    assert [n.depth for n in plan.path(2)] == [0, 1] and plan.side(plan.levels[1][1], 3) == 1
    with pytest.raises(ValueError):
        S.partition(1000, 64, 3)          # not a power of two
    with pytest.raises(ValueError):
        S.partition(256, 64, 8)           # depth-3 nodes would be leaves above the cut
