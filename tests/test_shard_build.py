"""Sharded compression of the top-level couplings (hmat_shard.build_top_sharded), run as
2 and 4 gloo ranks on the CPU.  No rank forms more than its own rows of the operator:
each compresses its rows of the coupling blocks above its subtree with distributed
range finding (Gram and projection all-reduces), builds its own subtree alone (the
oracle's HODLR restatement on its diagonal block), and the sharded factor + solve runs on
the result.  The operator is the headline's kind at a CPU size: 2-D Coulomb, ranks <= 96,
tolerance 1e-10, which the top couplings do not reach at these ranks.  Checked:
* every top coupling A12 = U1 B12 V2^T and A21 = U2 B21 V1^T, assembled from the ranks'
  rows, against the best approximation of its rank (the truncated SVD of the dense
  block): Frobenius error <= 10x the optimal tail (a randomized range finder with one
  power iteration and 10 oversampling columns is near-optimal);
* the sharded factor + solve against a dense LAPACK solve of the operator the ranks built
  (their subtrees expanded, the couplings assembled): <= 1e-10;
* the same number of collectives and one rank table on every rank.
Both array back ends run it: numpy, and torch tensors (the device path's code, here on
the CPU) with torch.distributed's all-reduce."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, LEAF, TOL, MAXR = 2048, 64, 1e-10, 96


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _matrix():
    import hmat_b200 as H
    import hmat_oracle as O
    p = np.random.default_rng(3).random((N, 2))
    p = p[H.morton_order(p)]
    return O.coulomb_matrix(p, 1e-3, 4.0)


class _LocalSolver:
    """A_g^{-1} of this rank's subtree, built by the rank alone from its diagonal block."""

    def __init__(self, Ag):
        import hmat_oracle as O
        o = O.HodlrOracle(TOL, 48, oversample=10)
        o.build_from_dense(Ag, LEAF, O.SketchSource(7, "normal"))
        self.o = o
        self.F = o.factor()

    def solve(self, Y):
        return self.F.solve(Y)


def _worker(rank, world, port, backend, q):
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200"), os.path.join(ROOT, "oracle")]
    import torch.distributed as dist

    import hmat_shard as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    try:
        A = _matrix()
        plan = S.partition(N, LEAF, world)
        s, e = plan.owner_range(rank)

        if backend == "torch":
            import torch
            At = torch.from_numpy(A)
            ops, allreduce = S.TorchOps("cpu"), S.torch_allreduce
        else:
            At, ops, allreduce = A, S.NumpyOps(), S.numpy_allreduce_gloo

        def block_product(r0, r1, c0, c1, X, trans):
            assert (r0, r1) == (s, e)       # only this rank's rows are ever asked for
            blk = At[r0:r1, c0:c1]
            return blk.T @ X if trans else blk @ X

        top, table, nc = S.build_top_sharded(plan, rank, block_product, TOL, MAXR, oversample=10, power_iters=1,
                                             seed=5, ops=ops, allreduce=allreduce)
        np_of = (lambda t: t.numpy()) if backend == "torch" else (lambda t: t)
        top = {d: S.TopCoupling(*(np_of(t) for t in (c.B12, c.B21, c.U, c.V))) for d, c in top.items()}
        local = _LocalSolver(A[s:e, s:e])
        sh = S.ShardedHODLR(plan, rank, local, top, table, S.NumpyOps(), S.numpy_allreduce_gloo)
        b = np.random.default_rng(11).standard_normal((N, 3))
        x = sh.solve(b[s:e])
        dist.barrier()
        share = {d: (c.U, c.V, c.B12, c.B21) for d, c in top.items()}
        dense = local.o.multiply(np.eye(e - s))            # the subtree operator, expanded
        q.put((rank, s, e, x, nc, sh.collectives, share, table, dense))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,backend", [(2, "numpy"), (4, "numpy"), (2, "torch")])
def test_sharded_build_and_solve(world, backend):
    import torch.multiprocessing as mp
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200"), os.path.join(ROOT, "oracle")]
    import hmat_oracle as O
    import hmat_shard as S
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, backend, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert len({o[4] for o in out}) == 1 and len({o[5] for o in out}) == 1
    assert len({tuple(sorted(o[7].items())) for o in out}) == 1     # one rank table everywhere
    A = _matrix()
    At = np.zeros_like(A)          # the operator the ranks built
    for rank, s, e, *_, dense in out:
        At[s:e, s:e] = dense
    plan = S.partition(N, LEAF, world)
    # every top coupling, assembled from the ranks' rows
    for d, lvl in enumerate(plan.levels):
        for m in lvl:
            parts = {0: {}, 1: {}}
            for rank, s, e, _, _, _, share, _, _ in out:
                if m.start <= s and e <= m.end:
                    parts[plan.side(m, rank)][s] = share[d]
            U1 = np.vstack([parts[0][s][0] for s in sorted(parts[0])])
            V1 = np.vstack([parts[0][s][1] for s in sorted(parts[0])])
            U2 = np.vstack([parts[1][s][0] for s in sorted(parts[1])])
            V2 = np.vstack([parts[1][s][1] for s in sorted(parts[1])])
            B12, B21 = next(iter(parts[0].values()))[2], next(iter(parts[0].values()))[3]
            for blk, approx in ((A[m.start:m.mid, m.mid:m.end], U1 @ B12 @ V2.T),
                                (A[m.mid:m.end, m.start:m.mid], U2 @ B21 @ V1.T)):
                r = approx.shape[1] and np.linalg.matrix_rank(approx)
                sv = np.linalg.svd(blk, compute_uv=False)
                tail = np.sqrt(np.sum(sv[r:] ** 2))
                err = np.linalg.norm(blk - approx)
                assert err <= 10 * tail + 1e-10 * sv[0] * np.sqrt(len(sv)), (d, m.slot, r, err, tail)
            At[m.start:m.mid, m.mid:m.end] = U1 @ B12 @ V2.T
            At[m.mid:m.end, m.start:m.mid] = U2 @ B21 @ V1.T
    x = np.zeros((N, 3))
    for rank, s, e, xr, *_ in out:
        x[s:e] = xr
    b = np.random.default_rng(11).standard_normal((N, 3))
    err = O.rel_err(np.linalg.solve(At, b), x)
    assert err <= 1e-10, err
