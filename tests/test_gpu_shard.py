"""Subtree sharding on the device (hmat_shard.py with the CUDA engine as each rank's
local solver): two ranks as two processes on one GPU, collectives through gloo on host
copies (no kernel waits on the other process).  Rank 0 builds the operator matrix-free
and saves it (hm_save); rank 1 loads the file, so both hold identical factors.  Each rank
imports its depth-1 subtree into its own handle (hm_hodlr_import) and runs the sharded
factor and solve; the assembled solution must match the single-handle FP64 solve of the
whole operator to 1e-12.

The second test builds nothing whole: each rank builds its own subtree from its points
(hm_hodlr_build_from_kernel) and compresses its rows of the top couplings with
build_top_sharded, whose block products run on the device with generated entries
(hm_kernel_block_product_device).  Checked against the dense operator the ranks built
(1e-10) and each coupling against the truncated SVD of its dense block."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _allreduce_host(buf):
    import torch
    import torch.distributed as dist
    h = buf.cpu()
    dist.all_reduce(h)
    buf.copy_(h)
    return buf


def _worker(rank, world, port, path, q):
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200")]
    import torch
    import torch.distributed as dist

    import hmat_b200 as H
    import hmat_shard as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=300))
    try:
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        N, leaf = 4096, 128
        if rank == 0:
            p = np.random.default_rng(3).random((N, 2))
            p = np.ascontiguousarray(p[H.morton_order(p)])
            h = H.HODLRMatrix(1e-9, rsvd_rank=32, max_rank=32, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=0)
            h.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], leaf)
            h.save(path)
        dist.barrier()
        if rank != 0:
            h = H.load_operator(path, 1e-9)
        plan = S.partition(N, leaf, world)
        s, e = plan.owner_range(rank)
        nodes = S.nodes_from_handle(h, (s, e))
        sub, top, table = S.rank_share(plan, rank, nodes)
        local = S.EngineLocalSolver(sub, s, leaf)
        sh = S.ShardedHODLR(plan, rank, local, S.to_torch_share(top, dev), table, S.TorchOps(dev), _allreduce_host)
        b = np.random.default_rng(12).standard_normal((N, 3))
        x = sh.solve(torch.from_numpy(b[s:e].copy()).to(dev)).cpu().numpy()
        ref = h.solve(b) if rank == 0 else None
        dist.barrier()
        q.put((rank, s, e, x, ref, sh.collectives))
        local.close()
        h.close()
    finally:
        dist.destroy_process_group()


def test_sharded_solve_on_the_engine_matches_single_handle():
    import torch.multiprocessing as mp
    sys.path[:0] = [os.path.join(ROOT, "oracle")]
    import hmat_oracle as O
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "op.hmb")
        procs = [ctx.Process(target=_worker, args=(r, world, port, path, q)) for r in range(world)]
        for p in procs:
            p.start()
        out = sorted((q.get(timeout=600) for _ in procs), key=lambda t: t[0])
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    N = 4096
    x = np.zeros((N, 3))
    for rank, s, e, xr, _, _ in out:
        x[s:e] = xr
    ref = out[0][4]
    assert len({o[5] for o in out}) == 1
    assert O.rel_err(ref, x) < 1e-12, O.rel_err(ref, x)


def _worker_build(rank, world, port, q):
    sys.path[:0] = [os.path.join(ROOT, "hmat-omp_b200")]
    import torch
    import torch.distributed as dist

    import hmat_b200 as H
    import hmat_shard as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=300))
    try:
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.current_stream().cuda_stream or 1
        N, leaf, tol, maxr = 4096, 128, 1e-10, 64
        p = np.random.default_rng(3).random((N, 2))
        p = np.ascontiguousarray(p[H.morton_order(p)])
        params = [1e-3, 4.0]
        plan = S.partition(N, leaf, world)
        s, e = plan.owner_range(rank)
        dense = H.Dense()
        dense.set_stream(stream)
        top, table, nc = S.build_top_sharded(plan, rank, S.device_block_product(dense, H.KERNEL_COULOMB, p, params),
                                             tol, maxr, oversample=10, power_iters=1, seed=5, ops=S.TorchOps(dev),
                                             allreduce=_allreduce_host)
        h = H.HODLRMatrix(tol, rsvd_rank=maxr, max_rank=maxr, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
        h.set_stream(stream)
        h.build_from_kernel(H.KERNEL_COULOMB, p[s:e], params, leaf)      # this rank's subtree only
        local = S.EngineLocalSolver.from_handle(h)
        sh = S.ShardedHODLR(plan, rank, local, top, table, S.TorchOps(dev), _allreduce_host)
        b = np.random.default_rng(12).standard_normal((N, 3))
        x = sh.solve(torch.from_numpy(b[s:e].copy()).to(dev)).cpu().numpy()
        dense_local = h.multiply(np.eye(e - s))
        share = {d: tuple(t.cpu().numpy() for t in (c.U, c.V, c.B12, c.B21)) for d, c in top.items()}
        dist.barrier()
        q.put((rank, s, e, x, nc, sh.collectives, share, dense_local))
        h.close()
        dense.close()
    finally:
        dist.destroy_process_group()


def test_sharded_build_on_the_engine():
    import torch.multiprocessing as mp
    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "hmat-omp_b200")]
    import hmat_b200 as H
    import hmat_oracle as O
    import hmat_shard as S
    world, N, leaf = 2, 4096, 128
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_build, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert len({o[4] for o in out}) == 1 and len({o[5] for o in out}) == 1
    pts = np.random.default_rng(3).random((N, 2))
    pts = pts[H.morton_order(pts)]
    A = O.coulomb_matrix(pts, 1e-3, 4.0)
    At = np.zeros_like(A)
    for rank, s, e, *_, dl in out:
        At[s:e, s:e] = dl
    plan = S.partition(N, leaf, world)
    m = plan.levels[0][0]
    (_, _, _, _, _, _, sh0, _), (_, _, _, _, _, _, sh1, _) = out
    U1, V1, B12, B21 = sh0[0]
    U2, V2 = sh1[0][0], sh1[0][1]
    for blk, approx in ((A[m.start:m.mid, m.mid:m.end], U1 @ B12 @ V2.T),
                        (A[m.mid:m.end, m.start:m.mid], U2 @ B21 @ V1.T)):
        r = np.linalg.matrix_rank(approx)
        sv = np.linalg.svd(blk, compute_uv=False)
        err = np.linalg.norm(blk - approx)
        assert err <= 10 * np.sqrt(np.sum(sv[r:] ** 2)) + 1e-10 * sv[0] * np.sqrt(len(sv)), (r, err)
    At[m.start:m.mid, m.mid:m.end] = U1 @ B12 @ V2.T
    At[m.mid:m.end, m.start:m.mid] = U2 @ B21 @ V1.T
    x = np.zeros((N, 3))
    for rank, s, e, xr, *_ in out:
        x[s:e] = xr
    b = np.random.default_rng(12).standard_normal((N, 3))
    err = O.rel_err(np.linalg.solve(At, b), x)
    assert err <= 1e-10, err
