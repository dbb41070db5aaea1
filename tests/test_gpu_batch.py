"""Many independent HODLR systems in shared launches (the batched configuration's
kernel: Gaussian, h log-uniform in [0.01, 0.2], shift 1e-2, leaf 64, ranks <= 48, 1-64
right-hand sides each), at sizes a dense check finishes quickly."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def make_batch(nsys, nmin, nmax, seed=4):
    rng = np.random.default_rng(seed)
    Ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys)).astype(int)
    hs = np.exp(rng.uniform(np.log(0.01), np.log(0.2), nsys))
    ss = rng.integers(1, 65, nsys)
    pts = [np.sort(rng.random(n)) for n in Ns]
    return Ns, hs, ss, pts


def test_batch_matches_dense_per_system():
    Ns, hs, ss, pts = make_batch(24, 256, 3000)
    # smooth kernels (h up to 0.2) with shift 1e-2 reach cond ~1e6: one FP64 refinement
    # step restores the backward error that the explicit-inverse Woodbury sweep loses
    B = H.HODLRBatch(1e-12, rsvd_rank=48, max_rank=48, sketch=H.SKETCH_DEVICE_NORMAL, seed=2, refine_steps=1)
    B.build_from_kernel(H.KERNEL_GAUSSIAN, pts, [[h, 1e-2] for h in hs], 64)
    rng = np.random.default_rng(5)
    bs = [rng.standard_normal((n, s)) for n, s in zip(Ns, ss)]
    xs = B.solve(bs)
    ys = B.multiply(xs)
    for k in range(len(Ns)):
        # backward error against the compressed operator (after one refinement step it
        # sits at ~1e-12, the FP64 rounding of the sweep at cond ~1e6; the workload's
        # bar is 1e-10) and forward error vs dense FP64
        assert O.rel_err(bs[k], ys[k]) < 1e-11, (k, O.rel_err(bs[k], ys[k]))
        A = O.gaussian_matrix(pts[k], hs[k], 1e-2)
        xd = np.linalg.solve(A, bs[k])
        assert O.rel_err(xd, xs[k]) < 1e-6, (k, O.rel_err(xd, xs[k]))


def test_batch_equals_single_system_handles():
    """A batch of one system and the single-system API give the same operator."""
    Ns, hs, ss, pts = make_batch(1, 2048, 2048, seed=7)
    kw = dict(rsvd_rank=48, max_rank=48, sketch=H.SKETCH_DEVICE_NORMAL, seed=3)
    B = H.HODLRBatch(1e-10, **kw)
    B.build_from_kernel(H.KERNEL_GAUSSIAN, pts, [[hs[0], 1e-2]], 64)
    S = H.HODLRMatrix(1e-10, **kw)
    S.build_from_kernel(H.KERNEL_GAUSSIAN, pts[0].reshape(-1, 1), [hs[0], 1e-2], 64)
    b = np.random.default_rng(1).standard_normal((Ns[0], 3))
    # same operator (multiply agrees to rounding); the solves agree to rounding times cond
    # (split-K sums are accumulated in a nondeterministic order; cond reaches ~1e6 here)
    assert O.rel_err(S.multiply(b), B.multiply([b])[0]) < 1e-12
    assert O.rel_err(S.solve(b), B.solve([b])[0]) < 1e-8


def test_batch_zero_rhs_systems_are_skipped():
    Ns, hs, ss, pts = make_batch(5, 300, 900, seed=9)
    B = H.HODLRBatch(1e-10, rsvd_rank=48, max_rank=48, sketch=H.SKETCH_DEVICE_NORMAL)
    B.build_from_kernel(H.KERNEL_GAUSSIAN, pts, [[h, 1e-2] for h in hs], 64)
    rng = np.random.default_rng(2)
    bs = [rng.standard_normal((n, 2)) if k % 2 == 0 else None for k, n in enumerate(Ns)]
    xs = B.solve(bs)
    for k, (b, x) in enumerate(zip(bs, xs)):
        if b is None:
            assert x is None
        else:
            A = O.gaussian_matrix(pts[k], hs[k], 1e-2)
            assert O.rel_err(np.linalg.solve(A, b), x) < 1e-6
