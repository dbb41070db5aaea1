"""Parameters of the golden cases (inputs are regenerated from these).

Each case names the reference class it exercises, the operator, the tree and
compression options, the sketch seed, and the seeds of the vectors.  The operators are
the benchmark configurations' kernels at sizes the CPU reference finishes in seconds,
plus the reference drivers' own operator (include/kernel.h:30-48, main_hodlr.cpp:38-51)
and ragged/edge trees.
"""
from __future__ import annotations

import numpy as np

CASES = {
    # configuration-1 operator: Cauchy 1/(x_i - y_j), x_i = i/N, y_j = (j+0.5)/N
    "hodlr_cauchy_4096": dict(kind="hodlr", op="cauchy", N=4096, leaf=64, tol=1e-8, rsvd_rank=16,
                              seed=11, xseed=1, nrhs=1),
    # the reference HODLR driver's operator: 1/(x_i + x_j + 1) + I on i/(N-1)
    "hodlr_driver_2048": dict(kind="hodlr", op="driver_cauchy", N=2048, leaf=512, tol=1e-8,
                              rsvd_rank=64, seed=12, xseed=2, nrhs=1),
    # Gaussian sketch variant (N(0,1) through the same mt19937 stream)
    "hodlr_cauchy_gauss_1024": dict(kind="hodlr", op="cauchy", N=1024, leaf=64, tol=1e-8,
                                    rsvd_rank=16, seed=13, xseed=3, nrhs=1, sketch="normal"),
    # ragged tree: leaves at several depths, full-SVD and RSVD blocks mixed
    "hodlr_gauss_ragged_1543": dict(kind="hodlr", op="gaussian", N=1543, leaf=96, tol=1e-9,
                                    rsvd_rank=32, seed=14, xseed=4, nrhs=3, h=0.05, shift=1e-2,
                                    pseed=2),
    # 2-D Coulomb (configuration-3 operator), Morton-sorted points
    "hodlr_coulomb_2048": dict(kind="hodlr", op="coulomb", N=2048, leaf=128, tol=1e-10,
                               rsvd_rank=64, seed=15, xseed=5, nrhs=2, pseed=3),
    # single leaf: the root is a leaf (N <= leaf)
    "hodlr_single_leaf_50": dict(kind="hodlr", op="gaussian", N=50, leaf=64, tol=1e-8,
                                 rsvd_rank=64, seed=16, xseed=6, nrhs=1, h=0.05, shift=1e-2,
                                 pseed=7),
    # non-symmetric leaves of 256 whose leading 128 x 128 block is zero (singular) while the
    # leaf is regular: getrf's partial pivoting handles them (matrix.h:120-131)
    "hodlr_pivot_leaf_1024": dict(kind="hodlr", op="pivot_leaf", N=1024, leaf=256, tol=1e-10,
                                  rsvd_rank=32, seed=17, xseed=9, nrhs=2, pseed=11),
    # HSS: configuration-2 operator (Gaussian h = 0.05 + 1e-2 I, sorted uniform points)
    "hss_gauss_512": dict(kind="hss", op="gaussian", N=512, leaf=64, tol=1e-10, rsvd_rank=64,
                          seed=21, xseed=7, nrhs=1, h=0.05, shift=1e-2, pseed=2),
    # HSS with leaves >= 256: the RSVD path of the leaf strips
    "hss_gauss_rsvd_1024": dict(kind="hss", op="gaussian", N=1024, leaf=256, tol=1e-9,
                                rsvd_rank=64, seed=22, xseed=8, nrhs=1, h=0.05, shift=1e-2,
                                pseed=2),
}


def points(c, N):
    rng = np.random.default_rng(c.get("pseed", 0))
    if c["op"] == "coulomb":
        import hmat_oracle as O
        p = rng.random((N, 2))
        return p[O.morton_order(p)]
    return np.sort(rng.random(N))


def make_matrix(c) -> np.ndarray:
    import hmat_oracle as O
    N = c["N"]
    if c["op"] == "cauchy":
        return O.cauchy_matrix(N)
    if c["op"] == "driver_cauchy":
        x = np.arange(N) / (N - 1)
        A = 1.0 / (x[:, None] + x[None, :] + 1.0)
        A[np.diag_indices(N)] += 1.0
        return A
    if c["op"] == "gaussian":
        return O.gaussian_matrix(points(c, N), c["h"], c["shift"])
    if c["op"] == "pivot_leaf":
        # smooth off-diagonal part (the reference driver's kernel), leaf diagonal blocks
        # [[0, B], [C, E]]: singular leading half, regular leaf
        x = np.arange(N) / (N - 1)
        A = 1.0 / (x[:, None] + x[None, :] + 1.0)
        rng = np.random.default_rng(c["pseed"])
        L, h = c["leaf"], c["leaf"] // 2
        for s0 in range(0, N, L):
            B = 2.0 * np.eye(h) + 0.3 * rng.standard_normal((h, h)) / np.sqrt(h)
            C = 2.0 * np.eye(h) + 0.3 * rng.standard_normal((h, h)) / np.sqrt(h)
            E = 0.3 * rng.standard_normal((h, h)) / np.sqrt(h)
            A[s0:s0 + L, s0:s0 + L] = np.block([[np.zeros((h, h)), B], [C, E]])
        return A
    if c["op"] == "coulomb":
        return O.coulomb_matrix(points(c, N))
    raise ValueError(c["op"])


def make_vectors(c, N):
    rng = np.random.default_rng(c["xseed"])
    x = rng.standard_normal(N)
    b = rng.standard_normal((N, c["nrhs"]))
    if c["nrhs"] == 1:
        b = b[:, 0]
    if c["kind"] == "hss":
        b = b if b.ndim == 1 else b[:, 0]
    return x, b
