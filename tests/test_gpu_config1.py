"""Configuration 1 on the device path: plain HODLR in FP64 on the Cauchy kernel
A_ij = 1/(x_i - y_j), x_i = i/N, y_j = (j + 0.5)/N, N = 4096, leaf 64, fixed rank 16
(rank cap 16, truncation tolerance 0), oversampling 10, one power iteration, Gaussian
sketch drawn on the host from mt19937(seed 0) in the reference's draw order.

Checked against the oracle's compress_rsvd (oracle/hmat_oracle.py, compression.h:67-99
plus the power-iteration and rank-cap extensions) built on the same sketch stream: tree
and ranks exact, multiply and solve within 1e-10 relative.  The error against dense
LAPACK (numpy solve of the full matrix) is stated and bounded: the rank-16 truncation
leaves ~5e-10 on this operator."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu

N, LEAF, RANK, OVERSAMPLE, POWER, SEED = 4096, 64, 16, 10, 1, 0


@pytest.fixture(scope="module")
def config1():
    A = O.cauchy_matrix(N)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(N)
    b = rng.standard_normal(N)
    o = O.HodlrOracle(0.0, RANK, oversample=OVERSAMPLE, power_iters=POWER, max_rank=RANK)
    o.build_from_dense(A, LEAF, O.SketchSource(SEED, "normal"))
    h = H.HODLRMatrix(0.0, rsvd_rank=RANK, oversample=OVERSAMPLE, power_iters=POWER, max_rank=RANK,
                      sketch=H.SKETCH_REFERENCE_NORMAL, seed=SEED)
    h.build_from_dense(A, LEAF)
    yield A, x, b, o, h
    h.close()


def test_config1_tree_and_fixed_ranks(config1):
    A, x, b, o, h = config1
    t = h.tree()
    assert list(t["start"]) == [n.start for n in o.nodes]
    assert list(t["end"]) == [n.end for n in o.nodes]
    internal = t["is_leaf"] == 0
    assert np.all(t["rank12"][internal] == RANK) and np.all(t["rank21"][internal] == RANK)
    assert list(t["rank12"]) == [0 if n.is_leaf else n.B12.shape[0] for n in o.nodes]


def test_config1_multiply_and_solve_vs_oracle(config1):
    A, x, b, o, h = config1
    assert O.rel_err(o.multiply(x), h.multiply(x)) < 1e-10
    assert O.rel_err(o.factor().solve(b), h.solve(b)) < 1e-10


def test_config1_error_vs_dense_lapack(config1):
    A, x, b, o, h = config1
    e_mv = O.rel_err(A @ x, h.multiply(x))
    e_sv = O.rel_err(np.linalg.solve(A, b), h.solve(b))
    print(f"config 1: multiply vs dense {e_mv:.2e}, solve vs dense LAPACK {e_sv:.2e}")
    assert e_mv < 5e-9 and e_sv < 5e-9
