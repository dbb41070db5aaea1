"""The oracle (numpy restatement of the reference) against the reference's own answers:
the golden fixtures made by tests/golden/make_golden.py from the compiled reference,
and, where oracle/_ref is built, the reference library itself."""
import os

import numpy as np
import pytest

import hmat_oracle as O
import ref
from cases import CASES, make_matrix, make_vectors


def load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, f"{name}.npz")))


def oracle_build(c, A):
    kind = "normal" if c.get("sketch") == "normal" else "uniform"
    src = O.SketchSource(c["seed"], kind)
    if c["kind"] == "hodlr":
        o = O.HodlrOracle(c["tol"], c["rsvd_rank"])
    else:
        o = O.HssOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], src)
    return o


@pytest.mark.parametrize("name", [n for n in CASES if CASES[n]["kind"] == "hodlr"])
def test_hodlr_oracle_matches_reference(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    o = oracle_build(c, A)
    # tree layout: bit-exact
    assert np.array_equal(g["start"], [n.start for n in o.nodes])
    assert np.array_equal(g["end"], [n.end for n in o.nodes])
    assert np.array_equal(g["is_leaf"], [int(n.is_leaf) for n in o.nodes])
    assert np.array_equal(g["depth"], [n.depth for n in o.nodes])
    # ranks: exact
    r12 = [0 if n.is_leaf else n.B12.shape[0] for n in o.nodes]
    r21 = [0 if n.is_leaf else n.B21.shape[0] for n in o.nodes]
    assert np.array_equal(g["rank12"], r12)
    assert np.array_equal(g["rank21"], r21)
    # multiply (column 0, as the reference) and the recursive solve
    assert O.rel_err(g["y"], o.multiply(x)) < 1e-13
    assert O.rel_err(g["xs"], o.solve_recursive(b)) < 1e-11
    # the level-synchronous factorization that the GPU runs
    assert O.rel_err(g["xs"], o.factor().solve(b)) < 1e-11


@pytest.mark.parametrize("name", [n for n in CASES if CASES[n]["kind"] == "hss"])
def test_hss_oracle_matches_reference(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    o = oracle_build(c, A)
    assert np.array_equal(g["start"], [n.start for n in o.nodes])
    assert np.array_equal(g["left"], [n.left.id if n.left else -1 for n in o.nodes])
    assert np.array_equal(g["parent"], [n.parent.id if n.parent else -1 for n in o.nodes])
    assert np.array_equal(g["rank_U"], [n.rank_U for n in o.nodes])
    assert np.array_equal(g["rank_V"], [n.rank_V for n in o.nodes])
    assert O.rel_err(g["y"], o.multiply(x)) < 1e-13
    assert O.rel_err(g["xs"], o.factor().solve(b)) < 1e-9


def test_rng_stream_matches_reference():
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    for seed in (0, 5, 123456789):
        for shape in ((7, 3), (300, 26)):
            assert np.array_equal(ref.random(seed, *shape), O.RefStream(seed).uniform(*shape))
            if ref.available(gaussian=True):
                assert np.array_equal(ref.random(seed, *shape, gaussian=True),
                                      O.RefStream(seed).normal(*shape))


def test_compress_rsvd_matches_reference():
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    A = O.cauchy_matrix(1024)[:512, 512:]
    U, V, S = ref.compress_rsvd(A, 1e-9, 20, seed=9)
    lr = O.compress_rsvd(A, 1e-9, 20, O.SketchSource(9))
    assert lr.rank == S.shape[0]
    assert np.allclose(lr.S, S, rtol=1e-12, atol=1e-14 * S[0])
    assert O.rel_err(U * S @ V.T, lr.U * lr.S @ lr.V.T) < 1e-13


def test_transpose_solve_is_adjoint():
    c = CASES["hodlr_cauchy_gauss_1024"]
    A = make_matrix(c)
    o = oracle_build(c, A)
    F = o.factor()
    N = A.shape[0]
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal(N), rng.standard_normal(N)
    # <A^{-1} u, v> == <u, A^{-T} v>
    lhs = F.solve(u) @ v
    rhs = u @ F.solve_transpose(v)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
