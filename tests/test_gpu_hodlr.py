"""Device path against the reference (golden fixtures from the compiled reference, and
the oracle restatement pinned to them).  Tolerances: tree layout bit-exact, ranks exact,
multiply and solve within 1e-10 relative (FP64); mixed precision refined to 1e-10."""
import os

import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix, make_vectors

pytestmark = pytest.mark.gpu

HODLR_CASES = [n for n in CASES if CASES[n]["kind"] == "hodlr"]


def load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, f"{name}.npz")))


def device_build(c, A, **kw):
    sketch = H.SKETCH_REFERENCE_NORMAL if c.get("sketch") == "normal" else H.SKETCH_REFERENCE_UNIFORM
    h = H.HODLRMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"], sketch=sketch, **kw)
    h.build_from_dense(A, c["leaf"])
    return h


def rank_flip_allowed(c, A, node, which, rank_dev, rank_ref):
    """A rank may differ only at a near-tie of S_r / S_0 with tol (compression.h:44)."""
    return abs(rank_dev - rank_ref) <= 1  # refined below by the caller when it happens


@pytest.mark.parametrize("name", HODLR_CASES)
def test_build_tree_and_ranks(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    h = device_build(c, A)
    t = h.tree()
    for k in ("start", "end", "is_leaf", "depth"):
        assert np.array_equal(t[k], g[k]), k
    assert np.array_equal(t["rank12"], g["rank12"])
    assert np.array_equal(t["rank21"], g["rank21"])


@pytest.mark.parametrize("name", HODLR_CASES)
def test_multiply_and_solve_parity(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    h = device_build(c, A)
    y = h.multiply(x)
    assert O.rel_err(g["y"], y) < 1e-10
    xs = h.solve(b)
    assert O.rel_err(g["xs"], xs) < 1e-10


@pytest.mark.parametrize("name", ["hodlr_cauchy_4096", "hodlr_gauss_ragged_1543"])
def test_imported_reference_factors(golden_dir, name):
    """Factors computed by the reference's algorithm, uploaded: the device multiply and
    solve must reproduce the reference's outputs on exactly those factors."""
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    o = O.HodlrOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))
    h = H.HODLRMatrix(c["tol"])
    h.import_factors(A.shape[0], c["leaf"], o.nodes)
    assert O.rel_err(g["y"], h.multiply(x)) < 1e-12
    assert O.rel_err(g["xs"], h.solve(b)) < 1e-10
    # factor download round-trips
    for i in (1, 2, len(o.nodes) - 1):
        n = o.nodes[i]
        if n.is_leaf:
            assert np.array_equal(h.get_factor(i, H.HODLRMatrix.D), n.D)
        assert np.array_equal(h.get_factor(i, H.HODLRMatrix.U), n.U)
        assert np.array_equal(h.get_factor(i, H.HODLRMatrix.V), n.V)


def test_multi_rhs_and_multiply_columns(golden_dir):
    c = CASES["hodlr_coulomb_2048"]
    A = make_matrix(c)
    N = A.shape[0]
    h = device_build(c, A)
    o = O.HodlrOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))
    X = np.random.default_rng(5).standard_normal((N, 7))
    assert O.rel_err(o.multiply(X), h.multiply(X)) < 1e-10
    assert O.rel_err(o.factor().solve(X), h.solve(X)) < 1e-10


def test_mixed_precision_refines_to_tolerance(golden_dir):
    c = CASES["hodlr_coulomb_2048"]
    g = load(golden_dir, "hodlr_coulomb_2048")
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    h = device_build(c, A, precision=H.MIXED, ir_tol=1e-10)
    xs, st = h.solve(b, stats=True)
    assert st.rel_residual <= 1e-10
    assert st.ir_iters >= 1
    assert O.rel_err(g["xs"], xs) < 1e-9


def test_singular_leaf_reports_error():
    c = CASES["hodlr_cauchy_gauss_1024"]
    A = make_matrix(c)
    o = O.HodlrOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"], "normal"))
    leaf = next(n for n in o.nodes if n.is_leaf)
    leaf.D = np.zeros_like(leaf.D)
    h = H.HODLRMatrix(c["tol"])
    h.import_factors(A.shape[0], c["leaf"], o.nodes)
    with pytest.raises(H.HmError) as e:
        h.solve(np.ones(A.shape[0]))
    assert e.value.code == H.HM_ERR_SINGULAR


def test_nonfinite_input_rejected():
    A = np.eye(300)
    A[7, 9] = np.nan
    h = H.HODLRMatrix(1e-8)
    with pytest.raises(H.HmError) as e:
        h.build_from_dense(A, 64)
    assert e.value.code == H.HM_ERR_NONFINITE


def test_calls_out_of_order():
    h = H.HODLRMatrix(1e-8)
    h.N = 10
    with pytest.raises(H.HmError) as e:
        h.solve(np.ones(10))
    assert e.value.code == H.HM_ERR_STATE
