"""The nested-basis HSS oracle (an extension: the reference's transfers are identities,
hss_routines.h:86-90) on CPU: its telescoping product equals its dense form, it
approximates A to the truncation tolerance, its transfers are orthonormal, and its ranks
stay at the strips' numerical ranks where the reference form's grow with the leaves."""
import numpy as np
import pytest

import hmat_oracle as O
from cases import CASES, make_matrix


def _pair(name):
    c = CASES[name]
    A = make_matrix(c)
    nested = O.HssNestedOracle(c["tol"], c["rsvd_rank"])
    nested.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))
    ref = O.HssOracle(c["tol"], c["rsvd_rank"])
    ref.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))
    return c, A, nested, ref


@pytest.mark.parametrize("name", ["hss_gauss_512", "hss_gauss_rsvd_1024"])
def test_nested_oracle_operator(name):
    c, A, o, ref = _pair(name)
    x = np.random.default_rng(1).standard_normal((A.shape[0], 3))
    y = o.multiply(x)
    assert O.rel_err(o.dense() @ x, y) < 1e-13
    # nested truncation errors add up over the levels: a few tol, like the reference form's
    assert O.rel_err(A @ x, y) < 20 * c["tol"]
    assert O.rel_err(A @ x, y) < 10 * O.rel_err(A @ x, ref.multiply(x)) + c["tol"]
    for n in o.nodes:
        if n.is_leaf:
            # leaf bases are the reference form's (same sketch stream)
            m = next(r for r in ref.nodes if r.id == n.id)
            assert n.U.shape == m.U.shape and n.V.shape == m.V.shape
            continue
        if n.parent is None:
            assert n.rank_U == 0 and n.rank_V == 0
            continue
        assert n.R.shape == (n.left.rank_U + n.right.rank_U, n.rank_U)
        assert np.allclose(n.R.T @ n.R, np.eye(n.rank_U), atol=1e-12)
        assert np.allclose(n.W.T @ n.W, np.eye(n.rank_V), atol=1e-12)
        m = next(r for r in ref.nodes if r.id == n.id)
        assert n.rank_U <= m.rank_U and n.rank_V <= m.rank_V


def test_nested_ranks_do_not_grow():
    """Gaussian kernel, 8 leaves under each depth-1 node: the reference form's rank there
    is the sum of its leaves' ranks, the nested rank is the strip's."""
    c, A, o, ref = _pair("hss_gauss_512")
    d1 = [n for n in o.nodes if n.depth == 1]
    r1 = [n for n in ref.nodes if n.depth == 1]
    assert max(n.rank_U for n in d1) * 2 < min(n.rank_U for n in r1)


def test_nested_oracle_solve():
    c, A, o, _ = _pair("hss_gauss_512")
    F = O.level_factor(o.nodes, *o.generic())
    b = np.random.default_rng(2).standard_normal((A.shape[0], 2))
    x = F.solve(b)
    assert O.rel_err(b, o.multiply(x)) < 1e-11
