"""Nested-basis HSS on the device (hm_hss_set_nested; no reference counterpart: the
reference's transfers are identities, hss_routines.h:86-90) against the nested oracle
on the same sketch stream: ranks node by node, the operator, the downloaded transfers
and couplings, the solve; kernel builds against dense builds; save/load; and the switch
back to the reference form."""
import numpy as np
import pytest
import scipy.linalg as sla

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix, make_vectors, points

pytestmark = pytest.mark.gpu

NESTED_CASES = ["hss_gauss_512", "hss_gauss_rsvd_1024"]


def _build(c, A, nested=True, **kw):
    h = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"], nested=nested, **kw)
    h.build_from_dense(A, c["leaf"])
    return h


def _oracle(c, A):
    o = O.HssNestedOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))
    return o


@pytest.mark.parametrize("name", NESTED_CASES)
def test_nested_ranks_and_operator_match_oracle(name):
    c = CASES[name]
    A = make_matrix(c)
    x, _ = make_vectors(c, A.shape[0])
    h = _build(c, A)
    o = _oracle(c, A)
    assert h.nested
    t = h.tree()
    assert np.array_equal(t["rank12"], [n.rank_U for n in o.nodes])
    assert np.array_equal(t["rank21"], [n.rank_V for n in o.nodes])
    X = np.random.default_rng(4).standard_normal((A.shape[0], 3))
    assert O.rel_err(o.multiply(X), h.multiply(X)) < 1e-10
    assert O.rel_err(o.multiply(x), h.multiply(x)) < 1e-10
    assert O.rel_err(A @ X, h.multiply(X)) < 20 * c["tol"]


def test_nested_factor_download():
    """Leaf U/V, R/W and B downloaded through hm_get_factor rebuild the device operator
    (telescoping product from the exported factors only) and match the oracle's."""
    c = CASES["hss_gauss_512"]
    A = make_matrix(c)
    h = _build(c, A)
    o = _oracle(c, A)
    F = {}
    for n in o.nodes:
        i = n.id
        if n.is_leaf:
            F[i] = dict(D=h.get_factor(i, H.HSSMatrix.D), U=h.get_factor(i, H.HSSMatrix.U),
                        V=h.get_factor(i, H.HSSMatrix.V))
            assert np.array_equal(F[i]["D"], n.D)
            assert F[i]["U"].shape == n.U.shape
            continue
        B = h.get_factor(i, H.HSSMatrix.B)
        lu, lv, ru, rv = n.left.rank_U, n.left.rank_V, n.right.rank_U, n.right.rank_V
        assert B.shape == (lu + ru, lv + rv)
        assert not B[:lu, :lv].any() and not B[lu:, lv:].any()
        F[i] = dict(B12=B[:lu, lv:], B21=B[lu:, :lv])
        if n.parent is None:
            assert h.get_factor(i, H.HSSMatrix.R).size == 0
            continue
        R, W = h.get_factor(i, H.HSSMatrix.R), h.get_factor(i, H.HSSMatrix.W)
        assert R.shape == n.R.shape and W.shape == n.W.shape
        assert np.allclose(R.T @ R, np.eye(R.shape[1]), atol=1e-12)
        assert np.allclose(W.T @ W, np.eye(W.shape[1]), atol=1e-12)
        # R itself is not compared with the oracle's: it is written in the children's
        # basis coordinates, which differ from the oracle's by column signs (and rotations
        # inside clusters of equal singular values); the blocks U B V^T below do not
        F[i].update(R=R, W=W)
    # expanded bases from the downloads, then every off-diagonal block vs the oracle's
    EU, EV = {}, {}
    for n in reversed(o.nodes):
        if n.is_leaf:
            EU[n.id], EV[n.id] = F[n.id]["U"], F[n.id]["V"]
        elif n.parent is not None:
            EU[n.id] = sla.block_diag(EU[n.left.id], EU[n.right.id]) @ F[n.id]["R"]
            EV[n.id] = sla.block_diag(EV[n.left.id], EV[n.right.id]) @ F[n.id]["W"]
    Y = np.zeros_like(A)
    for n in o.nodes:
        if n.is_leaf:
            Y[n.start:n.end, n.start:n.end] = F[n.id]["D"]
        else:
            a, b = n.left, n.right
            Y[a.start:a.end, b.start:b.end] = EU[a.id] @ F[n.id]["B12"] @ EV[b.id].T
            Y[b.start:b.end, a.start:a.end] = EU[b.id] @ F[n.id]["B21"] @ EV[a.id].T
    assert O.rel_err(o.dense(), Y) < 1e-10
    X = np.random.default_rng(5).standard_normal((A.shape[0], 2))
    assert O.rel_err(Y @ X, h.multiply(X)) < 1e-12


@pytest.mark.parametrize("name", NESTED_CASES)
def test_nested_solve(name):
    c = CASES[name]
    A = make_matrix(c)
    _, b = make_vectors(c, A.shape[0])
    h = _build(c, A)
    o = _oracle(c, A)
    xs = h.solve(b)
    assert np.linalg.norm(b - h.multiply(xs)) / np.linalg.norm(b) < 1e-10
    xo = O.level_factor(o.nodes, *o.generic()).solve(b)
    assert O.rel_err(xo, xs) < 1e-9
    hm = _build(c, A, precision=H.MIXED, ir_tol=1e-10, ir_max_iter=30)
    xm, st = hm.solve(b, stats=True)
    assert st.rel_residual <= 1e-10
    assert O.rel_err(xs, xm) < 1e-8


@pytest.mark.parametrize("name", NESTED_CASES)
def test_nested_kernel_build_matches_dense(name):
    c = CASES[name]
    A = make_matrix(c)
    hd = _build(c, A)
    hk = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"], nested=True)
    hk.build_from_kernel(H.KERNEL_GAUSSIAN, points(c, A.shape[0]), [c["h"], c["shift"]], c["leaf"])
    td, tk = hd.tree(), hk.tree()
    for key in ("start", "end", "is_leaf", "rank12", "rank21"):
        assert np.array_equal(td[key], tk[key]), key
    X = np.random.default_rng(6).standard_normal((A.shape[0], 2))
    assert O.rel_err(hd.multiply(X), hk.multiply(X)) < 1e-12


def test_nested_save_load(tmp_path):
    c = CASES["hss_gauss_rsvd_1024"]
    A = make_matrix(c)
    h = _build(c, A)
    f = str(tmp_path / "nested.hmat")
    h.save(f)
    r = H.load_operator(f, c["tol"])
    assert r.nested
    X = np.random.default_rng(7).standard_normal((A.shape[0], 2))
    assert np.array_equal(h.multiply(X), r.multiply(X))
    for key in ("rank12", "rank21"):
        assert np.array_equal(h.tree()[key], r.tree()[key])
    n = next(i for i, (d, leaf) in enumerate(zip(h.tree()["depth"], h.tree()["is_leaf"])) if d == 1 and not leaf)
    assert np.array_equal(h.get_factor(n, H.HSSMatrix.R), r.get_factor(n, H.HSSMatrix.R))


def test_mode_switch_and_rank_growth():
    """One handle: nested, then the reference form (rank sums, R = I), then nested again.
    On a 2-D Coulomb operator the reference form's ranks at depth 1 are the sums over 16
    leaves; the nested ones stay at the strips' numerical ranks."""
    p = np.random.default_rng(8).random((4096, 2))
    p = np.ascontiguousarray(p[O.morton_order(p)])
    A = O.coulomb_matrix(p, 1e-3, 4.0)
    h = H.HSSMatrix(1e-8, rsvd_rank=64, seed=3, nested=True)
    h.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    tn = h.tree()
    X = np.random.default_rng(9).standard_normal((4096, 2))
    en = O.rel_err(A @ X, h.multiply(X))
    h.set_nested(False)
    h.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    assert not h.nested
    tr = h.tree()
    er = O.rel_err(A @ X, h.multiply(X))
    d1 = (tn["depth"] == 1)
    assert tn["rank12"][d1].max() < tr["rank12"][d1].min()
    assert en < 20 * 1e-8 and er < 20 * 1e-8
    i = int(np.flatnonzero(d1)[0])
    assert np.array_equal(h.get_factor(i, H.HSSMatrix.R), np.eye(tr["rank12"][i]))
    h.set_nested(True)
    h.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    assert h.nested and np.array_equal(h.tree()["rank12"], tn["rank12"])
