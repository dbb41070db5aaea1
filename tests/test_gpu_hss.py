"""HSS device path against the reference (hss_routines.h): build_topo ids, leaf ranks and
their sums, multiply and solve on the golden cases (full-SVD and RSVD leaf strips)."""
import os

import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix, make_vectors

pytestmark = pytest.mark.gpu

HSS_CASES = [n for n in CASES if CASES[n]["kind"] == "hss"]


def load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, f"{name}.npz")))


def build(c, A):
    h = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    h.build_from_dense(A, c["leaf"])
    return h


@pytest.mark.parametrize("name", HSS_CASES)
def test_hss_tree_and_ranks(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    h = build(c, make_matrix(c))
    t = h.tree()
    assert np.array_equal(t["start"], g["start"])
    assert np.array_equal(t["end"], g["end"])
    assert np.array_equal(t["is_leaf"], g["is_leaf"])
    assert np.array_equal(t["rank12"], g["rank_U"])
    assert np.array_equal(t["rank21"], g["rank_V"])


@pytest.mark.parametrize("name", HSS_CASES)
def test_hss_multiply_and_solve(golden_dir, name):
    c = CASES[name]
    g = load(golden_dir, name)
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    h = build(c, A)
    assert O.rel_err(g["y"], h.multiply(x)) < 1e-10
    xs = h.solve(b)
    # the reference's HSS solve recurses per column (hss_routines.h:281-290); both solve
    # the same compressed operator, cond ~1e4: agreement to 1e-10
    assert O.rel_err(g["xs"], xs) < 1e-10
    # backward error against the device operator itself (explicit leaf/capacitance
    # inverses: measured ~2e-11 at cond ~1e4)
    r = b - h.multiply(xs)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10


def test_hss_factor_download_matches_oracle():
    import scipy.linalg as sla

    c = CASES["hss_gauss_512"]
    A = make_matrix(c)
    h = build(c, A)
    o = O.HssOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"]))

    def leaves(n):
        return [n] if n.is_leaf else leaves(n.left) + leaves(n.right)

    def basis(n, which):  # reconstruct_U/V (hss_routines.h:23-45) from downloaded leaf bases
        return sla.block_diag(*[h.get_factor(l.id, which) for l in leaves(n)])

    for n in o.nodes:
        if n.is_leaf:
            assert np.array_equal(h.get_factor(n.id, H.HSSMatrix.D), n.D)
            U = h.get_factor(n.id, H.HSSMatrix.U)
            assert U.shape == n.U.shape
            assert np.allclose(np.abs(U.T @ n.U), np.eye(U.shape[1]), atol=1e-8)  # up to column signs
        else:
            assert np.array_equal(h.get_factor(n.id, H.HSSMatrix.R), np.eye(n.rank_U))
            assert np.array_equal(h.get_factor(n.id, H.HSSMatrix.W), np.eye(n.rank_V))
            B = h.get_factor(n.id, H.HSSMatrix.B)
            assert B.shape == n.B.shape
            lu, lv = n.left.rank_U, n.left.rank_V
            ref_blk = o.reconstruct_U(n.left) @ n.B[:lu, lv:] @ o.reconstruct_V(n.right).T
            dev_blk = basis(n.left, H.HSSMatrix.U) @ B[:lu, lv:] @ basis(n.right, H.HSSMatrix.V).T
            assert O.rel_err(ref_blk, dev_blk) < 1e-10


@pytest.mark.parametrize("name", HSS_CASES)
def test_hss_kernel_build_matches_dense(name):
    """hm_hss_build_from_kernel (entries generated on the device, A never stored) gives
    the operator the dense build gives: same tree and ranks, multiply and solve equal to
    rounding (same sketch stream)."""
    c = CASES[name]
    A = make_matrix(c)
    x, b = make_vectors(c, A.shape[0])
    from cases import points
    hd = build(c, A)
    hk = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    hk.build_from_kernel(H.KERNEL_GAUSSIAN, points(c, A.shape[0]), [c["h"], c["shift"]], c["leaf"])
    td, tk = hd.tree(), hk.tree()
    for key in ("start", "end", "is_leaf", "rank12", "rank21"):
        assert np.array_equal(td[key], tk[key]), key
    assert O.rel_err(hd.multiply(x), hk.multiply(x)) < 1e-12
    assert O.rel_err(hd.solve(b), hk.solve(b)) < 1e-10
