"""Refinement against the exact kernel operator (hm_solve_exact): the compressed
factorization preconditions a refinement whose residual uses entries of A generated on
the device.  Checked against the dense FP64 solution (numpy LAPACK) of the same kernel
matrix: the compressed solve alone is off by the compression error times cond(A); the
exact refinement reaches the requested residual against A itself."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def _gaussian(N, tol, cls=H.HODLRMatrix, precision=H.FP64):
    x = np.sort(np.random.default_rng(2).random(N))
    m = cls(tol, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1,
            precision=precision, ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, x.reshape(-1, 1), [0.05, 1e-2], 128)
    return m, O.gaussian_matrix(x, 0.05, 1e-2)


def _coulomb(N, precision):
    p = np.random.default_rng(3).random((N, 2))
    p = np.ascontiguousarray(p[H.morton_order(p)])
    m = H.HODLRMatrix(1e-6, rsvd_rank=32, max_rank=32, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=0,
                      precision=precision, ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    return m, O.coulomb_matrix(p, 1e-3, 4.0)


def _resid(A, x, b):
    return np.linalg.norm(A @ x - b, axis=0).max() / np.linalg.norm(b, axis=0).min()


@pytest.mark.parametrize("cls", [H.HODLRMatrix, H.HSSMatrix])
def test_gaussian_exact_refinement_reaches_dense_solution(cls):
    N = 4096
    m, A = _gaussian(N, 1e-7, cls)
    b = np.random.default_rng(4).standard_normal((N, 3))
    xc = m.solve(b)
    x, st = m.solve_exact(b, tol=1e-12, max_iter=10, stats=True)
    assert st.rel_residual <= 1e-12 and 1 <= st.ir_iters <= 10
    assert _resid(A, x, b) < 2e-12                 # against A, measured on the host
    assert _resid(A, xc, b) > 100 * _resid(A, x, b)  # the compressed solve alone is not there
    xd = np.linalg.solve(A, b)
    assert O.rel_err(xd, x) < 5e-7                  # cond(A) ~5e4 times the residual
    assert O.rel_err(xd, x) < 1e-2 * O.rel_err(xd, xc)


def test_mixed_precision_coulomb_exact_refinement():
    N = 4096
    m, A = _coulomb(N, H.MIXED)
    b = np.random.default_rng(5).standard_normal((N, 17))   # > 16 columns: the wide tile path
    x, st = m.solve_exact(b, tol=1e-12, max_iter=20, stats=True)
    assert st.rel_residual <= 1e-12
    assert _resid(A, x, b) < 2e-12
    assert O.rel_err(np.linalg.solve(A, b), x) < 1e-8   # cond(A) ~1e3 times the residual


def test_exact_refinement_gives_up_with_ir_error():
    m, _ = _gaussian(2048, 1e-4)
    b = np.random.default_rng(6).standard_normal(2048)
    with pytest.raises(H.HmError) as e:
        m.solve_exact(b, tol=1e-14, max_iter=0)
    assert e.value.code == H.HM_ERR_IR


def test_dense_builds_are_refused():
    x = np.sort(np.random.default_rng(2).random(1024))
    A = O.gaussian_matrix(x, 0.05, 1e-2)
    m = H.HODLRMatrix(1e-10, rsvd_rank=32)
    m.build_from_dense(A, 128)
    with pytest.raises(H.HmError) as e:
        m.solve_exact(np.ones(1024))
    assert e.value.code == H.HM_ERR_STATE


def test_residual_exact_matches_dense_residual():
    """hm_residual_exact (generated entries, A never stored) against the host residual
    with the dense kernel matrix."""
    N = 2048
    m, A = _coulomb(N, H.FP64)
    b = np.random.default_rng(7).standard_normal((N, 5))
    x = m.solve(b)
    rel = m.residual_exact(b, x)
    ref = np.linalg.norm(b - A @ x, axis=0) / np.linalg.norm(b, axis=0)
    assert np.allclose(rel, ref, rtol=1e-6, atol=1e-15)
    assert rel.max() > 1e-9   # the compressed operator is not A: a visible residual
