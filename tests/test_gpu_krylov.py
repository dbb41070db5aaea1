"""Krylov solve against the exact operator (hm_solve_gmres): flexible GMRES on the exact
kernel matrix (entries generated on the device), right-preconditioned by the compressed
factorization.  Checked against the dense FP64 solution (numpy LAPACK) of the same kernel
matrix.

The hard case is a smooth Gaussian kernel (h = 0.2, shift 1e-3, cond(A) ~ 9e5) compressed
to rank 4: there ||A - A~|| ||A~^{-1}|| > 1, so the stationary refinement of
hm_solve_exact diverges (its residual grows ~2.5x per sweep, measured with the oracle),
while GMRES with the same factorization as preconditioner converges (13 iterations in the
oracle's numpy restatement)."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def _gaussian(N, h, shift, rank, precision=H.FP64):
    x = np.sort(np.random.default_rng(2).random(N))
    m = H.HODLRMatrix(1e-14, rsvd_rank=rank, max_rank=rank, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1,
                      precision=precision, ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, x.reshape(-1, 1), [h, shift], 128)
    return m, O.gaussian_matrix(x, h, shift)


def _resid(A, x, b):
    return float((np.linalg.norm(b - A @ x, axis=0) / np.linalg.norm(b, axis=0)).max())


def test_gmres_converges_where_refinement_diverges():
    N = 2048
    m, A = _gaussian(N, 0.2, 1e-3, 4)
    b = np.random.default_rng(5).standard_normal((N, 3))
    with pytest.raises(H.HmError) as e:      # stationary refinement: diverges
        m.solve_exact(b, tol=1e-10, max_iter=8)
    assert e.value.code == H.HM_ERR_IR
    x, st = m.solve_gmres(b, tol=1e-10, restart=40, max_iter=120, stats=True)
    assert st.rel_residual <= 1e-10 and st.ir_iters <= 60, (st.rel_residual, st.ir_iters)
    assert _resid(A, x, b) <= 1.5e-10                     # against A, measured on the host
    xd = np.linalg.solve(A, b)
    assert O.rel_err(xd, x) < 1e-3                         # cond(A) ~9e5 times the residual


def test_gmres_few_iterations_with_a_good_preconditioner():
    N = 2048
    m, A = _gaussian(N, 0.05, 1e-2, 32)
    b = np.random.default_rng(6).standard_normal((N, 2))
    x, st = m.solve_gmres(b, tol=1e-12, restart=10, max_iter=20, stats=True)
    assert st.rel_residual <= 1e-12 and st.ir_iters <= 4, (st.rel_residual, st.ir_iters)
    assert _resid(A, x, b) <= 2e-12


def test_gmres_mixed_precision_preconditioner():
    N = 2048
    m, A = _gaussian(N, 0.2, 1e-3, 4, precision=H.MIXED)
    b = np.random.default_rng(7).standard_normal(N)
    x, st = m.solve_gmres(b, tol=1e-10, restart=40, max_iter=120, stats=True)
    assert st.rel_residual <= 1e-10
    assert _resid(A, x.reshape(-1, 1), b.reshape(-1, 1)) <= 1.5e-10


def test_gmres_refuses_dense_builds_and_gives_up_with_ir_error():
    x = np.sort(np.random.default_rng(2).random(512))
    A = O.gaussian_matrix(x, 0.05, 1e-2)
    d = H.HODLRMatrix(1e-10, rsvd_rank=32)
    d.build_from_dense(A, 128)
    with pytest.raises(H.HmError) as e:
        d.solve_gmres(np.ones(512))
    assert e.value.code == H.HM_ERR_STATE
    m, _ = _gaussian(2048, 0.2, 1e-3, 4)
    with pytest.raises(H.HmError) as e:
        m.solve_gmres(np.ones(2048), tol=1e-14, restart=5, max_iter=3)
    assert e.value.code == H.HM_ERR_IR
