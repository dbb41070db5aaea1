"""hm_factor_solve: the reference's solve(b) (factor + solve in one call), with a host b
copied to the device while the factorization runs.  Same answer as factor() then
solve(), for host (pageable and page-locked) and device buffers, FP64 and mixed."""
import ctypes

import numpy as np
import pytest
import torch

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix

pytestmark = pytest.mark.gpu


def _op(precision):
    p = np.random.default_rng(3).random((8192, 2))
    p = np.ascontiguousarray(p[H.morton_order(p)])
    m = H.HODLRMatrix(1e-10, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=0,
                      precision=precision, ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    return m


@pytest.mark.parametrize("precision", [H.FP64, H.MIXED])
def test_factor_solve_matches_factor_then_solve(precision):
    m = _op(precision)
    b = np.random.default_rng(4).standard_normal((m.N, 6))
    m.factor()
    ref = m.solve(b)
    x, st = m.factor_solve(b, stats=True)          # pageable host b
    assert O.rel_err(ref, x) < 1e-9
    if precision == H.MIXED:
        assert st.rel_residual <= 1e-10
    # page-locked host buffers and device buffers through the C ABI
    bp = torch.from_numpy(np.ascontiguousarray(b.T)).pin_memory()
    xp = torch.empty_like(bp).pin_memory()
    dp = ctypes.POINTER(ctypes.c_double)
    m._check(m._L.hm_factor_solve(m._h, ctypes.cast(bp.data_ptr(), dp), 6, m.N, ctypes.cast(xp.data_ptr(), dp),
                                  m.N, None))
    assert O.rel_err(ref, xp.numpy().T) < 1e-9
    bd, xd = bp.cuda(), torch.empty_like(bp, device="cuda")
    m._check(m._L.hm_factor_solve(m._h, ctypes.cast(bd.data_ptr(), dp), 6, m.N, ctypes.cast(xd.data_ptr(), dp),
                                  m.N, None))
    assert O.rel_err(ref, xd.cpu().numpy().T) < 1e-9


def test_factor_solve_reports_singular_leaf():
    c = CASES["hodlr_cauchy_gauss_1024"]
    A = make_matrix(c)
    o = O.HodlrOracle(c["tol"], c["rsvd_rank"])
    o.build_from_dense(A, c["leaf"], O.SketchSource(c["seed"], "normal"))
    next(n for n in o.nodes if n.is_leaf).D[:] = 0.0
    h = H.HODLRMatrix(c["tol"])
    h.import_factors(A.shape[0], c["leaf"], o.nodes)
    with pytest.raises(H.HmError) as e:
        h.factor_solve(np.ones(A.shape[0]))
    assert e.value.code == H.HM_ERR_SINGULAR
