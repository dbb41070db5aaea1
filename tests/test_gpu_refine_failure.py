"""Refinement that cannot converge is reported, never returned as a result.

A Gaussian kernel with h = 0.05 and shift 1e-2 on 4096 sorted points has leaf blocks
within ~1e-2 of singular (cond ~5e4 overall). Its FP32 factorization is too inaccurate
for the refinement to contract: the residual grows by orders of magnitude per sweep and
can overflow in some columns. The mixed solve must then fail with HM_ERR_IR. A column
whose residual is NaN must not drop out of the max-over-columns test: that would accept
non-finite x as converged. The FP64 solve of the same operator is fine."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("profiled", [False, True])
def test_diverging_mixed_refinement_raises(profiled):
    rng = np.random.default_rng(0)
    N = 4096
    pts = np.sort(rng.random(N))
    b = rng.standard_normal((N, 8))
    m = H.HODLRMatrix(1e-10, rsvd_rank=48, max_rank=64, sketch=H.SKETCH_DEVICE_NORMAL, precision=H.FP64,
                      ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, pts, [0.05, 1e-2], 128)
    x64 = m.solve(b)
    assert np.isfinite(x64).all()
    assert O.rel_err(b, O.gaussian_matrix(pts, 0.05, 1e-2) @ x64) < 1e-6
    m.set_precision(H.MIXED)
    H.profile_enable(profiled)
    try:
        with pytest.raises(H.HmError) as e:
            m.solve(b)
    finally:
        H.profile_enable(False)
    assert e.value.code == H.HM_ERR_IR, str(e.value)
    m.close()
