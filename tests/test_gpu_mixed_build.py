"""The mixed-precision matrix-free build: sketch, power-iteration and projection products
in FP32 on the tensor cores (tcgen05, A's entries generated inside the kernel, TF32 hi/lo
products accumulated in FP32), the sketch's basis by shifted CholeskyQR3 in FP64, the
small SVDs in FP64 (compression.h:67-99 with those substitutions).

Checked against the FP64 build of the same operator: the two compressed operators agree
to the FP32 level of the sketch (relative 1e-5 on products with random vectors, both
checked against the dense kernel matrix), the mixed solve still refines to 1e-10 against
its own operator, and the profile shows the tensor-core sketch launches."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def _points(N):
    p = np.random.default_rng(3).random((N, 2))
    return np.ascontiguousarray(p[H.morton_order(p)])


def _build(pts, precision, power_iters=0, rank=48):
    m = H.HODLRMatrix(1e-9, rsvd_rank=rank, max_rank=rank, oversample=10, power_iters=power_iters,
                      sketch=H.SKETCH_DEVICE_NORMAL, seed=0, precision=precision, ir_tol=1e-10, ir_max_iter=30)
    m.build_from_kernel(H.KERNEL_COULOMB, pts, [1e-3, 4.0], 256)
    return m


@pytest.mark.parametrize("power_iters", [0, 1])
def test_mixed_build_matches_fp64_build(power_iters):
    N = 8192
    pts = _points(N)
    H.profile_enable(True)
    mm = _build(pts, H.MIXED, power_iters)
    prof = H.profile_report()
    H.profile_enable(False)
    assert any(k.startswith("tc_tf32x4_gen:build.sketch") for k in prof), sorted(prof)
    assert any(k.startswith("tc_tf32x4_gen:build.project") for k in prof), sorted(prof)
    assert "cholesky_rinv" in prof
    m64 = _build(pts, H.FP64, power_iters)
    A = O.coulomb_matrix(pts, 1e-3, 4.0)
    x = np.random.default_rng(5).standard_normal((N, 3))
    y64, ymx = m64.multiply(x), mm.multiply(x)
    assert O.rel_err(y64, ymx) < 1e-5, O.rel_err(y64, ymx)
    e64, emx = O.rel_err(A @ x, y64), O.rel_err(A @ x, ymx)
    assert emx < 2 * e64 + 1e-5, (e64, emx)   # the rank-48 compression error dominates both
    b = np.random.default_rng(6).standard_normal((N, 4))
    xs, st = mm.solve(b, stats=True)
    assert st.rel_residual <= 1e-10
    assert O.rel_err(mm.multiply(xs), b) <= 1e-10
