"""Plan replays through CUDA graphs: a plan's first run launches its steps one by one,
the second captures them into a graph and later runs replay it.  Every replay must give
what the first (eager) run gave, for the factorization, the FP64 and the mixed solve,
the multiply and the transpose solve."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def build(precision, N=8192):
    """FP64: the Gaussian operator of the differentiation workload (cond ~1e5).  Mixed:
    the 2-D Coulomb operator of the mixed-precision workload (FP32 factors of the Gaussian
    one do not contract under refinement at this conditioning)."""
    m = H.HODLRMatrix(1e-12, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
    rng = np.random.default_rng(3)
    if precision == 0:
        m.build_from_kernel(H.KERNEL_GAUSSIAN, np.sort(rng.random(N)).reshape(-1, 1), [0.05, 1e-2], 128)
    else:
        p = rng.random((N, 2))
        m.build_from_kernel(H.KERNEL_COULOMB, p[H.morton_order(p)], [1e-3, 4.0], 128)
    return m


@pytest.mark.parametrize("precision", [0, 1])
def test_replays_match_the_eager_run(precision):
    m = build(precision)
    m.set_precision(precision)
    b = np.random.default_rng(4).standard_normal((m.N, 5))
    m.factor()
    first = m.solve(b)
    runs = [m.solve(b) for _ in range(3)]
    for _ in range(2):
        m.factor()
    runs.append(m.solve(b))
    # run-to-run differences are rounding (split-K accumulation order) amplified by
    # cond(A) ~ 1e5; the mixed runs each stop at their own refinement residual <= 1e-10
    tol = 1e-10 if precision == 0 else 1e-5
    for x in runs:
        assert O.rel_err(first, x) < tol
        assert np.linalg.norm(m.multiply(x) - b) / np.linalg.norm(b) < 5e-9
    # A x ~ b with |A| |x| ~ 1e5 |b|: rounding of the products shows at ~1e-11 relative
    y0 = m.multiply(first)
    for _ in range(3):
        assert O.rel_err(y0, m.multiply(first)) < 1e-11
    l0 = m.solve_transpose(b)
    for _ in range(3):
        assert O.rel_err(l0, m.solve_transpose(b)) < 1e-10
