"""Adjoint solve and gradients (the differentiation configuration: Gaussian kernel
h = 0.05 + 1e-2 I on sorted uniform points, HODLR leaf 128, ranks <= 64, FP64;
L = ||A^{-1} b - t||^2).  Checked against a dense FP64 gradient, central finite
differences of the whole pipeline (rebuild at h +- eps), and finite differences of the
factors."""
import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu

H0, SHIFT, LEAF, RANK = 0.05, 1e-2, 128, 64


def points(N, seed=5):
    return np.sort(np.random.default_rng(seed).random(N))


def build(N, h=H0, tol=1e-12, pts=None):
    pts = points(N) if pts is None else pts
    m = H.HODLRMatrix(tol, rsvd_rank=RANK, max_rank=RANK, oversample=10, power_iters=1,
                      sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, pts.reshape(-1, 1), [h, SHIFT], LEAF)
    return m


def loss_and_grad(m, b, t):
    x = m.solve(b)
    g = 2.0 * (x - t)
    lam = m.solve_transpose(g)
    dp = m.gradients(x, lam)
    return float(((x - t) ** 2).sum()), x, lam, dp


def test_transpose_solve_is_the_adjoint():
    N = 4096
    m = build(N)
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal((N, 3)), rng.standard_normal((N, 3))
    lhs = np.sum(m.solve(u) * v)
    rhs = np.sum(u * m.solve_transpose(v))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_gradients_against_dense_fp64():
    N = 4096
    pts = points(N)
    m = build(N, pts=pts)
    rng = np.random.default_rng(1)
    b, t = rng.standard_normal(N), rng.standard_normal(N)
    L, x, lam, dp = loss_and_grad(m, b, t)
    A = O.gaussian_matrix(pts, H0, SHIFT)
    xd = np.linalg.solve(A, b)
    lamd = np.linalg.solve(A.T, 2.0 * (xd - t))
    d = pts[:, None] - pts[None, :]
    dA = np.exp(-d * d / (2 * H0 * H0)) * d * d / H0 ** 3
    dh_dense = -lamd @ dA @ xd
    assert O.rel_err(lamd, lam) < 1e-6          # dL/db
    assert abs(dp[0] - dh_dense) <= 1e-6 * abs(dh_dense)   # dL/dh
    assert abs(dp[1] - (-lamd @ xd)) <= 1e-6 * abs(lamd @ xd)  # dL/d(shift)


def _richardson(central, e):
    """Two central differences at e and e/2 combined to cancel the O(e^2) term."""
    return (4.0 * central(e / 2) - central(e)) / 3.0


def test_dh_against_dense_central_differences():
    """Central differences of the exact loss (dense FP64 LAPACK solves of A(h +- eps))
    against the device adjoint: the 1e-6 bar."""
    N = 4096
    pts = points(N)
    rng = np.random.default_rng(2)
    b, t = rng.standard_normal(N), rng.standard_normal(N)
    _, _, _, dp = loss_and_grad(build(N, pts=pts), b, t)

    def central(eps):
        def L(h):
            x = np.linalg.solve(O.gaussian_matrix(pts, h, SHIFT), b)
            return ((x - t) ** 2).sum()
        return (L(H0 + eps) - L(H0 - eps)) / (2 * eps)

    fd = _richardson(central, 2e-4 * H0)
    assert abs(dp[0] - fd) <= 1e-6 * abs(fd), (dp[0], fd)


def test_dh_against_pipeline_central_differences():
    """Central differences through the whole device pipeline (rebuild, factor, solve at
    h +- eps).  Each rebuild re-truncates the compression (relative jumps ~1e-15 of the
    operator, the smallest singular value the SVD keeps), which moves L by about
    cond(A) * 1e-15 * L; with L ~ 8e7, dL/dh ~ 7.6e6 and cond ~1e4 this puts a noise floor
    of ~1e-6 on any step size, so the bound here is 3e-6 (the dense check above holds the
    adjoint itself to 1e-6, and it matches the dense adjoint to ~1e-8)."""
    N = 8192
    pts = points(N)
    rng = np.random.default_rng(2)
    b, t = rng.standard_normal(N), rng.standard_normal(N)
    tol = 1e-15
    _, _, _, dp = loss_and_grad(build(N, pts=pts, tol=tol), b, t)

    def central(eps):
        Lp = loss_and_grad(build(N, H0 + eps, pts=pts, tol=tol), b, t)[0]
        Lm = loss_and_grad(build(N, H0 - eps, pts=pts, tol=tol), b, t)[0]
        return (Lp - Lm) / (2 * eps)

    fd = _richardson(central, 2e-3 * H0)
    assert abs(dp[0] - fd) <= 3e-6 * abs(fd), (dp[0], fd)


def test_db_through_autograd_against_central_differences():
    torch = pytest.importorskip("torch")
    from hodlr_autograd import HodlrSolve

    N = 4096
    m = build(N)
    rng = np.random.default_rng(3)
    b = torch.tensor(rng.standard_normal(N), requires_grad=True)
    t = torch.tensor(rng.standard_normal(N))
    L = ((HodlrSolve.apply(b, m) - t) ** 2).sum()
    L.backward()
    for i in (0, 1234, N - 1):
        e = np.zeros(N)
        e[i] = 1e-3
        bp, bm = b.detach().numpy() + e, b.detach().numpy() - e
        fd = (((m.solve(bp) - t.numpy()) ** 2).sum() - ((m.solve(bm) - t.numpy()) ** 2).sum()) / 2e-3
        assert abs(b.grad[i].item() - fd) <= 1e-6 * max(1.0, abs(fd))


def test_factor_gradients_against_finite_differences():
    """dL/dD, dL/dU, dL/dV, dL/dB12 of the HODLR representation, by perturbing one entry
    of each imported factor."""
    N = 2048
    pts = points(N)
    A = O.gaussian_matrix(pts, H0, SHIFT)
    o = O.HodlrOracle(1e-12, RANK)
    o.build_from_dense(A, LEAF, O.SketchSource(4, "normal"))
    rng = np.random.default_rng(4)
    b, t = rng.standard_normal(N), rng.standard_normal(N)

    def handle():
        m = H.HODLRMatrix(1e-12)
        m.import_factors(N, LEAF, o.nodes)
        return m

    m = handle()
    L, x, lam, _ = loss_and_grad(m, b, t)
    leaf = next(n for n in o.nodes if n.is_leaf)
    inner = o.nodes[0]
    child = o.nodes[1]
    checks = [(leaf, "D", H.HODLRMatrix.D, (3, 5)), (child, "U", H.HODLRMatrix.U, (7, 0)),
              (child, "V", H.HODLRMatrix.V, (11, 1)), (inner, "B12", H.HODLRMatrix.B12, (0, 0))]
    for node, attr, which, (i, j) in checks:
        G = m.get_gradient(node.index, which)
        M0 = getattr(node, attr)
        # Richardson-extrapolated central differences (steps e and 2e): with L ~ 2e7 and
        # cond(A) ~ 1e4, a plain central difference at e = 1e-6 carries ~1e-5 relative
        # rounding noise (measured with LAPACK inverses on the CPU), as large as the bar.
        # Each perturbation changes A by a rank-one term of norm e (unit basis columns).
        eps = 1e-4

        def central(e):
            vals = []
            for sgn in (1, -1):
                Mp = M0.copy()
                Mp[i, j] += sgn * e
                setattr(node, attr, Mp)
                vals.append(loss_and_grad(handle(), b, t)[0])
            return (vals[0] - vals[1]) / (2 * e)

        fd = (4 * central(eps) - central(2 * eps)) / 3
        setattr(node, attr, M0)
        assert abs(G[i, j] - fd) <= 1e-5 * max(abs(fd), 1e-3 * abs(L)), (attr, G[i, j], fd)


def test_rank_profile_freezes_ranks():
    """hm_set_rank_profile: a rebuild at a perturbed length scale keeps the ranks of the
    h0 build exactly; a raised profile is honoured up to the sketch width; a profile for
    another tree is refused."""
    N = 8192
    pts = points(N)
    m = build(N, pts=pts)
    tr = m.tree()
    r12, r21 = tr["rank12"].copy(), tr["rank21"].copy()
    m2 = H.HODLRMatrix(1e-12, rsvd_rank=RANK, max_rank=RANK, oversample=10, power_iters=1,
                       sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
    m2.set_rank_profile(r12, r21)
    m2.build_from_kernel(H.KERNEL_GAUSSIAN, pts.reshape(-1, 1), [H0 * 1.01, SHIFT], LEAF)
    t2 = m2.tree()
    assert np.array_equal(t2["rank12"], r12) and np.array_equal(t2["rank21"], r21)
    inner = tr["is_leaf"] == 0
    up12, up21 = r12.copy(), r21.copy()
    up12[inner] += 3
    up21[inner] += 3
    m2.set_rank_profile(up12, up21)
    m2.build_from_kernel(H.KERNEL_GAUSSIAN, pts.reshape(-1, 1), [H0, SHIFT], LEAF)
    t3 = m2.tree()
    assert np.all(t3["rank12"][inner] == np.minimum(up12[inner], RANK + 10))
    # the raised ranks keep (tiny) extra singular triplets: same operator to ~1e-12
    x = np.random.default_rng(3).standard_normal(N)
    assert O.rel_err(m.multiply(x), m2.multiply(x)) < 1e-10
    m2.set_rank_profile(r12[:-1], r21[:-1])
    with pytest.raises(H.HmError) as e:
        m2.build_from_kernel(H.KERNEL_GAUSSIAN, pts.reshape(-1, 1), [H0, SHIFT], LEAF)
    assert e.value.code == H.HM_ERR_ARG
