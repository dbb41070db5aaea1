"""Why the HSS solve recompresses its coupling blocks (host-only numpy restatement).

The reference's HSS has identity transfers (hss_routines.h:86-90): a node's basis is the
block diagonal of its leaves' bases, so the coupling blocks B12 = U_L^T A12 V_R are as
wide as the sums of the leaves' ranks while their numerical rank is much smaller.  A
Woodbury solve over that wide form (the reference's, with an LU of the capacitance
matrix, hss_routines.h:205-279) leaves a residual far above rounding; recompressing each
coupling block to its numerical rank first (B = F H^T, what the device path does in
Engine::reduce_hss_coupling) gives the same operator and a residual at rounding level.
Gaussian h = 0.05 + 1e-2 I on sorted uniform points, leaf 64, tolerance 1e-10."""
import numpy as np
import scipy.linalg as sl

N, LEAF, TOL = 1024, 64, 1e-10


def _operator():
    x = np.sort(np.random.default_rng(2).random(N))
    A = np.exp(-(x[:, None] - x[None, :]) ** 2 / (2 * 0.05 ** 2))
    A[np.diag_indices(N)] += 1e-2
    return A


def _leaf_bases(A):
    def basis(S):
        u, s, _ = np.linalg.svd(S, full_matrices=False)
        return u[:, : max(1, int((s > TOL * s[0]).sum()))]
    U, V = {}, {}
    for a in range(0, N, LEAF):
        S = A[a:a + LEAF].copy()
        S[:, a:a + LEAF] = 0
        U[a] = basis(S)
        S = A[:, a:a + LEAF].T.copy()
        S[:, a:a + LEAF] = 0
        V[a] = basis(S)
    return U, V


class _Node:
    """Woodbury factor/solve of [[A1, U1 B12 V2^T], [U2 B21 V1^T, A2]] with LU of the
    capacitance matrix I + K B^ (K = blockdiag(V1^T A1^-1 U1, V2^T A2^-1 U2))."""

    def __init__(self, A, a, b, U, V, recompress):
        self.a, self.b = a, b
        if b - a <= LEAF:
            self.lu = sl.lu_factor(A[a:b, a:b])
            return
        m = (a + b) // 2
        self.L, self.R = _Node(A, a, m, U, V, recompress), _Node(A, m, b, U, V, recompress)
        bd = lambda d, lo, hi: sl.block_diag(*[d[s] for s in range(lo, hi, LEAF)])
        U1, U2, V1, V2 = bd(U, a, m), bd(U, m, b), bd(V, a, m), bd(V, m, b)
        B12, B21 = U1.T @ A[a:m, m:b] @ V2, U2.T @ A[m:b, a:m] @ V1
        self.width = B12.shape[0]
        if recompress:
            def red(Ux, B, Vy):
                f, s, gt = np.linalg.svd(B)
                r = int((s > 1e-15 * s[0]).sum())
                return Ux @ f[:, :r], np.diag(s[:r]), Vy @ gt[:r].T
            U1, B12, V2 = red(U1, B12, V2)
            U2, B21, V1 = red(U2, B21, V1)
        self.U1, self.U2, self.V1, self.V2, self.B12, self.B21 = U1, U2, V1, V2, B12, B21
        self.Q1, self.Q2 = self.L.solve(U1), self.R.solve(U2)
        X, Y = (V1.T @ self.Q1) @ B12, (V2.T @ self.Q2) @ B21
        self.M = sl.lu_factor(np.block([[np.eye(X.shape[0]), X], [Y, np.eye(Y.shape[0])]]))

    def solve(self, B):
        if self.b - self.a <= LEAF:
            return sl.lu_solve(self.lu, B)
        m = (self.a + self.b) // 2 - self.a
        z = np.vstack([self.L.solve(B[:m]), self.R.solve(B[m:])])
        w = sl.lu_solve(self.M, np.vstack([self.V1.T @ z[:m], self.V2.T @ z[m:]]))
        q1 = self.V1.shape[1]
        return z - np.vstack([self.Q1 @ (self.B12 @ w[q1:]), self.Q2 @ (self.B21 @ w[:q1])])

    def multiply(self, X):
        if self.b - self.a <= LEAF:
            return self.Adiag @ X
        m = (self.a + self.b) // 2 - self.a
        y = np.vstack([self.L.multiply(X[:m]), self.R.multiply(X[m:])])
        y[:m] += self.U1 @ (self.B12 @ (self.V2.T @ X[m:]))
        y[m:] += self.U2 @ (self.B21 @ (self.V1.T @ X[:m]))
        return y


def _build(A, U, V, recompress):
    root = _Node(A, 0, N, U, V, recompress)

    def attach(n):
        if n.b - n.a <= LEAF:
            n.Adiag = A[n.a:n.b, n.a:n.b]
        else:
            attach(n.L)
            attach(n.R)
    attach(root)
    return root


def test_recompressed_coupling_solves_the_same_operator_to_rounding():
    A = _operator()
    U, V = _leaf_bases(A)
    wide = _build(A, U, V, recompress=False)
    slim = _build(A, U, V, recompress=True)
    b = np.random.default_rng(5).standard_normal((N, 2))
    x = np.random.default_rng(6).standard_normal((N, 2))
    # the two forms are the same operator
    assert np.linalg.norm(wide.multiply(x) - slim.multiply(x)) <= 1e-13 * np.linalg.norm(wide.multiply(x))
    r_wide = np.linalg.norm(wide.multiply(wide.solve(b)) - b) / np.linalg.norm(b)
    r_slim = np.linalg.norm(slim.multiply(slim.solve(b)) - b) / np.linalg.norm(b)
    assert wide.width > 4 * slim.B12.shape[0]      # the top coupling is mostly redundant width
    assert r_slim < 1e-11
    assert r_wide > 10 * r_slim                    # the wide Woodbury form loses digits
