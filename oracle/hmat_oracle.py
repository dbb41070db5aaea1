"""TEST INFRASTRUCTURE ONLY — the oracle.

A CPU restatement (numpy + scipy LAPACK, FP64) of the reference's hot path
(chenxinye/hmat-omp, include/*.h).  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg import this module, and only to check or time; the
product library never calls it.

Pinned against the reference itself: ``oracle/_ref/libhmatref.so`` is the reference's
own serial/OpenMP code compiled by ``oracle/Makefile`` (see ``oracle/ref.py``); the
fixtures in ``tests/golden`` were produced from it by ``tests/golden/make_golden.py``
and ``tests/test_oracle.py`` checks this restatement against them.

Contents (each function cites the reference lines it restates):
  * ``RefStream``   — the sketch stream of ``Matrix::Random`` (matrix.h:50-57) under a
                      fixed seed: std::mt19937 + libstdc++ ``generate_canonical``.
  * ``compress_svd`` / ``compress_rsvd`` — compression.h:18-99.
  * ``HodlrOracle`` — hodlr_routines.h: build (post-order), multiply, recursive
                      Woodbury solve; plus the level-synchronous factor / solve /
                      adjoint that the GPU path implements.
  * ``HssOracle``   — hss_routines.h: build_topo, leaf compression, identity
                      transfers, up/down-sweep multiply, stable Woodbury solve.
  * ``HssNestedOracle`` — the nested-basis HSS extension (compressed transfers; no
                      reference counterpart): the specification its device build and
                      telescoping multiply are checked against.
  * kernel generators for the benchmark configurations.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

# ----------------------------------------------------------------------------------
# Random sketches exactly as the reference draws them
# ----------------------------------------------------------------------------------

_TWO32 = 4294967296.0
_TWO64 = 18446744073709551616.0
_ONE_MINUS = np.nextafter(1.0, 0.0)


class RefStream:
    """The draw sequence of ``Matrix::Random`` (include/matrix.h:50-57) for one
    thread whose generator was seeded with ``seed``.

    ``std::mt19937(seed)`` is numpy's MT19937 after ``init_genrand(seed)`` (the
    legacy ``RandomState(seed)`` seeding).  ``uniform_real_distribution<double>(0,1)``
    in libstdc++ is ``generate_canonical<double,53>``: two 32-bit words g0, g1,
    ``(g0 + g1 * 2^32) / 2^64`` evaluated in double, clamped below 1.
    ``normal(...)`` restates libstdc++'s ``normal_distribution`` (Marsaglia polar
    method, the second value of each pair cached) with a fresh distribution object
    per ``Matrix::Random`` call (matrix.h:53), i.e. the cache is dropped per block.
    """

    def __init__(self, seed: int):
        rs = np.random.RandomState(seed & 0xFFFFFFFF)
        key, pos = rs.get_state()[1], rs.get_state()[2]
        self._bg = np.random.MT19937()
        self._bg.state = {"bit_generator": "MT19937", "state": {"key": key, "pos": pos}}

    def _words(self, n: int) -> np.ndarray:
        return self._bg.random_raw(n).astype(np.uint64)

    def canonical(self, n: int) -> np.ndarray:
        w = self._words(2 * n).reshape(n, 2).astype(np.float64)
        v = (w[:, 0] + w[:, 1] * _TWO32) / _TWO64
        return np.where(v >= 1.0, _ONE_MINUS, v)

    def uniform(self, rows: int, cols: int) -> np.ndarray:
        """Matrix::Random(rows, cols): column-major fill."""
        return self.canonical(rows * cols).reshape(cols, rows).T.copy()

    def normal(self, rows: int, cols: int) -> np.ndarray:
        """Matrix::Random(rows, cols) built with normal_distribution (the
        Gaussian-sketch variant of the oracle library)."""
        n = rows * cols
        out = np.empty(n)
        i = 0
        saved = None
        while i < n:
            if saved is not None:
                out[i] = saved
                saved = None
                i += 1
                continue
            while True:
                x, y = 2.0 * self.canonical(2) - 1.0
                r2 = x * x + y * y
                if r2 <= 1.0 and r2 != 0.0:
                    break
            mult = math.sqrt(-2.0 * math.log(r2) / r2)
            saved = x * mult
            out[i] = y * mult
            i += 1
        return out.reshape(cols, rows).T.copy()


class SketchSource:
    """Hands out Ω matrices in draw order; ``kind`` is 'uniform' (reference) or
    'normal' (Gaussian variant)."""

    def __init__(self, seed: int, kind: str = "uniform"):
        self.stream = RefStream(seed)
        self.kind = kind
        self.log: list[tuple[int, int]] = []

    def __call__(self, rows: int, cols: int) -> np.ndarray:
        self.log.append((rows, cols))
        if self.kind == "uniform":
            return self.stream.uniform(rows, cols)
        return self.stream.normal(rows, cols)


# ----------------------------------------------------------------------------------
# Compression (include/compression.h)
# ----------------------------------------------------------------------------------


@dataclass
class LowRank:
    U: np.ndarray
    V: np.ndarray
    S: np.ndarray  # the diagonal of B (compression.h:57-63)

    @property
    def rank(self) -> int:
        return self.S.shape[0]


def truncation_rank(S: np.ndarray, tol: float, max_rank: int = 0) -> int:
    """compression.h:42-46: #{S_i > tol*S_0} when S_0 > 1e-15, at least 1.
    ``max_rank`` > 0 is an extension (not in the reference): a cap."""
    rank = 0
    if S.shape[0] > 0 and S[0] > 1e-15:
        rank = int(np.count_nonzero(S > tol * S[0]))
    if rank == 0:
        rank = 1
    if max_rank > 0:
        rank = min(rank, max_rank)
    return rank


def compress_svd(A: np.ndarray, tol: float, max_rank: int = 0) -> LowRank:
    """compression.h:18-64: thin dgesvd('S','S'), truncate, B = diag(S)."""
    m, n = A.shape
    if m == 0 or n == 0:
        return LowRank(np.zeros((0, 0)), np.zeros((0, 0)), np.zeros(0))
    U, S, Vt = sla.svd(A, full_matrices=False, lapack_driver="gesvd")
    r = truncation_rank(S, tol, max_rank)
    return LowRank(U[:, :r].copy(), Vt[:r, :].T.copy(), S[:r].copy())


def compress_rsvd(A: np.ndarray, tol: float, rank_guess: int, sketch, oversample: int = 10,
                  min_dim: int = 256, power_iters: int = 0, max_rank: int = 0) -> LowRank:
    """compression.h:67-99.  ``sketch(n, k)`` returns Ω in the reference's draw order.
    ``power_iters`` and ``max_rank`` are extensions (0 = the reference)."""
    m, n = A.shape
    if m < min_dim or n < min_dim:  # compression.h:72
        return compress_svd(A, tol, max_rank)
    k = min(rank_guess + oversample, min(m, n))  # compression.h:74-75
    Omega = sketch(n, k)  # compression.h:78
    Y = A @ Omega  # compression.h:79
    Q = compress_svd(Y, -1.0).U  # compression.h:83-84
    for _ in range(power_iters):
        Z = np.linalg.qr(A.T @ Q)[0]
        Q = np.linalg.qr(A @ Z)[0]
    Bs = Q.T @ A  # compression.h:87
    lr = compress_svd(Bs, tol, max_rank)  # compression.h:90
    return LowRank(Q @ lr.U, lr.V, lr.S)  # compression.h:94-98


# ----------------------------------------------------------------------------------
# HODLR (include/hodlr_routines.h)
# ----------------------------------------------------------------------------------


@dataclass
class HNode:
    start: int
    end: int
    depth: int
    is_leaf: bool = False
    left: "HNode | None" = None
    right: "HNode | None" = None
    index: int = -1  # pre-order position
    D: np.ndarray | None = None
    U: np.ndarray | None = None
    V: np.ndarray | None = None
    B12: np.ndarray | None = None  # diag(S) of A12's compression
    B21: np.ndarray | None = None

    @property
    def mid(self) -> int:
        return (self.start + self.end) // 2


def hodlr_tree(N: int, leaf: int) -> list[HNode]:
    """Pre-order node list of the reference's split (hodlr_routines.h:27-45):
    leaf iff len <= leaf, mid = (start+end)/2."""
    nodes: list[HNode] = []

    def rec(s, e, d):
        n = HNode(s, e, d)
        n.index = len(nodes)
        nodes.append(n)
        if e - s <= leaf:
            n.is_leaf = True
        else:
            m = (s + e) // 2
            n.left = rec(s, m, d + 1)
            n.right = rec(m, e, d + 1)
        return n

    rec(0, N, 0)
    return nodes


class HodlrOracle:
    """Restatement of HODLRMatrix (hodlr_routines.h:8-176)."""

    def __init__(self, tol: float = 1e-6, rsvd_rank: int = 64, oversample: int = 10,
                 min_dim: int = 256, power_iters: int = 0, max_rank: int = 0):
        self.tol = tol
        self.rsvd_rank = rsvd_rank
        self.oversample = oversample
        self.min_dim = min_dim
        self.power_iters = power_iters
        self.max_rank = max_rank
        self.nodes: list[HNode] = []
        self.N = 0

    @property
    def root(self) -> HNode:
        return self.nodes[0]

    # -- build (hodlr_routines.h:20-63) --
    def build_from_dense(self, A: np.ndarray, leaf: int, sketch) -> None:
        self.N = A.shape[0]
        self.nodes = hodlr_tree(self.N, leaf)

        def comp(blk):
            return compress_rsvd(blk, self.tol, self.rsvd_rank, sketch, self.oversample,
                                 self.min_dim, self.power_iters, self.max_rank)

        def rec(n: HNode):  # post-order: left, right, then A12, A21 (hodlr_routines.h:43-53)
            if n.is_leaf:
                n.D = A[n.start:n.end, n.start:n.end].copy()
                return
            rec(n.left)
            rec(n.right)
            m = n.mid
            lr12 = comp(A[n.start:m, m:n.end])
            lr21 = comp(A[m:n.end, n.start:m])
            n.left.U, n.right.V, n.B12 = lr12.U, lr12.V, np.diag(lr12.S)
            n.right.U, n.left.V, n.B21 = lr21.U, lr21.V, np.diag(lr21.S)

        rec(self.root)

    def set_factors_from(self, other) -> None:
        """Copy a tree's factors (e.g. downloaded from the reference library)."""
        self.nodes = other.nodes
        self.N = other.N

    # -- multiply (hodlr_routines.h:66-105), any number of columns --
    def multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        vec = x.ndim == 1
        X = x.reshape(self.N, -1)

        def rec(n: HNode, xs: np.ndarray) -> np.ndarray:
            if n.is_leaf:
                return n.D @ xs
            ll = n.mid - n.start
            xl, xr = xs[:ll], xs[ll:]
            yl = rec(n.left, xl)
            yr = rec(n.right, xr)
            yl = yl + n.left.U @ (n.B12 @ (n.right.V.T @ xr))
            yr = yr + n.right.U @ (n.B21 @ (n.left.V.T @ xl))
            return np.vstack([yl, yr])

        Y = rec(self.root, X)
        return Y.ravel() if vec else Y

    # -- recursive Woodbury solve (hodlr_routines.h:108-175); O(N^2), small N --
    def solve_recursive(self, b: np.ndarray) -> np.ndarray:
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        Bm = b.reshape(self.N, -1)

        def rec(n: HNode, bl: np.ndarray) -> np.ndarray:
            if n.is_leaf:
                return sla.lu_solve(sla.lu_factor(n.D), bl)
            ll = n.mid - n.start
            z1 = rec(n.left, bl[:ll])
            z2 = rec(n.right, bl[ll:])
            vz1 = n.right.V.T @ z2
            vz2 = n.left.V.T @ z1
            Q1 = rec(n.left, n.left.U)
            Q2 = rec(n.right, n.right.U)
            r1, r2 = n.B12.shape[0], n.B21.shape[0]
            C = np.zeros((r1 + r2, r1 + r2))
            C[:r1, :r1] = np.linalg.inv(n.B12)
            C[r1:, r1:] = np.linalg.inv(n.B21)
            C[:r1, r1:] = n.right.V.T @ Q2
            C[r1:, :r1] = n.left.V.T @ Q1
            g = sla.lu_solve(sla.lu_factor(C), np.vstack([vz1, vz2]))
            return np.vstack([z1 - Q1 @ g[:r1], z2 - Q2 @ g[r1:]])

        X = rec(self.root, Bm)
        return X.ravel() if vec else X

    # -- level-synchronous factorization: the algorithm of the GPU path --
    def factor(self) -> "HodlrFactors":
        return level_factor(self.nodes, *_hodlr_generic(self.nodes))


def _hodlr_generic(nodes: list[HNode]):
    """Per internal node: (U1, V1, U2, V2, B12, B21) with A12 = U1 B12 V2^T and
    A21 = U2 B21 V1^T (hodlr_routines.h:55-61)."""
    gen = {}
    for n in nodes:
        if n.is_leaf:
            continue
        gen[n.index] = (n.left.U, n.left.V, n.right.U, n.right.V, n.B12, n.B21)
    leaves = {n.index: n.D for n in nodes if n.is_leaf}
    return leaves, gen


@dataclass
class HodlrFactors:
    """Output of ``level_factor``.  Q1/Q2 = A_child^{-1} U_child, P = B^ M^{-1}
    with M = I + K B^ (the stable capacitance form of hss_routines.h:253-254)."""
    nodes: list
    Dinv: dict = field(default_factory=dict)
    Q: dict = field(default_factory=dict)  # node -> (Q1, Q2)
    V: dict = field(default_factory=dict)  # node -> (V1, V2)
    P: dict = field(default_factory=dict)
    M: dict = field(default_factory=dict)
    B: dict = field(default_factory=dict)  # node -> B^ = [[0, B12], [B21, 0]]

    def _levels(self):
        inner = [n for n in self.nodes if not n.is_leaf]
        depth = max((n.depth for n in inner), default=-1)
        return inner, depth

    def solve(self, b: np.ndarray) -> np.ndarray:
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        z = b.reshape(b.shape[0], -1).copy()
        for n in self.nodes:
            if n.is_leaf:
                z[n.start:n.end] = self.Dinv[n.index] @ z[n.start:n.end]
        inner, depth = self._levels()
        for d in range(depth, -1, -1):
            for n in inner:
                if n.depth != d:
                    continue
                _apply_woodbury(self, n, z)
        return z.ravel() if vec else z

    def solve_transpose(self, g: np.ndarray) -> np.ndarray:
        """A^T lam = g with the same factors: the transposed sweeps in reverse order."""
        g = np.asarray(g, dtype=np.float64)
        vec = g.ndim == 1
        lam = g.reshape(g.shape[0], -1).copy()
        inner, depth = self._levels()
        for d in range(0, depth + 1):
            for n in inner:
                if n.depth != d:
                    continue
                Q1, Q2 = self.Q[n.index]
                V1, V2 = self.V[n.index]
                m = n.mid
                p1 = Q1.shape[1]
                q1 = V1.shape[1]
                t = np.vstack([Q1.T @ lam[n.start:m], Q2.T @ lam[m:n.end]])
                gam = self.P[n.index].T @ t
                lam[n.start:m] -= V1 @ gam[:q1]
                lam[m:n.end] -= V2 @ gam[q1:]
        for n in self.nodes:
            if n.is_leaf:
                lam[n.start:n.end] = self.Dinv[n.index].T @ lam[n.start:n.end]
        return lam.ravel() if vec else lam


def _apply_woodbury(F: HodlrFactors, n, W: np.ndarray) -> None:
    """W[rows of n] <- A_n^{-1} applied, given blockdiag(A_c1, A_c2)^{-1} W already:
    t = V~^T W, delta = P t, W_i -= Q_i delta_i."""
    Q1, Q2 = F.Q[n.index]
    V1, V2 = F.V[n.index]
    m = n.mid
    p1 = Q1.shape[1]
    t = np.vstack([V1.T @ W[n.start:m], V2.T @ W[m:n.end]])
    delta = F.P[n.index] @ t
    W[n.start:m] -= Q1 @ delta[:p1]
    W[m:n.end] -= Q2 @ delta[p1:]


def level_factor(nodes, leaves: dict, gen: dict) -> HodlrFactors:
    """Bottom-up factorization (Ambikasaran & Darve 2013) in the form the GPU runs:
    leaf inverses applied to every ancestor basis block, then one Woodbury update per
    level.  Equivalent to the reference's recursive solve (hodlr_routines.h:112-175),
    which recomputes the same quantities on every call."""
    F = HodlrFactors(nodes)
    N = nodes[0].end
    # child basis blocks, keyed by child node index: Qcur[c] (len_c x p)
    parent = {}
    for n in nodes:
        if not n.is_leaf:
            parent[n.left.index] = n
            parent[n.right.index] = n
    Qcur = {}
    for ni, (U1, V1, U2, V2, B12, B21) in gen.items():
        n = nodes[ni]
        Qcur[n.left.index] = U1.copy()
        Qcur[n.right.index] = U2.copy()

    def ancestors_children(n):
        """(child-on-path c, offset of n inside c) for every ancestor level."""
        out = []
        c = n
        while c.index in parent:
            out.append(c)
            c = parent[c.index]
        return out

    for n in nodes:
        if n.is_leaf:
            Dinv = np.linalg.inv(leaves[n.index])
            F.Dinv[n.index] = Dinv
            for c in ancestors_children(n):
                o = n.start - c.start
                Qcur[c.index][o:o + (n.end - n.start)] = Dinv @ Qcur[c.index][o:o + (n.end - n.start)]
    inner = [n for n in nodes if not n.is_leaf]
    depth = max((n.depth for n in inner), default=-1)
    for d in range(depth, -1, -1):
        for n in inner:
            if n.depth != d:
                continue
            U1, V1, U2, V2, B12, B21 = gen[n.index]
            Q1, Q2 = Qcur[n.left.index], Qcur[n.right.index]
            p1, p2 = U1.shape[1], U2.shape[1]
            q1, q2 = V1.shape[1], V2.shape[1]
            Bh = np.zeros((p1 + p2, q1 + q2))
            Bh[:p1, q1:] = B12
            Bh[p1:, :q1] = B21
            K = np.zeros((q1 + q2, p1 + p2))
            K[:q1, :p1] = V1.T @ Q1
            K[q1:, p1:] = V2.T @ Q2
            M = np.eye(q1 + q2) + K @ Bh
            F.Q[n.index] = (Q1, Q2)
            F.V[n.index] = (V1, V2)
            F.B[n.index] = Bh
            F.M[n.index] = M
            F.P[n.index] = Bh @ np.linalg.inv(M)
            # update every ancestor basis block restricted to n's rows
            for c in ancestors_children(n):
                o = n.start - c.start
                W = Qcur[c.index][o:o + (n.end - n.start)]
                Wv = W.copy()
                sub = _Shift(n, Wv)
                _apply_woodbury(F, sub, Wv)
                Qcur[c.index][o:o + (n.end - n.start)] = Wv
    return F


class _Shift:
    """A node view whose row range starts at 0 (for updating a row slice)."""

    def __init__(self, n, W):
        self.index = n.index
        self.start = 0
        self.end = n.end - n.start
        self.mid = n.mid - n.start


# ----------------------------------------------------------------------------------
# HSS (include/hss_routines.h) — identity transfer matrices
# ----------------------------------------------------------------------------------


@dataclass
class SNode:
    id: int
    start: int
    end: int
    depth: int
    is_leaf: bool = False
    left: "SNode | None" = None
    right: "SNode | None" = None
    parent: "SNode | None" = None
    rank_U: int = 0
    rank_V: int = 0
    D: np.ndarray | None = None
    U: np.ndarray | None = None
    V: np.ndarray | None = None
    B: np.ndarray | None = None

    @property
    def mid(self) -> int:
        return (self.start + self.end) // 2

    @property
    def index(self) -> int:
        return self.id


def hss_tree(N: int, leaf: int) -> list[SNode]:
    """build_topo (hss_routines.h:293-306): children get ids when the parent is
    visited, then the recursion descends left, then right."""
    nodes = [SNode(0, 0, N, 0)]

    def rec(n: SNode):
        if n.end - n.start <= leaf:
            n.is_leaf = True
            return
        m = (n.start + n.end) // 2
        n.left = SNode(len(nodes), n.start, m, n.depth + 1, parent=n)
        nodes.append(n.left)
        n.right = SNode(len(nodes), m, n.end, n.depth + 1, parent=n)
        nodes.append(n.right)
        rec(n.left)
        rec(n.right)

    rec(nodes[0])
    return nodes


class HssOracle:
    """Restatement of HSSMatrix (hss_routines.h:10-307)."""

    def __init__(self, tol: float = 1e-9, rsvd_rank: int = 64, oversample: int = 10,
                 min_dim: int = 256, max_rank: int = 0):
        self.tol = tol
        self.rsvd_rank = rsvd_rank
        self.oversample = oversample
        self.min_dim = min_dim
        self.max_rank = max_rank
        self.nodes: list[SNode] = []
        self.N = 0

    @property
    def root(self) -> SNode:
        return self.nodes[0]

    def reconstruct_U(self, n: SNode) -> np.ndarray:
        """hss_routines.h:23-33 with R = I: block diagonal of the leaf bases."""
        if n.is_leaf:
            return n.U
        return sla.block_diag(self.reconstruct_U(n.left), self.reconstruct_U(n.right))

    def reconstruct_V(self, n: SNode) -> np.ndarray:
        if n.is_leaf:
            return n.V
        return sla.block_diag(self.reconstruct_V(n.left), self.reconstruct_V(n.right))

    def build_from_dense(self, A: np.ndarray, leaf: int, sketch) -> None:
        """hss_routines.h:50-113: leaves in reverse id order compress the row strip
        then the transposed column strip (diagonal block zeroed); internal nodes sum
        ranks, take R = W = I and B12 = UL^T A12 VR, B21 = UR^T A21 VL."""
        self.N = N = A.shape[0]
        self.nodes = hss_tree(N, leaf)

        def comp(blk):
            return compress_rsvd(blk, self.tol, self.rsvd_rank, sketch, self.oversample,
                                 self.min_dim, 0, self.max_rank)

        for n in reversed(self.nodes):
            s, e = n.start, n.end
            if n.is_leaf:
                n.D = A[s:e, s:e].copy()
                row = A[s:e, :].copy()
                row[:, s:e] = 0.0
                n.U = comp(row).U
                n.rank_U = n.U.shape[1]
                col = A[:, s:e].T.copy()
                col[:, s:e] = 0.0
                n.V = comp(col).U
                n.rank_V = n.V.shape[1]
            else:
                lc, rc = n.left, n.right
                n.rank_U = lc.rank_U + rc.rank_U
                n.rank_V = lc.rank_V + rc.rank_V
                if n.rank_U > 0 and n.rank_V > 0:
                    m = lc.end
                    B12 = self.reconstruct_U(lc).T @ A[s:m, m:e] @ self.reconstruct_V(rc)
                    B21 = self.reconstruct_U(rc).T @ A[m:e, s:m] @ self.reconstruct_V(lc)
                    n.B = np.zeros((n.rank_U, n.rank_V))
                    n.B[:lc.rank_U, lc.rank_V:] = B12
                    n.B[lc.rank_U:, :lc.rank_V] = B21
                else:
                    n.B = np.zeros((0, 0))

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """Up-sweep g = V^T x, down-sweep f_child = f + B g, y = D x + U f
        (hss_routines.h:118-192), any number of columns."""
        x = np.asarray(x, dtype=np.float64)
        vec = x.ndim == 1
        X = x.reshape(self.N, -1)
        s_ = X.shape[1]
        g = {}
        for n in reversed(self.nodes):
            if n.is_leaf:
                g[n.id] = n.V.T @ X[n.start:n.end]
            else:
                g[n.id] = np.vstack([g[n.left.id], g[n.right.id]])
        f = {0: np.zeros((self.root.rank_U, s_))}
        for n in self.nodes:
            if n.is_leaf:
                continue
            if n.rank_U == 0 or n.rank_V == 0:
                ft = np.zeros((n.rank_U, s_))
            else:
                ft = f[n.id] + n.B @ g[n.id]
            f[n.left.id] = ft[:n.left.rank_U]
            f[n.right.id] = ft[n.left.rank_U:]
        Y = np.zeros_like(X)
        for n in self.nodes:
            if n.is_leaf:
                Y[n.start:n.end] = n.D @ X[n.start:n.end] + n.U @ f[n.id]
        return Y.ravel() if vec else Y

    def generic(self):
        """The HSS operator in the generic two-block form of ``level_factor``."""
        leaves = {n.id: n.D for n in self.nodes if n.is_leaf}
        gen = {}
        for n in self.nodes:
            if n.is_leaf:
                continue
            lc, rc = n.left, n.right
            U1, V1 = self.reconstruct_U(lc), self.reconstruct_V(lc)
            U2, V2 = self.reconstruct_U(rc), self.reconstruct_V(rc)
            if n.B.size:
                B12 = n.B[:lc.rank_U, lc.rank_V:]
                B21 = n.B[lc.rank_U:, :lc.rank_V]
            else:
                B12 = np.zeros((lc.rank_U, rc.rank_V))
                B21 = np.zeros((rc.rank_U, lc.rank_V))
            gen[n.id] = (U1, V1, U2, V2, B12, B21)
        return leaves, gen

    def factor(self) -> HodlrFactors:
        return level_factor(self.nodes, *self.generic())


class HssNestedOracle(HssOracle):
    """Nested-basis HSS: an extension with no reference counterpart (the reference's
    transfers are identities, hss_routines.h:86-90), stated here as the specification the
    device build is checked against.

    Leaves: the reference form's strip bases (``HssOracle.build_from_dense``).  Internal
    node t (children a, b), bottom-up: R_t = the leading left singular vectors of the
    projected strip [U_a^T A[I_a, I_t^c]; U_b^T A[I_b, I_t^c]] kept by
    ``truncation_rank`` (W_t from the column strip likewise), U_t = diag(U_a, U_b) R_t
    (expanded, ``EU``), and B12 = U_a^T A[I_a, I_b] V_b, B21 = U_b^T A[I_b, I_a] V_a at the
    nested ranks.  The root has no strip: rank 0, no transfer."""

    def build_from_dense(self, A: np.ndarray, leaf: int, sketch) -> None:
        self.N = N = A.shape[0]
        self.nodes = hss_tree(N, leaf)

        def comp(blk):
            return compress_rsvd(blk, self.tol, self.rsvd_rank, sketch, self.oversample,
                                 self.min_dim, 0, self.max_rank)

        for n in reversed(self.nodes):   # children have larger ids than their parent
            s, e = n.start, n.end
            if n.is_leaf:
                n.D = A[s:e, s:e].copy()
                row = A[s:e, :].copy()
                row[:, s:e] = 0.0
                n.U = n.EU = comp(row).U
                col = A[:, s:e].T.copy()
                col[:, s:e] = 0.0
                n.V = n.EV = comp(col).U
                n.rank_U, n.rank_V = n.U.shape[1], n.V.shape[1]
                continue
            lc, rc = n.left, n.right
            m = lc.end
            n.B12 = lc.EU.T @ A[s:m, m:e] @ rc.EV
            n.B21 = rc.EU.T @ A[m:e, s:m] @ lc.EV
            if n.parent is None:
                n.rank_U = n.rank_V = 0
                n.R = n.W = None
                continue
            out = np.r_[0:s, e:N]
            SU = np.vstack([lc.EU.T @ A[s:m][:, out], rc.EU.T @ A[m:e][:, out]])
            SV = np.vstack([lc.EV.T @ A[out][:, s:m].T, rc.EV.T @ A[out][:, m:e].T])
            Ru, su, _ = sla.svd(SU, full_matrices=False, lapack_driver="gesvd")
            Rv, sv, _ = sla.svd(SV, full_matrices=False, lapack_driver="gesvd")
            n.R = Ru[:, :truncation_rank(su, self.tol, self.max_rank)].copy()
            n.W = Rv[:, :truncation_rank(sv, self.tol, self.max_rank)].copy()
            n.rank_U, n.rank_V = n.R.shape[1], n.W.shape[1]
            n.EU = sla.block_diag(lc.EU, rc.EU) @ n.R
            n.EV = sla.block_diag(lc.EV, rc.EV) @ n.W

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """Telescoping product: up-sweep g_leaf = V^T x, g_t = W_t^T [g_a; g_b];
        down-sweep [f_a; f_b] = R_t f_t + [B12 g_b; B21 g_a]; y = D x + U f."""
        x = np.asarray(x, dtype=np.float64)
        vec = x.ndim == 1
        X = x.reshape(self.N, -1)
        s_ = X.shape[1]
        g = {}
        for n in reversed(self.nodes):
            if n.is_leaf:
                g[n.id] = n.V.T @ X[n.start:n.end]
            elif n.parent is not None:
                g[n.id] = n.W.T @ np.vstack([g[n.left.id], g[n.right.id]])
        f = {}
        for n in self.nodes:
            if n.is_leaf:
                continue
            lc, rc = n.left, n.right
            fa = n.B12 @ g[rc.id]
            fb = n.B21 @ g[lc.id]
            if n.parent is not None:
                t = n.R @ f[n.id]
                fa = fa + t[:lc.rank_U]
                fb = fb + t[lc.rank_U:]
            f[lc.id], f[rc.id] = fa, fb
        Y = np.zeros_like(X)
        for n in self.nodes:
            if n.is_leaf:
                Y[n.start:n.end] = n.D @ X[n.start:n.end] + (n.U @ f[n.id] if n.id in f else 0.0)
        return Y.ravel() if vec else Y

    def generic(self):
        """The operator in the two-block form of ``level_factor`` (expanded bases)."""
        leaves = {n.id: n.D for n in self.nodes if n.is_leaf}
        gen = {n.id: (n.left.EU, n.left.EV, n.right.EU, n.right.EV, n.B12, n.B21)
               for n in self.nodes if not n.is_leaf}
        return leaves, gen

    def dense(self) -> np.ndarray:
        """The compressed operator as a dense matrix."""
        Y = np.zeros((self.N, self.N))
        for n in self.nodes:
            if n.is_leaf:
                Y[n.start:n.end, n.start:n.end] = n.D
            else:
                lc, rc = n.left, n.right
                Y[lc.start:lc.end, rc.start:rc.end] = lc.EU @ n.B12 @ rc.EV.T
                Y[rc.start:rc.end, lc.start:lc.end] = rc.EU @ n.B21 @ lc.EV.T
        return Y


# ----------------------------------------------------------------------------------
# Dense operators for the configurations (generators; not reference code)
# ----------------------------------------------------------------------------------


def cauchy_matrix(N: int) -> np.ndarray:
    """A_ij = 1/(x_i - y_j), x_i = i/N, y_j = (j + 0.5)/N."""
    x = np.arange(N) / N
    y = (np.arange(N) + 0.5) / N
    return 1.0 / (x[:, None] - y[None, :])


def gaussian_matrix(x: np.ndarray, h: float, shift: float) -> np.ndarray:
    """A_ij = exp(-(x_i - x_j)^2 / (2 h^2)) + shift * delta_ij (1-D points)."""
    d = x[:, None] - x[None, :]
    A = np.exp(-(d * d) / (2.0 * h * h))
    A[np.diag_indices_from(A)] += shift
    return A


def coulomb_matrix(p: np.ndarray, eps: float = 1e-3, shift: float = 4.0) -> np.ndarray:
    """A_ij = 1/(|p_i - p_j| + eps) + shift * delta_ij (2-D points)."""
    d = np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1))
    A = 1.0 / (d + eps)
    A[np.diag_indices_from(A)] += shift
    return A


def morton_order(p: np.ndarray, bits: int = 16) -> np.ndarray:
    """Permutation sorting 2-D points in [0,1)^2 along the Z-order curve."""
    q = np.clip((p * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)

    def spread(v):
        v = v.astype(np.uint64)
        out = np.zeros_like(v)
        for b in range(bits):
            out |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b)
        return out

    key = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1))
    return np.argsort(key, kind="stable")


def rel_err(ref: np.ndarray, val: np.ndarray) -> float:
    """calc_rel_error of the drivers (main_hodlr.cpp:26-35): ||ref - val|| / ||ref||."""
    den = np.linalg.norm(ref)
    return 0.0 if den == 0 else float(np.linalg.norm(ref - val) / den)
