"""TEST INFRASTRUCTURE ONLY — ctypes access to the compiled reference.

``oracle/_ref/libhmatref.so`` (and ``libhmatref_gauss.so``) are the reference's own
serial and OpenMP classes (hodlr_routines{,_omp}.h, hss_routines{,_omp}.h) compiled
by ``oracle/Makefile`` with seed injection (``oracle/ref_harness.cpp``).  Tests use them
as the checker and bench.py's reference arm times them; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


_libs: dict[str, C.CDLL] = {}


def available(gaussian: bool = False) -> bool:
    name = "libhmatref_gauss.so" if gaussian else "libhmatref.so"
    return os.path.exists(os.path.join(REF_DIR, name))


def lib(gaussian: bool = False) -> C.CDLL:
    name = "libhmatref_gauss.so" if gaussian else "libhmatref.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    L = C.CDLL(path)
    L.hmref_random.argtypes = [C.c_uint, C.c_int, C.c_int, _dp]
    L.hmref_compress_svd.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
    L.hmref_compress_svd.restype = C.c_int
    L.hmref_compress_rsvd.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                      C.c_uint, _dp, _dp, _dp]
    L.hmref_compress_rsvd.restype = C.c_int
    for kind in ("hodlr", "hss"):
        b = getattr(L, f"hmref_{kind}_build")
        b.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint, C.c_int]
        b.restype = C.c_void_p
        getattr(L, f"hmref_{kind}_free").argtypes = [C.c_void_p]
        getattr(L, f"hmref_{kind}_num_nodes").argtypes = [C.c_void_p]
        getattr(L, f"hmref_{kind}_num_nodes").restype = C.c_int
        getattr(L, f"hmref_{kind}_factor_shape").argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip]
        getattr(L, f"hmref_{kind}_factor").argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        getattr(L, f"hmref_{kind}_multiply").argtypes = [C.c_void_p, _dp, _dp]
        getattr(L, f"hmref_{kind}_solve").argtypes = [C.c_void_p, _dp, C.c_int, _dp]
    L.hmref_hodlr_tree.argtypes = [C.c_void_p] + [_ip] * 6
    L.hmref_hodlr_solve_omp.argtypes = [C.c_void_p, _dp, C.c_int, _dp]
    L.hmref_omp_max_threads.argtypes = []
    L.hmref_omp_max_threads.restype = C.c_int
    L.hmref_hss_tree.argtypes = [C.c_void_p] + [_ip] * 9
    _libs[name] = L
    return L


def random(seed: int, rows: int, cols: int, gaussian: bool = False) -> np.ndarray:
    out = np.zeros(rows * cols)
    lib(gaussian).hmref_random(seed, rows, cols, _d(out))
    return out.reshape(cols, rows).T.copy()


def compress_rsvd(A: np.ndarray, tol: float, rank_guess: int, seed: int, gaussian=False):
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    mx = min(m, n)
    U = np.zeros(m * mx)
    V = np.zeros(n * mx)
    S = np.zeros(mx)
    r = lib(gaussian).hmref_compress_rsvd(_d(A), m, n, m, tol, rank_guess, seed, _d(U), _d(V), _d(S))
    return U[: m * r].reshape(r, m).T.copy(), V[: n * r].reshape(r, n).T.copy(), S[:r].copy()


def _shape(L, kind, h, node, which):
    r, c = C.c_int(), C.c_int()
    getattr(L, f"hmref_{kind}_factor_shape")(h, node, which, C.byref(r), C.byref(c))
    return r.value, c.value


def _factor(L, kind, h, node, which):
    r, c = _shape(L, kind, h, node, which)
    out = np.zeros(r * c)
    if r * c:
        getattr(L, f"hmref_{kind}_factor")(h, node, which, _d(out))
    return out.reshape(c, r).T.copy()


@dataclass
class HodlrTree:
    start: np.ndarray
    end: np.ndarray
    is_leaf: np.ndarray
    depth: np.ndarray
    rank12: np.ndarray
    rank21: np.ndarray


class RefHODLR:
    """The reference HODLRMatrix / HODLRMatrixOMP on a dense host matrix."""

    def __init__(self, A: np.ndarray, leaf: int, tol: float, rsvd_rank: int = 64, seed: int = 0,
                 omp: bool = False, gaussian: bool = False):
        self.L = lib(gaussian)
        A = np.asfortranarray(A, dtype=np.float64)
        self.N = A.shape[0]
        self.h = self.L.hmref_hodlr_build(_d(A), self.N, self.N, leaf, tol, rsvd_rank, seed,
                                          1 if omp else 0)

    def close(self):
        if self.h:
            self.L.hmref_hodlr_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tree(self) -> HodlrTree:
        n = self.L.hmref_hodlr_num_nodes(self.h)
        arrs = [np.zeros(n, dtype=np.int32) for _ in range(6)]
        self.L.hmref_hodlr_tree(self.h, *[_i(a) for a in arrs])
        return HodlrTree(*arrs)

    def factor(self, node: int, which: str) -> np.ndarray:
        w = {"D": 0, "U": 1, "V": 2, "B12": 3, "B21": 4}[which]
        return _factor(self.L, "hodlr", self.h, node, w)

    def multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.zeros(self.N)
        self.L.hmref_hodlr_multiply(self.h, _d(x), _d(y))
        return y

    def solve(self, b: np.ndarray) -> np.ndarray:
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        self.L.hmref_hodlr_solve(self.h, _d(B), B.shape[1], _d(X))
        return X.ravel() if vec else X

    def solve_omp(self, b: np.ndarray) -> np.ndarray:
        """HODLRMatrixOMP::solve on this (serially built) tree."""
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        self.L.hmref_hodlr_solve_omp(self.h, _d(B), B.shape[1], _d(X))
        return X.ravel() if vec else X

    def to_oracle(self):
        """Download the factors into an oracle HodlrOracle tree (pre-order)."""
        from hmat_oracle import HodlrOracle, hodlr_tree
        t = self.tree()
        leaf_len = int((t.end - t.start)[t.is_leaf.astype(bool)].max())
        o = HodlrOracle()
        o.N = self.N
        nodes = hodlr_tree(self.N, leaf_len)
        assert len(nodes) == len(t.start)
        for i, n in enumerate(nodes):
            if n.is_leaf:
                n.D = self.factor(i, "D")
            else:
                n.B12 = self.factor(i, "B12")
                n.B21 = self.factor(i, "B21")
            if i > 0:
                n.U = self.factor(i, "U")
                n.V = self.factor(i, "V")
        o.nodes = nodes
        return o


class RefHSS:
    """The reference HSSMatrix / HSSMatrixOMP on a dense host matrix."""

    def __init__(self, A: np.ndarray, leaf: int, tol: float, rsvd_rank: int = 64, seed: int = 0,
                 omp: bool = False, gaussian: bool = False):
        self.L = lib(gaussian)
        A = np.asfortranarray(A, dtype=np.float64)
        self.N = A.shape[0]
        self.omp = omp
        self.h = self.L.hmref_hss_build(_d(A), self.N, self.N, leaf, tol, rsvd_rank, seed,
                                        1 if omp else 0)

    def close(self):
        if self.h:
            self.L.hmref_hss_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tree(self) -> dict:
        n = self.L.hmref_hss_num_nodes(self.h)
        names = ["id", "start", "end", "is_leaf", "left", "right", "parent", "rank_U", "rank_V"]
        arrs = [np.zeros(n, dtype=np.int32) for _ in names]
        self.L.hmref_hss_tree(self.h, *[_i(a) for a in arrs])
        return dict(zip(names, arrs))

    def factor(self, node: int, which: str) -> np.ndarray:
        w = {"D": 0, "U": 1, "V": 2, "R": 3, "W": 4, "B": 5}[which]
        return _factor(self.L, "hss", self.h, node, w)

    def multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.zeros(self.N)
        self.L.hmref_hss_multiply(self.h, _d(x), _d(y))
        return y

    def solve(self, b: np.ndarray) -> np.ndarray:
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        self.L.hmref_hss_solve(self.h, _d(B), B.shape[1], _d(X))
        return X.ravel() if vec else X

    def to_oracle(self):
        from hmat_oracle import HssOracle, hss_tree
        t = self.tree()
        leaf_len = int((t["end"] - t["start"])[t["is_leaf"].astype(bool)].max())
        o = HssOracle()
        o.N = self.N
        nodes = hss_tree(self.N, leaf_len)
        for n in nodes:
            n.rank_U = int(t["rank_U"][n.id])
            n.rank_V = int(t["rank_V"][n.id])
            if n.is_leaf:
                n.D = self.factor(n.id, "D")
                n.U = self.factor(n.id, "U")
                n.V = self.factor(n.id, "V")
            else:
                n.B = self.factor(n.id, "B")
        o.nodes = nodes
        return o
