"""ctypes binding of libhmat_b200.so (the C ABI in include/hmat_b200.h).

The classes mirror the reference's C++ API (chenxinye/hmat-omp
include/hodlr_routines.h:8-176, include/hss_routines.h:10-307): a constructor taking the
tolerance, public ``tolerance``/``rsvd_rank`` fields, ``build_from_dense(A, leaf_size)``,
``multiply(x)`` and ``solve(b)``.  Host arrays are numpy FP64; ``*_device`` methods take
raw device pointers (e.g. ``torch.Tensor.data_ptr()``).  There is no CPU fallback: if the
library is missing or no GPU is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhmat_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hmat_b200.h")

HM_OK, HM_ERR_ARG, HM_ERR_CUDA, HM_ERR_SINGULAR, HM_ERR_NO_CONVERGE = 0, 1, 2, 3, 4
HM_ERR_NONFINITE, HM_ERR_STATE, HM_ERR_UNSUPPORTED, HM_ERR_IR, HM_ERR_TIMEOUT = 5, 6, 7, 8, 9
GEMM_AUTO, GEMM_TENSOR_CORES, GEMM_FMA, GEMM_TEST_STALL = 0, 1, 2, 16
OP_N, OP_T = 0, 1   # opA / opB of Dense.gemm: as stored, or transposed
SKETCH_REFERENCE_UNIFORM, SKETCH_REFERENCE_NORMAL, SKETCH_DEVICE_NORMAL = 0, 1, 2
FP64, MIXED = 0, 1
KERNEL_CAUCHY, KERNEL_GAUSSIAN, KERNEL_COULOMB = 1, 2, 3


class HmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Opts(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("rsvd_rank", C.c_int),
        ("oversample", C.c_int),
        ("rsvd_min_dim", C.c_int),
        ("power_iters", C.c_int),
        ("max_rank", C.c_int),
        ("sketch", C.c_int),
        ("seed", C.c_ulonglong),
        ("precision", C.c_int),
        ("ir_tol", C.c_double),
        ("ir_max_iter", C.c_int),
        ("refine_steps", C.c_int),
    ]


class SolveStats(C.Structure):
    _fields_ = [("ir_iters", C.c_int), ("rel_residual", C.c_double)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built: run `make -C hmat-omp_b200`")
    L = C.CDLL(LIB_PATH)
    L.hm_opts_default.argtypes = [C.POINTER(Opts)]
    L.hm_opts_default.restype = None
    L.hm_create.argtypes = [C.POINTER(Opts), C.POINTER(C.c_void_p)]
    L.hm_destroy.argtypes = [C.c_void_p]
    L.hm_last_error.argtypes = [C.c_void_p]
    L.hm_last_error.restype = C.c_char_p
    L.hm_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    for f in ("hm_hodlr_build_from_dense", "hm_hss_build_from_dense"):
        getattr(L, f).argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, C.c_int]
    for f in ("hm_hodlr_build_from_kernel", "hm_hss_build_from_kernel"):
        getattr(L, f).argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    L.hm_hodlr_build_from_dense_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    PP = C.POINTER(C.c_void_p)
    L.hm_set_rank_profile.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
    L.hm_hss_set_nested.argtypes = [C.c_void_p, C.c_int]
    L.hm_hss_is_nested.argtypes = [C.c_void_p]
    L.hm_hodlr_import.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, PP, PP, PP, PP, PP]
    L.hm_num_nodes.argtypes = [C.c_void_p]
    L.hm_export_tree.argtypes = [C.c_void_p] + [_ip] * 6
    L.hm_get_factor.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _ip, _ip]
    L.hm_multiply.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_int]
    L.hm_multiply_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
    L.hm_factor.argtypes = [C.c_void_p]
    L.hm_solve.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_int, C.POINTER(SolveStats)]
    L.hm_factor_solve.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_int, C.POINTER(SolveStats)]
    L.hm_solve_exact.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_int, C.c_double, C.c_int,
                                 C.POINTER(SolveStats)]
    L.hm_solve_exact_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double,
                                        C.c_int, C.POINTER(SolveStats)]
    L.hm_solve_gmres.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_int,
                                 C.c_int, C.POINTER(SolveStats)]
    L.hm_residual_exact.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, _dp]
    L.hm_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                  C.POINTER(SolveStats)]
    L.hm_batch_build_from_kernel.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, _ip, _dp, C.c_int]
    L.hm_num_systems.argtypes = [C.c_void_p]
    L.hm_batch_solve.argtypes = [C.c_void_p, C.c_void_p, _ip, C.c_void_p]
    L.hm_batch_multiply.argtypes = [C.c_void_p, C.c_void_p, _ip, C.c_void_p]
    L.hm_solve_transpose.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_int]
    L.hm_solve_transpose_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
    L.hm_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, _dp]
    L.hm_get_gradient.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _ip, _ip]
    L.hm_set_precision.argtypes = [C.c_void_p, C.c_int]
    L.hm_launch_count.argtypes = []
    L.hm_launch_count.restype = C.c_longlong
    L.hm_profile_enable.argtypes = [C.c_int]
    L.hm_profile_enable.restype = None
    for f in ("hm_profile_report", "hm_profile_sequence"):
        getattr(L, f).argtypes = [C.c_char_p, C.c_size_t]
        getattr(L, f).restype = C.c_size_t
    L.hm_save.argtypes = [C.c_void_p, C.c_char_p]
    L.hm_load.argtypes = [C.c_void_p, C.c_char_p]
    PPd = C.POINTER(C.c_void_p)
    for f, T in (("hm_gemm_batched_f32_device", C.c_float), ("hm_gemm_batched_f64_device", C.c_double)):
        getattr(L, f).argtypes = [C.c_void_p, C.c_int, _ip, _ip, _ip, T, PPd, _ip, C.c_int, PPd, _ip, C.c_int, T,
                                  PPd, _ip, C.c_int, C.c_int]
    L.hm_inverse_batched_device.argtypes = [C.c_void_p, C.c_int, _ip, PPd, _ip, PPd, _ip]
    L.hm_kernel_block_product_device.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                 C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                                 C.c_int, C.c_int, C.c_void_p, C.c_int]
    L.hm_tile_table_load.argtypes = [C.c_char_p]
    L.hm_tile_table_size.argtypes = []
    _lib = L
    return L


def launch_count() -> int:
    """Kernels this library has launched in the process."""
    return int(load().hm_launch_count())


def profile_enable(on: bool) -> None:
    load().hm_profile_enable(1 if on else 0)


def profile_report() -> dict:
    """{step: (launches, ms, algorithmic flops, algorithmic bytes)} since profile_enable(True)."""
    import json
    L = load()
    n = L.hm_profile_report(None, 0)
    buf = C.create_string_buffer(int(n))
    L.hm_profile_report(buf, n)
    return {k: tuple(v) for k, v in json.loads(buf.value.decode()).items()}


def tile_table_load(path: str | None) -> None:
    """Replace the batched-GEMM tile table (autotune.py's JSON); None or "" clears it."""
    rc = load().hm_tile_table_load((path or "").encode())
    if rc != HM_OK:
        raise HmError(rc, f"cannot read tile table {path!r}")


def tile_table_size() -> int:
    return load().hm_tile_table_size()


def profile_sequence() -> list:
    """[(step, launches, ms, algorithmic flops, algorithmic bytes, tuning), ...] in launch
    order; tuning = "signature#bn,small,tc" for batched-GEMM steps, else ""."""
    import json
    L = load()
    n = L.hm_profile_sequence(None, 0)
    buf = C.create_string_buffer(int(n))
    L.hm_profile_sequence(buf, n)
    return [tuple(r) for r in json.loads(buf.value.decode())]


def header_functions() -> list[str]:
    """Names of the functions declared in include/hmat_b200.h."""
    import re
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^HM_API\s+[\w\s\*]+?\b(hm_\w+)\(", txt, flags=re.M)))


def default_opts() -> Opts:
    o = Opts()
    load().hm_opts_default(C.byref(o))
    return o


def morton_order(points: np.ndarray, bits: int = 16) -> np.ndarray:
    """Permutation that sorts 2-D points of [0,1)^2 along the Z-order (Morton) curve.

    A kernel operator over points in this order has numerically low-rank off-diagonal
    blocks at every level of the bisection tree (the ordering the 2-D Coulomb workload
    uses); quantises each coordinate to `bits` bits and interleaves them (x in the even
    bits)."""
    p = np.asarray(points, dtype=np.float64)
    q = np.clip((p * (1 << bits)).astype(np.uint64), 0, (1 << bits) - 1)

    def spread(v):   # bit i of v -> bit 2i (magic-number interleave of a 16-bit value)
        v = v & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v

    if bits > 16:
        raise ValueError("morton_order: at most 16 bits per coordinate")
    key = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1))
    return np.argsort(key, kind="stable")


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class _Handle:
    def __init__(self, tol: float, **kw):
        self._L = load()
        self.opts = default_opts()
        self.opts.tol = tol
        for k, v in kw.items():
            setattr(self.opts, k, v)
        self._h = C.c_void_p()
        self._check(self._L.hm_create(C.byref(self.opts), C.byref(self._h)), create=True)
        self.N = 0

    # reference public fields
    @property
    def tolerance(self) -> float:
        return self.opts.tol

    @property
    def rsvd_rank(self) -> int:
        return self.opts.rsvd_rank

    def _check(self, rc: int, create: bool = False):
        if rc != HM_OK:
            msg = "hm_create failed" if create else self._L.hm_last_error(self._h).decode()
            raise HmError(rc, msg)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.hm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, precision: int):
        self._check(self._L.hm_set_precision(self._h, precision))
        self.opts.precision = precision

    def set_stream(self, stream_ptr: int):
        self._check(self._L.hm_set_stream(self._h, C.c_void_p(stream_ptr)))

    def multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(self.N, -1))
        Y = np.zeros_like(X, order="F")
        self._check(self._L.hm_multiply(self._h, _d(X), X.shape[1], self.N, _d(Y), self.N))
        return Y.ravel() if vec else Y

    def multiply_device(self, dx: int, nrhs: int, ldx: int, dy: int, ldy: int):
        self._check(self._L.hm_multiply_device(self._h, C.c_void_p(dx), nrhs, ldx, C.c_void_p(dy), ldy))

    def factor(self):
        self._check(self._L.hm_factor(self._h))

    def solve(self, b: np.ndarray, stats: bool = False):
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        st = SolveStats()
        self._check(self._L.hm_solve(self._h, _d(B), B.shape[1], self.N, _d(X), self.N, C.byref(st)))
        out = X.ravel() if vec else X
        return (out, st) if stats else out

    def solve_device(self, db: int, nrhs: int, ldb: int, dx: int, ldx: int) -> SolveStats:
        st = SolveStats()
        self._check(self._L.hm_solve_device(self._h, C.c_void_p(db), nrhs, ldb, C.c_void_p(dx), ldx,
                                            C.byref(st)))
        return st

    def factor_solve(self, b: np.ndarray, stats: bool = False):
        """Factor, then solve (the reference's solve(b)); b's copy overlaps the factor."""
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        st = SolveStats()
        self._check(self._L.hm_factor_solve(self._h, _d(B), B.shape[1], self.N, _d(X), self.N, C.byref(st)))
        out = X.ravel() if vec else X
        return (out, st) if stats else out

    def solve_exact(self, b: np.ndarray, tol: float = 1e-12, max_iter: int = 10, stats: bool = False):
        """Solve with the exact kernel operator (matrix-free builds): refinement whose
        residual uses generated entries of A, corrections from the compressed factors."""
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        st = SolveStats()
        self._check(self._L.hm_solve_exact(self._h, _d(B), B.shape[1], self.N, _d(X), self.N, tol, max_iter,
                                           C.byref(st)))
        out = X.ravel() if vec else X
        return (out, st) if stats else out

    def solve_gmres(self, b: np.ndarray, tol: float = 1e-12, restart: int = 30, max_iter: int = 200,
                    stats: bool = False):
        """Flexible GMRES against the exact kernel operator, preconditioned by the
        compressed factorization (matrix-free builds)."""
        b = np.asarray(b, dtype=np.float64)
        vec = b.ndim == 1
        B = np.asfortranarray(b.reshape(self.N, -1))
        X = np.zeros_like(B, order="F")
        st = SolveStats()
        self._check(self._L.hm_solve_gmres(self._h, B.ctypes.data, B.shape[1], self.N, X.ctypes.data, self.N, tol,
                                           restart, max_iter, C.byref(st)))
        out = X.ravel() if vec else X
        return (out, st) if stats else out

    def residual_exact(self, b, x, nrhs: int | None = None, ld: int | None = None) -> np.ndarray:
        """Per-column ||b - A x|| / ||b|| against the exact kernel operator (matrix-free
        builds).  b, x: numpy arrays (N or N x nrhs) or device pointers with nrhs and ld."""
        if isinstance(b, np.ndarray):
            B = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(self.N, -1))
            X = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(self.N, -1))
            rel = np.zeros(B.shape[1])
            self._check(self._L.hm_residual_exact(self._h, B.ctypes.data, B.shape[1], self.N, X.ctypes.data,
                                                  self.N, _d(rel)))
            return rel
        rel = np.zeros(nrhs)
        self._check(self._L.hm_residual_exact(self._h, C.c_void_p(b), nrhs, ld, C.c_void_p(x), ld, _d(rel)))
        return rel

    def solve_transpose(self, g: np.ndarray) -> np.ndarray:
        """lam = A^{-T} g (the adjoint solve)."""
        g = np.asarray(g, dtype=np.float64)
        vec = g.ndim == 1
        G = np.asfortranarray(g.reshape(self.N, -1))
        Lm = np.zeros_like(G, order="F")
        self._check(self._L.hm_solve_transpose(self._h, _d(G), G.shape[1], self.N, _d(Lm), self.N))
        return Lm.ravel() if vec else Lm

    def gradients(self, x: np.ndarray, lam: np.ndarray) -> np.ndarray:
        """Accumulate dL/d(factors) from x and lam = A^{-T} dL/dx; returns [dL/dp0, dL/dp1]
        of the kernel (NaN for dense builds)."""
        X = np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(self.N, -1))
        Lm = np.asfortranarray(np.asarray(lam, dtype=np.float64).reshape(self.N, -1))
        out = np.zeros(2)
        self._check(self._L.hm_gradients(self._h, X.ctypes.data, self.N, Lm.ctypes.data, self.N, X.shape[1],
                                         _d(out)))
        return out

    def get_gradient(self, node: int, which: int) -> np.ndarray:
        r, c = C.c_int(), C.c_int()
        self._check(self._L.hm_get_gradient(self._h, node, which, None, C.byref(r), C.byref(c)))
        out = np.zeros(r.value * c.value)
        if out.size:
            self._check(self._L.hm_get_gradient(self._h, node, which, _d(out), C.byref(r), C.byref(c)))
        return out.reshape(c.value, r.value).T.copy()

    def set_rank_profile(self, rank12=None, rank21=None) -> None:
        """Fix each block's kept rank for the next builds (None clears): node i keeps
        rank12[i] / rank21[i] singular triplets, e.g. tree()["rank12"] of an earlier build."""
        if rank12 is None:
            self._check(self._L.hm_set_rank_profile(self._h, 0, None, None))
            return
        a = np.ascontiguousarray(rank12, dtype=np.int32)
        b = np.ascontiguousarray(rank21, dtype=np.int32)
        self._check(self._L.hm_set_rank_profile(self._h, a.size, a.ctypes.data_as(_ip), b.ctypes.data_as(_ip)))

    def save(self, path: str) -> None:
        """Write the built operator to `path` (hm_save)."""
        self._check(self._L.hm_save(self._h, str(path).encode()))

    def num_nodes(self) -> int:
        return self._L.hm_num_nodes(self._h)

    def tree(self) -> dict:
        n = self.num_nodes()
        names = ["start", "end", "is_leaf", "depth", "rank12", "rank21"]
        arrs = [np.zeros(n, dtype=np.int32) for _ in names]
        self._check(self._L.hm_export_tree(self._h, *[a.ctypes.data_as(_ip) for a in arrs]))
        return dict(zip(names, arrs))

    def get_factor(self, node: int, which: int) -> np.ndarray:
        r, c = C.c_int(), C.c_int()
        self._check(self._L.hm_get_factor(self._h, node, which, None, C.byref(r), C.byref(c)))
        out = np.zeros(r.value * c.value)
        if out.size:
            self._check(self._L.hm_get_factor(self._h, node, which, _d(out), C.byref(r), C.byref(c)))
        return out.reshape(c.value, r.value).T.copy()


class Dense(_Handle):
    """Batched dense building blocks on the device (no tree): the products of
    Matrix::operator* (matrix.h:93-104) and the inverses of Matrix::inverse
    (matrix.h:133-149) for many independent matrices per launch.  Arguments are lists of
    device pointers (e.g. ``torch.Tensor.data_ptr()``) and sizes."""

    def __init__(self):
        super().__init__(0.0)

    @staticmethod
    def _ia(v):
        return np.ascontiguousarray(v, dtype=np.int32)

    def gemm(self, m, n, k, alpha, A, lda, opA, B, ldb, opB, beta, Cs, ldc, ksplit=0, flags=GEMM_AUTO,
             dtype="f32"):
        cnt = len(m)
        PP = C.c_void_p * max(cnt, 1)
        arrs = [self._ia(v) for v in (m, n, k, lda, ldb, ldc)]
        ip = [a.ctypes.data_as(_ip) for a in arrs]
        f = self._L.hm_gemm_batched_f32_device if dtype == "f32" else self._L.hm_gemm_batched_f64_device
        self._check(f(self._h, cnt, ip[0], ip[1], ip[2], alpha, PP(*A), ip[3], opA, PP(*B), ip[4], opB, beta,
                      PP(*Cs), ip[5], ksplit, flags))

    def inverse(self, n, A, lda, X, ldx):
        cnt = len(n)
        PP = C.c_void_p * max(cnt, 1)
        na, la, lx = self._ia(n), self._ia(lda), self._ia(ldx)
        self._check(self._L.hm_inverse_batched_device(self._h, cnt, na.ctypes.data_as(_ip), PP(*A),
                                                      la.ctypes.data_as(_ip), PP(*X), lx.ctypes.data_as(_ip)))

    def kernel_block_product(self, kernel, points, params, r0, r1, c0, c1, X, ldx, nrhs, Y, ldy, trans=False):
        """Y = A[r0:r1, c0:c1] X (or its transpose times X) with A generated from `points`
        (host, hm_hodlr_build_from_kernel's layout); X, Y device pointers, column-major."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        if kernel == KERNEL_CAUCHY:
            N, dim = pts.size // 2, 1
        else:
            N, dim = pts.reshape(pts.shape[0], -1).shape
        prm = np.ascontiguousarray(params, dtype=np.float64)
        self._check(self._L.hm_kernel_block_product_device(self._h, kernel, pts.ctypes.data, dim, N, prm.ctypes.data,
                                                           len(prm), r0, r1, c0, c1, int(bool(trans)), C.c_void_p(X),
                                                           ldx, nrhs, C.c_void_p(Y), ldy))


class HODLRMatrix(_Handle):
    """Mirror of HODLRMatrix (hodlr_routines.h:8-176) on the device path."""

    D, U, V, B12, B21 = 0, 1, 2, 3, 4

    def __init__(self, tol: float = 1e-6, **kw):
        super().__init__(tol, **kw)

    def build_from_dense(self, A: np.ndarray, leaf_size: int):
        A = np.asfortranarray(A, dtype=np.float64)
        self.N = A.shape[0]
        self._check(self._L.hm_hodlr_build_from_dense(self._h, _d(A), self.N, self.N, leaf_size))

    def build_from_dense_device(self, dA: int, N: int, lda: int, leaf_size: int):
        self.N = N
        self._check(self._L.hm_hodlr_build_from_dense_device(self._h, C.c_void_p(dA), N, lda, leaf_size))

    _kernel_build = "hm_hodlr_build_from_kernel"

    def build_from_kernel(self, kernel: int, points: np.ndarray, params, leaf_size: int, N: int | None = None):
        """Matrix-free build.  Cauchy: points = concat(x, y) (1-D); Gaussian/Coulomb:
        points N x dim."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        if kernel == KERNEL_CAUCHY:
            N = pts.size // 2 if N is None else N
            dim = 1
        else:
            pts2 = pts.reshape(pts.shape[0], -1)
            N, dim = pts2.shape
        pr = np.ascontiguousarray(params, dtype=np.float64)
        self.N = N
        self._check(getattr(self._L, self._kernel_build)(self._h, kernel, _d(pts), dim, N, _d(pr), pr.size,
                                                         leaf_size))

    def import_factors(self, N: int, leaf_size: int, nodes) -> None:
        """Upload a tree of reference factors; ``nodes`` in pre-order with attributes
        D/U/V/B12/B21 (numpy or None), as oracle.hmat_oracle.HNode holds them."""
        self.N = N
        n = len(nodes)
        keep = []

        def arr(m):
            if m is None or m.size == 0:
                return None
            a = np.asfortranarray(m, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data

        PP = C.c_void_p * n
        D = PP(*[arr(x.D) if x.is_leaf else None for x in nodes])
        U = PP(*[arr(x.U) if i > 0 else None for i, x in enumerate(nodes)])
        V = PP(*[arr(x.V) if i > 0 else None for i, x in enumerate(nodes)])
        B12 = PP(*[arr(x.B12) if not x.is_leaf else None for x in nodes])
        B21 = PP(*[arr(x.B21) if not x.is_leaf else None for x in nodes])
        r12 = np.array([0 if x.is_leaf else x.B12.shape[0] for x in nodes], dtype=np.int32)
        r21 = np.array([0 if x.is_leaf else x.B21.shape[0] for x in nodes], dtype=np.int32)
        self._check(self._L.hm_hodlr_import(self._h, N, leaf_size, r12.ctypes.data_as(_ip),
                                            r21.ctypes.data_as(_ip), D, U, V, B12, B21))


class HSSMatrix(_Handle):
    """Mirror of HSSMatrix (hss_routines.h:10-307) on the device path.

    ``nested=True`` selects the nested-basis form (hm_hss_set_nested): compressed
    transfers R / W instead of the reference's identities, the same leaf bases."""

    D, U, V, R, W, B = 0, 1, 2, 3, 4, 5

    def __init__(self, tol: float = 1e-9, nested: bool = False, **kw):
        super().__init__(tol, **kw)
        if nested:
            self.set_nested(True)

    def set_nested(self, on: bool) -> None:
        """Form of the next builds: nested bases (True) or the reference's identity
        transfers (False)."""
        self._check(self._L.hm_hss_set_nested(self._h, 1 if on else 0))

    @property
    def nested(self) -> bool:
        """Whether the current operator is a nested-basis HSS."""
        return bool(self._L.hm_hss_is_nested(self._h))

    def build_from_dense(self, A: np.ndarray, leaf_size: int):
        A = np.asfortranarray(A, dtype=np.float64)
        self.N = A.shape[0]
        self._check(self._L.hm_hss_build_from_dense(self._h, _d(A), self.N, self.N, leaf_size))

    _kernel_build = "hm_hss_build_from_kernel"
    build_from_kernel = HODLRMatrix.build_from_kernel


def load_operator(path: str, tol: float = 1e-10, **kw):
    """Read an operator written by save() into a new HODLRMatrix or HSSMatrix (the kind
    stored in the file); tol/kw are the handle's options (precision, refinement...)."""
    import struct
    with open(path, "rb") as f:
        head = f.read(16)
    if len(head) < 16 or head[:8] != b"HMATB200":
        raise HmError(HM_ERR_ARG, f"{path}: not an hmat_b200 operator file")
    kind = struct.unpack("<I", head[12:16])[0]
    m = (HSSMatrix if kind == 1 else HODLRMatrix)(tol, **kw)
    m._check(m._L.hm_load(m._h, str(path).encode()))
    m.N = int(m.tree()["end"].max())
    return m


class HODLRBatch(_Handle):
    """Many independent HODLR systems sharing every launch (hm_batch_*)."""

    def __init__(self, tol: float = 1e-10, **kw):
        super().__init__(tol, **kw)
        self.sizes: list[int] = []

    def build_from_kernel(self, kernel: int, points: list, params: list, leaf_size: int):
        pts = [np.asarray(p, dtype=np.float64).reshape(len(p), -1) for p in points]
        dim = pts[0].shape[1]
        self.sizes = [p.shape[0] for p in pts]
        allp = np.ascontiguousarray(np.vstack(pts))
        Ns = np.array(self.sizes, dtype=np.int32)
        pr = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        self.N = int(Ns.sum())
        self._check(self._L.hm_batch_build_from_kernel(self._h, kernel, _d(allp), dim, len(pts),
                                                       Ns.ctypes.data_as(_ip), _d(pr), leaf_size))

    def _packed(self, blocks):
        cols = np.array([0 if b is None else (1 if np.ndim(b) == 1 else np.shape(b)[1]) for b in blocks],
                        dtype=np.int32)
        parts = [np.asarray(b, dtype=np.float64).reshape(n, -1, order="F").ravel(order="F")
                 for b, n in zip(blocks, self.sizes) if b is not None]
        return cols, np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(0))

    def _unpack(self, flat, cols):
        out, p = [], 0
        for n, c in zip(self.sizes, cols):
            out.append(flat[p:p + n * c].reshape(c, n).T.copy() if c else None)
            p += n * c
        return out

    def solve(self, blocks: list) -> list:
        cols, b = self._packed(blocks)
        x = np.zeros_like(b)
        self._check(self._L.hm_batch_solve(self._h, b.ctypes.data, cols.ctypes.data_as(_ip), x.ctypes.data))
        return self._unpack(x, cols)

    def multiply(self, blocks: list) -> list:
        cols, xin = self._packed(blocks)
        y = np.zeros_like(xin)
        self._check(self._L.hm_batch_multiply(self._h, xin.ctypes.data, cols.ctypes.data_as(_ip), y.ctypes.data))
        return self._unpack(y, cols)
