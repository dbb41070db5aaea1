"""The dense building blocks through the C ABI, against FP64 references.

* hm_gemm_batched_f32_device on the tcgen05 kernel (HM_GEMM_TENSOR_CORES) and on the FMA
  kernel: K-major and MN-major operands (every opA/opB combination), beta != 0,
  split-K reduce-add, and outputs whose row count is not a multiple of 4 (the row-by-row
  store) or whose leading dimension is not TMA-addressable.  Elementwise bound of an FP32
  GEMM: |C - C64| <= 8 k u32 (|alpha| |A||B| + |beta| |C0|), u32 = 2^-24.
* the FP64 MMA kernel against an FP64 product (1e-13 relative).
* the warp-tiled kernel's 96-row tiles at every tile width, FP32 and FP64, forced by a
  tile-table entry.
* hm_kernel_block_product_device (a generated kernel block times X, and its transpose)
  against the dense FP64 matrix, for the three kernels.
* the tcgen05 kernel's bounded waits: HM_GEMM_TEST_STALL makes them run out, the call
  returns HM_ERR_TIMEOUT, and the next call on the same handle is correct.
* hm_inverse_batched_device (Matrix::inverse, matrix.h:133-149) with pivoting at every
  size: matrices whose leading half-block is singular, in place and out of place;
  X A - I within 50 n cond(A) u64 (normwise); a singular matrix gives HM_ERR_SINGULAR.
"""
import os

import numpy as np
import pytest

import hmat_b200 as H

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


# (m, n, k, opA, opB, beta, ksplit, ld pad): pads keep ld % 4 == 0 except where noted
GEMM_CASES = [
    (256, 96, 512, 0, 0, 0.0, 1, 0),     # MN-major A, K-major B
    (130, 64, 384, 1, 0, 0.5, 1, 2),     # K-major A, m % 4 != 0: last tile stored row by row
    (77, 128, 640, 0, 1, 1.0, 1, 3),     # MN-major B, beta = 1
    (200, 32, 1024, 1, 1, 0.0, 4, 0),    # split-K (TMA reduce-add), both operands transposed
    (128, 96, 2048, 0, 0, 1.0, 8, 0),    # split-K with beta = 1 (adds into C)
    (255, 40, 256, 0, 0, -2.0, 1, 1),    # ldc = 256 (m 255): row-by-row tail, n not a multiple of 32
]


def _gemm_problem(torch, rng, m, n, k, opA, opB, beta, pad, dtype):
    ar, ac = (m, k) if opA == 0 else (k, m)
    br, bc = (k, n) if opB == 0 else (n, k)
    lda, ldb, ldc = ar + (-ar % 4), br + (-br % 4), m + pad
    Ah = rng.standard_normal((ar, ac))
    Bh = rng.standard_normal((br, bc))
    Ch = rng.standard_normal((m, n))
    # column-major storage with padded leading dimensions (a torch tensor of shape (cols, ld))
    def dev(X, ld):
        t = torch.zeros((X.shape[1], ld), dtype=dtype, device="cuda")
        t[:, :X.shape[0]] = torch.from_numpy(X.T.copy()).to(dtype)
        return t
    A, B, C = dev(Ah, lda), dev(Bh, ldb), dev(Ch, ldc)
    opa = Ah if opA == 0 else Ah.T
    opb = Bh if opB == 0 else Bh.T
    # reference from the values actually stored (FP32 rounding of the inputs)
    Ar = A[:, :ar].T.double().cpu().numpy()
    Br = B[:, :br].T.double().cpu().numpy()
    Cr = C[:, :m].T.double().cpu().numpy()
    opa = Ar if opA == 0 else Ar.T
    opb = Br if opB == 0 else Br.T
    return dict(A=A, B=B, C=C, lda=lda, ldb=ldb, ldc=ldc, opa=opa, opb=opb, C0=Cr)


@pytest.mark.parametrize("kernel", [H.GEMM_TENSOR_CORES, H.GEMM_FMA])
def test_gemm_f32_vs_fp64(kernel):
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(7)
    alpha = 0.75
    for (m, n, k, opA, opB, beta, ksplit, pad) in GEMM_CASES:
        # one batch of three problems of the same shape (a batched launch)
        probs = [_gemm_problem(torch, rng, m, n, k, opA, opB, beta, pad, torch.float32) for _ in range(3)]
        d.gemm([m] * 3, [n] * 3, [k] * 3, alpha, [p["A"].data_ptr() for p in probs], [p["lda"] for p in probs], opA,
               [p["B"].data_ptr() for p in probs], [p["ldb"] for p in probs], opB, beta,
               [p["C"].data_ptr() for p in probs], [p["ldc"] for p in probs], ksplit=ksplit, flags=kernel)
        torch.cuda.synchronize()
        for p in probs:
            ref = alpha * p["opa"] @ p["opb"] + beta * p["C0"]
            bound = 8 * k * U32 * (abs(alpha) * np.abs(p["opa"]) @ np.abs(p["opb"]) + abs(beta) * np.abs(p["C0"]))
            got = p["C"][:, :m].T.double().cpu().numpy()
            err = np.abs(got - ref)
            assert np.all(err <= bound), (m, n, k, opA, opB, beta, ksplit, float((err / bound).max()))
            # rows past m in the padded leading dimension are untouched
            if p["ldc"] > m:
                assert torch.count_nonzero(p["C"][:, m:]).item() == 0


def _gemm_signature(dtype, count, m, n, k):
    """The tuning signature GemmBatch::finalize gives a C-ABI batch of `count` problems
    of one shape: tag|type|p(count, next power of 2)|m(next power of 2)|n(multiple of 32)|
    k(median, next power of 2)."""
    def p2(v):
        q = 1
        while q < v:
            q <<= 1
        return q
    return f"gemm_batched|{dtype}|p{p2(count)}|m{p2(m)}|n{-(-n // 32) * 32}|k{p2(k)}"


# (m, n, k, opA, opB, beta, ksplit, ld pad) for the 96-row tiles: whole tiles (m = 96,
# 192), a ragged last tile (m = 290), split-K with beta 0 and 1, both operand layouts
TILE96_CASES = [
    (96, 64, 2048, 1, 0, 0.0, 0, 0),     # the projection shape V^T x: automatic split-K
    (192, 96, 300, 0, 1, 1.0, 1, 0),
    (290, 40, 256, 1, 1, -2.0, 1, 1),
    (96, 128, 4096, 0, 0, 1.0, 4, 0),
]


@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_gemm_tile96_vs_fp64(dtype, tmp_path):
    """The warp-tiled kernel's 96-row tile shape (shape 3) at every tile width, forced by a
    tile-table entry, against FP64 products (FP32: the elementwise bound above; FP64:
    1e-13 normwise)."""
    import json
    torch = _torch()
    tdt = torch.float32 if dtype == "f32" else torch.float64
    d = H.Dense()
    rng = np.random.default_rng(10)
    alpha = 0.75
    try:
        for bn in (32, 64, 96, 128):
            for (m, n, k, opA, opB, beta, ksplit, pad) in TILE96_CASES:
                f = tmp_path / f"t{bn}.json"
                f.write_text(json.dumps({_gemm_signature(dtype, 3, m, n, k): [bn, 3, 0]}))
                H.tile_table_load(str(f))
                probs = [_gemm_problem(torch, rng, m, n, k, opA, opB, beta, pad, tdt) for _ in range(3)]
                d.gemm([m] * 3, [n] * 3, [k] * 3, alpha, [p["A"].data_ptr() for p in probs],
                       [p["lda"] for p in probs], opA, [p["B"].data_ptr() for p in probs], [p["ldb"] for p in probs],
                       opB, beta, [p["C"].data_ptr() for p in probs], [p["ldc"] for p in probs], ksplit=ksplit,
                       flags=H.GEMM_FMA, dtype=dtype)
                torch.cuda.synchronize()
                for p in probs:
                    ref = alpha * p["opa"] @ p["opb"] + beta * p["C0"]
                    got = p["C"][:, :m].T.double().cpu().numpy()
                    if dtype == "f32":
                        bound = 8 * k * U32 * (abs(alpha) * np.abs(p["opa"]) @ np.abs(p["opb"]) +
                                               abs(beta) * np.abs(p["C0"]))
                        assert np.all(np.abs(got - ref) <= bound), (bn, m, n, k)
                    else:
                        assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref), (bn, m, n, k)
                    if p["ldc"] > m:
                        assert torch.count_nonzero(p["C"][:, m:]).item() == 0
    finally:   # the library's own table again
        H.tile_table_load(os.environ.get("HM_TILE_TABLE") or
                          os.path.join(os.path.dirname(os.path.abspath(H.__file__)), "tile_table.json"))


@pytest.mark.parametrize("kernel", [H.KERNEL_COULOMB, H.KERNEL_GAUSSIAN, H.KERNEL_CAUCHY])
def test_kernel_block_product_vs_dense(kernel):
    """hm_kernel_block_product_device: A[r0:r1, c0:c1] X and its transpose product with A
    generated on the device, against the dense FP64 matrix (1e-13 normwise): off-diagonal
    blocks, a block across the diagonal (the shift), skinny and wide right-hand sides."""
    import hmat_oracle as O
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(12)
    N = 3000
    if kernel == H.KERNEL_COULOMB:
        pts, params = rng.random((N, 2)), [1e-3, 4.0]
        A = O.coulomb_matrix(pts, 1e-3, 4.0)
    elif kernel == H.KERNEL_GAUSSIAN:
        pts, params = np.sort(rng.random(N)).reshape(-1, 1), [0.05, 1e-2]
        A = O.gaussian_matrix(pts[:, 0], 0.05, 1e-2)
    else:
        pts, params = np.concatenate([np.arange(N) / N, (np.arange(N) + 0.5) / N]), [0.0, 0.0]
        A = O.cauchy_matrix(N)
    for (r0, r1, c0, c1) in [(0, 1000, 1500, 3000), (1500, 3000, 0, 1500), (200, 900, 100, 800)]:
        for nrhs in (5, 70):
            for trans in (False, True):
                blk = A[r0:r1, c0:c1]
                op = blk.T if trans else blk
                m, k = op.shape
                X = rng.standard_normal((k, nrhs))
                Xd = torch.from_numpy(np.asfortranarray(X).T.copy()).cuda()      # column-major k x nrhs
                Yd = torch.full((nrhs, m + 3), 7.0, dtype=torch.float64, device="cuda")   # ld = m + 3
                d.kernel_block_product(kernel, pts, params, r0, r1, c0, c1, Xd.data_ptr(), k, nrhs,
                                       Yd.data_ptr(), m + 3, trans=trans)
                torch.cuda.synchronize()
                Y = Yd[:, :m].T.cpu().numpy()
                ref = op @ X
                assert np.linalg.norm(Y - ref) <= 1e-13 * np.linalg.norm(ref), (r0, r1, c0, c1, nrhs, trans)
                assert torch.all(Yd[:, m:] == 7.0).item()      # rows past m untouched
    with pytest.raises(H.HmError):
        d.kernel_block_product(kernel, pts, params, 0, N + 1, 0, 10, Xd.data_ptr(), 10, 1, Yd.data_ptr(), N + 1)


def test_gemm_tc_rejects_unaligned():
    torch = _torch()
    d = H.Dense()
    A = torch.zeros(64 * 130, dtype=torch.float32, device="cuda")
    B = torch.zeros(64 * 130, dtype=torch.float32, device="cuda")
    C = torch.zeros(64 * 130, dtype=torch.float32, device="cuda")
    with pytest.raises(H.HmError) as e:   # lda = 130 is not a multiple of 4 floats
        d.gemm([128], [64], [128], 1.0, [A.data_ptr()], [130], 0, [B.data_ptr()], [128], 0, 0.0,
               [C.data_ptr()], [128], flags=H.GEMM_TENSOR_CORES)
    assert e.value.code == H.HM_ERR_UNSUPPORTED


def test_gemm_f64_mma_vs_fp64():
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(8)
    for (m, n, k, opA, opB, beta, ksplit, pad) in GEMM_CASES[:4]:
        p = _gemm_problem(torch, rng, m, n, k, opA, opB, beta, pad, torch.float64)
        d.gemm([m], [n], [k], 1.5, [p["A"].data_ptr()], [p["lda"]], opA, [p["B"].data_ptr()], [p["ldb"]], opB, beta,
               [p["C"].data_ptr()], [p["ldc"]], ksplit=ksplit, flags=H.GEMM_TENSOR_CORES, dtype="f64")
        torch.cuda.synchronize()
        ref = 1.5 * p["opa"] @ p["opb"] + beta * p["C0"]
        got = p["C"][:, :m].T.cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)


def test_gemm_tc_wait_timeout_then_recovers():
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(9)
    m, n, k = 256, 64, 512
    p = _gemm_problem(torch, rng, m, n, k, 0, 0, 0.0, 0, torch.float32)
    args = ([m], [n], [k], 1.0, [p["A"].data_ptr()], [p["lda"]], 0, [p["B"].data_ptr()], [p["ldb"]], 0, 0.0,
            [p["C"].data_ptr()], [p["ldc"]])
    with pytest.raises(H.HmError) as e:
        d.gemm(*args, flags=H.GEMM_TENSOR_CORES | H.GEMM_TEST_STALL)
    assert e.value.code == H.HM_ERR_TIMEOUT
    # the context is intact: the same product on the same handle, without the stall
    d.gemm(*args, flags=H.GEMM_TENSOR_CORES)
    torch.cuda.synchronize()
    ref = p["opa"] @ p["opb"]
    got = p["C"][:, :m].T.double().cpu().numpy()
    bound = 8 * k * U32 * (np.abs(p["opa"]) @ np.abs(p["opb"]))
    assert np.all(np.abs(got - ref) <= bound)


def _pivot_needing(rng, n):
    """Regular n x n matrix whose leading half-block is singular (zero), non-symmetric."""
    h = n // 2
    A = rng.standard_normal((n, n)) / np.sqrt(n)
    A[:h, :h] = 0.0
    A[:h, h:2 * h] += 2.0 * np.eye(h)
    A[h:2 * h, :h] += 2.0 * np.eye(h)
    if n % 2:
        A[n - 1, n - 1] += 2.0
    return A


@pytest.mark.parametrize("inplace", [False, True])
def test_inverse_batched_pivoting(inplace):
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(10)
    sizes = [1, 5, 33, 64, 65, 100, 128, 200, 256, 300, 512]
    mats = [_pivot_needing(rng, n) if n > 1 else np.array([[3.0]]) for n in sizes]
    As = [torch.from_numpy(M.T.copy()).cuda() for M in mats]        # column-major
    Xs = As if inplace else [torch.empty_like(a) for a in As]
    d.inverse(sizes, [a.data_ptr() for a in As], sizes, [x.data_ptr() for x in Xs], sizes)
    torch.cuda.synchronize()
    for n, M, X in zip(sizes, mats, Xs):
        Xh = X.T.cpu().numpy()
        res = np.linalg.norm(Xh @ M - np.eye(n)) / np.sqrt(n)
        assert res <= 50 * n * np.linalg.cond(M) * 2.0 ** -52, (n, res)


def test_inverse_batched_singular():
    torch = _torch()
    d = H.Dense()
    rng = np.random.default_rng(11)
    for n in (40, 150):
        M = rng.standard_normal((n, n))
        M[:, 3] = 0.0    # exactly singular: a zero column stays zero through the elimination
        A = torch.from_numpy(M.T.copy()).cuda()
        X = torch.empty_like(A)
        with pytest.raises(H.HmError) as e:
            d.inverse([n], [A.data_ptr()], [n], [X.data_ptr()], [n])
        assert e.value.code == H.HM_ERR_SINGULAR
