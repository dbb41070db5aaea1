"""hm_multiply_device_noalloc: the multiply for callers that may not allocate device
memory when they multiply (a real-time or callback thread that must not block in the
allocator, or an application whose memory pool owns the whole GPU).  It keeps its intermediates in a
fixed device array instead of allocating, and must give the same result as
hm_multiply_device.  This file is collected last so that a failure here cannot hide
the other tests' results."""
import ctypes as C

import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix

pytestmark = pytest.mark.gpu


def _noalloc(L):
    f = L.hm_multiply_device_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
    f.restype = C.c_int
    return f


def test_noalloc_multiply_matches_multiply_twice():
    import torch

    c = CASES["hodlr_cauchy_4096"]
    A = make_matrix(c)
    N = A.shape[0]
    h = H.HODLRMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    h.build_from_dense(A, c["leaf"])
    stream = torch.cuda.current_stream()
    h.set_stream(stream.cuda_stream)
    f = _noalloc(h._L)
    rng = np.random.default_rng(11)
    for call, nrhs in enumerate((3, 5)):  # two calls in a row, different inputs
        X = torch.from_numpy(rng.standard_normal((nrhs, N))).cuda()  # column-major N x nrhs
        Y_ref = torch.empty_like(X)
        Y_new = torch.full_like(X, float("nan"))
        h.multiply_device(X.data_ptr(), nrhs, N, Y_ref.data_ptr(), N)
        rc = f(h._h, C.c_void_p(X.data_ptr()), nrhs, N, C.c_void_p(Y_new.data_ptr()), N)
        assert rc == H.HM_OK, h._L.hm_last_error(h._h).decode()
        torch.cuda.synchronize()
        ref, new = Y_ref.cpu().numpy(), Y_new.cpu().numpy()
        assert np.isfinite(new).all()
        assert O.rel_err(ref, new) < 1e-10, (call, O.rel_err(ref, new))


def test_noalloc_rejects_oversized_operator():
    """A multiply whose intermediates exceed the fixed array is refused with a clear
    error instead of allocating."""
    c = CASES["hodlr_cauchy_4096"]
    A = make_matrix(c)
    N = A.shape[0]
    h = H.HODLRMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    h.build_from_dense(A, c["leaf"])
    import torch
    nrhs = 4096  # (ranks of every node) x 4096 columns does not fit in 32 MiB
    X = torch.zeros((nrhs, N), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    f = _noalloc(h._L)
    rc = f(h._h, C.c_void_p(X.data_ptr()), nrhs, N, C.c_void_p(Y.data_ptr()), N)
    assert rc == H.HM_ERR_UNSUPPORTED
    assert "scratch" in h._L.hm_last_error(h._h).decode()
