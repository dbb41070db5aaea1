"""Serialized operators (hm_save / hm_load): a reloaded operator multiplies, factors and
solves like the one that was saved, exports the same reference-form factors, keeps its
kernel (exact-operator refinement, dL/dh), and bad files are refused with HM_ERR_ARG."""
import os
import struct

import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O
from cases import CASES, make_matrix, make_vectors

pytestmark = pytest.mark.gpu


def _gauss(N=4096):
    x = np.sort(np.random.default_rng(2).random(N))
    m = H.HODLRMatrix(1e-10, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, x.reshape(-1, 1), [0.05, 1e-2], 128)
    return m


def test_hodlr_roundtrip(tmp_path):
    m = _gauss()
    f = str(tmp_path / "op.hmat")
    m.save(f)
    r = H.load_operator(f, 1e-10)
    assert isinstance(r, H.HODLRMatrix) and r.N == m.N
    for k, v in m.tree().items():
        assert np.array_equal(v, r.tree()[k]), k
    rng = np.random.default_rng(3)
    x, b = rng.standard_normal((m.N, 4)), rng.standard_normal((m.N, 4))
    assert O.rel_err(m.multiply(x), r.multiply(x)) < 1e-14
    assert O.rel_err(m.solve(b), r.solve(b)) < 1e-10
    for node in (1, 2, 5):
        for w in (H.HODLRMatrix.U, H.HODLRMatrix.V):
            assert np.array_equal(m.get_factor(node, w), r.get_factor(node, w))
    # the kernel travels with the operator
    xe, st = r.solve_exact(b, tol=1e-11, stats=True)
    assert st.rel_residual <= 1e-11
    g = 2.0 * (m.solve(b[:, 0]) - 1.0)
    dp_m = m.gradients(m.solve(b[:, 0]), m.solve_transpose(g))
    dp_r = r.gradients(r.solve(b[:, 0]), r.solve_transpose(g))
    assert abs(dp_m[0] - dp_r[0]) <= 1e-8 * abs(dp_m[0])


def test_mixed_precision_after_load(tmp_path):
    p = np.random.default_rng(3).random((8192, 2))
    p = np.ascontiguousarray(p[H.morton_order(p)])
    m = H.HODLRMatrix(1e-10, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=0)
    m.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 128)
    f = str(tmp_path / "c.hmat")
    m.save(f)
    r = H.load_operator(f, 1e-10, precision=H.MIXED, ir_tol=1e-10, ir_max_iter=30)
    b = np.random.default_rng(4).standard_normal((8192, 8))
    x, st = r.solve(b, stats=True)
    assert st.rel_residual <= 1e-10
    assert O.rel_err(m.solve(b), x) < 1e-8


def test_hss_roundtrip_keeps_reference_factors(tmp_path):
    c = CASES["hss_gauss_512"]
    A = make_matrix(c)
    h = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    h.build_from_dense(A, c["leaf"])
    f = str(tmp_path / "h.hmat")
    h.save(f)
    r = H.load_operator(f, c["tol"])
    assert isinstance(r, H.HSSMatrix)
    for k, v in h.tree().items():
        assert np.array_equal(v, r.tree()[k]), k
    for node in range(h.num_nodes()):
        for w in (H.HSSMatrix.D, H.HSSMatrix.U, H.HSSMatrix.V, H.HSSMatrix.B):
            assert np.array_equal(h.get_factor(node, w), r.get_factor(node, w)), (node, w)
    x, b = make_vectors(c, A.shape[0])
    assert O.rel_err(h.multiply(x), r.multiply(x)) < 1e-14
    assert O.rel_err(h.solve(b), r.solve(b)) < 1e-12


def test_version1_files_load(tmp_path):
    """Files of the first format version (no nested-basis section) still load: a HODLR file
    differs only in its version word; a reference-form HSS file also lacks the trailing
    nested flag of version 2."""
    x = np.random.default_rng(4).standard_normal((1024, 3))
    m = _gauss(1024)
    f = tmp_path / "hodlr.hmat"
    m.save(str(f))
    data = f.read_bytes()
    g = tmp_path / "hodlr_v1.hmat"
    g.write_bytes(data[:8] + struct.pack("<I", 1) + data[12:])
    r = H.load_operator(str(g), 1e-10)
    assert np.array_equal(m.multiply(x), r.multiply(x))
    c = CASES["hss_gauss_512"]
    A = make_matrix(c)
    h = H.HSSMatrix(c["tol"], rsvd_rank=c["rsvd_rank"], seed=c["seed"])
    h.build_from_dense(A, c["leaf"])
    f = tmp_path / "hss.hmat"
    h.save(str(f))
    data = f.read_bytes()
    assert struct.unpack("<I", data[-4:])[0] == 0   # version 2: the nested flag ends the file
    g = tmp_path / "hss_v1.hmat"
    g.write_bytes(data[:8] + struct.pack("<I", 1) + data[12:-4])
    r = H.load_operator(str(g), c["tol"])
    xs = x[:512]
    assert not r.nested and np.array_equal(h.multiply(xs), r.multiply(xs))


def test_bad_files_are_refused(tmp_path):
    m = _gauss(1024)
    f = tmp_path / "op.hmat"
    m.save(str(f))
    data = f.read_bytes()
    h = H.HODLRMatrix(1e-10)
    cases = {
        "truncated": data[: len(data) // 2],
        "magic": b"XXXXXXXX" + data[8:],
        "version": data[:8] + struct.pack("<I", 99) + data[12:],
        "N": data[:16] + struct.pack("<q", 2048) + data[24:],     # tree no longer matches
        "empty": b"",
    }
    for name, blob in cases.items():
        g = tmp_path / f"{name}.hmat"
        g.write_bytes(blob)
        assert h._L.hm_load(h._h, str(g).encode()) == H.HM_ERR_ARG, name
    assert h._L.hm_load(h._h, str(tmp_path / "missing.hmat").encode()) == H.HM_ERR_ARG
    os.remove(f)
