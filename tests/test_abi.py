"""The C-ABI library: it loads, exports every function include/hmat_b200.h declares,
and reports errors (no compute without a GPU)."""
import ctypes as C
import subprocess

import pytest

import hmat_b200 as H
from conftest import gpu_available


def test_library_exports_every_header_symbol():
    L = H.load()
    names = H.header_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", H.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in names:
        assert getattr(L, n) is not None


def test_library_has_no_torch_dependency():
    out = subprocess.run(["ldd", H.LIB_PATH], capture_output=True, text=True).stdout
    assert "torch" not in out and "c10" not in out


def test_default_opts_mirror_reference():
    o = H.default_opts()
    assert o.tol == 1e-6 and o.rsvd_rank == 64 and o.oversample == 10 and o.rsvd_min_dim == 256
    assert o.power_iters == 0 and o.max_rank == 0 and o.precision == H.FP64


def test_create_without_gpu_fails_cleanly():
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(H.HmError) as e:
        H.HODLRMatrix(1e-8)
    assert e.value.code == H.HM_ERR_CUDA


def test_invalid_options_rejected_before_device_use():
    L = H.load()
    o = H.default_opts()
    o.precision = 7
    h = C.c_void_p()
    assert L.hm_create(C.byref(o), C.byref(h)) == H.HM_ERR_ARG
    o = H.default_opts()
    o.rsvd_rank = 500
    assert L.hm_create(C.byref(o), C.byref(h)) == H.HM_ERR_UNSUPPORTED
