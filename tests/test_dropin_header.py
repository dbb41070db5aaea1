"""The drop-in C++ header compiles against the reference's own headers (no GPU needed)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_INC = os.path.join(os.environ.get("HMAT_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference")),
                       "include")


def test_dropin_header_compiles(tmp_path):
    if not os.path.isdir(REF_INC):
        pytest.skip("reference headers not present")
    src = tmp_path / "t.cpp"
    src.write_text('#include "hodlr_routines_cuda.h"\n'
                   'int main(){ HODLRMatrixCUDA m(1e-8); m.rsvd_rank = 16;\n'
                   '            HSSMatrixCUDA h(1e-9); h.rsvd_rank = 32; return m.N + h.N; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", REF_INC, "-I", os.path.join(ROOT, "include"),
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
