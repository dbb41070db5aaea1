"""The C++ drop-in (include/hodlr_routines_cuda.h) inside a driver shaped like the
reference's src/main_hodlr.cpp and src/main_hss.cpp: HODLRMatrix / HSSMatrix and
HODLRMatrixCUDA / HSSMatrixCUDA on the same operators, same sketch seed (oracle/dropin_driver.cpp, built into oracle/_ref by oracle/Makefile)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_hodlr")

pytestmark = pytest.mark.gpu


def test_dropin_matches_reference_class():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/dropin_hodlr not built (needs the reference headers)")
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=600, check=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    assert r["nodes_ref"] == r["nodes_gpu"]
    assert r["tree_mismatches"] == 0
    assert r["root_children_linked"] == 1
    assert r["multiply_rel"] < 1e-10
    assert r["solve_rel"] < 1e-10
    # HSSMatrix against HSSMatrixCUDA (build_topo ids, ranks, parents, factor shapes)
    assert r["hss_nodes_ref"] == r["hss_nodes_gpu"]
    assert r["hss_tree_mismatches"] == 0
    assert r["hss_multiply_rel"] < 1e-10
    assert r["hss_solve_rel"] < 1e-10
