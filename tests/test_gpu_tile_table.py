"""Tile-table entries change the kernels a batched GEMM step runs, not its results:
an operator planned under a table that forces 32-wide, 64-row tiles (and no tensor
cores) on every step reports that choice in the profile and solves to the same answer."""
import json
import os

import numpy as np
import pytest

import hmat_b200 as H
import hmat_oracle as O

pytestmark = pytest.mark.gpu


def _op():
    x = np.sort(np.random.default_rng(3).random(8192))
    m = H.HODLRMatrix(1e-12, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=1)
    m.build_from_kernel(H.KERNEL_GAUSSIAN, x.reshape(-1, 1), [0.05, 1e-2], 128)
    return m


def _profiled(m, b):
    H.profile_enable(True)
    try:
        m.factor()
        x = m.solve(b)
        seq = H.profile_sequence()
    finally:
        H.profile_enable(False)
    return x, {r[5].split("#")[0]: r[5].split("#")[1] for r in seq if "#" in r[5]}


@pytest.mark.skipif(bool(os.environ.get("HM_TILE_FORCE") or os.environ.get("HM_FP64_DMMA")),
                    reason="a forced tile choice overrides the table")
def test_table_entries_apply_and_keep_results(tmp_path):
    b = np.random.default_rng(4).standard_normal((8192, 3))
    H.tile_table_load("")
    try:
        x0, choices0 = _profiled(_op(), b)
        tiled = [s for s, c in choices0.items() if not c.startswith("0,")]
        assert tiled
        f = tmp_path / "t.json"
        f.write_text(json.dumps({s: [32, 1, 0] for s in tiled}))
        H.tile_table_load(str(f))
        assert H.tile_table_size() == len(tiled)
        x1, choices1 = _profiled(_op(), b)
        for s in tiled:
            assert choices1[s] == "32,1,0", (s, choices1[s])
        # other tile shapes sum in another order: rounding (~1e-16) amplified by
        # cond(A) ~5e4 of this Gaussian operator
        assert O.rel_err(x0, x1) < 1e-9
    finally:
        H.tile_table_load("")
